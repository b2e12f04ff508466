"""Warm-start MLP: tcgen05 forward against the CPU reference."""
import numpy as np
import pytest

import mlp_reference as R


def test_reference_gradient_matches_finite_differences():
    rng = np.random.default_rng(1)
    p = R.init_params(3).astype(np.float64)
    x = rng.normal(0, 1, (16, R.IN))
    tgt = rng.uniform(0, 1, 16)
    loss, g = R.loss_and_grad(p, x, tgt, quantize=False)
    idx = rng.choice(R.NPARAM, 60, replace=False)
    for i in idx:
        e = 1e-6
        pp, pm = p.copy(), p.copy()
        pp[i] += e
        pm[i] -= e
        fd = (R.loss_and_grad(pp, x, tgt, quantize=False)[0] - R.loss_and_grad(pm, x, tgt, quantize=False)[0]) / (2 * e)
        assert abs(fd - g[i]) <= 1e-6 * max(1.0, abs(fd)) + 1e-9, (i, fd, g[i])


@pytest.mark.gpu
def test_tensor_core_forward_matches_reference():
    from sesmesh_b200 import native
    rng = np.random.default_rng(2)
    p = R.init_params(5)
    x = rng.normal(0, 1, (1000, R.IN)).astype(np.float32)
    dev = native.Device(0)
    m = native.Mlp(dev, p)
    t = m.forward(x)
    want, _ = R.forward(p, x)
    err = np.abs(t - want)
    assert err.max() < 2e-3 and err.mean() < 1e-4, (err.max(), err.mean())
    assert np.array_equal(m.params(), p)


@pytest.mark.gpu
def test_tensor_core_gradient_matches_reference():
    """Backward pass (all products on tcgen05) against the CPU reference with
    the same bf16 quantization points; tolerance from bf16 rounding of the
    quantized intermediates and f32 accumulation."""
    from sesmesh_b200 import native
    rng = np.random.default_rng(4)
    p = R.init_params(7)
    x = rng.normal(0, 1, (700, R.IN)).astype(np.float32)
    tgt = rng.uniform(0, 1, 700).astype(np.float32)
    dev = native.Device(0)
    m = native.Mlp(dev, p)
    loss, g = m.gradient(x, tgt)
    want_loss, want = R.loss_and_grad(p, x, tgt)
    assert abs(loss - want_loss) <= 1e-4 * want_loss + 1e-7
    scale = np.abs(want).max()
    err = np.abs(g - want)
    assert err.max() <= 2e-2 * scale, (err.max(), scale)
    # Per block, the relative error of the gradient vector.
    for lo, hi in ((R.W1, R.B1), (R.B1, R.W2), (R.W2, R.B2), (R.B2, R.W3), (R.W3, R.B3)):
        rel = np.linalg.norm(g[lo:hi] - want[lo:hi]) / max(np.linalg.norm(want[lo:hi]), 1e-12)
        assert rel < 1e-2, (lo, rel)


@pytest.mark.gpu
def test_training_reduces_the_loss():
    from sesmesh_b200 import native
    rng = np.random.default_rng(8)
    x = rng.normal(0, 1, (16384, R.IN)).astype(np.float32)
    w = rng.normal(0, 0.3, R.IN)
    tgt = (1.0 / (1.0 + np.exp(-(x @ w)))).astype(np.float32)
    dev = native.Device(0)
    m = native.Mlp(dev, R.init_params(9))
    first = m.train_epoch(x, tgt, batch=1024, lr=3e-3)
    for _ in range(4):
        last = m.train_epoch(x, tgt, batch=1024, lr=3e-3)
    assert last.mean() < 0.2 * first[:4].mean(), (first[:4], last[-4:])
