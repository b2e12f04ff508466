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
