"""Learned warm start of fast-mode refinement: training rows, training and
the committed weights.

The MLP (32 -> 64 -> 64 -> 1, GELU, sigmoid; BF16 weights on the tensor
cores, FP32 accumulation) chooses where each crossing edge's root search
begins.  For the sphere candidate whose contact sphere best explains the
edge's two samples, the refinement kernel runs the refinement iteration on
that sphere alone, without evaluating the field (t_c); where the MLP
answers >= 0.5 the edge starts at t_c, else at the linear guess
t_lin = fa / (fa - fb).  The reference's bracketed Newton / Illinois /
bisection iteration then runs unchanged (smb_refine_warm): a start the
field judges within the tolerance is accepted after one evaluation, any
other falls back to the bracketed refinement.  The reference's fast mode
(crates/sesmesh/src/field/gpu.rs:207-221 with the iteration of
crates/sesmesh/src/mesh/extract.rs:425-535) always starts at t_lin.  Where
the sphere is the surface's nearest feature along the whole edge, t_c is
where that iteration would stop, so the warm start keeps fast mode's
vertices (and its area and volume against exact mode) while it saves the
evaluations.

Training rows come from seeded synthetic globules (none of them the
330-atom globule or the ring assemblies the tests and the benchmark use):
features from the device feature pass (smb_batch_edge_features) and the
root parameter that exact mode's f64 host refinement finds on the same edge
(smb_engine_warm_start_rows).  The label is 1 where t_c lies within
2e-6 A of that root, else 0 (mean squared error on the sigmoid output).

    python -m sesmesh_b200.warm_start            # on a B200: rewrites data/warm_start.f32
"""
import argparse
import json
import os
import time

import numpy as np

from . import native, workloads
from .surface import SurfaceEngine, SurfaceParams, _device

WEIGHTS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "warm_start.f32")

# (seed, atoms, spacing): globules of 150-1200 atoms, probe 1.4 A, brick 10,
# at the spacings fast mode is used at.
TRAIN_SET = [(7000 + k, n, h) for k, (n, h) in enumerate(
    [(150, 0.5), (300, 0.5), (600, 0.5), (1200, 0.5),
     (150, 0.35), (300, 0.35), (600, 0.35), (1200, 0.35),
     (150, 0.25), (300, 0.25), (600, 0.25), (800, 0.25)])]
PROBE = 1.4


def init_params(seed=0):
    """He-style initial parameters (W1 [64][32], b1, W2 [64][64], b2, w3, b3)."""
    rng = np.random.default_rng(seed)
    p = np.zeros(native.MLP_NPARAM, np.float32)
    w1, b1 = 0, 64 * 32
    w2, b2 = b1 + 64, b1 + 64 + 64 * 64
    w3 = b2 + 64
    p[w1:b1] = rng.normal(0, 1 / np.sqrt(32), 64 * 32)
    p[w2:b2] = rng.normal(0, 1 / np.sqrt(64), 64 * 64)
    p[w3:w3 + 64] = rng.normal(0, 0.1 / np.sqrt(64), 64)
    return p


def load(path=WEIGHTS):
    """The committed warm-start parameters (SMB_MLP_NPARAM f32, little endian)."""
    p = np.fromfile(path, dtype="<f4")
    if p.size != native.MLP_NPARAM:
        raise ValueError("%s holds %d values, not %d" % (path, p.size, native.MLP_NPARAM))
    return p


def save(params, path=WEIGHTS):
    os.makedirs(os.path.dirname(path), exist_ok=True)
    np.asarray(params, "<f4").tofile(path)


def rows(spheres, spacing, probe=PROBE, brick=10):
    """(features, exact t) of every edge the device refines for one input."""
    params = SurfaceParams.ses(probe).with_spacing(spacing).with_brick_size(brick)
    eng = SurfaceEngine(spheres, params)
    try:
        return eng.warm_start_rows()
    finally:
        eng.close()


def contact_start(x):
    """t_c as the features give it (-1 where it is half an edge or more from
    t_lin, which the kernel does not take)."""
    d = x[:, 26].astype(np.float64) / 8.0
    return np.where(np.abs(d) < 0.5, x[:, 27].astype(np.float64) + d, -1.0)


def target_of(x, t_exact, spacing=None):
    """1 where the contact iteration's result lies within 2e-6 A of the
    exact root, else 0 (spacing per row: feature 28)."""
    h = x[:, 28].astype(np.float64) if spacing is None else spacing
    tc = contact_start(x)
    return ((tc >= 0) & (np.abs(tc - t_exact) * h <= 2e-6)).astype(np.float32)


def training_rows(train_set=TRAIN_SET, log=None):
    xs, ts = [], []
    for seed, n, h in train_set:
        x, t = rows(workloads.globule(seed, n), h)
        xs.append(x)
        ts.append(t)
        if log:
            log("seed %d: %d atoms at %.2f A -> %d rows" % (seed, n, h, len(x)))
    return np.concatenate(xs), np.concatenate(ts)


def train(x, target, epochs=40, batch=4096, lr=2e-3, seed=0, device=0, log=None):
    """Adam on the device (smb_mlp_train_epoch), cosine-decayed step size,
    rows shuffled per epoch with a seeded generator."""
    dev = _device(device)
    mlp = native.Mlp(dev, init_params(seed))
    rng = np.random.default_rng(seed + 1)
    n = len(x) // batch * batch
    hist = []
    for ep in range(epochs):
        order = rng.permutation(len(x))[:n]
        step = lr * 0.5 * (1 + np.cos(np.pi * ep / epochs)) + lr * 0.02
        losses = mlp.train_epoch(x[order], target[order], batch=batch, lr=float(step))
        hist.append(float(np.mean(losses)))
        if log:
            log("epoch %d: lr %.2e loss %.3e" % (ep, step, hist[-1]))
    return mlp.params(), hist


def evaluate(params, x, t_exact, device=0):
    """How the MLP's choices compare with the labels: the fraction of edges
    sent to t_c, the fraction whose label is 1, precision and recall."""
    mlp = native.Mlp(_device(device), params)
    y = mlp.forward(x) >= 0.5
    lab = target_of(x, t_exact) > 0.5
    tp = float(np.sum(y & lab))
    return dict(rows=int(len(x)), sent_to_contact=float(y.mean()), label_rate=float(lab.mean()),
                precision=tp / max(1.0, float(y.sum())), recall=tp / max(1.0, float(lab.sum())))


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--out", default=WEIGHTS)
    ap.add_argument("--epochs", type=int, default=40)
    ap.add_argument("--batch", type=int, default=4096)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--seed", type=int, default=0)
    a = ap.parse_args(argv)
    log = lambda m: print(m, flush=True)
    t0 = time.time()
    x, t = training_rows(log=log)
    log("%d rows in %.1f s" % (len(x), time.time() - t0))
    params, hist = train(x, target_of(x, t), epochs=a.epochs, batch=a.batch, lr=a.lr, seed=a.seed, log=log)
    save(params, a.out)
    held = workloads.globule330()
    xh, th = rows(held["spheres"], held["spacing"], held["probe"], held["brick"])
    summary = dict(train=evaluate(params, x, t), held_out_globule330=evaluate(params, xh, th),
                   final_loss=hist[-1], seconds=time.time() - t0, out=a.out)
    print(json.dumps(summary))


if __name__ == "__main__":
    main()
