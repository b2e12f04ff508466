"""Learned warm start of fast-mode refinement: training rows, training and
the committed weights.

The MLP (32 -> 64 -> 64 -> 1, GELU, sigmoid; BF16 weights on the tensor
cores, FP32 accumulation) chooses where each crossing edge's root search
begins.  The sampler records every sample's nearest feature; at an edge's
two samples it names one candidate (a sphere, a circle or a SAS vertex),
and the refinement iteration run on that candidate alone, without
evaluating the field, gives t_c.  With the gate head (the default, weights
data/warm_start.f32) the edge starts at t_c where both samples name the
candidate and the MLP answers >= 0.5, and at the linear guess
t_lin = fa / (fa - fb) elsewhere; with the root
head (data/warm_root.f32, smb_mlp_set_use ROOT) it starts at the MLP's
output itself.  The reference's bracketed Newton / Illinois / bisection
iteration then runs unchanged (smb_refine_warm): a start at which the field is
within the tolerance is accepted after one evaluation, any other falls back
to the bracketed refinement.  The reference's fast mode
(crates/sesmesh/src/field/gpu.rs:207-221 with the iteration of
crates/sesmesh/src/mesh/extract.rs:425-535) always starts at t_lin.  Where
the candidate is the surface's nearest feature at the iterates, t_c is
where that iteration would stop, so the gate keeps fast mode's vertices (and
its area and volume against exact mode) while it saves evaluations.

Training rows come from 200 seeded synthetic globules of 300-30,000 atoms
(log-uniform; none of them the 330-atom globule, the ring assemblies or the
shell that the tests and the benchmark use) at 0.1, 0.25, 0.35, 0.5 and
1 A (0.1 A for globules of at most 8,000 atoms),
at most ROWS_PER_GLOBULE rows each (about 1e7 in all): features from the
device feature pass (smb_batch_edge_features) and, as the label source,
the root parameter that exact mode's f64 refinement finds on the same edge
(smb_engine_warm_start_rows), with the root plain f32 refinement stops at.
Gate label: 1 where both samples name the candidate, t_c is that plain f32
root (the candidate's iteration followed the field's own) and lies within
2e-6 A of the exact root, else 0; the gate trains on the rows where both
samples name the candidate (the only rows it decides), those labelled 0
repeated NEG_REPEAT times.  Root head: the exact root itself, every row
(mean squared error on the sigmoid output for both).

    python -m sesmesh_b200.warm_start [--out-dir DIR]   # on a B200: writes
                                                      # warm_start.f32, warm_root.f32
"""
import argparse
import json
import os
import time

import numpy as np

from . import native, workloads
from .surface import SurfaceEngine, SurfaceParams, _device

DATA = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data")
WEIGHTS = os.path.join(DATA, "warm_start.f32")
ROOT_WEIGHTS = os.path.join(DATA, "warm_root.f32")

PROBE = 1.4
N_GLOBULES = 200
ROWS_PER_GLOBULE = 50000
SPACINGS = (0.1, 0.25, 0.35, 0.5, 1.0)
NEG_REPEAT = 10
FINE_ATOMS = 8000  # above it a 0.1 A turn takes 0.25 A (the edge count grows as 1 / h^2)


def train_set(n=N_GLOBULES, seed=7000):
    """(seed, atoms, spacing) of the training globules: atoms log-uniform in
    300..30,000, spacing cycling through SPACINGS (the spacings of the
    benchmark configurations and fast mode's usual ones)."""
    rng = np.random.default_rng(seed)
    atoms = np.exp(rng.uniform(np.log(300), np.log(30000), n)).round().astype(int)
    out = []
    for k in range(n):
        h = SPACINGS[k % len(SPACINGS)]
        if h < 0.25 and atoms[k] > FINE_ATOMS:
            h = 0.25
        out.append((seed + k, int(atoms[k]), h))
    return out


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
    """The committed warm-start parameters (SMB_MLP_NPARAM f32, little
    endian): the gate head by default, ROOT_WEIGHTS for the root head."""
    p = np.fromfile(path, dtype="<f4")
    if p.size != native.MLP_NPARAM:
        raise ValueError("%s holds %d values, not %d" % (path, p.size, native.MLP_NPARAM))
    return p


def save(params, path=WEIGHTS):
    os.makedirs(os.path.dirname(path) or ".", exist_ok=True)
    np.asarray(params, "<f4").tofile(path)


def rows(spheres, spacing, probe=PROBE, brick=10):
    """(features, exact t, plain f32 t) of every edge the device refines for
    one input."""
    params = SurfaceParams.ses(probe).with_spacing(spacing).with_brick_size(brick)
    eng = SurfaceEngine(spheres, params)
    try:
        return eng.warm_start_rows()
    finally:
        eng.close()


# Feature columns (smb_batch_edge_features): both samples name the same
# feature, t_c's iteration converged, t_c (t_lin where it did not), spacing.
F_AGREE, F_CONV, F_TC, F_H = 12, 14, 17, 25


def contact_start(x):
    """t_c as the features give it (-1 where the candidate's iteration did
    not converge or there is no candidate)."""
    return np.where(x[:, F_CONV] > 0.5, x[:, F_TC].astype(np.float64), -1.0)


def eligible(x):
    """Rows on which the gate decides: the candidate's iteration converged
    and both samples name the candidate (k_warm_starts sends every other row
    to t_lin whatever the gate answers)."""
    return (contact_start(x) >= 0) & (x[:, F_AGREE] > 0.5)


def target_of(x, t_exact, t_plain):
    """Gate label: 1 on an eligible row where t_c is where plain f32
    refinement stops (the same f32 value: the candidate's iteration followed
    the field's own) and lies within 2e-6 A of the exact root.  Accepting t_c
    there keeps plain fast mode's vertex, so area and volume keep their
    distance to exact mode's."""
    h = x[:, F_H].astype(np.float64)
    tc = contact_start(x)
    same = np.asarray(x[:, F_TC], np.float32) == np.asarray(t_plain, np.float32)
    return (eligible(x) & same & (np.abs(tc - t_exact) * h <= 2e-6)).astype(np.float32)


def training_rows(sets=None, per=ROWS_PER_GLOBULE, log=None):
    sets = train_set() if sets is None else sets
    rng = np.random.default_rng(1)
    xs, ts, ps = [], [], []
    for seed, n, h in sets:
        x, t, tp = rows(workloads.globule(seed, n), h)
        if len(x) > per:
            keep = np.sort(rng.choice(len(x), per, replace=False))
            x, t, tp = x[keep], t[keep], tp[keep]
        xs.append(x)
        ts.append(t)
        ps.append(tp)
        if log:
            log("seed %d: %d atoms at %.2f A -> %d rows" % (seed, n, h, len(x)))
    return np.concatenate(xs), np.concatenate(ts), np.concatenate(ps)


def gate_rows(x, t_exact, t_plain, neg_repeat=None):
    """The gate's training rows: the eligible rows alone (the gate decides
    no other), those labelled 0 repeated neg_repeat times.  Sending a row to
    t_c that the label rejects can move a vertex to another root on its edge,
    while the reverse costs only evaluations, so the repetition weights the
    first error above the second."""
    neg_repeat = NEG_REPEAT if neg_repeat is None else neg_repeat
    keep = eligible(x)
    xg, yg = x[keep], target_of(x, t_exact, t_plain)[keep]
    neg = np.nonzero(yg < 0.5)[0]
    if neg_repeat > 1 and len(neg):
        extra = np.tile(neg, neg_repeat - 1)
        xg, yg = np.concatenate([xg, xg[extra]]), np.concatenate([yg, yg[extra]])
    return xg, yg


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


def evaluate(params, x, t_exact, t_plain, device=0):
    """How the gate's choices compare with the labels: the fraction of edges
    sent to t_c, the fraction whose label is 1, precision and recall."""
    mlp = native.Mlp(_device(device), params)
    y = (mlp.forward(x) >= 0.5) & eligible(x)
    lab = target_of(x, t_exact, t_plain) > 0.5
    tp = float(np.sum(y & lab))
    return dict(rows=int(len(x)), sent_to_contact=float(y.mean()), label_rate=float(lab.mean()),
                precision=tp / max(1.0, float(y.sum())), recall=tp / max(1.0, float(lab.sum())))


def evaluate_root(params, x, t_exact, device=0):
    """The root head's error against the exact root, in A (median, 90th
    percentile)."""
    mlp = native.Mlp(_device(device), params)
    d = np.abs(mlp.forward(x).astype(np.float64) - t_exact) * x[:, F_H]
    return dict(rows=int(len(x)), median_A=float(np.median(d)), p90_A=float(np.percentile(d, 90)))


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--out-dir", default=DATA)
    ap.add_argument("--epochs", type=int, default=20)
    ap.add_argument("--batch", type=int, default=8192)
    ap.add_argument("--lr", type=float, default=2e-3)
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--globules", type=int, default=N_GLOBULES)
    ap.add_argument("--neg-repeat", type=int, default=NEG_REPEAT)
    a = ap.parse_args(argv)
    log = lambda m: print(m, flush=True)
    t0 = time.time()
    x, t, tp = training_rows(train_set(a.globules), log=log)
    log("%d rows in %.1f s" % (len(x), time.time() - t0))
    t1 = time.time()
    xg, yg = gate_rows(x, t, tp, a.neg_repeat)
    log("gate: %d eligible rows, %d labelled 0 (each repeated %d times)" % (len(xg), int((yg < 0.5).sum()) //
                                                                         max(1, a.neg_repeat), a.neg_repeat))
    gate, hist = train(xg, yg, epochs=a.epochs, batch=a.batch, lr=a.lr, seed=a.seed, log=log)
    save(gate, os.path.join(a.out_dir, "warm_start.f32"))
    root, hist_r = train(x, t.astype(np.float32), epochs=a.epochs, batch=a.batch, lr=a.lr, seed=a.seed + 7, log=log)
    save(root, os.path.join(a.out_dir, "warm_root.f32"))
    t_train = time.time() - t1
    held = workloads.globule330()
    xh, th, tph = rows(held["spheres"], held["spacing"], held["probe"], held["brick"])
    summary = dict(rows=int(len(x)), globules=a.globules, train_gate=evaluate(gate, x, t, tp),
                   held_out_globule330_gate=evaluate(gate, xh, th, tph),
                   held_out_globule330_root=evaluate_root(root, xh, th),
                   final_loss_gate=hist[-1], final_loss_root=hist_r[-1], seconds_rows=t1 - t0, seconds_train=t_train,
                   out_dir=a.out_dir)
    print(json.dumps(summary), flush=True)


if __name__ == "__main__":
    main()
