"""Learned warm start of fast-mode refinement (no counterpart in the
reference, whose fast mode starts every edge at the linear guess).

CPU: the committed weights (gate and root heads) load and are finite; the
gate's training label.
GPU:
* recording the nearest features leaves every sample value bit-identical
  to the oracle's, and each recorded feature is a candidate of the sample's
  own sub-block lists whose distance gives the sample's value;
* the feature pass covers exactly the edges the device refines, and its
  features equal a numpy restatement from the batch's own sample values,
  edge values, recorded features and the arrangement (the candidate's
  iteration in f64, compared with tolerances);
* a gate that answers below 0.5 everywhere (zero last layer, negative
  bias: the linear start) gives smb_refine's results bit for bit;
* training rows: labels are the exact refiner's roots, within the
  tolerance band of the device's own converged roots;
* with the committed gate, fast mode meets the fast-mode bounds against
  exact mode (same triangles, area and volume within 4e-7 relative, worst
  |F| at most exact's + 1e-5 A, at most 0.1 % of vertices beyond 1e-4 A;
  mean |F| printed) and its device refinement takes fewer field evaluations
  than the linear start on inputs outside the training set; the root head
  keeps the triangles and the |F| bounds (its area drift and evaluation
  count are printed beside the gate's).
"""
import numpy as np
import pytest

import oracle as O
from helpers import arrangement_from_oracle, lattice_from_oracle, random_chain


def test_committed_weights_load():
    from sesmesh_b200 import warm_start, native
    for path in (warm_start.WEIGHTS, warm_start.ROOT_WEIGHTS):
        p = warm_start.load(path)
        assert p.shape == (native.MLP_NPARAM,) and np.all(np.isfinite(p))


def test_target_marks_contact_starts_at_the_root():
    from sesmesh_b200 import warm_start
    x = np.zeros((6, 32), np.float32)
    x[:, warm_start.F_CONV] = [1, 1, 0, 1, 1, 1]
    x[:, warm_start.F_AGREE] = [1, 1, 1, 1, 1, 0]
    x[:, warm_start.F_TC] = [0.25, 0.4, 0.5, 0.9, 0.3, 0.25]
    x[:, warm_start.F_H] = 0.25
    t = np.array([0.25 + 4e-6, 0.5, 0.5, 0.1, 0.3, 0.25])
    # The fifth: plain stops elsewhere; the sixth: the samples name two features.
    tp = np.array([0.25, 0.4, 0.5, 0.9, 0.3 + 1e-7, 0.25], np.float32)
    assert np.array_equal(warm_start.target_of(x, t, tp), [1.0, 0.0, 0.0, 0.0, 0.0, 0.0])
    assert np.array_equal(warm_start.eligible(x), [True, True, False, True, True, False])
    xg, yg = warm_start.gate_rows(x, t, tp, neg_repeat=3)
    # Eligible rows 0, 1, 3, 4; the three labelled 0 twice more each.
    assert len(xg) == 4 + 2 * 3 and yg.sum() == 1.0
    assert np.array_equal(xg[:4], x[[0, 1, 3, 4]])


def test_training_set_spans_the_stated_sizes():
    from sesmesh_b200 import warm_start
    s = warm_start.train_set()
    assert len(s) == 200
    atoms = np.array([n for _, n, _ in s])
    assert atoms.min() >= 300 and atoms.max() <= 30000
    assert {h for _, _, h in s} == set(warm_start.SPACINGS)
    assert all(n <= warm_start.FINE_ATOMS for _, n, h in s if h < 0.25)
    assert 330 not in atoms


def _batch(device, spheres, probe, spacing, brick=10, record=True):
    from sesmesh_b200 import native
    eng = O.Engine(spheres, probe, spacing, brick)
    arr = arrangement_from_oracle(eng)
    arr["probe"] = probe
    res = native.Resident(device, arr, lattice_from_oracle(eng, spacing, brick))
    res.classify()
    b = native.Batch(res)
    if record:
        b.record_features(True)
    b.run()
    return eng, arr, res, b


SHIFT = 29


def _cand_eval(kind, cand, probe, band, x):
    """The candidate's part of the field at x (f64): value, closest point,
    found."""
    best = probe + band
    if kind == 2:
        c, R = cand
        d = x - c
        ln = np.sqrt(d @ d)
        lb = abs(ln - R)
        if not (lb >= best or ln < 1e-12):
            return probe - lb, c + d * (R / ln), True
    elif kind == 3:
        m, u, e1, r = cand
        y = x - m
        along = y @ u
        w = y - u * along
        wl = np.sqrt(w @ w)
        dist = np.sqrt(along * along + (wl - r) ** 2)
        if not dist >= best:
            q = m + (w / wl) * r if wl > 1e-12 else m + e1 * r
            return probe - dist, q, True
    elif kind == 4:
        p = cand
        v = np.sqrt((x - p) @ (x - p))
        if v < best:
            return probe - v, p, True
    return probe - best, x, False


def _cand_iteration(kind, cand, probe, band, a, ax, h, fa, fb, tol=1e-5, max_iter=8):
    """The refinement's Newton / Illinois steps on the candidate alone (f64)."""
    t = min(max(fa / (fa - fb), 0.0), 1.0)
    t0, g0, t1, g1, side = 0.0, fa, 1.0, fb, 0
    g = fa
    it = 0
    conv = False
    while it < max_iter:
        x = a.copy()
        x[ax] += h * t
        g, q, found = _cand_eval(kind, cand, probe, band, x)
        it += 1
        if abs(g) <= tol:
            conv = True
            break
        if (g < 0) == (g0 < 0):
            t0, g0 = t, g
            if side == -1:
                g1 *= 0.5
            side = -1
        else:
            t1, g1 = t, g
            if side == 1:
                g0 *= 0.5
            side = 1
        slope = 0.0
        if found:
            w = q - x
            ln = np.sqrt(w @ w)
            if ln > 1e-12:
                slope = w[ax] / ln * h
        newton = t - g / slope if slope != 0 else np.inf
        if abs(slope) > 1e-3 * h and t0 < newton < t1:
            t = newton
        else:
            sec = (t0 * g1 - t1 * g0) / (g1 - g0)
            t = sec if np.isfinite(sec) and t0 < sec < t1 else 0.5 * (t0 + t1)
    return t, it, abs(g), conv


def _owner(x, y, z, sub, states):
    """Engine::assign's owner of a sample (first non-uniform sub-block
    containing it, faces shared) or -1."""
    for q in range(8):
        ox, oy, oz = (q & 1) * sub, ((q >> 1) & 1) * sub, (q >> 2) * sub
        if ox <= x <= ox + sub and oy <= y <= oy + sub and oz <= z <= oz + sub and states[q] == 0:
            return q
    return -1


def _features_np(arr, probe, h, brick, bricks, vals, feats, mc, rec):
    s = brick + 1
    sub = brick // 2
    h32, p32 = np.float32(h), np.float32(probe)
    band = np.sqrt(3.0) * h * 1.01
    n_e = len(mc["edges"])
    F = np.zeros((n_e, 32), np.float64)
    cov = np.zeros(n_e, bool)
    for i in range(len(bricks)):
        v = vals[i].reshape(s, s, s)
        fw = feats[i].reshape(s, s, s)
        states = rec[8 * i:8 * i + 8, 0]
        origin = np.asarray(bricks[i], np.float64) * brick * h
        for k in range(mc["edge_off"][i], mc["edge_off"][i + 1]):
            cell, ax = divmod(int(mc["edges"][k]), 3)
            x, y, z = cell % brick, (cell // brick) % brick, cell // (brick * brick)
            sb = min(x // sub, 1) + 2 * min(y // sub, 1) + 4 * min(z // sub, 1)
            j = 8 * i + sb
            if rec[j, 0] != 0 or rec[j, 11] != 0:
                continue
            cov[k] = True
            fa, fb = np.float32(mc["edge_vals"][k, 0]), np.float32(mc["edge_vals"][k, 1])
            f = F[k]

            def grad(c):
                g = np.zeros(3, np.float32)
                for d in range(3):
                    lo, hi = list(c), list(c)
                    lo[d] -= 1
                    hi[d] += 1
                    V = lambda q: v[q[2], q[1], q[0]]
                    if lo[d] >= 0 and hi[d] <= brick:
                        g[d] = (V(hi) - V(lo)) / (np.float32(2.0) * h32)
                    elif hi[d] <= brick:
                        g[d] = (V(hi) - V(c)) / h32
                    else:
                        g[d] = (V(c) - V(lo)) / h32
                return g

            def word(c):
                o = _owner(c[0], c[1], c[2], sub, states)
                if o < 0 or rec[8 * i + o, 11] != 0:
                    return 1 << SHIFT
                return int(fw[c[2], c[1], c[0]])

            ca, cb = [x, y, z], [x + (ax == 0), y + (ax == 1), z + (ax == 2)]
            wa, wb = word(ca), word(cb)
            ka, kb = wa >> SHIFT, wb >> SHIFT
            prim = wa if ka >= 2 else (wb if kb >= 2 else 1 << SHIFT)
            kind, cid = prim >> SHIFT, prim & ((1 << SHIFT) - 1)
            f[0], f[1] = fa / h32, fb / h32
            f[2:5] = grad(ca)
            f[5:8] = grad(cb)
            t_lin = np.float32(min(max(fa / (fa - fb), np.float32(0)), np.float32(1)))
            f[8] = t_lin
            f[9], f[10], f[11] = kind == 2, kind == 3, kind == 4
            f[12] = wa == wb
            f[13] = ka >= 2 and kb >= 2 and wa != wb
            a = np.array([x, y, z], np.float64) * h
            if kind == 2:
                cand = (arr["center"][cid] - origin, arr["expanded"][cid])
                centre, size = cand[0], arr["expanded"][cid] - probe
            elif kind == 3:
                c = arr["circle"][cid]
                cand = (c[0:3] - origin, c[3:6], c[6:9], c[9])
                centre, size = cand[0], c[9]
            elif kind == 4:
                cand = arr["vertex"][cid] - origin
                centre, size = cand, 0.0
            if kind >= 2:
                tc, it, lg, conv = _cand_iteration(kind, cand, probe, band, a, ax, h, float(fa), float(fb))
                f[14], f[15] = conv, it / 8
                f[16] = np.clip(tc - float(t_lin), -0.5, 0.5) * 8
                f[17] = tc if conv else t_lin
                phi = lambda u: np.log10(max(u, 1e-9)) / 9 + 1
                f[18] = phi(lg)
                b_ = a.copy()
                b_[ax] += h
                f[19] = phi(abs(_cand_eval(kind, cand, probe, band, a)[0] - float(fa)))
                f[20] = phi(abs(_cand_eval(kind, cand, probe, band, b_)[0] - float(fb)))
                mid = a.copy()
                mid[ax] += 0.5 * h
                f[21:24] = (centre - mid) * 0.25
                f[24] = size * 0.25
            else:
                f[14:21] = [0, 0, 0, t_lin, 1, 1, 1]
            f[25], f[26] = h32, p32
            inv = h32 / (fb - fa)
            f[27] = np.clip(np.float32(f[2 + ax]) * inv, -10, 10)
            f[28] = np.clip(np.float32(f[5 + ax]) * inv, -10, 10)
            f[29] = np.clip(np.linalg.norm(f[2:5]) - 1, -4, 4)
            f[30] = np.clip(np.linalg.norm(f[5:8]) - 1, -4, 4)
            f[31] = (kb if prim == wa else ka) / 4
    return F, cov


@pytest.fixture(scope="module")
def device():
    from sesmesh_b200 import native
    return native.Device(0)


def _cases():
    from sesmesh_b200 import workloads
    s, p = random_chain(5, 40)
    g = workloads.globule330()
    return [("chain5", s, p, 0.3), ("globule330", g["spheres"], 1.4, 0.5)]


@pytest.mark.gpu
@pytest.mark.parametrize("case", _cases(), ids=lambda c: c[0])
def test_recorded_features_keep_values_and_name_the_nearest_candidate(device, case):
    name, spheres, probe, h = case
    eng, arr, res, b = _batch(device, spheres, probe, h)
    want = eng.values(res.bricks())
    vals = b.values()
    assert np.array_equal(vals.view(np.uint32), want.view(np.uint32))
    feats = b.sample_features()
    rec = b.records()
    ids = b.ids()
    brick, s, sub = 10, 11, 5
    bricks = res.bricks()
    band = np.sqrt(3.0) * h * 1.01
    checked = 0
    for i in range(0, len(bricks), max(1, len(bricks) // 60)):
        states = rec[8 * i:8 * i + 8, 0]
        origin = np.asarray(bricks[i], np.float64) * brick * h
        for idx in range(0, s ** 3, 7):
            x, y, z = idx % s, (idx // s) % s, idx // (s * s)
            o = _owner(x, y, z, sub, states)
            if o < 0 or rec[8 * i + o, 11] != 0:
                continue
            w = int(feats[i, idx])
            kind, cid = w >> SHIFT, w & ((1 << SHIFT) - 1)
            assert kind <= 4
            if kind < 2:
                continue
            lists = b.lists(rec[8 * i + o], ids)
            assert cid in {2: lists["s"], 3: lists["c"], 4: lists["v"]}[kind]
            p = np.array([x, y, z], np.float64) * h
            if kind == 2:
                cand = (arr["center"][cid] - origin, arr["expanded"][cid])
            elif kind == 3:
                c = arr["circle"][cid]
                cand = (c[0:3] - origin, c[3:6], c[6:9], c[9])
            else:
                cand = arr["vertex"][cid] - origin
            val = _cand_eval(kind, cand, probe, band, p)[0]
            assert abs(val - float(vals[i, idx])) <= 1e-4, (i, idx, kind, val, vals[i, idx])
            checked += 1
    assert checked > 100


@pytest.mark.gpu
@pytest.mark.parametrize("case", _cases(), ids=lambda c: c[0])
def test_features_match_restatement(device, case):
    name, spheres, probe, h = case
    eng, arr, res, b = _batch(device, spheres, probe, h)
    b.refine()
    _, _, _, ev = b.edges()
    x, cov = b.edge_features()
    assert np.array_equal(cov, ev != 0)
    F, cov_np = _features_np(arr, probe, h, 10, res.bricks(), b.values(), b.sample_features(), b.mc(), b.records())
    assert np.array_equal(cov, cov_np)
    assert np.all(x[~cov] == 0)
    xs, Fs = x[cov].astype(np.float64), F[cov]
    exact_cols = [0, 1, 2, 3, 4, 5, 6, 7, 8, 25, 26, 27, 28, 29, 30]
    np.testing.assert_allclose(xs[:, exact_cols], Fs[:, exact_cols], rtol=1e-5, atol=1e-6)
    np.testing.assert_array_equal(xs[:, [9, 10, 11, 12, 13, 31]], Fs[:, [9, 10, 11, 12, 13, 31]])
    has = Fs[:, 9] + Fs[:, 10] + Fs[:, 11] > 0
    assert has.mean() > 0.5
    np.testing.assert_allclose(xs[has][:, 21:25], Fs[has][:, 21:25], rtol=0, atol=2e-5)
    # The candidate's iteration: f32 on the device against f64 here (an
    # acceptance test at the tolerance can go either way): converged flags
    # and t_c for 99 % of the edges.
    agree = xs[has][:, 14] == Fs[has][:, 14]
    assert agree.mean() >= 0.99, agree.mean()
    both = has & (xs[:, 14] == 1) & (Fs[:, 14] == 1)
    d = np.abs(xs[both][:, 17] - Fs[both][:, 17])
    assert np.percentile(d, 99) <= 1e-3, np.percentile(d, 99)


@pytest.mark.gpu
def test_neutral_gate_reproduces_plain_refinement(device):
    from sesmesh_b200 import native, warm_start, workloads
    g = workloads.globule330()
    _, _, res, b = _batch(device, g["spheres"], 1.4, 0.25)
    b.refine()
    plain = b.edges()
    p = warm_start.init_params(3)
    p[-65:] = 0.0
    p[-1] = -20.0  # w3 = 0, b3 = -20: output below 0.5 everywhere, linear start
    mlp = native.Mlp(device, p)
    b.refine(mlp)
    warm = b.edges()
    for a, w in zip(plain, warm):
        assert np.array_equal(a.view(np.uint32), w.view(np.uint32))


@pytest.mark.gpu
def test_warm_refinement_needs_recorded_features(device):
    from sesmesh_b200 import native, warm_start, workloads
    g = workloads.globule330()
    _, _, res, b = _batch(device, g["spheres"], 1.4, 0.5, record=False)
    mlp = native.Mlp(device, warm_start.load())
    with pytest.raises(native.SmbError) as e:
        b.refine(mlp)
    assert e.value.code == 7


@pytest.mark.gpu
def test_training_rows_are_exact_roots(device):
    from sesmesh_b200 import surface as S
    s, probe = random_chain(11, 60)
    h = 0.3
    eng = S.SurfaceEngine(s, S.SurfaceParams.ses(probe).with_spacing(h))
    x, t, tp = eng.warm_start_rows()
    eng.close()
    assert len(x) > 100 and np.all((t >= 0) & (t <= 1))
    _, _, res, b = _batch(device, s, probe, h)
    b.refine()
    td, _, _, ev = b.edges()
    xf, cov = b.edge_features()
    assert len(x) <= cov.sum() and len(x) >= 0.99 * cov.sum()
    conv = (ev[cov] >> 31) == 1
    if len(x) == cov.sum():
        assert np.array_equal(xf[cov], x)
        # The plain roots are this batch's own converged f32 roots.
        assert np.array_equal(tp[conv].view(np.uint32), td[cov][conv].view(np.uint32))
        assert np.all(np.isnan(tp[~conv]))
        dt = np.abs(td[cov] - t)[conv] * h
        assert np.percentile(dt, 99) <= 1e-4, np.percentile(dt, 99)


WARM_CASES = [("globule330@0.5", 0.5), ("globule330@0.25", 0.25)]


@pytest.mark.gpu
@pytest.mark.parametrize("case", WARM_CASES, ids=lambda c: c[0])
def test_trained_warm_start_saves_evaluations(device, case):
    from sesmesh_b200 import native, surface as S, warm_start, workloads
    name, h = case
    g = workloads.globule330()
    base = S.SurfaceParams.ses(1.4).with_spacing(h)
    exact = S.compute_surface(g["spheres"], base)
    plain = S.compute_surface(g["spheres"], base.with_refine("fast"))
    ref = O.Engine(g["spheres"], 1.4, h)
    fe = np.abs(ref.field(exact.positions.astype(np.float64)))
    out = {}
    for head, path in (("gate", warm_start.WEIGHTS), ("root", warm_start.ROOT_WEIGHTS)):
        eng = S.SurfaceEngine(g["spheres"], base.with_refine("fast"))
        mlp = native.Mlp(eng.dev, warm_start.load(path))
        mlp.set_use(head)
        eng.set_warm_start(mlp)
        warm = eng.mesh()
        eng.close()
        assert np.array_equal(warm.triangles, exact.triangles)
        rel = {k: abs(warm.stats[k] - exact.stats[k]) / abs(exact.stats[k]) for k in ("area", "volume")}
        fw = np.abs(ref.field(warm.positions.astype(np.float64)))
        assert fw.max() <= fe.max() + 1e-5
        assert np.count_nonzero(fw > 1e-4) <= max(1, len(fw) // 1000)
        out[head] = (warm.stats["refine_evaluations"], rel, fw.mean())
    e_plain = plain.stats["refine_evaluations"]
    for head, (e_warm, rel, fmean) in out.items():
        print("%s %s: evaluations linear start %d, warm start %d (%.1f %% saved); area %.1e, volume %.1e of exact; "
              "mean |F| exact %.2e, warm %.2e" % (name, head, e_plain, e_warm, 100 * (1 - e_warm / e_plain),
                                                  rel["area"], rel["volume"], fe.mean(), fmean))
    e_gate, rel_gate, _ = out["gate"]
    for k in ("area", "volume"):
        assert rel_gate[k] <= 4e-7, (k, rel_gate[k])
    assert e_gate < 0.85 * e_plain
