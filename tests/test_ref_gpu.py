"""The reference's own CUDA kernels (crates/sesmesh-gpu/kernels/sesmesh.cuh,
built from their source into oracle/_ref by `make -C oracle ref-gpu`) on the
same surface bricks as this library: their sample values must equal ours
bit for bit except the +-band values of uniform sub-blocks (the reference's
device parity rule, crates/sesmesh/src/field/gpu.rs:846-1070), and the test
prints both sides' device times (the GPU bar of the benchmark).
"""
import numpy as np
import pytest

import oracle as O
from helpers import arrangement_from_oracle, lattice_from_oracle

pytestmark = pytest.mark.gpu


def _cases():
    from sesmesh_b200 import workloads
    g = workloads.globule330()
    u = workloads.globule2800()
    r = workloads.rings58800()
    return [("globule330@0.5", g["spheres"], 1.4, 0.5), ("globule2800@0.25", u["spheres"], 1.4, 0.25),
            ("rings58800@0.25", r["spheres"], 1.4, 0.25)]


@pytest.mark.skipif(not O.ref_gpu_available(), reason="oracle/_ref not built (make -C oracle ref-gpu)")
@pytest.mark.parametrize("case", _cases(), ids=lambda c: c[0])
def test_reference_kernels_give_our_values(case):
    from sesmesh_b200 import native
    name, spheres, probe, h = case
    eng = O.Engine(spheres, probe, h, 10)
    bricks, _ = eng.classify()
    ref, t = O.ref_gpu_run(eng, bricks, h, 10, probe, reps=4)
    dev = native.Device(0)
    arr = arrangement_from_oracle(eng)
    arr["probe"] = probe
    res = native.Resident(dev, arr, lattice_from_oracle(eng, h, 10))
    res.classify()
    assert np.array_equal(res.bricks(), bricks)
    b = native.Batch(res)
    ours = []
    for _ in range(4):
        ours.append(b.run())
    vals = b.values()
    band = np.float32(eng.info["band"])
    sel = (np.abs(ref) != band) & (np.abs(vals) != band)
    assert sel.sum() > 0.3 * sel.size
    assert np.array_equal(ref[sel].view(np.uint32), vals[sel].view(np.uint32))
    # Signs agree everywhere (the mesh is the same).
    assert np.array_equal(ref < 0, vals < 0)
    o = min(ours[1:], key=lambda x: x["total"])
    print("%s: reference kernels count %.3f + scan %.3f (host) + fill %.3f + sample %.3f ms; "
          "ours sub-block states %.3f + gather %.3f + sample %.3f (+ marching cubes %.3f) ms"
          % (name, t["count_ms"], t["scan_ms"], t["fill_ms"], t["sample_ms"], o["substates"], o["gather"],
             o["sample"], o["mc"]))


def _reference_edge_keys(vals, b, edge_off):
    """Brick-global keys (brick * 3 b^3 + ((z b + y) b + x) 3 + axis) of the
    edges the reference's refine pass wrote, in its slot order: per
    sub-block, the crossing edges whose lower sample lies in it, in
    crossing_edge's z, y, x, axis order (sesmesh.cuh:624-637, 756-800).
    Sub-blocks the pass skipped (no slots) contribute nothing; the count of
    crossing edges in every other sub-block must equal its slots."""
    side, sub = b + 1, b // 2
    n = len(vals)
    v = vals.reshape(n, side, side, side) < 0                          # [brick, z, y, x]
    keys, sbs = [], []
    z, y, x = np.meshgrid(np.arange(b), np.arange(b), np.arange(b), indexing="ij")
    for axis in range(3):
        lo = v[:, :b, :b, :b]
        hi = [v[:, :b, :b, 1:side], v[:, :b, 1:side, :b], v[:, 1:side, :b, :b]][axis]
        cross = lo != hi
        bi, zi, yi, xi = np.nonzero(cross)
        keys.append(bi.astype(np.int64) * 3 * b ** 3 + ((zi * b + yi) * b + xi) * 3 + axis)
        sbs.append(bi.astype(np.int64) * 8 + (xi >= sub) + 2 * (yi >= sub) + 4 * (zi >= sub))
    keys, sbs = np.concatenate(keys), np.concatenate(sbs)
    order = np.lexsort((keys, sbs))
    keys, sbs = keys[order], sbs[order]
    counts = np.diff(edge_off.astype(np.int64))
    have = np.bincount(sbs, minlength=8 * n)
    written = counts > 0
    assert np.array_equal(have[written], counts[written])
    return keys[written[sbs]], int(have[~written].sum())


@pytest.mark.skipif(not O.ref_gpu_available(), reason="oracle/_ref not built (make -C oracle ref-gpu)")
@pytest.mark.parametrize("case", _cases(), ids=lambda c: c[0])
def test_reference_refine_gives_our_roots(case):
    """Fast mode: the reference's edge count + refine kernels (its f32
    Newton/Illinois iteration, sesmesh.cuh:669-754) and this library's
    smb_refine on the same bricks.  Every edge the reference refines is one
    of ours; where both ends' samples are the same bits on both sides the
    root parameter, feature word and evaluation count equal ours; prints
    both sides' device times."""
    from sesmesh_b200 import native
    name, spheres, probe, h = case
    b = 10
    eng = O.Engine(spheres, probe, h, b)
    bricks, _ = eng.classify()
    ref, t, fr = O.ref_gpu_run(eng, bricks, h, b, probe, reps=4, fast=True)
    dev = native.Device(0)
    arr = arrangement_from_oracle(eng)
    arr["probe"] = probe
    res = native.Resident(dev, arr, lattice_from_oracle(eng, h, b))
    res.classify()
    bt = native.Batch(res)
    bt.run()
    ms = [bt.refine() for _ in range(4)]
    vals = bt.values()
    t_o, feat_o, q_o, ev_o = bt.edges()
    m = bt.mc()
    per = np.diff(m["edge_off"].astype(np.int64))
    ours = np.repeat(np.arange(len(per), dtype=np.int64), per) * 3 * b ** 3 + m["edges"].astype(np.int64)
    assert np.all(np.diff(ours) > 0)
    rkeys, skipped = _reference_edge_keys(ref, b, fr["edge_off"])
    assert len(rkeys) == len(fr["t"])
    pos = np.searchsorted(ours, rkeys)
    pos = np.minimum(pos, len(ours) - 1)
    found = ours[pos] == rkeys
    assert found.all(), "reference refined %d edges this library does not own" % (~found).sum()
    # Same sample bits at both ends: the same start, so the same root.
    side = b + 1
    loc = rkeys % (3 * b ** 3)
    bi = rkeys // (3 * b ** 3)
    ax = loc % 3
    cell = loc // 3
    xi, yi, zi = cell % b, (cell // b) % b, cell // (b * b)
    i0 = xi + side * (yi + side * zi)
    i1 = i0 + np.where(ax == 0, 1, np.where(ax == 1, side, side * side))
    rv, ov = ref.view(np.uint32), vals.view(np.uint32)
    same = (rv[bi, i0] == ov[bi, i0]) & (rv[bi, i1] == ov[bi, i1])
    assert same.mean() > 0.95
    conv = (fr["evals"] >> 31).astype(bool) & (ev_o[pos] >> 31).astype(bool)
    sel = same & conv
    dt = np.abs(fr["t"][sel].astype(np.float64) - t_o[pos][sel].astype(np.float64)) * h
    far = dt > 4e-5
    assert far.mean() < 1e-3, (far.sum(), dt.max())
    kind_r, kind_o = fr["feat"][sel] >> 29, feat_o[pos][sel] >> 29
    assert (kind_r != kind_o).mean() < 2e-3
    bit_t = (fr["t"][sel].view(np.uint32) == t_o[pos][sel].view(np.uint32)).mean()
    # On B200 both iterations run the same f32 operations in the same order:
    # every same-start edge ends on the same bits, feature and evaluation
    # count (measured on all three workloads).
    assert bit_t == 1.0
    assert np.array_equal(fr["feat"][same], feat_o[pos][same])
    assert np.array_equal(fr["evals"][same], ev_o[pos][same])
    ev_r = (fr["evals"] & 0x7FFFFFFF).astype(np.int64).sum()
    ev_ours = (ev_o & 0x7FFFFFFF).astype(np.int64).sum()
    print("%s: %d edges refined by the reference (%d crossing edges in sub-blocks it skips), %d by this library; "
          "same-start roots: %.4f bit-equal t, max |dt| %.2e A; evaluations reference %d, ours %d; "
          "reference edge count %.3f + scan %.3f (host) + refine %.3f ms; ours refine %.3f ms"
          % (name, len(rkeys), skipped, len(ours), bit_t, dt.max() if len(dt) else 0.0, ev_r, ev_ours,
             t["edge_count_ms"], t["edge_scan_ms"], t["refine_ms"], min(ms[1:])))
