"""The benchmark configurations through the device path against the CPU oracle.

tests/golden/configs.json holds the oracle's exact-mode meshes of the
benchmark configurations (made by tests/golden/make_config_golden.py): the
58,800-sphere rings at 0.25 A, the 2.4 M-sphere icosahedral shell at 1 A and
every 16th structure of the 512-structure batch at its own probe and
spacing.  Here:

* exact mode (compute_surface, --refine exact): OBJ bytes, mesh arrays and
  statistics equal the oracle's (sha256 of the bytes, counts, area and
  volume bit for bit, refinement evaluations) -- the reference's
  device_meshes_equal_cpu_meshes contract (field/gpu.rs:906-962);
* fast mode, plain f32 refinement and the learned warm start: the rules of
  fast_meshes_match_exact_meshes (field/gpu.rs:996-1070) against the
  oracle's exact mesh: the same triangles, area and volume within 4e-7
  relative, worst |F| (exact f64 field, every k-th vertex) at most the
  exact mesh's worst + 1e-5 A, at most 0.1 % of those vertices beyond
  1e-4 A;
* the batch (one device pass over all 512 structures, fast mode, warm
  start, 16-sample bricks): each pinned structure by the fast-mode rules;
  and each pinned structure alone through compute_surface in exact mode
  at the same brick edge, equal to the oracle.  (The brick order sets the
  vertex order, so the pins are made at the brick edge the batch runs;
  tests/test_multi_gpu.py shows tuned and fixed configurations give the
  single-structure path's meshes.)
"""
import hashlib
import json
import os

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "configs.json")
CFG = json.load(open(GOLD)) if os.path.exists(GOLD) else {}


def _sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def _check_input(spheres, rec):
    got = _sha(np.ascontiguousarray(spheres, "<f8").reshape(-1, 4))
    assert got == rec["spheres_sha256"], "the seeded generator gives other spheres than the fixture's"


def _check_exact(out, rec):
    st = out.stats
    for k in ("vertices", "triangles", "components", "surface_bricks", "refine_evaluations"):
        assert st[k] == rec[k], k
    assert st["touched_bricks"] == rec["touched"]
    assert st["area"] == float.fromhex(rec["area"]) and st["volume"] == float.fromhex(rec["volume"])
    assert _sha(out.triangles.astype("<u4")) == rec["triangles_sha256"]
    assert _sha(out.positions.astype("<f4")) == rec["positions_sha256"]
    assert _sha(out.normals.astype("<f4")) == rec["normals_sha256"]
    assert _sha(out.vertex_atom.astype("<u4")) == rec["atoms_sha256"]
    assert _sha(out.vertex_patch.astype("u1")) == rec["patches_sha256"]
    obj = out.obj()
    assert len(obj) == rec["obj_bytes"]
    assert hashlib.sha256(obj).hexdigest() == rec["obj_sha256"]


def _check_fast(out, rec, field):
    st = out.stats
    assert st["vertices"] == rec["vertices"] and st["triangles"] == rec["triangles"]
    assert _sha(out.triangles.astype("<u4")) == rec["triangles_sha256"], "fast mode changed the triangles"
    for k in ("area", "volume"):
        want = float.fromhex(rec[k])
        rel = abs(st[k] - want) / abs(want)
        assert rel <= 4e-7, (k, rel)
    pick = out.positions[:: rec["F_stride"]].astype(np.float64)
    f = np.abs(field(pick))
    assert f.max() <= rec["F_max"] + 1e-5, (f.max(), rec["F_max"])
    assert np.count_nonzero(f > 1e-4) <= max(1, len(f) // 1000)
    assert st["refine_evaluations"] > 0
    return f


def _workload(name):
    from sesmesh_b200 import workloads
    return getattr(workloads, name)()


@pytest.mark.parametrize("name", [n for n in ("rings58800", "shell2400k") if n in CFG])
def test_exact_mode_equals_oracle(name):
    from sesmesh_b200 import surface as S
    rec = CFG[name]
    w = _workload(name)
    _check_input(w["spheres"], rec)
    p = S.SurfaceParams.ses(w["probe"]).with_spacing(w["spacing"]).with_brick_size(w["brick"])
    out = S.compute_surface(w["spheres"], p)
    assert out.stats["refine_cpu_edges"] == 0
    _check_exact(out, rec)


@pytest.mark.parametrize("name", [n for n in ("rings58800", "shell2400k") if n in CFG])
@pytest.mark.parametrize("warm", [False, True], ids=["plain", "warm"])
def test_fast_mode_within_bounds_of_oracle(name, warm):
    from sesmesh_b200 import native, warm_start
    from sesmesh_b200 import surface as S
    rec = CFG[name]
    w = _workload(name)
    p = S.SurfaceParams.ses(w["probe"]).with_spacing(w["spacing"]).with_brick_size(w["brick"]).with_refine("fast")
    eng = S.SurfaceEngine(w["spheres"], p)
    if warm:
        eng.set_warm_start(native.Mlp(eng.dev, warm_start.load()))
    out = eng.mesh()
    _check_fast(out, rec, eng.field)
    out.close()
    eng.close()


@pytest.fixture(scope="module")
def batch_run():
    from sesmesh_b200 import native, warm_start, workloads
    from sesmesh_b200 import surface as S
    items = workloads.batch512()
    structs = [(it["spheres"], S.SurfaceParams.ses(it["probe"]).with_spacing(it["spacing"])) for it in items]
    b = S.MultiBatch(structs, config=(CFG["batch512"]["brick"], 0, 4))
    b.set_warm_start(native.Mlp(b.dev, warm_start.load()))
    r = b.run()
    yield items, b, r
    b.close()


@pytest.mark.skipif("batch512" not in CFG, reason="no batch fixture")
def test_batch_structures_within_bounds_of_oracle(batch_run):
    from sesmesh_b200 import surface as S
    items, b, r = batch_run
    pinned = CFG["batch512"]["items"]
    assert len(pinned) == 32
    for key, rec in sorted(pinned.items(), key=lambda kv: int(kv[0])):
        i = int(key)
        it = items[i]
        _check_input(it["spheres"], rec)
        out = b.surface(i)
        if rec["vertices"] == 0:
            assert out.stats["triangles"] == 0
            continue
        eng = S.SurfaceEngine(it["spheres"], S.SurfaceParams.ses(it["probe"]).with_spacing(it["spacing"])
                              .with_brick_size(rec["brick"]))
        _check_fast(out, rec, eng.field)
        eng.close()


@pytest.mark.skipif("batch512" not in CFG, reason="no batch fixture")
def test_batch_structures_exact_equal_oracle():
    from sesmesh_b200 import surface as S, workloads
    items = workloads.batch512()
    for key, rec in sorted(CFG["batch512"]["items"].items(), key=lambda kv: int(kv[0])):
        it = items[int(key)]
        p = S.SurfaceParams.ses(it["probe"]).with_spacing(it["spacing"]).with_brick_size(rec["brick"])
        out = S.compute_surface(it["spheres"], p)
        _check_exact(out, rec)
