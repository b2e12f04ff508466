"""Many structures in one device pass (smb_multi_*).

Each structure's mesh must be the single-structure device path's at the
same brick edge: the batch runs the same kernels per (structure, brick)
item, so the OBJ bytes and statistics are compared for equality, with the
linear start and with the learned warm start.  The tuned configuration must
give the single path's meshes at the brick edge it chose, the pass must run
from a captured CUDA graph once recorded, and every structure must report a
latency within the run; finishing each structure on the device and on the
host threads gives the same bytes.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _structures():
    from sesmesh_b200 import surface as S, workloads
    rng = np.random.default_rng(24)
    out = []
    for k, n in enumerate([1, 20, 35, 60, 120, 200, 330, 500]):
        sph = workloads.globule(9000 + k, n) if n > 1 else np.array([[0.3, -0.2, 0.1, 1.7]])
        probe = float(rng.uniform(1.2, 1.4))
        h = [0.25, 0.5, 0.35][k % 3]
        out.append((sph, S.SurfaceParams.ses(probe).with_spacing(h)))
    return out


def _single(sph, params, brick, mlp=None):
    from sesmesh_b200 import surface as S
    eng = S.SurfaceEngine(sph, params.with_refine("fast").with_brick_size(brick))
    if mlp is not None:
        eng.set_warm_start(mlp)
    out = eng.mesh()
    res = (out.obj(), out.stats)
    out.close()
    eng.close()
    return res


def _check(batch, structs, brick, mlp=None):
    for i, (sph, params) in enumerate(structs):
        got = batch.surface(i)
        obj, st = _single(sph, params, brick, mlp)
        for k in ("vertices", "triangles", "components", "surface_bricks", "area", "volume", "refine_evaluations"):
            assert got.stats[k] == st[k], (i, k, got.stats[k], st[k])
        assert got.obj() == obj, i


@pytest.mark.parametrize("warm", [False, True], ids=["linear", "warm"])
def test_batch_equals_single_structure_path(warm):
    from sesmesh_b200 import native, surface as S, warm_start
    structs = _structures()
    mlp = None
    b = S.MultiBatch(structs, config=(10, 0, 4))
    if warm:
        mlp = native.Mlp(b.dev, warm_start.load())
        b.set_warm_start(mlp)
    t = b.run()
    assert t["structures"] == len(structs) and t["redone"] == 0
    _check(b, structs, 10, mlp)
    t2 = b.run()  # replay of the recorded pass
    assert t2["graph"] == 1
    _check(b, structs, 10, mlp)
    lat = b.latency()
    assert np.all(lat > 0) and np.all(lat <= t2["t_total"] + 1e-6)
    b.close()


def test_tuned_batch_equals_single_structure_path():
    from sesmesh_b200 import surface as S
    structs = _structures()
    b = S.MultiBatch(structs)
    cfg = b.tune()
    assert cfg["brick"] in (8, 16) and cfg["caps_level"] in (0, 1) and cfg["gather_warps"] in (2, 4)
    t = b.run()
    assert t["structures"] == len(structs)
    _check(b, structs, cfg["brick"])
    b.close()


def test_device_finish_equals_host_finish():
    from sesmesh_b200 import surface as S
    structs = _structures()
    outs = []
    for on in (True, False):
        b = S.MultiBatch(structs, config=(10, 0, 4))
        b.set_device_finish(on)
        t = b.run()
        assert t["structures"] == len(structs) and t["redone"] == 0
        outs.append([(b.surface(i).obj(), b.surface(i).stats) for i in range(len(structs))])
        b.close()
    for (obj_d, st_d), (obj_h, st_h) in zip(*outs):
        for k in ("vertices", "triangles", "components", "area", "volume", "refine_evaluations", "refine_cpu_edges"):
            assert st_d[k] == st_h[k], (k, st_d[k], st_h[k])
        assert obj_d == obj_h
