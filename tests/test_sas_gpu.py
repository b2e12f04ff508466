"""The SAS arrangement built on the device equals the host build bit for
bit (the host build is pinned to the oracle by test_arrangement.py), and
meshes made over it equal meshes made over the host build byte for byte.
"""
import numpy as np
import pytest

from helpers import random_chain

pytestmark = pytest.mark.gpu

KEYS = ("orig", "center", "expanded", "status", "circle", "circle_ij", "vertex", "vertex_atoms", "nb_off",
        "nb_items", "cb_off", "cb_items")


def _sets():
    from sesmesh_b200 import workloads
    out = [("pair", np.array([[0, 0, 0, 1.7], [2.5, 0, 0, 1.5]]), 1.4),
           ("one", np.array([[0.3, -0.2, 0.1, 1.7]]), 1.4),
           ("zero radii", np.array([[0, 0, 0, 0.0], [1.0, 0, 0, 1.2], [5, 5, 5, 0.0], [1.5, 0.5, 0, 1.1]]), 1.2)]
    for seed, n in ((3, 30), (9, 50), (21, 120)):
        s, p = random_chain(seed, n)
        out.append(("chain%d" % seed, s, p))
    s, p = random_chain(4, 40)
    dup = np.concatenate([s, s[::4], [[s[0, 0] + 0.1, s[0, 1], s[0, 2], s[0, 3] * 0.3]]])
    out.append(("duplicates", dup, p))
    g = np.array([[x * 3.0, y * 3.0, z * 3.0, 1.6] for x in range(4) for y in range(4) for z in range(4)])
    out.append(("lattice", g, 1.4))
    out.append(("globule330", workloads.globule330()["spheres"], 1.4))
    out.append(("globule2800", workloads.globule2800()["spheres"], 1.4))
    out.append(("rings58800", workloads.rings58800()["spheres"], 1.4))
    return out


def _device_built(spheres, params):
    from sesmesh_b200 import surface as S
    S.set_device_arrangement_min(0)
    try:
        eng = S.SurfaceEngine(spheres, params)
        a = S.engine_arrangement(eng)
        eng.close()
        return a
    finally:
        S.set_device_arrangement_min(16384)


@pytest.mark.parametrize("case", _sets(), ids=lambda c: c[0])
def test_device_arrangement_equals_host(case):
    from sesmesh_b200 import surface as S
    name, spheres, probe = case
    p = S.SurfaceParams.ses(probe).with_spacing(0.5)
    got = _device_built(spheres, p)
    want = S.host_arrangement(spheres, p)
    assert got["built_on_device"]
    for k in KEYS:
        a, b = np.asarray(got[k]), np.asarray(want[k])
        assert a.shape == b.shape, (k, a.shape, b.shape)
        assert np.array_equal(a.view(np.uint8), b.view(np.uint8)), k
    for k in ("n_contained", "max_expanded", "rho_max"):
        assert got[k] == want[k], k


@pytest.mark.parametrize("refine", ["exact", "fast"])
@pytest.mark.parametrize("name,h", [("globule2800", 0.25), ("globule330", 0.5)])
def test_meshes_over_device_arrangement_equal_host(name, h, refine):
    from sesmesh_b200 import surface as S, workloads
    w = getattr(workloads, name)()
    p = S.SurfaceParams.ses(1.4).with_spacing(h).with_refine(refine)
    outs = []
    for threshold in (0, None):
        S.set_device_arrangement_min(threshold)
        try:
            o = S.compute_surface(w["spheres"], p)
            outs.append((o.obj(), dict(o.stats)))
            o.close()
        finally:
            S.set_device_arrangement_min(16384)
    (obj_d, st_d), (obj_h, st_h) = outs
    for k in ("vertices", "triangles", "components", "area", "volume", "refine_evaluations"):
        assert st_d[k] == st_h[k], (k, st_d[k], st_h[k])
    assert obj_d == obj_h
