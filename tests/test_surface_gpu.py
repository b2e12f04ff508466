"""compute_surface through the B200 back end against the CPU oracle.

Exact mode: OBJ bytes identical to the CPU back end's (the reference's
`--backend cuda --refine exact` contract, docs/06-gpu-cuda.md), plus equal
statistics.  Fast mode (field/gpu.rs:996-1070 rules): the same triangles,
area and volume within 4e-7 relative of exact mode, worst |F| at most the
exact worst + 1e-5 A, at most 0.1 % of vertices more than 1e-4 A off the
surface (FP64 evaluation of the exact field).
"""
import json
import os

import numpy as np
import pytest

import oracle as O
from helpers import random_chain

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _cases():
    from sesmesh_b200 import workloads
    out = []
    for row in json.load(open(os.path.join(GOLD, "analytic.json"))):
        if row["spacing"] in (0.5, 0.25):
            out.append(("%s@%g" % (row["case"], row["spacing"]), np.array(row["spheres"]), row["probe"],
                        row["spacing"]))
    for seed, n in ((5, 40), (11, 60), (31, 30)):
        s, p = random_chain(seed, n)
        out.append(("chain%d" % seed, s, p, 0.3))
    g = workloads.globule330()
    out.append(("globule330@0.5", g["spheres"], 1.4, 0.5))
    out.append(("globule330@0.25", g["spheres"], 1.4, 0.25))
    # Non-monotone edges where Newton stalls (tests/surface.rs:202-240 sets).
    out.append(("stall4", np.array([[42.580, -79.518, -23.569, 1.52], [45.767, -76.655, -20.023, 1.7],
                                    [46.735, -77.095, -22.324, 1.7], [45.949, -76.134, -21.455, 1.7]]), 1.4, 0.25))
    out.append(("stall3", np.array([[-6.673, 27.709, 45.944, 1.7], [-7.086, 29.017, 45.404, 1.7],
                                    [-5.941, 27.687, 40.494, 1.7]]), 1.4, 0.25))
    return out


CASES = _cases()


@pytest.mark.parametrize("case", CASES, ids=lambda c: c[0])
def test_exact_mode_obj_is_byte_identical(case):
    from sesmesh_b200 import surface as S
    name, spheres, probe, h = case
    out = S.compute_surface(spheres, S.SurfaceParams.ses(probe).with_spacing(h))
    ref = O.Surface(spheres, probe, h)
    st = out.stats
    for k in ("vertices", "triangles", "components", "surface_bricks"):
        assert st[k] == int(ref.stats[k]), k
    assert st["touched_bricks"] == int(ref.stats["touched"])
    assert st["area"] == ref.stats["area"] and st["volume"] == ref.stats["volume"]
    assert st["refine_evaluations"] == int(ref.stats["refine_evaluations"])
    assert out.obj() == ref.obj()


@pytest.mark.parametrize("case", [c for c in CASES if c[0].startswith(("chain", "globule", "pair r=1.7"))],
                         ids=lambda c: c[0])
def test_fast_mode_matches_exact_within_bounds(case):
    from sesmesh_b200 import surface as S
    name, spheres, probe, h = case
    base = S.SurfaceParams.ses(probe).with_spacing(h)
    exact = S.compute_surface(spheres, base)
    fast = S.compute_surface(spheres, base.with_refine("fast"))
    assert np.array_equal(fast.triangles, exact.triangles)
    for k in ("area", "volume"):
        rel = abs(fast.stats[k] - exact.stats[k]) / abs(exact.stats[k])
        assert rel <= 4e-7, (k, rel)
    eng = O.Engine(spheres, probe, h)
    fe = np.abs(eng.field(exact.positions.astype(np.float64)))
    ff = np.abs(eng.field(fast.positions.astype(np.float64)))
    assert ff.max() <= fe.max() + 1e-5
    assert np.count_nonzero(ff > 1e-4) <= max(1, len(ff) // 1000)
    assert fast.stats["refine_evaluations"] > 0


def test_engine_reuse_gives_the_same_mesh():
    from sesmesh_b200 import surface as S, workloads
    g = workloads.globule330()
    eng = S.SurfaceEngine(g["spheres"], S.SurfaceParams.ses(1.4).with_spacing(0.5))
    a = eng.mesh().obj()
    b = eng.mesh().obj()
    assert a == b


def test_invalid_parameters_are_rejected():
    from sesmesh_b200 import surface as S, native
    s = np.array([[0.0, 0.0, 0.0, 1.0]])
    for p in (S.SurfaceParams.ses(1.4).with_spacing(0.0), S.SurfaceParams.ses(1.4).with_spacing(float("nan")),
              S.SurfaceParams.ses(-1.0), S.SurfaceParams.ses(1.4).with_brick_size(1),
              S.SurfaceParams.ses(1.4).with_brick_size(9)):
        with pytest.raises(native.SmbError):
            S.compute_surface(s, p)


def test_empty_input_gives_an_empty_mesh():
    from sesmesh_b200 import surface as S
    out = S.compute_surface(np.zeros((0, 4)), S.SurfaceParams.ses(1.4))
    assert out.stats["triangles"] == 0 and out.stats["components"] == 0


def test_engine_field_equals_oracle_field():
    """smb_engine_field (the exact f64 field on the host, used for vertex
    distances) gives the CPU back end's SesField::value bit for bit within
    the refinement band around the surface, where it is defined."""
    from sesmesh_b200 import surface as S, workloads
    g = workloads.globule330()
    eng = S.SurfaceEngine(g["spheres"], S.SurfaceParams.ses(1.4).with_spacing(0.5))
    rng = np.random.default_rng(7)
    verts = eng.mesh().positions.astype(np.float64)
    pts = verts[::7] + rng.uniform(-0.3, 0.3, size=(len(verts[::7]), 3))
    got = eng.field(pts)
    want = O.Engine(g["spheres"], 1.4, 0.5).field(pts)
    eng.close()
    band = np.sqrt(3.0) * 0.5 * 1.01
    near = np.abs(want) < 0.9 * band
    assert near.sum() > 1000
    assert np.array_equal(got[near].view(np.uint64), want[near].view(np.uint64))
