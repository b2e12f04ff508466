"""SAS and vdW surfaces through the device path against the CPU oracle.

A sphere field (SurfaceKind::Sas / Vdw, crates/sesmesh/src/field/mod.rs:
33-41) is min(|x - c| - R) over the spheres, R = r + probe for the SAS and r
for the vdW surface (SurfaceParams::effective_probe, surface.rs:411-417),
meshed by the same pipeline with the simpler field: brick classification on
the sign of s_sas (lattice.rs:213-215), the near spheres alone gathered
(gather_spheres, kernel.rs:651-654), sphere_kernel sampling
(kernel.rs:957-981), sphere-field refinement and attributes
(point.rs:566-579, 723-736; extract.rs:539-549, 583-587) and, in fast mode,
eval_point's sphere branch (sesmesh.cuh:486-503, 599-618).

* classification, sub-block states and every sample value equal the
  oracle's bit for bit;
* exact mode: OBJ bytes and statistics equal the oracle's;
* fast mode keeps the triangles, area and volume within 4e-7 relative of
  exact mode, worst |F| within exact's + 1e-5 A (the oracle's sphere field);
* tests/surface.rs:55-82 known answers (one sphere, all kinds) through the
  device path.
"""
import numpy as np
import pytest

import oracle as O
from helpers import arrangement_from_oracle, lattice_from_oracle, random_chain

pytestmark = pytest.mark.gpu


def _cases():
    from sesmesh_b200 import workloads
    out = [("single", np.array([[0.1, 0.2, 0.3, 1.8]]), 0.25),
           ("pair", np.array([[0, 0, 0, 1.7], [2.5, 0, 0, 1.5]]), 0.25),
           ("pair_far", np.array([[0, 0, 0, 1.5], [5.6, 0, 0, 1.5]]), 0.5)]
    s, _ = random_chain(5, 40)
    out.append(("chain5", s, 0.3))
    g = workloads.globule330()
    out.append(("globule330@0.5", g["spheres"], 0.5))
    out.append(("globule330@0.25", g["spheres"], 0.25))
    return out


CASES = [(kind, c) for kind in ("sas", "vdw") for c in _cases()]


def _params(kind, h):
    from sesmesh_b200 import surface as S
    return (S.SurfaceParams.sas(1.4) if kind == "sas" else S.SurfaceParams.vdw()).with_spacing(h)


@pytest.fixture(scope="module")
def device():
    from sesmesh_b200 import native
    return native.Device(0)


@pytest.mark.parametrize("kind,case", CASES, ids=lambda x: x if isinstance(x, str) else x[0])
def test_classification_and_values_equal_oracle(device, kind, case):
    from sesmesh_b200 import native
    name, spheres, h = case
    probe = 1.4 if kind == "sas" else 0.0
    eng = O.Engine(spheres, probe, h, 10, kind=kind)
    arr = arrangement_from_oracle(eng)
    arr["probe"] = probe
    arr["kind"] = kind
    assert len(arr["circle"]) == 0 and len(arr["vertex"]) == 0
    res = native.Resident(device, arr, lattice_from_oracle(eng, h, 10))
    touched, _ = res.classify()
    want_bricks, want_touched = eng.classify()
    assert touched == want_touched
    bricks = res.bricks()
    assert np.array_equal(bricks, want_bricks)
    b = native.Batch(res)
    b.run()
    st = eng.sub_states(bricks).reshape(-1)
    rec = b.records()
    assert np.array_equal(rec[:, 0].astype(np.int64), np.where(st < 0, 0, np.where(st == 1, 1, 2)))
    vals = b.values()
    want = eng.values(bricks)
    assert np.array_equal(vals.view(np.uint32), want.view(np.uint32))


@pytest.mark.parametrize("kind,case", CASES, ids=lambda x: x if isinstance(x, str) else x[0])
def test_exact_mode_obj_equals_oracle(kind, case):
    from sesmesh_b200 import surface as S
    name, spheres, h = case
    out = S.compute_surface(spheres, _params(kind, h))
    ref = O.Surface(spheres, 1.4 if kind == "sas" else 0.0, h, kind=kind)
    st = out.stats
    for k in ("vertices", "triangles", "components", "surface_bricks"):
        assert st[k] == int(ref.stats[k]), k
    assert st["area"] == ref.stats["area"] and st["volume"] == ref.stats["volume"]
    assert st["refine_evaluations"] == int(ref.stats["refine_evaluations"])
    assert out.obj() == ref.obj()


@pytest.mark.parametrize("kind,case", [c for c in CASES if c[1][0] in ("chain5", "globule330@0.25")],
                         ids=lambda x: x if isinstance(x, str) else x[0])
def test_fast_mode_within_bounds(kind, case):
    from sesmesh_b200 import surface as S
    name, spheres, h = case
    exact = S.compute_surface(spheres, _params(kind, h))
    fast = S.compute_surface(spheres, _params(kind, h).with_refine("fast"))
    assert np.array_equal(fast.triangles, exact.triangles)
    for k in ("area", "volume"):
        rel = abs(fast.stats[k] - exact.stats[k]) / abs(exact.stats[k])
        assert rel <= 4e-7, (k, rel)
    eng = O.Engine(spheres, 1.4 if kind == "sas" else 0.0, h, kind=kind)
    fe = np.abs(eng.field(exact.positions.astype(np.float64)))
    ff = np.abs(eng.field(fast.positions.astype(np.float64)))
    assert ff.max() <= fe.max() + 1e-5
    assert np.count_nonzero(ff > 1e-4) <= max(1, len(ff) // 1000)


def test_single_sphere_all_kinds_known_answers():
    """tests/surface.rs:55-82 through the device path."""
    from sesmesh_b200 import surface as S
    s = np.array([[0.3, -0.2, 0.1, 1.8]])
    for params, r, kind, probe in ((S.SurfaceParams.ses(1.4), 1.8, "ses", 1.4),
                                   (S.SurfaceParams.sas(1.4), 3.2, "sas", 1.4),
                                   (S.SurfaceParams.vdw(), 1.8, "vdw", 0.0)):
        out = S.compute_surface(s, params.with_spacing(0.25))
        st = out.stats
        assert st["components"] == 1 and st["euler"] == 2, kind
        area, vol = 4 * np.pi * r * r, 4.0 / 3.0 * np.pi * r ** 3
        assert abs(st["area"] - area) / area < 5e-3, kind
        assert abs(st["volume"] - vol) / vol < 1.2e-2, kind
        f, nrm, has = O.Engine(s, probe, 0.25, kind=kind).field_normals(out.positions.astype(np.float64))
        assert np.abs(f).max() < 1e-4 * 0.25 + 2e-6, kind
        a, b = nrm[has], out.normals.astype(np.float64)[has]
        ang = np.degrees(np.arctan2(np.linalg.norm(np.cross(a, b), axis=1), (a * b).sum(1)))
        assert ang.max() < 0.01, (kind, ang.max())


def test_ses_with_probe_zero_is_the_vdw_surface():
    from sesmesh_b200 import surface as S, workloads
    g = workloads.globule330()
    a = S.compute_surface(g["spheres"], S.SurfaceParams.ses(0.0).with_spacing(0.5))
    b = S.compute_surface(g["spheres"], S.SurfaceParams.vdw().with_spacing(0.5))
    assert a.obj() == b.obj()
