"""Vertex refinement, placement and the mesh's finish on the device
(smb_refine_exact in exact mode, smb_place_fast in fast mode).

The device restates the host's exact refinement operation by operation, so
the mesh must be byte-identical whichever side refines: OBJ bytes, counts,
area, volume and evaluation counts are compared for equality with the
host-refined mesh (and, through test_surface_gpu.py, with the CPU oracle).
The device must refine nearly every edge itself, and its whole-block path
(taken by sub-blocks whose lists exceed a warp's share of shared memory)
must give the same vertices as the warp path.  In fast mode the device's
placement of the f32 roots (and exact refinement of the edges they do not
settle) must equal the host placement byte for byte, with and without the
learned warm start.  The f32 refinement's second pass (whole blocks for
the sub-blocks whose lists outgrow a warp's region) must give the same mesh
as one pass with regions for every sub-block, and groups of 8 or 32 lanes
per edge the same mesh as each other; so must 1, 8 or 32 lanes per edge in
the exact refinement, in shared memory and in the global slabs, and the
sampling's second pass (sub-blocks over the first pass's shared memory).
"""
import ctypes as C

import numpy as np
import pytest

from helpers import random_chain

pytestmark = pytest.mark.gpu


def _cases():
    from sesmesh_b200 import workloads
    out = []
    for seed, n in ((5, 40), (11, 60)):
        s, p = random_chain(seed, n)
        out.append(("chain%d" % seed, s, p, 0.3))
    g = workloads.globule330()
    out.append(("globule330@0.5", g["spheres"], 1.4, 0.5))
    out.append(("globule330@0.25", g["spheres"], 1.4, 0.25))
    out.append(("globule330@1", g["spheres"], 1.4, 1.0))
    u = workloads.globule2800()
    out.append(("globule2800@0.25", u["spheres"], 1.4, 0.25))
    out.append(("one sphere", np.array([[0.3, -0.2, 0.1, 1.7]]), 1.4, 0.25))
    out.append(("stall4", np.array([[42.580, -79.518, -23.569, 1.52], [45.767, -76.655, -20.023, 1.7],
                                    [46.735, -77.095, -22.324, 1.7], [45.949, -76.134, -21.455, 1.7]]), 1.4, 0.25))
    return out


def _mesh(spheres, probe, h, on_device, region=None, brick=10, refine="exact", warm=None, refine_region=None,
          refine_group=None, exact_group=None, sample_region=None, exact_hint=None):
    from sesmesh_b200 import surface as S
    from sesmesh_b200.native import lib
    eng = S.SurfaceEngine(spheres, S.SurfaceParams.ses(probe).with_spacing(h).with_brick_size(brick)
                          .with_refine(refine))
    if warm is not None:
        eng.set_warm_start(warm)
    eng.set_exact_on_device(on_device)
    if region is not None:
        assert lib().smb_batch_set_exact_region(lib().smb_engine_batch(eng.h), C.c_size_t(region)) == 0
    if refine_region is not None:
        assert lib().smb_batch_set_refine_region(lib().smb_engine_batch(eng.h), C.c_size_t(refine_region)) == 0
    if refine_group is not None:
        assert lib().smb_batch_set_refine_group(lib().smb_engine_batch(eng.h), refine_group) == 0
    if exact_group is not None:
        assert lib().smb_batch_set_exact_group(lib().smb_engine_batch(eng.h), exact_group) == 0
    if exact_hint is not None:
        assert lib().smb_batch_set_exact_hint(lib().smb_engine_batch(eng.h), exact_hint) == 0
    if sample_region is not None:
        assert lib().smb_batch_set_sample_region(lib().smb_engine_batch(eng.h), C.c_size_t(sample_region)) == 0
    out = eng.mesh()
    res = (out.obj(), dict(out.stats))
    out.close()
    eng.close()
    return res


KEYS = ("vertices", "triangles", "components", "surface_bricks", "area", "volume", "euler", "refine_evaluations")


@pytest.mark.parametrize("case", _cases(), ids=lambda c: c[0])
def test_device_exact_equals_host_exact(case):
    name, spheres, probe, h = case
    obj_d, st_d = _mesh(spheres, probe, h, True)
    obj_h, st_h = _mesh(spheres, probe, h, False)
    for k in KEYS:
        assert st_d[k] == st_h[k], (k, st_d[k], st_h[k])
    assert obj_d == obj_h
    assert st_h["refine_cpu_edges"] == 0
    # The host refines only the edges the device leaves to it.
    if st_d["vertices"] > 1000:
        assert st_d["refine_cpu_edges"] < 0.01 * st_d["vertices"], st_d["refine_cpu_edges"]


@pytest.mark.parametrize("brick", [10, 16])
def test_block_path_equals_warp_path(brick):
    from sesmesh_b200 import workloads
    g = workloads.globule330()
    obj_w, st_w = _mesh(g["spheres"], 1.4, 0.35, True, brick=brick)
    obj_b, st_b = _mesh(g["spheres"], 1.4, 0.35, True, region=1024, brick=brick)
    for k in KEYS + ("refine_cpu_edges",):
        assert st_w[k] == st_b[k], (k, st_w[k], st_b[k])
    assert obj_w == obj_b


@pytest.mark.parametrize("case", [c for c in _cases() if c[0] in ("chain5", "globule330@0.5", "globule2800@0.25",
                                                                   "globule330@1", "stall4")], ids=lambda c: c[0])
def test_fast_device_placement_equals_host(case):
    name, spheres, probe, h = case
    obj_d, st_d = _mesh(spheres, probe, h, True, refine="fast")
    obj_h, st_h = _mesh(spheres, probe, h, False, refine="fast")
    for k in KEYS + ("refine_cpu_edges",):
        assert st_d[k] == st_h[k], (k, st_d[k], st_h[k])
    assert obj_d == obj_h


def test_fast_device_placement_with_warm_start_equals_host():
    from sesmesh_b200 import native, warm_start, workloads
    from sesmesh_b200 import surface as S
    g = workloads.globule2800()
    mlp = native.Mlp(S._device(0), warm_start.load())
    obj_d, st_d = _mesh(g["spheres"], 1.4, 0.25, True, refine="fast", warm=mlp)
    obj_h, st_h = _mesh(g["spheres"], 1.4, 0.25, False, refine="fast", warm=mlp)
    for k in KEYS + ("refine_cpu_edges",):
        assert st_d[k] == st_h[k], (k, st_d[k], st_h[k])
    assert obj_d == obj_h


@pytest.mark.parametrize("variant", [dict(refine_region=2048), dict(refine_group=32),
                                     dict(refine_group=32, refine_region=4096), dict(sample_region=2048)], ids=str)
@pytest.mark.parametrize("case", [c for c in _cases() if c[0] in ("globule330@0.5", "globule2800@0.25")],
                         ids=lambda c: c[0])
def test_fast_refine_variants_give_one_mesh(case, variant):
    name, spheres, probe, h = case
    obj_1, st_1 = _mesh(spheres, probe, h, True, refine="fast", refine_group=8)
    obj_2, st_2 = _mesh(spheres, probe, h, True, refine="fast", **variant)
    for k in KEYS + ("refine_cpu_edges",):
        assert st_1[k] == st_2[k], (k, st_1[k], st_2[k])
    assert obj_1 == obj_2


@pytest.mark.parametrize("group", [8, 32])
@pytest.mark.parametrize("region", [None, 1024], ids=["shared", "slab"])
@pytest.mark.parametrize("case", [c for c in _cases() if c[0] in ("chain5", "globule330@0.5", "globule2800@0.25",
                                                                   "stall4")], ids=lambda c: c[0])
def test_exact_groups_give_one_mesh(case, region, group):
    name, spheres, probe, h = case
    obj_1, st_1 = _mesh(spheres, probe, h, True, region=region, exact_group=1)
    obj_2, st_2 = _mesh(spheres, probe, h, True, region=region, exact_group=group)
    for k in KEYS + ("refine_cpu_edges",):
        assert st_1[k] == st_2[k], (k, st_1[k], st_2[k])
    assert obj_1 == obj_2


@pytest.mark.parametrize("hint", [0, 2])
@pytest.mark.parametrize("region", [None, 1024], ids=["shared", "slab"])
@pytest.mark.parametrize("case", [c for c in _cases() if c[0] in ("chain5", "globule330@0.5", "globule2800@0.25",
                                                                   "stall4")], ids=lambda c: c[0])
def test_exact_list_layouts_give_one_mesh(case, region, hint):
    name, spheres, probe, h = case
    obj_1, st_1 = _mesh(spheres, probe, h, True, region=region)
    obj_2, st_2 = _mesh(spheres, probe, h, True, region=region, exact_hint=hint)
    for k in KEYS + ("refine_cpu_edges",):
        assert st_1[k] == st_2[k], (k, st_1[k], st_2[k])
    assert obj_1 == obj_2
