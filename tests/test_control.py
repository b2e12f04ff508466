"""Cooperative cancellation, progress and the device-memory guard
(Control, crates/sesmesh/src/control.rs:54-131; SurfaceParams::
with_max_memory / with_auto_coarsen, surface.rs:226-236, 776-890).

CPU (no device): the host arrangement build under a control polls the
cancel flag per sphere and returns SMB_ERR_CANCELLED, whether the flag is
set before the call or from another thread while it runs, and reports the
geometry stage's start and end; the device-memory estimate grows with the
surface bricks and is monotone in the spacing.  Two gloo ranks cancel their
own builds independently (one rank cancelled, the other finishes).
GPU: compute_surface_with reports every stage in order with the surface
bricks as the mesh stage's total; a flag set from the progress callback at
the mesh stage stops the computation with SMB_ERR_CANCELLED and the next
computation runs normally; a limit below the estimate refuses with
SMB_ERR_MEMORY before any mesh-stage buffer is taken, and with auto_coarsen
meshes at a coarser spacing whose estimate fits; the estimate bounds the
device bytes a run actually took; a batch run stops between groups when
cancelled.
"""
import threading
import time

import numpy as np
import pytest


def _spheres():
    from sesmesh_b200 import workloads
    return workloads.globule(4242, 20000)


def test_host_build_cancelled_before_start():
    from sesmesh_b200 import native, surface as S
    c = S.Control()
    c.cancel()
    with pytest.raises(native.SmbError) as e:
        S.host_arrangement(_spheres(), S.SurfaceParams.ses(1.4), control=c)
    assert e.value.code == 9


def test_host_build_cancelled_while_running():
    from sesmesh_b200 import native, surface as S
    sph = _spheres()
    t0 = time.perf_counter()
    S.host_arrangement(sph, S.SurfaceParams.ses(1.4))
    full = time.perf_counter() - t0
    c = S.Control()
    timer = threading.Timer(full * 0.2, c.cancel)
    timer.start()
    t0 = time.perf_counter()
    with pytest.raises(native.SmbError) as e:
        S.host_arrangement(sph, S.SurfaceParams.ses(1.4), control=c)
    took = time.perf_counter() - t0
    timer.cancel()
    assert e.value.code == 9
    assert took < full  # returned before a full build


def test_host_build_reports_geometry_progress():
    from sesmesh_b200 import surface as S
    seen = []
    c = S.Control(progress=lambda stage, done, total: seen.append((stage, done, total)))
    a = S.host_arrangement(_spheres()[:500], S.SurfaceParams.ses(1.4), control=c)
    assert seen == [("geometry", 0, 1), ("geometry", 1, 1)]
    assert len(a["center"]) == 500


def test_device_bytes_estimate_scales():
    from sesmesh_b200.native import lib
    est = lib().smb_device_bytes_estimate
    a = est(1000, 10, 0.25, 1.4, 100000, 0, 148)
    fixed = est(0, 10, 0.25, 1.4, 100000, 0, 148)
    assert fixed == 148 * 4 * 4 * (256 << 10) + (224 << 20)
    assert est(2000, 10, 0.25, 1.4, 100000, 0, 148) - fixed == 2 * (a - fixed)
    assert est(1000, 10, 1.0, 1.4, 100000, 0, 148) > a  # larger sub-blocks gather more candidates
    assert est(1000, 10, 1.0, 1.4, 50, 0, 148) < est(1000, 10, 1.0, 1.4, 100000, 0, 148)  # at most every sphere
    assert est(1000, 16, 0.25, 1.4, 100000, 0, 148) > a


def _rank(rank, world, port, q):
    import os
    import torch.distributed as dist
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    from sesmesh_b200 import native, surface as S
    c = S.Control()
    if rank == 1:
        c.cancel()
    try:
        S.host_arrangement(_spheres()[:2000], S.SurfaceParams.ses(1.4), control=c)
        got = 0
    except native.SmbError as e:
        got = e.code
    import torch
    t = torch.tensor([got])
    out = [torch.zeros(1, dtype=t.dtype) for _ in range(world)]
    dist.all_gather(out, t)
    q.put((rank, [int(x) for x in out]))
    dist.destroy_process_group()


def test_two_ranks_cancel_independently():
    import multiprocessing as mp
    import socket
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    ps = [ctx.Process(target=_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in ps:
        p.start()
    res = dict(q.get(timeout=120) for _ in ps)
    for p in ps:
        p.join(timeout=60)
    assert res[0] == [0, 9] and res[1] == [0, 9]


@pytest.mark.gpu
def test_progress_reports_every_stage():
    from sesmesh_b200 import surface as S, workloads
    g = workloads.globule330()
    seen = []
    c = S.Control(progress=lambda stage, done, total: seen.append((stage, done, total)))
    out = S.compute_surface_with(g["spheres"], S.SurfaceParams.ses(1.4).with_spacing(0.5), c)
    stages = [x[0] for x in seen]
    assert stages == ["geometry", "geometry", "classify", "classify", "mesh", "mesh", "assemble", "assemble",
                      "measure", "measure"]
    nb = out.stats["surface_bricks"]
    assert ("mesh", 0, nb) in seen and ("mesh", nb, nb) in seen
    assert out.stats["spacing_used"] == 0.5


@pytest.mark.gpu
def test_cancel_at_mesh_stage_then_run_again():
    from sesmesh_b200 import native, surface as S, workloads
    g = workloads.globule330()
    p = S.SurfaceParams.ses(1.4).with_spacing(0.25)
    holder = {}

    def on(stage, done, total):
        if stage == "mesh" and done == 0:
            holder["c"].cancel()

    c = S.Control(progress=on)
    holder["c"] = c
    with pytest.raises(native.SmbError) as e:
        S.compute_surface_with(g["spheres"], p, c)
    assert e.value.code == 9
    out = S.compute_surface_with(g["spheres"], p, S.Control())
    ref = S.compute_surface(g["spheres"], p)
    assert out.obj() == ref.obj()


@pytest.mark.gpu
def test_memory_guard_refuses_and_coarsens():
    from sesmesh_b200 import native, surface as S, workloads
    from sesmesh_b200.native import lib
    g = workloads.globule330()
    p = S.SurfaceParams.ses(1.4).with_spacing(0.1)
    ref = S.compute_surface(g["spheres"], p)
    est = ref.stats["device_bytes_estimate"]
    fixed = lib().smb_device_bytes_estimate(0, 10, 0.1, 1.4, 330, 0, S._device(0).multiprocessors)
    assert est > fixed
    limit = (est + fixed) // 2
    with pytest.raises(native.SmbError) as e:
        S.compute_surface_with(g["spheres"], p, S.Control(max_device_bytes=limit))
    assert e.value.code == 6 and "exceeds the limit" in str(e.value)
    out = S.compute_surface_with(g["spheres"], p, S.Control(max_device_bytes=limit, auto_coarsen=True))
    assert out.stats["spacing_used"] > 0.1
    assert out.stats["device_bytes_estimate"] <= limit
    want = S.compute_surface(g["spheres"], p.with_spacing(out.stats["spacing_used"]))
    assert out.obj() == want.obj()


@pytest.mark.gpu
@pytest.mark.parametrize("name,h", [("globule330", 0.25), ("globule2800", 0.25), ("globule2800", 1.0)])
def test_estimate_bounds_device_bytes_taken(name, h):
    from sesmesh_b200 import surface as S, workloads
    from sesmesh_b200.native import lib
    w = getattr(workloads, name)()
    for refine in ("exact", "fast"):
        eng = S.SurfaceEngine(w["spheres"], S.SurfaceParams.ses(1.4).with_spacing(h).with_refine(refine))
        out = eng.mesh()
        taken = lib().smb_engine_device_bytes(eng.h)
        est = out.stats["device_bytes_estimate"]
        print("%s@%g %s: estimate %.1f MB, taken %.1f MB" % (name, h, refine, est / 1e6, taken / 1e6))
        assert est >= taken
        eng.close()


@pytest.mark.gpu
def test_batch_run_cancelled_between_groups():
    from sesmesh_b200 import native, surface as S, workloads
    structs = [(workloads.globule(9100 + k, 60 + 20 * k), S.SurfaceParams.ses(1.4).with_spacing(0.5))
               for k in range(6)]
    b = S.MultiBatch(structs, config=(10, 0, 4))
    c = S.Control()
    c.cancel()
    b.set_control(c)
    with pytest.raises(native.SmbError) as e:
        b.run()
    assert e.value.code == 9
    b.set_control(None)
    t = b.run()
    assert t["structures"] == 6
    b.close()
