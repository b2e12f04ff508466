#!/usr/bin/env python3
"""Benchmark of the SES mesh stage on B200 (one JSON line on rank 0).

Workload (N=1): rings58800 -- 58,800 spheres (21 copies of a seeded
2,800-sphere globule on three stacked 7-fold rings), probe 1.4 A, spacing
0.25 A, brick 10: sesmesh's 1AON-at-0.25-A analogue, in fast mode with the
learned warm start (the configuration the metric compares with plain f32
refinement); --refine exact|fast|warm picks the main leg's mode.

* value -- device mesh-stage throughput in Mgridpts/s (grid points =
  surface bricks x (b+1)^3, as sesmesh counts samples) with the arrangement
  resident in HBM: brick classification, sub-block states, candidate gather,
  field sampling, marching-cubes compaction and the vertex refinement (the
  warm starts, f32 refinement and placement in fast mode; f64 in exact
  mode), timed with CUDA events on the library's stream; L2 flushed
  (256 MiB write) before every step.
* e2e -- the same metric through the public API from host sphere arrays
  (compute_surface; with the warm start, an engine with the model set):
  the arrangement (on the device for 16,384 spheres or more), the device
  stage, the mesh's assembly, validation, components, area and volume on
  the device, and the finished mesh copied back to page-locked host memory;
  wall clock.
* exact_mode -- the same assembly in exact mode (meshes byte-identical to
  the CPU back end), with its own value, e2e and roofline; fast_mode --
  plain f32 refinement against the warm start (end to end, device
  refinement, evaluations, area and volume against exact mode, vertex |F|).
* roofline -- the dominant kernel against its bound: counted operations of
  its evaluations per launch over the launch's CUDA-event time.
* cpu_baseline -- the CPU oracle (C++ restatement of sesmesh's CPU back end)
  meshing a sample of the same bricks on all host cores.

--impl reference runs that CPU path alone (the reference's own CPU back end
is Rust and cannot be built here; the oracle is its restatement).
Multi-GPU: independent replicas (one structure per GPU, no collective on the
data path); value = all ranks' grid points / max-over-ranks step time.
"""
import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

PEAKS_FALLBACK = {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}
# FP32 lanes x SMs x max clock, one operation per lane per cycle: the bound
# of kernels that may not contract multiply-adds (bit-exact f32).
FP32_NOFMA_TOPS = 148 * 128 * 1.965e9 / 1e12
FP64_NOFMA_TOPS = 148 * 64 * 1.965e9 / 1e12


def args_():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=5)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--workload", default="rings58800",
                   choices=["rings58800", "globule330", "globule2800", "shell2400k", "batch512"])
    p.add_argument("--refine", default=None, choices=[None, "exact", "fast", "warm"],
                   help="mode of the main leg (default: warm for rings58800, the workload's own otherwise)")
    p.add_argument("--spacing", type=float, default=None, help="override the workload's grid spacing")
    p.add_argument("--spheres", type=int, default=None,
                   help="keep the workload's first N spheres (smaller cases of the same kind, for ncu captures)")
    p.add_argument("--e2e-steps", type=int, default=2)
    p.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    p.add_argument("--no-fast", action="store_true", help="skip the fast-mode (plain vs warm start) leg")
    p.add_argument("--no-exact", action="store_true", help="skip the exact-mode block of a fast-mode line")
    p.add_argument("--no-configs", action="store_true",
                   help="skip the shell2400k and batch512 blocks of the default line")
    return p.parse_args()


def workload(name, refine=None, spacing=None, spheres=None):
    from sesmesh_b200 import workloads
    w = {"rings58800": workloads.rings58800, "globule330": workloads.globule330,
         "globule2800": workloads.globule2800, "shell2400k": workloads.shell2400k}[name]()
    if refine:
        w["refine"] = refine
    if spacing:
        w["spacing"] = spacing
    if spheres and spheres < len(w["spheres"]):
        w["spheres"] = w["spheres"][:spheres]
        w["name"] = "%s[:%d]" % (w["name"], spheres)
    return w


def describe(w):
    return ("%s: %d spheres, probe %.1f A, spacing %g A, brick %d, %s" %
            (w["name"], len(w["spheres"]), w["probe"], w["spacing"], w["brick"], w["refine"]))


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        d = json.load(open(path))
        return d, "measured"
    return PEAKS_FALLBACK, "fallback"


class Clocks:
    """nvidia-smi samples of SM clock and throttle reasons during a region."""

    def __init__(self, index):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(index), "--query-gpu=" + q, "--format=csv,noheader,nounits",
                                       "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.p.kill()
        self.f.seek(0)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.f.read().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        os.unlink(self.f.name)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def cpu_leg(w, budget_s=20.0):
    """CPU oracle on a deterministic sample of the workload's surface bricks
    (every k-th brick), all host threads: grid points per second."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    O.build()
    eng = O.Engine(w["spheres"], w["probe"], w["spacing"], w["brick"])
    bricks, _ = eng.classify()
    spb = (w["brick"] + 1) ** 3
    # Calibrate on a small sample, then size the sample to the time budget.
    k0 = max(1, len(bricks) // 500)
    t, _ = eng.mesh_sample(bricks[::k0])
    per_brick = t / max(1, len(bricks[::k0]))
    n_want = int(min(len(bricks), max(256, budget_s / max(per_brick, 1e-9))))
    k = max(1, len(bricks) // n_want)
    sample = bricks[::k]
    return eng, sample, spb, k, len(bricks)


def run_reference_batch(a):
    """The CPU restatement on every 16th structure of the batch (each one's
    mesh stage: classification, sampling, marching cubes, f64 refinement;
    the reference's CPU fast mode is its exact mode): structures/s."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    from sesmesh_b200 import workloads
    O.build()
    items = workloads.batch512()[::16]
    engs = []
    for it in items:
        e = O.Engine(it["spheres"], it["probe"], it["spacing"], 10)
        engs.append((e, e.classify()[0]))
    for _ in range(max(1, a.warmup)):
        engs[0][0].mesh_sample(engs[0][1])
    times = []
    for _ in range(a.steps):
        t = 0.0
        for e, bricks in engs:
            t0 = time.perf_counter()
            if len(bricks):
                e.mesh_sample(bricks)
            t += time.perf_counter() - t0
        times.append(t)
    value = len(engs) / float(np.mean(times))
    line = {
        "impl": "reference", "metric": "structures/s (batched SES meshes, fast mode + learned warm start)",
        "value": value, "unit": "structures/s", "n_gpus": a.gpus, "steps": a.steps, "warmup": a.warmup,
        "ms_per_step": 1e3 * float(np.mean(times)), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic (seeded)",
        "config": {"workload": "batch512 (every 16th structure: %d)" % len(engs)},
        "cpu_baseline": {"value": value, "unit": "structures/s", "cores": O.threads(), "kind": "port",
                         "sample": "every 16th of the 512 structures, whole mesh stage each"},
        "e2e": {"value": value, "unit": "structures/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def run_reference(a):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    if a.workload == "batch512":
        return run_reference_batch(a)
    w = workload(a.workload, None, a.spacing, a.spheres)
    mode = a.refine or ("warm" if a.workload == "rings58800" else w["refine"])
    w["refine"] = "exact" if mode == "exact" else "fast"
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    eng, sample, spb, k, nb = cpu_leg(w, budget_s=6.0)
    for _ in range(a.warmup):
        eng.mesh_sample(sample[: max(1, len(sample) // 4)])
    times = []
    for _ in range(a.steps):
        t, _ = eng.mesh_sample(sample)
        times.append(t)
    ms = 1e3 * float(np.mean(times))
    value = len(sample) * spb / (np.mean(times)) / 1e6
    cores = O.threads()
    line = {
        "impl": "reference", "metric": "Mgridpts/s (SES mesh stage, %s)" % MODE_NAMES[mode], "value": value,
        "unit": "Mgridpts/s",
        "n_gpus": a.gpus, "steps": a.steps, "warmup": a.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic (seeded)",
        "config": {"workload": describe(w) + ("" if mode != "warm" else " + learned warm start"),
                   "surface_bricks": nb, "sample": "every %d-th surface brick (%d bricks)" % (k, len(sample)),
                   "stage": "Engine::evaluate + mesh_brick per brick (exact f64 refinement: the reference's CPU "
                            "back end has no fast mode, its fast mode is the GPU's)"},
        "cpu_baseline": {"value": value, "unit": "Mgridpts/s", "cores": cores, "kind": "port",
                         "sample": "%d of %d surface bricks of %s" % (len(sample), nb, w["name"])},
        "e2e": {"value": value, "unit": "Mgridpts/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


MODE_NAMES = {"exact": "exact f64 refinement", "fast": "fast mode, plain f32 refinement",
              "warm": "fast mode, f32 refinement from the learned warm start"}


def rank_max(x, dist, device):
    """x's maximum over the ranks of the process group (x itself alone)."""
    import torch
    t = torch.tensor([float(x)], device=device, dtype=torch.float64)
    if dist is not None:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_value(grid_points, world, step_ms):
    """Whole-job throughput of N replicas (each rank meshes its own copy of
    the workload): all ranks' grid points over the slowest rank's step."""
    return world * grid_points / (step_ms / 1e3) / 1e6


def mode_params(w, mode, local):
    """SurfaceParams of a mode: exact, fast (plain f32) or warm (fast with
    the learned warm start)."""
    from sesmesh_b200 import surface as S
    p = S.SurfaceParams.ses(w["probe"]).with_spacing(w["spacing"]).with_brick_size(w["brick"]).with_refine(
        "exact" if mode == "exact" else "fast")
    return S.SurfaceParams(**{**p.__dict__, "device": local})


def new_engine(w, params, mlp):
    from sesmesh_b200 import surface as S
    eng = S.SurfaceEngine(w["spheres"], params)
    if mlp is not None:
        eng.set_warm_start(mlp)
    return eng


def mode_leg(a, w, mode, local, dev, barrier, max_over_ranks, world, flush, counted=True):
    """One mode of the workload: the device stage with the arrangement
    resident (CUDA events, L2 flushed before every step, max over ranks),
    then end to end through the public API, then the roofline of the
    dominant kernel."""
    from sesmesh_b200 import native, warm_start
    from sesmesh_b200 import surface as S
    import torch
    params = mode_params(w, mode, local)
    mlp = native.Mlp(S._device(local), warm_start.load()) if mode == "warm" else None
    eng = new_engine(w, params, mlp)
    for _ in range(max(3, a.warmup)):
        eng.run_device()
    n_bricks = eng.bricks
    spb = (w["brick"] + 1) ** 3
    grid_points = n_bricks * spb
    launches0 = native.lib().smb_kernel_launches()
    clocks = Clocks(local)
    barrier()
    step_ms, parts = [], []
    for _ in range(a.steps):
        flush.zero_()
        torch.cuda.synchronize(dev)
        t = eng.run_device()
        cls = eng.batch_info()["classify_ms"]
        step_ms.append(cls + t["total"])
        parts.append(dict(t, classify=cls))
    barrier()
    clk = clocks.stop()
    launches = native.lib().smb_kernel_launches() - launches0
    mean_ms = max_over_ranks(float(np.mean(step_ms)))
    value = replica_value(grid_points, world, mean_ms)
    stage = {k: float(np.mean([p[k] for p in parts])) for k in ("classify", "substates", "gather", "sample", "mc")}
    # Vertex refinement on the device: f64 in exact mode; in fast mode the
    # warm starts, the f32 refinement and the placement.
    stage["refine"] = float(np.mean([p["total"] - p["substates"] - p["gather"] - p["sample"] - p["mc"]
                                     for p in parts]))
    dominant = max(stage, key=stage.get)

    # End to end through the public API, host arrays in, mesh out: exact and
    # plain fast mode through compute_surface, the warm start through an
    # engine with the model set (arrangement, upload, device stage, finish,
    # copies back).  Two warm-up calls, so that the timed calls find the
    # memory caches in their steady state.
    def mesh_once():
        if mlp is None:
            return S.compute_surface(w["spheres"], params), None
        e = new_engine(w, params, mlp)
        return e.mesh(), e

    e2e_ms, st, out = [], None, None
    for _ in range(2 if a.e2e_steps else 0):
        out, e = mesh_once()
        if e is not None:
            out.close(), e.close()
    for _ in range(a.e2e_steps):
        if out is not None:
            out.close()
        barrier()
        t0 = time.perf_counter()
        out, e = mesh_once()
        torch.cuda.synchronize(dev)
        e2e_ms.append(1e3 * (time.perf_counter() - t0))
        if e is not None:
            st = dict(out.stats)
            out.close(), e.close()
            out = None
    if out is not None:
        st = dict(out.stats)
        out.close()
    e2e_mean = max_over_ranks(float(np.mean(e2e_ms)) if e2e_ms else float("nan"))
    info = eng.batch_info()
    st = st or {}
    # Host to device: the sphere rows when the device builds the arrangement,
    # else the uploaded arrangement (what the engine copied, counted by it).
    h2d = int(st.get("upload_bytes", 0))
    nv, nt = int(st.get("vertices", 0)), int(st.get("triangles", 0))
    if mode == "exact":
        # Finished on the device: the mesh alone (position, normal, atom,
        # component, patch per vertex; triangles) and 16 B of totals.
        d2h = nv * 33 + nt * 12 + 16
    else:
        d2h = n_bricks * 16 + (n_bricks + 1) * 8 + nv * 12 + nt * 12 + nv * 24
    pk, pk_kind = peaks()
    ops, owned = eng.count_ops() if counted else (0, 0)
    if counted and mode == "exact":
        rops = eng.count_exact_ops()
    elif counted:
        rops = eng.count_refine_ops(mlp)
    else:
        rops = 0
    roof = roofline(dominant, stage, info, ops, owned, w, pk, pk_kind, n_bricks, rops, mode)
    evals = int(st.get("refine_evaluations", 0))
    if roof.get("kernel", "").startswith("k_refine"):
        roof["evaluations"] = evals
    eng.close()
    leg = {
        "mode": mode, "value": value, "ms_per_step": mean_ms, "grid_points": int(grid_points),
        "surface_bricks": int(n_bricks), "stage_ms": stage,
        "lists": {"sampled_subblocks": int(info["sampled_subblocks"]), "ids_words": int(info["ids_words"]),
                  "pack_bytes_mean": float(info["pack_units"]) * 16 / max(1, info["sampled_subblocks"]),
                  "pack_bytes_max": int(info["max_pack_units"]) * 16, "edges": int(info["edges"]),
                  "triangles": int(info["triangles"])},
        "e2e": {"value": replica_value(grid_points, world, e2e_mean), "unit": "Mgridpts/s",
                "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": int(d2h), "ms_per_mesh": e2e_mean,
                "host_threads": st.get("host_threads"),
                "stages_ms": {k: st.get(k) for k in ("t_geometry", "t_upload", "t_device", "t_d2h", "t_host_refine",
                                                     "t_assemble", "t_measure", "t_total")},
                "mesh": {"vertices": nv, "triangles": nt, "area": st.get("area"), "volume": st.get("volume"),
                         "refine_evaluations": evals, "refine_cpu_edges": st.get("refine_cpu_edges")},
                "fallbacks": fallbacks(st)},
        "roofline": roof, "gpu_launches": int(launches), "clocks": clk,
    }
    return leg, st


def run_ours(a):
    import torch
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    else:
        torch.cuda.set_device(local)
    dev = torch.device("cuda", local)

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize(dev)

    def max_over_ranks(x):
        return rank_max(x, dist, dev)

    w = workload(a.workload, None, a.spacing, a.spheres)
    mode = a.refine or ("warm" if a.workload == "rings58800" else w["refine"])
    w["refine"] = "exact" if mode == "exact" else "fast"
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    leg, st = mode_leg(a, w, mode, local, dev, barrier, max_over_ranks, world, flush)
    line = {
        "metric": "Mgridpts/s (SES mesh stage, %s)" % MODE_NAMES[mode], "value": leg["value"], "unit": "Mgridpts/s",
        "n_gpus": world, "steps": a.steps, "warmup": max(3, a.warmup), "ms_per_step": leg["ms_per_step"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64" if mode == "exact" else "f32 (bf16 MLP)" if mode == "warm" else "f32",
        "data": "synthetic (seeded)",
        "config": {"workload": describe(w) + ("" if mode != "warm" else " + learned warm start"),
                   "spheres": int(len(w["spheres"])), "surface_bricks": leg["surface_bricks"],
                   "grid_points": leg["grid_points"], "refine": mode, "parallelism": "replicas x%d" % world,
                   "l2": "flushed before every step (256 MiB write)"},
        "stage_ms": leg["stage_ms"], "lists": leg["lists"], "e2e": leg["e2e"], "roofline": leg["roofline"],
        "gpu_launches": leg["gpu_launches"], "clocks": leg["clocks"],
    }
    exact_stats = st if mode == "exact" else None
    if rank == 0 and world == 1 and mode != "exact" and not a.no_exact:
        # Config 1: the same assembly in exact mode (byte-identical meshes).
        xleg, exact_stats = mode_leg(a, dict(w, refine="exact"), "exact", local, dev, barrier, max_over_ranks, 1,
                                     flush)
        line["exact_mode"] = {k: xleg[k] for k in ("value", "ms_per_step", "stage_ms", "e2e", "roofline",
                                                   "gpu_launches", "clocks")}
    if rank == 0 and world == 1 and not a.no_fast and exact_stats:
        line["fast_mode"] = fast_leg(w, mode_params(w, "fast", local), exact_stats, leg["grid_points"])
    if rank == 0 and world == 1 and not a.no_configs and a.workload == "rings58800" and not a.spheres:
        line["shell2400k"] = shell_leg(dev)
        line["batch512"] = batch_leg(dev)
        line["1AON"] = aon_leg(dev)
    if rank == 0 and world == 1 and not a.no_cpu:
        ceng, sample, spb_, k, nb = cpu_leg(w)
        t, _ = ceng.mesh_sample(sample)
        import oracle as O
        line["cpu_baseline"] = {"value": len(sample) * spb_ / t / 1e6, "unit": "Mgridpts/s", "cores": O.threads(),
                                "kind": "port",
                                "sample": "every %d-th of %d surface bricks (%d bricks, %.1f s): CPU oracle evaluate + "
                                          "mesh_brick (exact f64 refinement; the reference's CPU back end has no "
                                          "fast mode)" % (k, nb, len(sample), t)}
        # The same restatement on one core, on a smaller sample.
        cores = O.threads()
        O.set_threads(1)
        one = sample[:: max(1, 4 * cores)]
        t1, _ = ceng.mesh_sample(one)
        O.set_threads(cores)
        line["cpu_baseline_one_core"] = {"value": len(one) * spb_ / t1 / 1e6, "unit": "Mgridpts/s", "cores": 1,
                                         "kind": "port", "sample": "%d surface bricks (%.1f s)" % (len(one), t1)}
        if O.ref_gpu_available():
            stage_x = line.get("exact_mode", {}).get("stage_ms", line["stage_ms"])
            line["ref_kernels"] = ref_kernels_leg(ceng, w, stage_x, line.get("fast_mode"))
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


def fast_leg(w, params, exact_stats, grid_points, reps=2):
    """Fast mode on the same workload, plain f32 refinement against the
    learned warm start: end to end through the engine (arrangement, upload,
    device stage, copies, host placement, assembly, measure), device
    refinement time, field evaluations per edge, area and volume against
    exact mode, and vertex |F| from the exact f64 field on a sample of
    vertices."""
    from sesmesh_b200 import native
    from sesmesh_b200 import surface as S
    from sesmesh_b200 import warm_start
    fp = params.with_refine("fast")
    out = {}
    for mode in ("plain", "warm", "warm_root"):
        e2e, dev_refine = [], []
        st = None
        for r in range(reps + 1):
            t0 = time.perf_counter()
            eng = S.SurfaceEngine(w["spheres"], fp)
            mlp = None
            if mode == "warm":
                mlp = native.Mlp(eng.dev, warm_start.load())
                eng.set_warm_start(mlp)
            elif mode == "warm_root":
                mlp = native.Mlp(eng.dev, warm_start.load(warm_start.ROOT_WEIGHTS))
                mlp.set_use("root")
                eng.set_warm_start(mlp)
            mesh = eng.mesh()
            ms = 1e3 * (time.perf_counter() - t0)
            if r:  # the first is a warm-up
                e2e.append(ms)
            st = mesh.stats
            t = eng.run_device()
            dev_refine.append(t["total"] - t["substates"] - t["gather"] - t["sample"] - t["mc"])
            if r == reps:
                pos = mesh.positions
                pick = pos[:: max(1, len(pos) // 200000)].astype(np.float64)
                f = np.abs(eng.field(pick))
            mesh.close()
            eng.close()
        e2e_ms = float(np.mean(e2e))
        out[mode] = {
            "e2e_ms_per_mesh": e2e_ms, "e2e_Mgridpts_s": grid_points / (e2e_ms / 1e3) / 1e6,
            "device_refine_ms": float(np.median(dev_refine)),
            "evaluations": int(st["refine_evaluations"]), "edges": int(st["vertices"]),
            "evaluations_per_edge": st["refine_evaluations"] / max(1, st["vertices"]),
            "cpu_refined_edges": int(st["refine_cpu_edges"]),
            "area_rel_vs_exact": abs(st["area"] - exact_stats["area"]) / abs(exact_stats["area"]),
            "volume_rel_vs_exact": abs(st["volume"] - exact_stats["volume"]) / abs(exact_stats["volume"]),
            "vertex_F_max": float(f.max()) if len(f) else 0.0,
            "vertex_F_rms": float(np.sqrt(np.mean(f * f))) if len(f) else 0.0,
            "vertex_F_sample": int(len(f)),
            "stages_ms": {k: st[k] for k in ("t_geometry", "t_upload", "t_device", "t_d2h", "t_host_refine",
                                             "t_assemble", "t_measure")},
        }
    p = out["plain"]
    for mode in ("warm", "warm_root"):
        q = out[mode]
        out[mode + "_vs_plain"] = {"e2e_speedup": p["e2e_ms_per_mesh"] / q["e2e_ms_per_mesh"],
                                   "device_refine_speedup": p["device_refine_ms"] / max(q["device_refine_ms"], 1e-9),
                                   "evaluations_saved": 1.0 - q["evaluations"] / max(1, p["evaluations"])}
    # Amdahl: the warm start only changes the device refinement, so even a
    # free refinement bounds the end-to-end gain.
    out["e2e_ceiling_if_refine_free"] = p["e2e_ms_per_mesh"] / max(p["e2e_ms_per_mesh"] - p["device_refine_ms"], 1e-9)
    return out


def ref_kernels_leg(ceng, w, stage, fast, reps=5):
    """The reference's own CUDA kernels (sesmesh.cuh, built from their
    source into oracle/_ref) on every surface brick of the workload, pass by
    pass as cuda::Resident::run and ::refine issue them (64 threads per
    sub-block; the list-size and edge-count scans on the host), best of
    `reps` after a warm-up, beside this library's passes on the same bricks:
    list build (count + scan + fill against sub-block states + gather),
    sampling, crossing-edge enumeration (edge_count + scan against marching
    cubes with edge compaction) and the plain f32 refinement (fast mode)."""
    import oracle as O
    bricks, _ = ceng.classify()
    _, t, fr = O.ref_gpu_run(ceng, bricks, w["spacing"], w["brick"], w["probe"], reps=reps, fast=True)
    ref = {"count": t["count_ms"], "scan_host": t["scan_ms"], "fill": t["fill_ms"], "sample": t["sample_ms"],
           "edge_count": t["edge_count_ms"], "edge_scan_host": t["edge_scan_ms"], "refine": t["refine_ms"]}
    ours = {"substates": stage["substates"], "gather": stage["gather"], "sample": stage["sample"],
            "mc": stage["mc"]}
    if fast:
        ours["refine_f32"] = fast["plain"]["device_refine_ms"]
    # The passes do not split the work alike (this library's gather also
    # computes the keys, blockers and packed f32 blocks the reference's
    # sample pass derives per sample; its marching cubes also writes the
    # triangles, which the reference builds on the host), so the like-for-
    # like comparisons are the sampled values (lists + sampling) and the
    # refinement.
    ref_values = ref["count"] + ref["scan_host"] + ref["fill"] + ref["sample"]
    our_values = ours["substates"] + ours["gather"] + ours["sample"]
    out = {"bricks": int(len(bricks)), "edges_refined": int(len(fr["t"])),
           "evaluations": int((fr["evals"] & 0x7FFFFFFF).astype(np.int64).sum()),
           "reference_ms": ref, "ours_ms": ours,
           "speedup": {"values": ref_values / max(our_values, 1e-9),
                       "lists": (ref["count"] + ref["scan_host"] + ref["fill"]) /
                                max(ours["substates"] + ours["gather"], 1e-9),
                       "sample": ref["sample"] / max(ours["sample"], 1e-9),
                       "edges_vs_mc": (ref["edge_count"] + ref["edge_scan_host"]) / max(ours["mc"], 1e-9)}}
    if fast:
        out["speedup"]["refine_f32"] = ref["refine"] / max(ours["refine_f32"], 1e-9)
    return out


def fallbacks(st):
    """Work the device path handed to the host: the arrangement (1 built on
    the device, 0 on the host below the device threshold, 2 the device
    declined), meshes finished on the host and their host-refined edges.
    In fast mode the edges whose f32 search ends without converging go to
    the f64 refinement, as the reference sends them to its CPU refiner
    (refine_cpu_edges); on the device path that f64 pass runs on the
    device (f64_pass_edges)."""
    host = int(st.get("finished_on_host", 0))
    cpu = int(st.get("refine_cpu_edges", 0))
    return {"arrangement_where": int(st.get("arrangement_where", 0)), "finished_on_host": host,
            "host_refined_edges": cpu if host else 0, "f64_pass_edges": 0 if host else cpu}


# The reference's published wall times for 1AON at 0.25 A (CLI, best of 5,
# OBJ written to /dev/null, device open excluded; mesh stage in brackets):
# docs/05-gpu-hip.md:613 and docs/06-gpu-cuda.md:177.
AON_PUBLISHED_MS = {
    "cpu_16_zen5": {"total": 3403, "mesh_stage": 2504},
    "radeon_8060s_exact": {"total": 2366, "mesh_stage": 1463}, "radeon_8060s_fast": {"total": 1411, "mesh_stage": 534},
    "rtx2070_exact": {"total": 6984, "mesh_stage": 4497}, "rtx2070_fast": {"total": 4192, "mesh_stage": 1357},
}


def aon_leg(dev, reps=3):
    """1AON (GroEL-GroES, the reference's own data/1aon.pdb, 58,870 atoms
    after the default selection) at 0.25 A, timed as the reference's CLI
    numbers are: parse the PDB text, mesh, write the OBJ to /dev/null; exact
    mode, plain fast mode and fast mode with the learned warm start; best of
    `reps` after a warm-up.  Gzip decompression of the committed fixture is
    outside the timing (the reference reads the plain file)."""
    import gzip
    from sesmesh_b200 import native, structure, warm_start
    from sesmesh_b200 import surface as S
    with gzip.open(os.path.join(ROOT, "tests", "golden", "1AON.pdb.gz"), "rb") as f:
        text = f.read()
    out = {"workload": "1AON (58,870 atoms), probe 1.4 A, spacing 0.25 A, brick 10",
           "published_ms": AON_PUBLISHED_MS}
    mlp = None
    for mode in ("exact", "fast", "fast+warm"):
        p = S.SurfaceParams.ses(1.4).with_spacing(0.25).with_refine("exact" if mode == "exact" else "fast")
        best, st = None, None
        for r in range(reps + 1):
            t0 = time.perf_counter()
            spheres = structure.read_bytes(text, "pdb")
            t1 = time.perf_counter()
            if mode == "fast+warm":
                eng = S.SurfaceEngine(spheres, p)
                if mlp is None:
                    mlp = native.Mlp(eng.dev, warm_start.load())
                eng.set_warm_start(mlp)
                mesh = eng.mesh()
            else:
                eng = None
                mesh = S.compute_surface(spheres, p)
            t2 = time.perf_counter()
            mesh.write_obj(os.devnull)
            t3 = time.perf_counter()
            times = {"parse": 1e3 * (t1 - t0), "mesh": 1e3 * (t2 - t1), "obj": 1e3 * (t3 - t2),
                     "total": 1e3 * (t3 - t0)}
            if r and (best is None or times["total"] < best["total"]):
                best = times
            st = mesh.stats
            mesh.close()
            if eng is not None:
                eng.close()
        out[mode] = {"ms": best, "vertices": int(st["vertices"]), "triangles": int(st["triangles"]),
                     "area": st["area"], "volume": st["volume"], "refine_evaluations": int(st["refine_evaluations"])}
    return out


def shell_leg(dev, reps=2):
    """The 2.4 M-sphere icosahedral shell at 1 A (60 x 40,000 spheres on a
    380 A sphere), probe 1.4 A: exact and fast mode (plain f32 and the
    learned warm start) end to end through compute_surface / the engine
    (host sphere rows in, finished mesh in host memory out; wall clock,
    first call a warm-up), and the device stage with the arrangement
    resident (CUDA events, L2 flushed)."""
    import torch
    from sesmesh_b200 import native, warm_start
    from sesmesh_b200 import surface as S
    w = workload("shell2400k")
    base = S.SurfaceParams.ses(w["probe"]).with_spacing(w["spacing"]).with_brick_size(w["brick"])
    out = {"workload": describe(w)}
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    for mode in ("exact", "fast", "fast+warm"):
        p = base.with_refine("fast" if mode.startswith("fast") else "exact")
        times, st = [], None
        for r in range(reps + 1):
            torch.cuda.synchronize(dev)
            t0 = time.perf_counter()
            eng = S.SurfaceEngine(w["spheres"], p)
            if mode == "fast+warm":
                eng.set_warm_start(native.Mlp(eng.dev, warm_start.load()))
            mesh = eng.mesh()
            torch.cuda.synchronize(dev)
            ms = 1e3 * (time.perf_counter() - t0)
            if r:
                times.append(ms)
            st = mesh.stats
            if r == reps:
                dev_ms = []
                for _ in range(3):
                    flush.zero_()
                    torch.cuda.synchronize(dev)
                    t = eng.run_device()
                    dev_ms.append(eng.batch_info()["classify_ms"] + t["total"])
            mesh.close()
            eng.close()
        gp = st["samples"]
        e2e = float(np.mean(times))
        out[mode] = {"e2e_ms_per_mesh": e2e, "e2e_Mgridpts_s": gp / (e2e / 1e3) / 1e6,
                     "device_ms": float(np.median(dev_ms)), "device_Mgridpts_s": gp / (np.median(dev_ms) / 1e3) / 1e6,
                     "stages_ms": {k: st[k] for k in ("t_geometry", "t_upload", "t_device", "t_assemble", "t_measure")},
                     "vertices": int(st["vertices"]), "triangles": int(st["triangles"]),
                     "refine_evaluations": int(st["refine_evaluations"]), "area": st["area"], "volume": st["volume"],
                     "fallbacks": fallbacks(st)}
    ex = out["exact"]
    for mode in ("fast", "fast+warm"):
        out[mode]["area_rel_vs_exact"] = abs(out[mode]["area"] - ex["area"]) / abs(ex["area"])
        out[mode]["volume_rel_vs_exact"] = abs(out[mode]["volume"] - ex["volume"]) / abs(ex["volume"])
    out["cpu_baseline"] = ("not run here: the oracle's single-threaded arrangement of 2.4 M spheres alone takes "
                           "minutes; bench.py --workload shell2400k --impl reference times its mesh stage")
    return out


def batch_leg(dev, steps=2):
    """The 512-structure batch (fast mode, learned warm start, autotuned):
    structures/s over whole runs (wall clock; arrangements resident), p50/p99
    per-structure latency, structures redone alone."""
    import torch
    from sesmesh_b200 import native, warm_start, workloads
    from sesmesh_b200 import surface as S
    items = workloads.batch512()
    structs = [(it["spheres"], S.SurfaceParams.ses(it["probe"]).with_spacing(it["spacing"])) for it in items]
    b = S.MultiBatch(structs)
    b.set_warm_start(native.Mlp(b.dev, warm_start.load()))
    cfg = b.tune()
    b.run()
    runs, lats = [], []
    for _ in range(steps):
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        r = b.run()
        r["wall_ms"] = 1e3 * (time.perf_counter() - t0)
        runs.append(r)
        lats.append(b.latency())
    wall = float(np.mean([r["wall_ms"] for r in runs]))
    lat = np.concatenate(lats)
    last = runs[-1]
    out = {"workload": "batch512: 512 globules, atoms log-uniform 20-5000, probe U(1.2, 1.4), spacing in "
                       "{0.1, 0.25, 0.5} A, fast mode + learned warm start",
           "structures_per_s": len(items) / (wall / 1e3), "ms_per_batch": wall,
           "grid_Mpts_s": last["samples"] / (wall / 1e3) / 1e6,
           "latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99))},
           "tuned": cfg, "groups": int(last["groups"]), "graph": bool(last["graph"]),
           "redone": int(last["redone"]), "over_lists": int(last["over_lists"]), "over_memory": int(last["over_memory"]),
           "once_ms": {"t_setup": last["t_setup"], "t_tune": last["t_tune"]}}
    b.close()
    return out


def run_batch(a):
    """Config: 512 seeded structures in one device pass per group (fast mode,
    learned warm start, autotuned brick edge, caps and gather block)."""
    import torch
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    else:
        torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    from sesmesh_b200 import native, warm_start, workloads
    from sesmesh_b200 import surface as S
    items = workloads.batch512()
    structs = [(it["spheres"], S.SurfaceParams.ses(it["probe"]).with_spacing(it["spacing"])) for it in items]
    b = S.MultiBatch(structs, device=local)
    mlp = native.Mlp(b.dev, warm_start.load())
    b.set_warm_start(mlp)
    cfg = b.tune()
    for _ in range(max(3, a.warmup)):
        b.run()
    clocks = Clocks(local)
    runs, lats = [], []
    for _ in range(a.steps):
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        r = b.run()
        r["wall_ms"] = 1e3 * (time.perf_counter() - t0)
        runs.append(r)
        lats.append(b.latency())
    clk = clocks.stop()
    wall = float(np.mean([r["wall_ms"] for r in runs]))
    t = torch.tensor([wall], dtype=torch.float64, device=dev)
    if dist is not None:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    wall = float(t.item())
    lat = np.concatenate(lats)
    last = runs[-1]
    line = {
        "metric": "structures/s (batched SES meshes, fast mode + learned warm start)",
        "value": world * len(items) / (wall / 1e3), "unit": "structures/s", "n_gpus": world, "steps": a.steps,
        "warmup": max(3, a.warmup), "ms_per_step": wall, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic (seeded)",
        "config": {"workload": "batch512: 512 globules, atoms log-uniform 20-5000, probe U(1.2, 1.4), "
                               "spacing in {0.1, 0.25, 0.5} A", "atoms": int(sum(len(it["spheres"]) for it in items)),
                   "tuned": cfg, "groups": int(last["groups"]), "graph": bool(last["graph"]),
                   "parallelism": "replicas x%d" % world},
        "grid_Mpts_s": world * last["samples"] / (wall / 1e3) / 1e6,
        "latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99))},
        "stages_ms": {k: float(np.mean([r[k] for r in runs])) for k in ("t_classify", "t_device", "t_d2h", "t_host",
                                                                         "t_redo", "t_total")},
        "once_ms": {"t_setup": last["t_setup"], "t_tune": last["t_tune"]},
        "bricks": int(last["bricks"]), "samples": int(last["samples"]), "redone": int(last["redone"]),
        "e2e": {"value": world * len(items) / (wall / 1e3), "unit": "structures/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": None},
        "clocks": clk,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    b.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


# DRAM bytes (read + write) per step of the dominant kernel, from one ncu
# capture of the same workload (profiles/mc_item_edges_refine_exact_traffic_
# rings58800_h025.md: both passes of k_refine_exact; profiles/
# refine_f32_warm_rings58800_h025.md: k_refine from the warm starts).
TRAFFIC = {("rings58800", 0.25, "k_refine_exact"): 1152510464 + 277156352 + 216691712 + 104072448,
           ("rings58800", 0.25, "k_refine_warm"): 1360927744 + 193899264}


def roofline(dominant, stage, info, ops, owned, w, pk, pk_kind, n_bricks, xops=0, mode="exact"):
    """Roofline of the dominant kernel: its counted operations (or bytes) per
    launch over the launch's device time, against the matching peak."""
    ms = stage[dominant]
    hbm = pk.get("hbm_gbs", PEAKS_FALLBACK["hbm_gbs"])
    spb = (w["brick"] + 1) ** 3
    if dominant == "refine" and xops and mode != "exact":
        achieved = xops / (ms / 1e3) / 1e12
        return {"kernel": "k_refine", "bound": "fp32", "achieved": achieved, "peak": FP32_NOFMA_TOPS,
                "unit": "Tops/s", "frac": achieved / FP32_NOFMA_TOPS,
                "traffic": TRAFFIC.get((w["name"], w["spacing"], "k_refine_" + mode)),
                "peak_source": "nominal: 148 SMs x 128 FP32 lanes x 1965 MHz, one op per lane-cycle "
                               "(no FMA contraction, bit-exact f32; sqrt and division counted as one op)",
                "algorithmic_ops": xops,
                "ms": ms, "ms_note": "the refinement stage: edge lists, warm starts (warm mode), the f32 "
                                     "refinement and the vertex placement; the operations are those of the "
                                     "refinement's field evaluations",
                "sampler": roofline("sample", stage, info, ops, owned, w, pk, pk_kind, n_bricks)}
    if dominant == "refine" and xops:
        achieved = xops / (ms / 1e3) / 1e12
        return {"kernel": "k_refine_exact", "bound": "fp64", "achieved": achieved, "peak": FP64_NOFMA_TOPS,
                "unit": "Tops/s", "frac": achieved / FP64_NOFMA_TOPS,
                "traffic": TRAFFIC.get((w["name"], w["spacing"], "k_refine_exact")),
                "peak_source": "nominal: 148 SMs x 64 FP64 lanes x 1965 MHz, one op per lane-cycle "
                               "(no FMA contraction, bit-exact f64; sqrt and division counted as one op)",
                "algorithmic_ops": xops, "ms": ms,
                "sampler": roofline("sample", stage, info, ops, owned, w, pk, pk_kind, n_bricks)}
    if dominant == "sample":
        achieved = ops / (ms / 1e3) / 1e12
        return {"kernel": "k_sample", "bound": "fp32", "achieved": achieved, "peak": FP32_NOFMA_TOPS,
                "unit": "Tops/s", "frac": achieved / FP32_NOFMA_TOPS, "traffic": None,
                "peak_source": "nominal: 148 SMs x 128 FP32 lanes x 1965 MHz, one op per lane-cycle "
                               "(no FMA contraction, bit-exact f32)",
                "algorithmic_ops": ops, "evaluated_samples": owned, "ms": ms}
    if dominant == "gather":
        algo = info["ids_words"] * 4 + info["pack_units"] * 16
        kern = "k_gather"
    elif dominant == "mc":
        algo = n_bricks * spb * 4 + info["edges"] * 12 + info["triangles"] * 12
        kern = "k_mc"
    else:
        algo = n_bricks * spb * 4
        kern = "k_" + dominant
    achieved = algo / (ms / 1e3) / 1e9
    return {"kernel": kern, "bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
            "frac": achieved / hbm, "traffic": None, "peak_source": pk_kind, "algorithmic_bytes": algo, "ms": ms}


def main():
    a = args_()
    if a.impl == "reference":
        run_reference(a)
    elif a.workload == "batch512":
        run_batch(a)
    else:
        run_ours(a)


if __name__ == "__main__":
    main()
