#!/usr/bin/env python3
"""Writes configs.json: the CPU oracle's exact-mode meshes of the benchmark
configurations, as hashes and statistics.

    python tests/golden/make_config_golden.py [rings58800 shell2400k batch512]

The oracle (oracle/, the C++ restatement of sesmesh 1.3.2's CPU back end)
meshes, in exact mode with its default OBJ options:

* rings58800  -- 58,800 spheres, probe 1.4 A, spacing 0.25 A (the exact-mode
  large assembly, and the assembly the fast-mode comparison runs on);
* shell2400k  -- 2.4 M spheres on an icosahedral shell, probe 1.4 A,
  spacing 1 A;
* batch512    -- every 16th of the 512 batch structures (32 structures), each
  at its own probe and spacing, with 16-sample bricks (the brick edge the
  batch's tuner picks from 8 and 16: the brick order sets the vertex order,
  so the batch is compared at a fixed edge).

For each mesh: the sha256 of the input sphere rows (little-endian f64 x, y,
z, r), so a changed generator shows up as such; the statistics (counts, area
and volume as exact float hex); the sha256 of the OBJ bytes and of the mesh
arrays (positions, normals, triangles, vertex atoms, vertex patches, as
little-endian bytes); and max |F| of the exact f64 field over every k-th
vertex (with k), the exact-mode bound the fast-mode rules refer to.  The GPU
tests (tests/test_config_parity_gpu.py) compare the device path with these.
"""
import hashlib
import json
import os
import sys
import time

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
for p in (ROOT, os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)

import numpy as np  # noqa: E402

import oracle as O  # noqa: E402
from sesmesh_b200 import workloads  # noqa: E402

OUT = os.path.join(HERE, "configs.json")
F_SAMPLE = 200000  # vertices whose |F| is evaluated per mesh (every k-th)
BATCH_BRICK = 16


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def spheres_sha(spheres):
    return sha(np.ascontiguousarray(spheres, "<f8").reshape(-1, 4))


def record(name, spheres, probe, spacing, brick=10):
    t0 = time.time()
    s = O.Surface(spheres, probe, spacing, brick)
    m = s.mesh()
    obj = s.obj()
    st = s.stats
    nv = len(m["positions"])
    k = max(1, nv // F_SAMPLE)
    if nv:
        eng = O.Engine(spheres, probe, spacing, brick)
        f = np.abs(eng.field(m["positions"][::k].astype(np.float64)))
        fmax = float(f.max())
        del eng
    else:
        fmax = 0.0
    rec = dict(
        name=name, probe=float(probe), spacing=float(spacing), brick=int(brick), spheres=int(len(spheres)),
        spheres_sha256=spheres_sha(spheres),
        touched=int(st["touched"]), surface_bricks=int(st["surface_bricks"]), vertices=int(st["vertices"]),
        triangles=int(st["triangles"]), components=int(st["components"]), euler=int(st["euler"]),
        refine_evaluations=int(st["refine_evaluations"]),
        area=float(st["area"]).hex(), volume=float(st["volume"]).hex(),
        obj_sha256=hashlib.sha256(obj).hexdigest(), obj_bytes=len(obj),
        positions_sha256=sha(m["positions"].astype("<f4")), normals_sha256=sha(m["normals"].astype("<f4")),
        triangles_sha256=sha(m["triangles"].astype("<u4")), atoms_sha256=sha(m["atoms"].astype("<u4")),
        patches_sha256=sha(m["patches"].astype("u1")),
        F_stride=int(k), F_max=fmax)
    print("%-16s %8d spheres  %9d vertices  %9d triangles  %.1f s" %
          (name, len(spheres), rec["vertices"], rec["triangles"], time.time() - t0), flush=True)
    del obj, m, s
    return rec


def main(which):
    data = json.load(open(OUT)) if os.path.exists(OUT) else {}
    if "rings58800" in which:
        w = workloads.rings58800()
        data["rings58800"] = record("rings58800", w["spheres"], w["probe"], w["spacing"], w["brick"])
    if "shell2400k" in which:
        w = workloads.shell2400k()
        data["shell2400k"] = record("shell2400k", w["spheres"], w["probe"], w["spacing"], w["brick"])
    if "batch512" in which:
        items = workloads.batch512()
        data["batch512"] = {"stride": 16, "brick": BATCH_BRICK, "items": {
            str(i): record(items[i]["name"], items[i]["spheres"], items[i]["probe"], items[i]["spacing"],
                           BATCH_BRICK)
            for i in range(0, len(items), 16)}}
    data["generator"] = ("tests/golden/make_config_golden.py: CPU oracle (C++ restatement of sesmesh 1.3.2's "
                         "CPU back end), exact mode, default OBJ options")
    json.dump(data, open(OUT, "w"), indent=1, sort_keys=True)


if __name__ == "__main__":
    main(sys.argv[1:] or ["rings58800", "shell2400k", "batch512"])
