"""Pins of the CPU oracle against the reference's own known answers.

* paper/data/analytic.csv: counts, area and volume (6 dp) and max |F| of one
  sphere and four sphere pairs at four spacings (tests/golden/analytic.json).
* tests/surface.rs obj_snapshot: exact OBJ bytes.
* export/fmt.rs: number formatting identical to Rust's `{:.N}`.
* mesh/tables.rs: marching-cubes table invariants and the table digest.
"""
import hashlib
import json
import os
import struct

import numpy as np
import pytest

import oracle as O
import mc_table

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def _load(name):
    return json.load(open(os.path.join(GOLD, name)))


@pytest.mark.parametrize("row", _load("analytic.json"), ids=lambda r: "%s@%g" % (r["case"], r["spacing"]))
def test_analytic_counts_area_volume(row):
    s = O.Surface(row["spheres"], row["probe"], row["spacing"])
    st = s.stats
    assert int(st["vertices"]) == row["vertices"]
    assert int(st["triangles"]) == row["triangles"]
    assert int(st["components"]) == row["components"]
    assert "%.6f" % st["area"] == row["area"]
    assert "%.6f" % st["volume"] == row["volume"]


@pytest.mark.parametrize("row", [r for r in _load("analytic.json") if r["spacing"] >= 0.5],
                         ids=lambda r: "%s@%g" % (r["case"], r["spacing"]))
def test_analytic_max_abs_f(row):
    """max |F| at the vertices, by the exact f64 field (3 significant digits)."""
    s = O.Surface(row["spheres"], row["probe"], row["spacing"])
    e = O.Engine(row["spheres"], row["probe"], row["spacing"])
    f = np.abs(e.field(s.mesh()["positions"].astype(np.float64)))
    m, e = ("%.3e" % f.max()).split("e")
    assert "%se%d" % (m, int(e)) == row["max_abs_f"]  # Rust's {:.3e} form


def test_obj_snapshot():
    snap = _load("obj_snapshot.json")
    got = O.obj_of(snap["positions"], snap["normals"], snap["triangles"])
    assert got.decode() == snap["expected"]


def test_fmt_matches_rust_formatting():
    for c in _load("fmt_cases.json"):
        x = struct.unpack("<f", struct.pack("<I", c["bits"]))[0]
        assert O.push_fixed(x, c["prec"]) == c["expected"], (x, c["prec"])


def test_mc_table_digest():
    offs, tris = mc_table.load()
    want = _load("mc_table.json")
    h = hashlib.sha256()
    h.update(",".join(map(str, offs)).encode())
    h.update(b";")
    h.update(",".join("%d.%d.%d" % t for t in tris).encode())
    assert h.hexdigest() == want["sha256"] and len(tris) == want["triangles"]


def test_mc_table_cases_use_exactly_their_crossing_edges():
    offs, tris = mc_table.load()
    for case in range(256):
        crossing = {e for e in range(12)
                    if ((case >> mc_table.edge_corners(e)[0]) & 1) != ((case >> mc_table.edge_corners(e)[1]) & 1)}
        used = {e for t in tris[offs[case]:offs[case + 1]] for e in t}
        assert used == crossing, case


def test_mc_table_meshes_random_grids_closed_and_oriented():
    """Random sign grids padded with outside samples: every undirected edge
    is used once in each direction (closed, edge-manifold, consistently
    oriented) and the signed volume is positive (outward winding)."""
    rng = np.random.default_rng(7)
    for trial in range(20):
        n = 7
        inside = rng.random((n, n, n)) < rng.uniform(0.2, 0.8)
        inside[[0, -1], :, :] = False
        inside[:, [0, -1], :] = False
        inside[:, :, [0, -1]] = False
        vals = np.where(inside, -1.0, 1.0).astype(np.float32)
        b = n - 1
        # MC over the whole grid as one brick of b^3 cells.
        v = vals.transpose(2, 1, 0).copy()  # index [z][y][x] -> x fastest in memory
        edges, tri_refs = O.mc_brick(b, v.reshape(-1))
        assert len(tri_refs) > 0
        assert np.all((tri_refs >> 28) == 0)
        ids = tri_refs & ((1 << 28) - 1)
        vid = {int(e): i for i, e in enumerate(edges)}
        tris = np.vectorize(lambda e: vid[int(e)])(ids)
        uses = {}
        for t in tris:
            for k in range(3):
                a, c = int(t[k]), int(t[(k + 1) % 3])
                uses[(a, c)] = uses.get((a, c), 0) + 1
        for (a, c), m in uses.items():
            assert m == 1 and uses.get((c, a)) == 1
        # Midpoint vertices; signed volume.
        pos = []
        for e in edges:
            cell, axis = divmod(int(e), 3)
            x, y, z = cell % b, (cell // b) % b, cell // (b * b)
            p = [x, y, z]
            p[axis] += 0.5
            pos.append(p)
        pos = np.array(pos, float)
        p0, p1, p2 = pos[tris[:, 0]], pos[tris[:, 1]], pos[tris[:, 2]]
        vol = np.einsum("ij,ij->i", p0, np.cross(p1, p2)).sum() / 6.0
        assert vol > 0


def test_single_sphere_all_kinds():
    """tests/surface.rs:55-82 (single_sphere_all_kinds): one sphere of radius
    1.8 meshed as SES (probe 1.4), SAS (probe 1.4: radius 3.2) and vdW at
    0.25 A gives one component with Euler characteristic 2, area within
    5e-3 and volume within 1.2e-2 relative of the sphere's, every vertex
    within 1e-4 h + 2e-6 of the surface and normals within 0.01 degrees."""
    s = np.array([[0.3, -0.2, 0.1, 1.8]])
    h = 0.25
    for kind, probe, r in (("ses", 1.4, 1.8), ("sas", 1.4, 3.2), ("vdw", 0.0, 1.8)):
        out = O.Surface(s, probe, h, kind=kind)
        st = out.stats
        assert st["components"] == 1 and st["euler"] == 2, kind
        area, vol = 4 * np.pi * r * r, 4.0 / 3.0 * np.pi * r ** 3
        assert abs(st["area"] - area) / area < 5e-3, kind
        assert abs(st["volume"] - vol) / vol < 1.2e-2, kind
        m = out.mesh()
        f, nrm, has = O.Engine(s, probe, h, kind=kind).field_normals(m["positions"].astype(np.float64))
        assert np.abs(f).max() < 1e-4 * h + 2e-6, kind
        b = m["normals"].astype(np.float64)[has]
        a = nrm[has]
        ang = np.degrees(np.arctan2(np.linalg.norm(np.cross(a, b), axis=1), (a * b).sum(1)))
        assert has.sum() > 0.9 * len(has) and ang.max() < 0.01, (kind, ang.max())
