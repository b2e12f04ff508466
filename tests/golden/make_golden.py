#!/usr/bin/env python3
"""Writes the golden fixtures of this directory from the sesmesh sources.

Run where the reference tree is available (it is read as text only):

    python tests/golden/make_golden.py /path/to/sesmesh

Fixtures written:
* analytic.json -- paper/data/analytic.csv (mesh counts, area, volume and max
  |F| for one sphere and four sphere pairs at four spacings, probe 1.4) with
  the sphere sets of paper/scripts/analytic/src/main.rs:16-37.
* obj_snapshot.json -- the mesh and expected bytes of tests/surface.rs:341-355
  (the `{}` of the format string is the crate version, 1.3.2).
* fmt_cases.json -- the values of export/fmt.rs:81-101 and the strings Rust's
  `format!("{x:.prec$}")` gives for them, computed here from the exact decimal
  value of each f32 (round half to even, sign kept for negative values that
  round to zero), which is the behaviour fmt.rs:23-29 documents.
* mc_table.json -- the sha256 of the marching-cubes table data (see
  sesmesh_b200/csrc/gen_mc_table.py).
"""
import csv
import decimal
import json
import math
import os
import re
import struct
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def f32(x):
    return struct.unpack("<f", struct.pack("<f", x))[0]


def rust_fixed(x, prec):
    if math.isnan(x):
        return "NaN"
    if math.isinf(x):
        return "inf" if x > 0 else "-inf"
    d = decimal.Decimal(x)  # exact value of the f32 (held exactly in a double)
    q = d.quantize(decimal.Decimal(1).scaleb(-prec), rounding=decimal.ROUND_HALF_EVEN,
                   context=decimal.Context(prec=400))
    s = format(q.copy_abs(), "f")
    neg = math.copysign(1.0, x) < 0
    return ("-" if neg else "") + s


def main(root):
    rows = list(csv.DictReader(open(os.path.join(root, "paper/data/analytic.csv"))))
    cases = {"single r=1.8": [[0.1, 0.2, 0.3, 1.8]]}
    for r1, r2, d in [(1.7, 1.5, 2.5), (1.6, 1.6, 4.0), (1.8, 1.2, 5.0), (1.5, 1.5, 5.6)]:
        cases["pair r=%g/%g d=%g" % (r1, r2, d)] = [[0.0, 0.0, 0.0, r1], [d, 0.0, 0.0, r2]]
    out = []
    for r in rows:
        out.append(dict(case=r["case"], spheres=cases[r["case"]], probe=1.4, spacing=float(r["spacing"]),
                        vertices=int(r["vertices"]), triangles=int(r["triangles"]),
                        components=int(r["components"]), area=r["area"], volume=r["volume"],
                        max_abs_f=r["max_abs_f"]))
    json.dump(out, open(os.path.join(HERE, "analytic.json"), "w"), indent=1)

    src = open(os.path.join(root, "crates/sesmesh/tests/surface.rs")).read()
    body = src[src.index("fn obj_snapshot"):]
    lit = re.search(r'format!\(\s*"(.*?)",\s*sesmesh::VERSION', body, re.S).group(1)
    lit = re.sub(r"\\\n\s*", "", lit).replace("\\n", "\n").replace("{}", "1.3.2")
    snap = dict(positions=[[0.0, 0.0, 0.0], [1.0, -0.5, 0.0], [0.0, 1.25, -2.71849]],
                normals=[[0.0, 0.0, 1.0]] * 3, triangles=[[0, 1, 2]], expected=lit)
    json.dump(snap, open(os.path.join(HERE, "obj_snapshot.json"), "w"), indent=1)

    values = [0.0, -0.0, 0.5, 1.5, 2.5, -0.5, 0.25, 0.125, 0.375, 0.03125, -0.00001, 1e-9, 123456.79,
              -98765.43, 1.1754943508222875e-38, 1e15, -3e30, 3.4028234663852886e38, math.inf, -math.inf,
              math.nan]
    fmt = []
    for v in values:
        x = f32(v)
        for prec in range(10):
            fmt.append(dict(bits=struct.unpack("<I", struct.pack("<f", x))[0], prec=prec,
                            expected=rust_fixed(x, prec)))
    json.dump(fmt, open(os.path.join(HERE, "fmt_cases.json"), "w"))

    sys.path.insert(0, os.path.join(HERE, "..", "..", "sesmesh_b200", "csrc"))
    import gen_mc_table
    offs, tris = gen_mc_table.parse(open(os.path.join(root, "crates/sesmesh/src/mesh/mc_table.rs")).read())
    json.dump(dict(sha256=gen_mc_table.digest(offs, tris), triangles=len(tris)),
              open(os.path.join(HERE, "mc_table.json"), "w"))


if __name__ == "__main__":
    if len(sys.argv) > 1:
        main(sys.argv[1])
    elif os.environ.get("SESMESH_REFERENCE"):
        main(os.environ["SESMESH_REFERENCE"])
    else:
        sys.exit("usage: make_golden.py REFERENCE_TREE (or set SESMESH_REFERENCE)")
