#!/usr/bin/env python3
"""Writes the structure fixtures of this directory from the sesmesh sources.

    python tests/golden/make_structure_golden.py /path/to/sesmesh   (or set SESMESH_REFERENCE)

* 1CRN.cif.gz, 1L2Y.cif.gz, 1EJG.cif.gz and 1CRN.pdb.gz: copies of the
  reference's parser fixtures (tests/data/fixtures/, RCSB PDB entries, CC0);
* 1AON.pdb.gz: the reference's data/1aon.pdb, gzip-compressed;
* structures.json: the reference's published meshes of these entries --
  docs/validation/accuracy.csv rows (entry, atoms, spacing, vertices,
  triangles, components, area and volume to 3 decimals; probe 1.4 A, the
  default selection and Bondi radii) and the 1AON row of
  docs/validation/large.csv (58,870 atoms at 0.25 A: vertices, triangles,
  components) -- plus, for 1AON at 0.25 A, the sha256 of the CPU oracle's
  OBJ bytes (exact mode, default OBJ options).
"""
import csv
import gzip
import hashlib
import json
import os
import shutil
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
for p in (ROOT, os.path.join(ROOT, "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)

ENTRIES = ("1CRN", "1L2Y", "1EJG")


def main(ref):
    fx = os.path.join(ref, "tests", "data", "fixtures")
    for e in ENTRIES:
        shutil.copyfile(os.path.join(fx, e + ".cif.gz"), os.path.join(HERE, e + ".cif.gz"))
    shutil.copyfile(os.path.join(fx, "1CRN.pdb.gz"), os.path.join(HERE, "1CRN.pdb.gz"))
    with open(os.path.join(ref, "data", "1aon.pdb"), "rb") as f, \
            gzip.GzipFile(os.path.join(HERE, "1AON.pdb.gz"), "wb", compresslevel=9, mtime=0) as g:
        g.write(f.read())
    rows = []
    for r in csv.DictReader(open(os.path.join(ref, "docs", "validation", "accuracy.csv"))):
        if r["entry"] in ENTRIES:
            rows.append(dict(entry=r["entry"], atoms=int(r["atoms"]), spacing=float(r["spacing"]),
                             vertices=int(r["vertices"]), triangles=int(r["triangles"]),
                             components=int(r["components"]), area=r["area"], volume=r["volume"]))
    large = None
    for r in csv.DictReader(open(os.path.join(ref, "docs", "validation", "large.csv"))):
        if r["entry"] == "1AON":
            large = dict(entry="1AON", atoms=int(r["atoms"]), spacing=0.25, vertices=int(r["vertices"]),
                         triangles=int(r["triangles"]), components=int(r["components"]))
    import oracle as O
    from sesmesh_b200 import structure
    s = structure.read_path(os.path.join(HERE, "1AON.pdb.gz"))
    out = O.Surface(s, 1.4, 0.25)
    large["oracle_obj_sha256"] = hashlib.sha256(out.obj()).hexdigest()
    large["oracle_area"] = float(out.stats["area"]).hex()
    large["oracle_volume"] = float(out.stats["volume"]).hex()
    json.dump(dict(accuracy=rows, large=large,
                   source="docs/validation/accuracy.csv and large.csv of sesmesh; probe 1.4 A, brick 10, "
                          "default selection, Bondi radii"),
              open(os.path.join(HERE, "structures.json"), "w"), indent=1)


if __name__ == "__main__":
    if len(sys.argv) > 1:
        main(sys.argv[1])
    elif os.environ.get("SESMESH_REFERENCE"):
        main(os.environ["SESMESH_REFERENCE"])
    else:
        sys.exit("usage: make_structure_golden.py REFERENCE_TREE (or set SESMESH_REFERENCE)")
