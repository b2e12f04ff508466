"""Structure input (smb_read_structure) and the published meshes of real
structures.

CPU:
* the default selection keeps the reference's atom counts (RCSB deposited
  non-hydrogen counts of the first model, crates/sesmesh/tests/
  structures.rs:60-77): 1CRN 327, 1L2Y 154 (an NMR ensemble with explicit
  hydrogens: the first model, hydrogens dropped), 1EJG 327 (alternate
  locations resolved by occupancy), 1AON 58,870; the PDB and mmCIF files of
  1CRN give the same spheres; radii are Bondi's (C 1.70, N 1.55, O 1.52,
  S 1.80 A); model and hydrogen options; malformed input is refused;
* the CPU oracle meshes 1CRN, 1L2Y and 1EJG at 1, 0.7, 0.5, 0.35 and 0.25 A
  into the reference's published meshes (docs/validation/accuracy.csv:
  vertices, triangles and components exactly, area and volume to the 3
  decimals printed) -- real structures pinning the oracle beyond the
  synthetic inputs.
GPU: compute_surface (exact mode) gives the same numbers, and for 1AON at
0.25 A the published vertex, triangle and component counts
(docs/validation/large.csv) and the oracle's OBJ bytes.
"""
import hashlib
import json
import os

import numpy as np
import pytest

import oracle as O

GOLD = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
PINS = json.load(open(os.path.join(GOLD, "structures.json")))


def _read(name, **kw):
    from sesmesh_b200 import structure
    return structure.read_path(os.path.join(GOLD, name), **kw)


def test_default_selection_counts():
    assert len(_read("1CRN.cif.gz")) == 327
    assert len(_read("1L2Y.cif.gz")) == 154
    assert len(_read("1EJG.cif.gz")) == 327
    assert len(_read("1AON.pdb.gz")) == 58870


def test_pdb_and_mmcif_agree_and_radii_are_bondi():
    a = _read("1CRN.cif.gz")
    b = _read("1CRN.pdb.gz")
    assert np.array_equal(a, b)
    assert set(np.unique(a[:, 3]).tolist()) == {1.52, 1.55, 1.70, 1.80}


def test_selection_options():
    h = _read("1L2Y.cif.gz", hydrogens=True)
    assert len(h) == 304 and np.count_nonzero(h[:, 3] == 1.20) == 150
    m7 = _read("1L2Y.cif.gz", model=7)
    assert len(m7) == 154 and not np.array_equal(m7, _read("1L2Y.cif.gz"))
    from sesmesh_b200 import native, structure
    with pytest.raises(native.SmbError):
        structure.read_bytes(b"HEADER nothing here\n")
    with pytest.raises(native.SmbError):
        structure.read_bytes(b"ATOM      1  CA  ALA A   1      11.1\n")
    with pytest.raises(native.SmbError):
        _read("1L2Y.cif.gz", model=99)


@pytest.mark.parametrize("row", PINS["accuracy"], ids=lambda r: "%s@%g" % (r["entry"], r["spacing"]))
def test_oracle_meshes_equal_published(row):
    s = _read(row["entry"] + ".cif.gz")
    assert len(s) == row["atoms"]
    st = O.Surface(s, 1.4, row["spacing"]).stats
    assert (int(st["vertices"]), int(st["triangles"]), int(st["components"])) == \
        (row["vertices"], row["triangles"], row["components"])
    assert "%.3f" % st["area"] == row["area"] and "%.3f" % st["volume"] == row["volume"]


@pytest.mark.gpu
@pytest.mark.parametrize("row", PINS["accuracy"], ids=lambda r: "%s@%g" % (r["entry"], r["spacing"]))
def test_device_meshes_equal_published(row):
    from sesmesh_b200 import surface as S
    s = _read(row["entry"] + ".cif.gz")
    out = S.compute_surface(s, S.SurfaceParams.ses(1.4).with_spacing(row["spacing"]))
    st = out.stats
    assert (st["vertices"], st["triangles"], st["components"]) == (row["vertices"], row["triangles"],
                                                                  row["components"])
    assert "%.3f" % st["area"] == row["area"] and "%.3f" % st["volume"] == row["volume"]


@pytest.mark.gpu
def test_device_1aon_equals_published_counts_and_oracle_bytes():
    from sesmesh_b200 import surface as S
    pin = PINS["large"]
    s = _read("1AON.pdb.gz")
    out = S.compute_surface(s, S.SurfaceParams.ses(1.4).with_spacing(pin["spacing"]))
    st = out.stats
    assert (st["vertices"], st["triangles"], st["components"]) == (pin["vertices"], pin["triangles"],
                                                                  pin["components"])
    assert st["area"] == float.fromhex(pin["oracle_area"]) and st["volume"] == float.fromhex(pin["oracle_volume"])
    assert hashlib.sha256(out.obj()).hexdigest() == pin["oracle_obj_sha256"]
