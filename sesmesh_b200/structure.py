"""Structure input: PDB and mmCIF files to (x, y, z, r) sphere rows.

The Python face of smb_read_structure (include/sesmesh_b200_surface.h),
shaped like sesmesh's io::read_path + Structure::select + radii::assign
(crates/sesmesh/src/io/mod.rs:188, structure/select.rs:61-95,
radii/mod.rs:166): the first model by default, alternate locations resolved
by occupancy, hydrogens and waters dropped, hetero atoms kept, Bondi radii.
Gzip-compressed files (.gz) are read through the gzip module.
"""
import ctypes as C
import gzip
import os

import numpy as np

from . import native
from .native import _check, _p, lib

FORMATS = {"auto": 0, "pdb": 1, "cif": 2, "mmcif": 2}


def read_bytes(data, fmt="auto", model=None, hydrogens=False, waters=False, hetero=True):
    """Spheres (n, 4) of the selected atoms of PDB or mmCIF bytes."""
    sel = native.Selection_(int(model or 0), int(bool(hydrogens)), int(bool(waters)), int(bool(hetero)))
    err = C.create_string_buffer(1024)
    n = C.c_size_t(0)
    # One pass for the usual case: an atom record takes more than 32 bytes of
    # text, so this capacity holds every atom; a second pass only if not.
    out = np.zeros((len(data) // 32 + 16, 4))
    rc = lib().smb_read_structure(data, len(data), FORMATS[fmt], C.byref(sel), _p(out, C.c_double), len(out),
                                  C.byref(n), err, 1024)
    if rc == native.SMB_ERR_MEMORY:
        out = np.zeros((n.value, 4))
        rc = lib().smb_read_structure(data, len(data), FORMATS[fmt], C.byref(sel), _p(out, C.c_double), len(out),
                                      C.byref(n), err, 1024)
    _check(rc, err)
    return out[:n.value].copy()


def read_path(path, model=None, hydrogens=False, waters=False, hetero=True):
    """io::read_path: the format from the extension (.pdb / .ent, .cif /
    .mmcif, optionally .gz), else from the contents."""
    name = os.path.basename(path).lower()
    opener = gzip.open if name.endswith(".gz") else open
    if name.endswith(".gz"):
        name = name[:-3]
    fmt = "pdb" if name.endswith((".pdb", ".ent")) else ("cif" if name.endswith((".cif", ".mmcif")) else "auto")
    with opener(path, "rb") as f:
        data = f.read()
    return read_bytes(data, fmt, model, hydrogens, waters, hetero)
