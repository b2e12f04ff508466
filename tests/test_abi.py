"""The C ABI library loads, exports every entry point of include/*.h, and
its struct layouts agree with the ctypes bindings (no GPU needed)."""
import ctypes as C
import os
import re
import subprocess
import tempfile

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADERS = [os.path.join(ROOT, "include", h) for h in ("sesmesh_b200.h", "sesmesh_b200_surface.h")]


def declared():
    text = "".join(open(h).read() for h in HEADERS)
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(smb_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    from sesmesh_b200 import native
    lib = native.lib()
    names = declared()
    assert len(names) >= 19
    for n in names:
        assert hasattr(lib, n), n
    assert set(names) == set(native.SIGNATURES), "ctypes signatures must cover the header"


def test_struct_layouts_match_the_header():
    from sesmesh_b200 import native
    prog = r'''
#include <stdio.h>
#include <stddef.h>
#include "sesmesh_b200_surface.h"
int main(void) {
  printf("%zu %zu\n", sizeof(smb_surface_stats), offsetof(smb_surface_stats, upload_bytes));
  printf("%zu %zu %zu %zu %zu\n", sizeof(smb_grid_ref), sizeof(smb_arrangement_ref), sizeof(smb_lattice_ref),
         sizeof(smb_batch_times), sizeof(smb_device_info));
  printf("%zu %zu %zu %zu\n", offsetof(smb_arrangement_ref, sphere_grid), offsetof(smb_arrangement_ref, probe),
         offsetof(smb_arrangement_ref, kind), offsetof(smb_lattice_ref, band));
  return 0;
}
'''
    with tempfile.TemporaryDirectory() as d:
        src, exe = os.path.join(d, "l.c"), os.path.join(d, "l")
        open(src, "w").write(prog)
        subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), src, "-o", exe], check=True)
        out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout.split()
    got = [int(v) for v in out]
    want = [C.sizeof(native.SurfaceStats_), native.SurfaceStats_.upload_bytes.offset,
            C.sizeof(native.GridRef), C.sizeof(native.ArrangementRef), C.sizeof(native.LatticeRef),
            C.sizeof(native.BatchTimes), C.sizeof(native.DeviceInfo),
            native.ArrangementRef.sphere_grid.offset, native.ArrangementRef.probe.offset,
            native.ArrangementRef.kind.offset, native.LatticeRef.band.offset]
    assert got == want


def test_open_without_a_device_fails_loudly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a device is present")
    from sesmesh_b200 import native
    with pytest.raises(native.SmbError) as e:
        native.Device(0)
    assert e.value.code == 3


def test_synthetic_inputs_are_deterministic():
    from sesmesh_b200 import workloads
    a = workloads.globule330()["spheres"]
    b = workloads.globule330()["spheres"]
    assert a.shape == (330, 4) and np.array_equal(a, b)
    r = np.sqrt((a[:, :3] ** 2).sum(1))
    assert r.max() <= 11.5 + 1e-9
    d = np.sqrt(((a[:, None, :3] - a[None, :, :3]) ** 2).sum(-1))
    np.fill_diagonal(d, 9.0)
    assert d.min() >= 1.5 - 1e-9
