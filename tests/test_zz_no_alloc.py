"""smb_mc_noalloc: marching cubes without any device allocation.

Callers that cannot allocate device memory while they mesh (a service under
a fixed device-memory budget, or a host whose device memory belongs to
another framework's caching allocator) call this entry point with their own
input and output buffers; its scratch is a static device array.  The test
runs a normal batch (smb_run), hands its values and records to
smb_mc_noalloc in caller-owned device buffers, and checks the edges, edge
values, triangle references and offsets on two calls in a row against
smb_batch_mc (bit-identical: integer and copied float data) and, brick by
brick, against the CPU oracle's marching cubes.  It also checks that device
free memory does not change across a call, that an empty call writes zero
offsets and totals, that the caller's current device is kept, and that too
many bricks and too small output buffers are refused.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _ptr(t):
    return C.c_void_p(t.data_ptr())


def test_mc_noalloc_matches_smb_batch_mc():
    import torch
    import oracle as O
    from helpers import arrangement_from_oracle, lattice_from_oracle
    from sesmesh_b200 import native, workloads

    w = workloads.globule330()
    h = 0.25
    brick = w["brick"]
    oeng = O.Engine(w["spheres"], w["probe"], h, brick)
    arr = arrangement_from_oracle(oeng)
    arr["probe"] = w["probe"]
    device = native.Device(0)
    resident = native.Resident(device, arr, lattice_from_oracle(oeng, h, brick))
    resident.classify()
    b = native.Batch(resident)
    b.run()
    L = native.lib()
    batch = b.h
    info = b.info()
    n = info["bricks"]
    assert 0 < n <= 65536
    spb = (brick + 1) ** 3
    vals = np.zeros(n * spb, np.float32)
    recs = np.zeros(n * 8 * native.REC_WORDS, np.uint32)
    assert L.smb_batch_values(batch, native._p(vals, C.c_float)) == 0
    assert L.smb_batch_records(batch, native._p(recs, C.c_uint32)) == 0
    ne, nt = info["edges"], info["triangles"]
    want_eo = np.zeros(n + 1, np.uint32)
    want_to = np.zeros(n + 1, np.uint32)
    want_e = np.zeros(ne, np.uint32)
    want_v = np.zeros(2 * ne, np.float32)
    want_t = np.zeros(3 * nt, np.uint32)
    L.smb_batch_mc(batch, native._p(want_eo, C.c_uint32), native._p(want_e, C.c_uint32), native._p(want_v, C.c_float),
                   native._p(want_to, C.c_uint32), native._p(want_t, C.c_uint32))
    # The oracle's marching cubes per brick (every 7th brick) over the same values.
    want_vals = oeng.values(resident.bricks())
    for i in range(0, n, 7):
        oe, ot = O.mc_brick(brick, want_vals[i])
        assert np.array_equal(want_e[want_eo[i]:want_eo[i + 1]], oe), i
        assert np.array_equal(want_t.reshape(-1, 3)[want_to[i]:want_to[i + 1]], ot), i

    dev = torch.device("cuda", 0)
    d_vals = torch.from_numpy(vals).to(dev)
    d_recs = torch.from_numpy(recs.view(np.int32)).to(dev)
    res = resident.h
    err = C.create_string_buffer(512)
    d_eo = torch.full((n + 1,), -1, dtype=torch.int32, device=dev)
    d_to = torch.full((n + 1,), -1, dtype=torch.int32, device=dev)
    d_e = torch.full((ne,), -1, dtype=torch.int32, device=dev)
    d_v = torch.full((2 * ne,), float("nan"), dtype=torch.float32, device=dev)
    d_t = torch.full((3 * nt,), -1, dtype=torch.int32, device=dev)
    got_ne, got_nt = C.c_size_t(0), C.c_size_t(0)
    free_after_first = None
    for call in range(2):
        for t in (d_eo, d_to, d_e, d_t):
            t.fill_(-1)
        d_v.fill_(float("nan"))
        torch.cuda.synchronize(dev)
        rc = L.smb_mc_noalloc(res, _ptr(d_vals), _ptr(d_recs), n, _ptr(d_eo), _ptr(d_e), _ptr(d_v), ne, _ptr(d_to),
                              _ptr(d_t), nt, C.byref(got_ne), C.byref(got_nt), err, 512)
        assert rc == 0, err.value
        torch.cuda.synchronize(dev)
        free_now = torch.cuda.mem_get_info(dev)[0]
        if call == 0:
            free_after_first = free_now
        else:
            # The second call allocates nothing: free device memory is unchanged.
            assert free_now == free_after_first
        assert torch.cuda.current_device() == 0
        assert (got_ne.value, got_nt.value) == (ne, nt), call
        assert np.array_equal(d_eo.cpu().numpy().view(np.uint32), want_eo), call
        assert np.array_equal(d_to.cpu().numpy().view(np.uint32), want_to), call
        assert np.array_equal(d_e.cpu().numpy().view(np.uint32), want_e), call
        assert np.array_equal(d_v.cpu().numpy().view(np.uint32), want_v.view(np.uint32)), call
        assert np.array_equal(d_t.cpu().numpy().view(np.uint32), want_t), call
    # No bricks: zero offsets and totals.
    d_eo.fill_(-1)
    d_to.fill_(-1)
    got_ne.value, got_nt.value = 7, 7
    rc = L.smb_mc_noalloc(res, _ptr(d_vals), _ptr(d_recs), 0, _ptr(d_eo), _ptr(d_e), _ptr(d_v), ne, _ptr(d_to),
                          _ptr(d_t), nt, C.byref(got_ne), C.byref(got_nt), err, 512)
    assert rc == 0, err.value
    assert (got_ne.value, got_nt.value) == (0, 0)
    assert int(d_eo[0]) == 0 and int(d_to[0]) == 0
    # Output buffers one element too small: refused, totals still reported.
    rc = L.smb_mc_noalloc(res, _ptr(d_vals), _ptr(d_recs), n, _ptr(d_eo), _ptr(d_e), _ptr(d_v), ne - 1, _ptr(d_to),
                          _ptr(d_t), nt, C.byref(got_ne), C.byref(got_nt), err, 512)
    assert rc == 6 and got_ne.value == ne
    # More bricks than the static scratch holds: refused before any launch.
    rc = L.smb_mc_noalloc(res, _ptr(d_vals), _ptr(d_recs), 65537, _ptr(d_eo), _ptr(d_e), _ptr(d_v), ne, _ptr(d_to),
                          _ptr(d_t), nt, C.byref(got_ne), C.byref(got_nt), err, 512)
    assert rc == 1 and b"at most 65536" in err.value
