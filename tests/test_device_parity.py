"""Device path (C ABI) against the CPU oracle, bit for bit.

For each sphere set the oracle's arrangement is handed to smb_resident_new
(the reference's boundary passes the host-built arrangement the same way),
then every device output is compared with the oracle's CPU back end:

* surface bricks (lattice::touched_bricks + surface_bricks): same set, order;
* sub-block states (Engine::sub_states): equal;
* candidate lists of every sampled sub-block (Engine::gather_ses): equal
  ids in equal order, equal blocker lists;
* sample values (Engine::evaluate): equal bits, including +-band samples;
* marching-cubes edges and triangle references per brick (mesh_brick edge
  scan and cells()): equal.
"""
import numpy as np
import pytest

import oracle as O
from helpers import arrangement_from_oracle, lattice_from_oracle, random_chain

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def device():
    from sesmesh_b200 import native
    return native.Device(0)


def _cases():
    from sesmesh_b200 import workloads
    cases = [("single", np.array([[0.1, 0.2, 0.3, 1.8]]), 1.4, 0.25),
             ("pair", np.array([[0, 0, 0, 1.7], [2.5, 0, 0, 1.5]]), 1.4, 0.25),
             ("pair_far", np.array([[0, 0, 0, 1.5], [5.6, 0, 0, 1.5]]), 1.4, 0.5)]
    for seed, n in ((5, 40), (11, 60)):
        s, probe = random_chain(seed, n)
        cases.append(("chain%d" % seed, s, probe, 0.3))
    g = workloads.globule330()
    cases.append(("globule330", g["spheres"], g["probe"], g["spacing"]))
    cases.append(("globule330_fine", g["spheres"], g["probe"], 0.25))
    return cases


CASES = _cases() if __import__("os").path.exists(
    __import__("os").path.join(__import__("os").path.dirname(__file__), "..", "sesmesh_b200",
                               "libsesmesh_synth.so")) else []


@pytest.mark.parametrize("case", CASES, ids=lambda c: c[0])
def test_device_matches_oracle(device, case):
    from sesmesh_b200 import native
    name, spheres, probe, spacing = case
    brick = 10
    eng = O.Engine(spheres, probe, spacing, brick)
    arr = arrangement_from_oracle(eng)
    arr["probe"] = probe
    res = native.Resident(device, arr, lattice_from_oracle(eng, spacing, brick))
    touched, surface = res.classify()
    want_bricks, want_touched = eng.classify()
    assert touched == want_touched
    bricks = res.bricks()
    assert np.array_equal(bricks, want_bricks)
    if len(bricks) == 0:
        return
    batch = native.Batch(res)
    batch.run()
    rec = batch.records()
    # Sub-block states: oracle 1 out / 0 in / -1 sampled; device 1 out / 2 in / 0 sampled.
    st = eng.sub_states(bricks).reshape(-1)
    dev_state = rec[:, 0].astype(np.int64)
    want_state = np.where(st < 0, 0, np.where(st == 1, 1, 2))
    assert np.array_equal(dev_state, want_state)
    assert np.all(rec[:, 11] == 0)
    # Values, bit for bit.
    vals = batch.values()
    want_vals = eng.values(bricks)
    assert np.array_equal(vals.view(np.uint32), want_vals.view(np.uint32))
    # Candidate lists of sampled sub-blocks (all of them for small cases).
    ids = batch.ids()
    sampled = np.nonzero(dev_state == 0)[0]
    step = max(1, len(sampled) // 400)
    for j in sampled[::step]:
        got = batch.lists(rec[j], ids)
        want = eng.gather(bricks[j // 8], int(j % 8))
        assert got["n_inside"] == want["n_inside"], j
        for key in ("near", "s", "s_off", "s_blk", "c", "c_off", "c_blk", "v"):
            assert np.array_equal(got[key], want[key]), (j, key)
    # Marching cubes per brick.
    mc = batch.mc()
    for i in range(0, len(bricks), max(1, len(bricks) // 300)):
        e0, e1 = mc["edge_off"][i], mc["edge_off"][i + 1]
        t0, t1 = mc["tri_off"][i], mc["tri_off"][i + 1]
        want_e, want_t = O.mc_brick(brick, want_vals[i])
        assert np.array_equal(mc["edges"][e0:e1], want_e), i
        assert np.array_equal(mc["tris"][t0:t1], want_t), i
        v = want_vals[i]
        s = brick + 1
        st3 = [1, s, s * s]
        for k, e in enumerate(want_e):
            cell, ax = divmod(int(e), 3)
            x, y, z = cell % brick, (cell // brick) % brick, cell // (brick * brick)
            ia = (z * s + y) * s + x
            assert mc["edge_vals"][e0 + k, 0] == v[ia] and mc["edge_vals"][e0 + k, 1] == v[ia + st3[ax]]


def test_self_test_large(device):
    device.self_test(1 << 20)


def test_bad_tables_are_rejected(device):
    from sesmesh_b200 import native
    eng = O.Engine([[0, 0, 0, 1.5], [2.0, 0, 0, 1.5]], 1.4, 0.5, 10)
    arr = arrangement_from_oracle(eng)
    arr["probe"] = 1.4
    lat = lattice_from_oracle(eng, 0.5, 10)
    bad = dict(arr, nb_items=np.array([99], np.uint32), nb_off=np.array([0, 1, 1], np.uint32))
    with pytest.raises(native.SmbError):
        native.Resident(device, bad, lat)
    with pytest.raises(native.SmbError):
        native.Resident(device, arr, dict(lat, brick=9))
