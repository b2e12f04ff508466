"""The product's host arrangement equals the oracle's bit for bit (no GPU).

Both restate geom/arrangement.rs; the device path consumes this
arrangement, so its equality with the oracle's is the first link of the
byte-identical chain.
"""
import numpy as np
import pytest

import oracle as O
from helpers import random_chain

from sesmesh_b200 import surface as S


def _sets():
    out = [("pair", np.array([[0, 0, 0, 1.7], [2.5, 0, 0, 1.5]]), 1.4)]
    for seed, n in ((3, 30), (9, 50), (21, 120)):
        s, p = random_chain(seed, n)
        out.append(("chain%d" % seed, s, p))
    s, p = random_chain(4, 40)
    dup = np.concatenate([s, s[::4], [[s[0, 0] + 0.1, s[0, 1], s[0, 2], s[0, 3] * 0.3]]])
    out.append(("duplicates", dup, p))
    g = np.array([[x * 3.0, y * 3.0, z * 3.0, 1.6] for x in range(4) for y in range(4) for z in range(4)])
    out.append(("lattice", g, 1.4))
    from sesmesh_b200 import workloads
    out.append(("globule330", workloads.globule330()["spheres"], 1.4))
    return out


@pytest.mark.parametrize("case", _sets(), ids=lambda c: c[0])
def test_host_arrangement_matches_oracle(case):
    name, spheres, probe = case
    got = S.host_arrangement(spheres, S.SurfaceParams.ses(probe))
    eng = O.Engine(spheres, probe, 0.5)
    want = eng.arrangement()
    assert np.array_equal(got["orig"], want["orig"])
    assert np.array_equal(got["center"].view(np.uint64), want["spheres"][:, :3].copy().view(np.uint64))
    assert np.array_equal(got["expanded"].view(np.uint64), want["spheres"][:, 3].copy().view(np.uint64))
    assert np.array_equal(got["status"], want["status"].astype(np.uint32))
    assert got["n_contained"] == int(eng.info["n_contained"])
    wc = want["circles"]
    assert len(got["circle"]) == len(wc)
    if len(wc):
        assert np.array_equal(got["circle_ij"], wc[:, :2].astype(np.uint32))
        assert np.array_equal(got["circle"].view(np.uint64), wc[:, 2:].copy().view(np.uint64))
    wv = want["vertices"]
    assert len(got["vertex"]) == len(wv)
    if len(wv):
        assert np.array_equal(got["vertex"].view(np.uint64), wv[:, :3].copy().view(np.uint64))
        assert np.array_equal(got["vertex_atoms"], wv[:, 3:].astype(np.uint32))
    for which, key in ((0, "nb"), (1, "cb")):
        off, items = eng.csr(which)
        assert np.array_equal(got[key + "_off"], off)
        assert np.array_equal(got[key + "_items"], items)
    assert got["max_expanded"] == eng.info["max_expanded"] and got["rho_max"] == eng.info["rho_max"]
