"""Seeded synthetic workloads (no public dataset is involved).

Each function returns a dict with `spheres` ((n, 4) float64 rows x, y, z, r),
`probe`, `spacing`, `brick` and `refine`, plus a `name` and the generator
settings.  Globules are grown by libsesmesh_synth (a branching self-avoiding
walk, see csrc/synth.cpp); seeds are fixed here.

* globule330     -- 330 spheres in a ball of radius 11.5 A, spacing 0.5 A, exact.
* rings58800     -- 21 copies of a 2 800-sphere globule on three stacked 7-fold
                    rings (two rings of radius 60 A at z = -22.5 and +22.5 A,
                    a cap ring of radius 55 A at z = +67.5 A), spacing 0.25 A,
                    exact.  The globule's ball radius is the density radius
                    for 2 800 spheres at one sphere per 20 A^3, 23.7 A (a
                    ball of 19 A cannot hold 2 800 spheres 2.8 A apart).
* shell2400k     -- 60 copies of a 40 000-sphere globule (ball radius 57.6 A)
                    on an icosahedral shell of radius 380 A, spacing 1 A.
* batch512       -- 512 globules, sizes log-uniform in 20..5 000, probe
                    uniform in 1.2..1.4 A, spacing drawn from {0.1, 0.25, 0.5}.
"""
import ctypes as C
import math

import numpy as np

from . import native


def _p(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def globule(seed, n, radius=0.0):
    out = np.zeros((n, 4))
    m = native.synth().smb_synth_globule(seed, n, radius, _p(out))
    return out[:m]


def globule330(seed=330):
    return dict(name="globule330", spheres=globule(seed, 330, 11.5), probe=1.4, spacing=0.5, brick=10,
                refine="exact")


RING_Z = (-22.5, 22.5, 67.5)
RING_R = (60.0, 60.0, 55.0)
RING_OFF = (0.0, math.pi / 7.0, 0.0)


def rings58800(seed=58800, per=2800, spacing=0.25, refine="exact"):
    out = np.zeros((21 * per, 4))
    z = np.array(RING_Z)
    r = np.array(RING_R)
    o = np.array(RING_OFF)
    m = native.synth().smb_synth_rings(seed, per, 0.0, 3, _p(z), _p(r), _p(o), _p(out))
    return dict(name="rings58800", spheres=out[:m], probe=1.4, spacing=spacing, brick=10, refine=refine,
                copies=21, per_copy=per, ring_z=RING_Z, ring_r=RING_R)


def globule2800(seed=58800, spacing=0.25, refine="exact"):
    """One copy of the rings58800 unit (2,800 spheres): the profiling case."""
    r = rings58800(seed)
    return dict(name="globule2800", spheres=r["spheres"][:2800], probe=1.4, spacing=spacing, brick=10,
                refine=refine)


def shell2400k(seed=2400, per=40000, refine="exact"):
    out = np.zeros((60 * per, 4))
    m = native.synth().smb_synth_icosahedral(seed, per, 0.0, 380.0, _p(out))
    return dict(name="shell2400k", spheres=out[:m], probe=1.4, spacing=1.0, brick=10, refine=refine,
                copies=60, per_copy=per, shell_radius=380.0)


def batch512(seed=512, count=512):
    rng = np.random.default_rng(seed)
    items = []
    for k in range(count):
        n = int(round(math.exp(rng.uniform(math.log(20), math.log(5000)))))
        probe = float(rng.uniform(1.2, 1.4))
        spacing = float(rng.choice([0.1, 0.25, 0.5]))
        items.append(dict(name="batch512/%d" % k, spheres=globule(seed * 100003 + k, n), probe=probe,
                          spacing=spacing, brick=10, refine="fast"))
    return items
