"""Shared test helpers: oracle arrangement -> C-ABI arrangement arrays."""
import numpy as np


def arrangement_from_oracle(eng):
    """The oracle engine's arrangement in the layout of smb_arrangement_ref."""
    a = eng.arrangement()
    nb_off, nb_items = eng.csr(0)
    cb_off, cb_items = eng.csr(1)
    sph, circ, vert = a["spheres"], a["circles"], a["vertices"]
    arr = dict(center=sph[:, :3].copy(), expanded=sph[:, 3].copy(), radius=sph[:, 4].copy(),
               status=a["status"].astype(np.uint32), nb_off=nb_off, nb_items=nb_items,
               circle=circ[:, 2:12].copy() if len(circ) else np.zeros((0, 10)), cb_off=cb_off, cb_items=cb_items,
               vertex=vert[:, :3].copy() if len(vert) else np.zeros((0, 3)),
               sphere_grid=eng.grid(0), circle_grid=eng.grid(1), vertex_grid=eng.grid(2),
               max_expanded=eng.info["max_expanded"], rho_max=eng.info["rho_max"], probe=None)
    return arr


def lattice_from_oracle(eng, spacing, brick):
    i = eng.info
    return dict(spacing=spacing, brick=brick, frame=[int(i["frame_x"]), int(i["frame_y"]), int(i["frame_z"])],
                band=i["band"])


def random_chain(seed, n):
    """testkit::clusters::random_chain (crates/sesmesh-testkit/src/clusters.rs:73-88)."""
    s = [seed & 0xFFFFFFFFFFFFFFFF]
    M = 0xFFFFFFFFFFFFFFFF

    def nxt():
        s[0] = (s[0] + 0x9E3779B97F4A7C15) & M
        z = s[0]
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & M
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & M
        return z ^ (z >> 31)

    def uniform(lo, hi):
        return lo + (hi - lo) * float(nxt() >> 11) / float(1 << 53)

    def unit():
        while True:
            v = [uniform(-1.0, 1.0) for _ in range(3)]
            n2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2]
            if 0.01 <= n2 <= 1.0:
                n = n2 ** 0.5
                return [v[0] / n, v[1] / n, v[2] / n]

    centers = [[0.0, 0.0, 0.0]]
    while len(centers) < n:
        frm = centers[nxt() % len(centers)]
        step = uniform(1.3, 1.6)
        u = unit()
        centers.append([frm[0] + u[0] * step, frm[1] + u[1] * step, frm[2] + u[2] * step])
    radii = [uniform(1.2, 2.0) for _ in range(n)]
    probe = uniform(0.6, 1.8)
    return np.array([c + [r] for c, r in zip(centers, radii)]), probe
