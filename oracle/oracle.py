"""ctypes view of the CPU oracle (test infrastructure only).

The oracle is a C++ restatement of sesmesh 1.3.2's CPU back end for the SES
mesh stage (see oracle.hpp).  Only the tests, the smoke check and the
benchmark's CPU-baseline leg load it; the product never does.
"""
import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None


def build():
    """Builds liboracle.so with make (no-op when it is up to date)."""
    import subprocess
    subprocess.run(["make", "-s", "-C", _HERE], check=True)


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            build()
        L = C.CDLL(path)
        vp, sz, dp, fp = C.c_void_p, C.c_size_t, C.POINTER(C.c_double), C.POINTER(C.c_float)
        u32p, i32p = C.POINTER(C.c_uint32), C.POINTER(C.c_int32)
        L.orc_engine_new.restype = vp
        L.orc_engine_new.argtypes = [dp, sz, C.c_double, C.c_double, sz, C.c_int, C.c_char_p, sz]
        L.orc_engine_free.argtypes = [vp]
        L.orc_engine_info.argtypes = [vp, dp]
        L.orc_engine_arrangement.argtypes = [vp, dp, C.POINTER(C.c_uint8), u32p, dp, dp]
        L.orc_engine_csr.argtypes = [vp, C.c_int, u32p, u32p]
        L.orc_engine_grid.restype = sz
        L.orc_engine_grid.argtypes = [vp, C.c_int, dp, u32p, u32p, u32p]
        L.orc_engine_classify.restype = C.c_long
        L.orc_engine_classify.argtypes = [vp, i32p, sz, C.POINTER(sz), C.c_char_p, sz]
        L.orc_engine_sub_states.argtypes = [vp, i32p, sz, C.POINTER(C.c_int8)]
        L.orc_engine_values.argtypes = [vp, i32p, sz, fp]
        L.orc_engine_gather.restype = sz
        L.orc_engine_gather.argtypes = [vp, i32p, C.c_int, u32p, sz]
        L.orc_mc_brick.argtypes = [C.c_int, fp, u32p, u32p, C.POINTER(sz)]
        L.orc_engine_field.argtypes = [vp, dp, sz, dp]
        L.orc_engine_field_normals.restype = None
        L.orc_engine_field_normals.argtypes = [vp, dp, sz, dp, dp, C.POINTER(C.c_uint8)]
        L.orc_engine_mesh_sample.restype = C.c_double
        L.orc_engine_mesh_sample.argtypes = [vp, i32p, sz, C.POINTER(C.c_uint64)]
        L.orc_surface_new.restype = vp
        L.orc_surface_new.argtypes = [dp, sz, C.c_double, C.c_double, sz, C.c_int, C.c_char_p, sz]
        L.orc_surface_free.argtypes = [vp]
        L.orc_surface_stats.argtypes = [vp, dp]
        L.orc_surface_mesh.argtypes = [vp, fp, fp, u32p, u32p, C.POINTER(C.c_uint8)]
        L.orc_surface_obj.restype = sz
        L.orc_surface_obj.argtypes = [vp, C.c_char_p, sz]
        L.orc_obj_of.restype = sz
        L.orc_obj_of.argtypes = [fp, fp, sz, u32p, sz, C.c_int, C.c_char_p, sz]
        L.orc_push_fixed.restype = sz
        L.orc_push_fixed.argtypes = [C.c_float, C.c_int, C.c_char_p, sz]
        L.orc_set_threads.argtypes = [C.c_int]
        L.orc_threads.restype = C.c_int
        _LIB = L
    return _LIB


def _p(a, t):
    return a.ctypes.data_as(C.POINTER(t))


def _xyzr(spheres):
    a = np.ascontiguousarray(spheres, dtype=np.float64).reshape(-1, 4)
    return a


def set_threads(n):
    lib().orc_set_threads(int(n))


def threads():
    return lib().orc_threads()


INFO_KEYS = ("frame_x", "frame_y", "frame_z", "band", "coord_max", "f32_ok", "n_spheres", "n_contained",
             "n_circles", "n_vertices", "max_expanded", "rho_max", "nb_items", "cb_items", "sub", "nsub",
             "edge_clamp")

KINDS = {"ses": 0, "sas": 1, "vdw": 2}
STAT_KEYS = ("touched", "surface_bricks", "vertices", "triangles", "components", "area", "volume", "euler",
             "refine_evaluations", "t_geometry", "t_classify", "t_mesh", "t_assemble", "t_measure")


class Engine:
    """SesField + Engine of the oracle for one sphere set."""

    def __init__(self, spheres, probe, spacing, brick=10, kind="ses"):
        s = _xyzr(spheres)
        self._keep = s
        err = C.create_string_buffer(512)
        self.h = lib().orc_engine_new(_p(s, C.c_double), len(s), probe, spacing, brick, KINDS[kind], err, 512)
        if not self.h:
            raise ValueError(err.value.decode())
        self.brick = brick
        self.info = self._info()

    def _info(self):
        out = np.zeros(len(INFO_KEYS))
        lib().orc_engine_info(self.h, _p(out, C.c_double))
        return dict(zip(INFO_KEYS, out.tolist()))

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_engine_free(self.h)
            self.h = None

    def arrangement(self):
        n, nc, nv = int(self.info["n_spheres"]), int(self.info["n_circles"]), int(self.info["n_vertices"])
        sph = np.zeros((n, 5))
        st = np.zeros(n, np.uint8)
        orig = np.zeros(n, np.uint32)
        circ = np.zeros((nc, 12))
        vert = np.zeros((nv, 6))
        lib().orc_engine_arrangement(self.h, _p(sph, C.c_double), _p(st, C.c_uint8), _p(orig, C.c_uint32),
                                     _p(circ, C.c_double), _p(vert, C.c_double))
        return dict(spheres=sph, status=st, orig=orig, circles=circ, vertices=vert)

    def csr(self, which):
        rows = int(self.info["n_spheres"] if which == 0 else self.info["n_circles"])
        total = int(self.info["nb_items"] if which == 0 else self.info["cb_items"])
        off = np.zeros(rows + 1, np.uint32)
        items = np.zeros(max(total, 1), np.uint32)
        lib().orc_engine_csr(self.h, which, _p(off, C.c_uint32), _p(items, C.c_uint32))
        return off, items[:total]

    def grid(self, which):
        n_items = [self.info["n_spheres"], self.info["n_circles"], self.info["n_vertices"]][which]
        cells = lib().orc_engine_grid(self.h, which, None, None, None, None)
        oc = np.zeros(4)
        dims = np.zeros(3, np.uint32)
        starts = np.zeros(cells + 1, np.uint32)
        items = np.zeros(max(int(n_items), 1), np.uint32)
        lib().orc_engine_grid(self.h, which, _p(oc, C.c_double), _p(dims, C.c_uint32), _p(starts, C.c_uint32),
                              _p(items, C.c_uint32))
        return dict(origin=oc[:3].copy(), cell=float(oc[3]), dims=dims, starts=starts, items=items[:int(n_items)])

    def classify(self):
        err = C.create_string_buffer(512)
        touched = C.c_size_t(0)
        n = lib().orc_engine_classify(self.h, None, 0, C.byref(touched), err, 512)
        if n < 0:
            raise ValueError(err.value.decode())
        out = np.zeros((max(n, 1), 3), np.int32)
        lib().orc_engine_classify(self.h, _p(out, C.c_int32), n, C.byref(touched), err, 512)
        return out[:n], touched.value

    def sub_states(self, bricks):
        b = np.ascontiguousarray(bricks, np.int32).reshape(-1, 3)
        out = np.zeros((len(b), 8), np.int8)
        lib().orc_engine_sub_states(self.h, _p(b, C.c_int32), len(b), _p(out, C.c_int8))
        return out

    def values(self, bricks):
        b = np.ascontiguousarray(bricks, np.int32).reshape(-1, 3)
        s = self.brick + 1
        out = np.zeros((len(b), s * s * s), np.float32)
        lib().orc_engine_values(self.h, _p(b, C.c_int32), len(b), _p(out, C.c_float))
        return out

    def gather(self, brick, sb):
        b = np.ascontiguousarray(brick, np.int32).reshape(3)
        n = lib().orc_engine_gather(self.h, _p(b, C.c_int32), sb, None, 0)
        w = np.zeros(n, np.uint32)
        lib().orc_engine_gather(self.h, _p(b, C.c_int32), sb, _p(w, C.c_uint32), n)
        n_in, n_near, n_s, n_c, n_v, n_sb, n_cb = (int(x) for x in w[:7])
        pos = 7
        out = {"n_inside": n_in}
        for key, cnt in (("near", n_near), ("s", n_s), ("s_off", n_s + 1), ("s_blk", n_sb), ("c", n_c),
                         ("c_off", n_c + 1), ("c_blk", n_cb), ("v", n_v)):
            out[key] = w[pos:pos + cnt].copy()
            pos += cnt
        return out

    def mesh_sample(self, bricks):
        """Wall seconds of the CPU mesh stage (evaluate + mesh_brick) on the
        given bricks, all threads; and the refinement evaluations."""
        b = np.ascontiguousarray(bricks, np.int32).reshape(-1, 3)
        ev = C.c_uint64(0)
        s = lib().orc_engine_mesh_sample(self.h, _p(b, C.c_int32), len(b), C.byref(ev))
        return s, ev.value

    def field(self, pts):
        p = np.ascontiguousarray(pts, np.float64).reshape(-1, 3)
        out = np.zeros(len(p))
        lib().orc_engine_field(self.h, _p(p, C.c_double), len(p), _p(out, C.c_double))
        return out

    def field_normals(self, pts):
        """(values, normals (n, 3), has-normal mask) of SesField::sample."""
        p = np.ascontiguousarray(pts, np.float64).reshape(-1, 3)
        out = np.zeros(len(p))
        nrm = np.zeros((len(p), 3))
        has = np.zeros(len(p), np.uint8)
        lib().orc_engine_field_normals(self.h, _p(p, C.c_double), len(p), _p(out, C.c_double),
                                       _p(nrm, C.c_double), _p(has, C.c_uint8))
        return out, nrm, has.astype(bool)


def mc_brick(b, values):
    v = np.ascontiguousarray(values, np.float32)
    cap = 3 * b * b * b
    edges = np.zeros(cap, np.uint32)
    tris = np.zeros((5 * b * b * b, 3), np.uint32)
    n = (C.c_size_t * 2)()
    lib().orc_mc_brick(b, _p(v, C.c_float), _p(edges, C.c_uint32), _p(tris, C.c_uint32), n)
    return edges[:n[0]], tris[:n[1]]


class Surface:
    """The oracle's whole CPU pipeline (compute_surface, CPU back end)."""

    def __init__(self, spheres, probe, spacing, brick=10, kind="ses"):
        s = _xyzr(spheres)
        err = C.create_string_buffer(512)
        self.h = lib().orc_surface_new(_p(s, C.c_double), len(s), probe, spacing, brick, KINDS[kind], err, 512)
        if not self.h:
            raise ValueError(err.value.decode())
        out = np.zeros(len(STAT_KEYS))
        lib().orc_surface_stats(self.h, _p(out, C.c_double))
        self.stats = dict(zip(STAT_KEYS, out.tolist()))

    def __del__(self):
        if getattr(self, "h", None):
            lib().orc_surface_free(self.h)
            self.h = None

    def mesh(self):
        nv, nt = int(self.stats["vertices"]), int(self.stats["triangles"])
        pos = np.zeros((nv, 3), np.float32)
        nrm = np.zeros((nv, 3), np.float32)
        tris = np.zeros((nt, 3), np.uint32)
        atoms = np.zeros(nv, np.uint32)
        patches = np.zeros(nv, np.uint8)
        lib().orc_surface_mesh(self.h, _p(pos, C.c_float), _p(nrm, C.c_float), _p(tris, C.c_uint32),
                               _p(atoms, C.c_uint32), _p(patches, C.c_uint8))
        return dict(positions=pos, normals=nrm, triangles=tris, atoms=atoms, patches=patches)

    def obj(self):
        n = lib().orc_surface_obj(self.h, None, 0)
        buf = C.create_string_buffer(n)
        lib().orc_surface_obj(self.h, buf, n)
        return buf.raw[:n]


def obj_of(positions, normals, triangles, precision=4):
    p = np.ascontiguousarray(positions, np.float32)
    t = np.ascontiguousarray(triangles, np.uint32)
    nrm = None if normals is None else np.ascontiguousarray(normals, np.float32)
    n = lib().orc_obj_of(_p(p, C.c_float), None if nrm is None else _p(nrm, C.c_float), len(p),
                         _p(t, C.c_uint32), len(t), precision, None, 0)
    buf = C.create_string_buffer(n)
    lib().orc_obj_of(_p(p, C.c_float), None if nrm is None else _p(nrm, C.c_float), len(p),
                     _p(t, C.c_uint32), len(t), precision, buf, n)
    return buf.raw[:n]


def push_fixed(x, prec):
    buf = C.create_string_buffer(600)
    n = lib().orc_push_fixed(C.c_float(x), prec, buf, 600)
    return buf.raw[:n].decode()


# ---- the reference's own CUDA kernels (oracle/_ref, built by `make ref-gpu`) ----
_REFGPU = None


class _RefInput(C.Structure):
    _fields_ = [("n_spheres", C.c_uint), ("n_circles", C.c_uint), ("n_vertices", C.c_uint),
                ("sphere", C.c_void_p), ("status", C.c_void_p), ("nb_off", C.c_void_p), ("nb_items", C.c_void_p),
                ("nb_items_len", C.c_uint), ("circle", C.c_void_p), ("cb_off", C.c_void_p),
                ("cb_items", C.c_void_p), ("cb_items_len", C.c_uint), ("vertex", C.c_void_p),
                ("grid_f", C.c_void_p), ("grid_dims", C.c_void_p), ("grid_starts", C.c_void_p * 3),
                ("grid_items", C.c_void_p * 3), ("grid_n_items", C.c_uint * 3),
                ("max_expanded", C.c_float), ("rho_max", C.c_float), ("probe", C.c_float), ("band", C.c_float),
                ("cutoff2", C.c_float), ("rho", C.c_float), ("reach", C.c_float), ("margin", C.c_float),
                ("slack", C.c_float), ("cutoffc2", C.c_float), ("h", C.c_float), ("b", C.c_uint),
                ("sub", C.c_uint), ("bricks", C.c_void_p), ("n_bricks", C.c_uint)]


class _RefTimes(C.Structure):
    _fields_ = [("count_ms", C.c_double), ("scan_ms", C.c_double), ("fill_ms", C.c_double),
                ("sample_ms", C.c_double), ("total_ms", C.c_double), ("ids", C.c_ulonglong)]


class _RefFast(C.Structure):
    _fields_ = [("sphere_lo", C.c_void_p), ("circle_lo", C.c_void_p), ("vertex_lo", C.c_void_p),
                ("h_hi", C.c_float), ("h_lo", C.c_float), ("tol", C.c_float), ("max_iter", C.c_uint),
                ("max_bisect", C.c_uint), ("edge_off", C.c_void_p), ("t", C.c_void_p), ("feat", C.c_void_p),
                ("q", C.c_void_p), ("evals", C.c_void_p), ("cap", C.c_ulonglong), ("n_edges", C.c_ulonglong),
                ("edge_count_ms", C.c_double), ("scan_ms", C.c_double), ("refine_ms", C.c_double)]


def _residuals(points, fo):
    """(x - f64(f32(x))) as f32 of the frame-local points, x, y, z rows
    (Residuals::new, crates/sesmesh/src/field/gpu.rs:184-204)."""
    if len(points) == 0:
        return np.zeros((3, 1), np.float32)
    d = np.asarray(points, np.float64)[:, :3] - fo
    return np.ascontiguousarray((d - d.astype(np.float32).astype(np.float64)).T.astype(np.float32))


def ref_gpu_path():
    return os.path.join(_HERE, "_ref", "libsesmesh_refgpu.so")


def ref_gpu_available():
    return os.path.exists(ref_gpu_path())


def ref_gpu_run(eng, bricks, spacing, brick, probe, reps=3, fast=False, cap=None):
    """Sample values of the given surface bricks from the reference's own
    CUDA kernels (count, host scan, fill, sample, as cuda::Resident::run)
    with the inputs gpu.rs builds for them, and the best time of each pass
    over `reps` runs (the first a warm-up): ((n, (b+1)^3) f32, times).

    With fast, then cuda::Resident::refine's passes (edge count, host scan,
    refine; resident.rs:632-687) on those values with the refinement
    constants of Residuals::as_ref (gpu.rs:206-222), and a third result:
    dict(edge_off (8n + 1, per sub-block), t, feat, q (n_edges, 3), evals)
    in the kernels' order (sub-blocks in turn, each in crossing_edge's
    z, y, x, axis order)."""
    global _REFGPU
    if _REFGPU is None:
        L = C.CDLL(ref_gpu_path())
        L.refgpu_run.restype = C.c_int
        L.refgpu_run.argtypes = [C.POINTER(_RefInput), C.c_int, C.POINTER(C.c_float), C.POINTER(_RefTimes)]
        L.refgpu_run_fast.restype = C.c_int
        L.refgpu_run_fast.argtypes = [C.POINTER(_RefInput), C.c_int, C.POINTER(C.c_float), C.POINTER(_RefTimes),
                                      C.POINTER(_RefFast)]
        _REFGPU = L
    i = eng.info
    h, b = float(spacing), int(brick)
    sub = b // 2
    frame = np.array([i["frame_x"], i["frame_y"], i["frame_z"]], np.int64)
    fo = frame.astype(np.float64) * h                               # lattice.rs:62-64
    a = eng.arrangement()
    sph = a["spheres"]
    n = len(sph)
    r32 = sph[:, 3].astype(np.float32)
    rt = np.maximum(r32 - np.float32(2e-5), np.float32(0))           # kernel.rs:42 INSIDE_TOL
    sphere = np.stack([(sph[:, 0] - fo[0]).astype(np.float32), (sph[:, 1] - fo[1]).astype(np.float32),
                       (sph[:, 2] - fo[2]).astype(np.float32), r32, r32 * r32, rt * rt,
                       sph[:, 4].astype(np.float32)]).astype(np.float32).copy()
    status = np.ascontiguousarray(a["status"], np.uint32)
    nb_off, nb_items = eng.csr(0)
    cb_off, cb_items = eng.csr(1)
    circ = a["circles"]
    nc = len(circ)
    if nc:
        c = circ[:, 2:12].copy()
        c[:, 0:3] -= fo
        circle = np.ascontiguousarray(c.T.astype(np.float32))
    else:
        circle = np.zeros((10, 1), np.float32)
    vert = a["vertices"]
    nv = len(vert)
    vertex = np.ascontiguousarray((vert[:, :3] - fo).T.astype(np.float32)) if nv else np.zeros((3, 1), np.float32)
    grids = [eng.grid(g) for g in range(3)]
    grid_f = np.array([[*(gr["origin"] - fo), gr["cell"]] for gr in grids], np.float64).astype(np.float32)
    grid_dims = np.array([gr["dims"] for gr in grids], np.uint32)
    # batch_params (field/gpu.rs:369-400).
    band = float(i["band"])
    rho = 0.5 * np.sqrt(3.0) * sub * h
    reach = probe + band + rho
    margin = rho + 2e-3                                              # CLASSIFY_EPS
    cutoffc = np.float32(probe + margin + 2e-3)
    cutoff = np.float32(probe + band)
    m = np.float32(min(max(float(i["coord_max"]), 1.0), 1e6))
    ulp = np.nextafter(m, np.float32(np.inf)) - m
    slack = np.float32(1e-3) + np.float32(16.0) * ulp
    bk = np.asarray(bricks, np.int64).reshape(-1, 3) * b - frame      # frame_origins (gpu.rs:403-414)
    bk = np.ascontiguousarray(bk, np.int32)
    keep = [sphere, status, nb_off, nb_items, circle, cb_off, cb_items, vertex, grid_f, grid_dims, bk]
    ri = _RefInput()
    ri.n_spheres, ri.n_circles, ri.n_vertices = n, nc, nv
    ri.sphere, ri.status = sphere.ctypes.data, status.ctypes.data
    ri.nb_off, ri.nb_items, ri.nb_items_len = nb_off.ctypes.data, nb_items.ctypes.data, len(nb_items)
    ri.circle, ri.cb_off, ri.cb_items, ri.cb_items_len = circle.ctypes.data, cb_off.ctypes.data, \
        cb_items.ctypes.data, len(cb_items)
    ri.vertex, ri.grid_f, ri.grid_dims = vertex.ctypes.data, grid_f.ctypes.data, grid_dims.ctypes.data
    for g, gr in enumerate(grids):
        keep += [gr["starts"], gr["items"]]
        ri.grid_starts[g], ri.grid_items[g], ri.grid_n_items[g] = gr["starts"].ctypes.data, \
            gr["items"].ctypes.data, len(gr["items"])
    ri.max_expanded, ri.rho_max = float(i["max_expanded"]), float(i["rho_max"])
    ri.probe, ri.band, ri.cutoff2, ri.rho = probe, band, float(cutoff * cutoff), rho
    ri.reach, ri.margin, ri.slack, ri.cutoffc2, ri.h = reach, margin, float(slack), float(cutoffc * cutoffc), h
    ri.b, ri.sub, ri.bricks, ri.n_bricks = b, sub, bk.ctypes.data, len(bk)
    out = np.zeros((len(bk), (b + 1) ** 3), np.float32)
    t = _RefTimes()
    if not fast:
        rc = _REFGPU.refgpu_run(C.byref(ri), int(reps), _p(out, C.c_float), C.byref(t))
        if rc:
            raise RuntimeError("reference kernels failed (%d)" % rc)
        return out, {name: getattr(t, name) for name, _ in t._fields_}
    if cap is None:
        cap = 3 * b * b * b * len(bk)
    cap = max(int(cap), 1)
    lo = [_residuals(sph, fo), _residuals(circ[:, 2:5] if nc else circ, fo),
          _residuals(vert[:, :3] if nv else vert, fo)]
    fr = dict(edge_off=np.zeros(8 * len(bk) + 1, np.uint32), t=np.zeros(cap, np.float32),
              feat=np.zeros(cap, np.uint32), q=np.zeros((cap, 3), np.float32), evals=np.zeros(cap, np.uint32))
    f = _RefFast()
    f.sphere_lo, f.circle_lo, f.vertex_lo = (x.ctypes.data for x in lo)
    f.h_hi = float(np.float32(h))
    f.h_lo = float(np.float32(h - float(np.float32(h))))
    f.tol, f.max_iter, f.max_bisect = float(np.float32(1e-5)), 8, 64
    f.edge_off, f.t, f.feat = fr["edge_off"].ctypes.data, fr["t"].ctypes.data, fr["feat"].ctypes.data
    f.q, f.evals, f.cap = fr["q"].ctypes.data, fr["evals"].ctypes.data, cap
    rc = _REFGPU.refgpu_run_fast(C.byref(ri), int(reps), _p(out, C.c_float), C.byref(t), C.byref(f))
    if rc:
        raise RuntimeError("reference kernels failed (%d)" % rc)
    ne = int(f.n_edges)
    for k in ("t", "feat", "q", "evals"):
        fr[k] = fr[k][:ne]
    times = {name: getattr(t, name) for name, _ in t._fields_}
    times.update(edge_count_ms=f.edge_count_ms, edge_scan_ms=f.scan_ms, refine_ms=f.refine_ms)
    return out, times, fr
