"""ctypes bindings of the C ABI in include/sesmesh_b200.h.

Loads the in-tree libsesmesh_b200.so (built by `make -C sesmesh_b200`); there
is no fallback: without the library, or without a CUDA device, the calls
raise.
"""
import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libsesmesh_b200.so")
SYNTH_PATH = os.path.join(_HERE, "libsesmesh_synth.so")

SMB_OK = 0
SMB_ERR_MEMORY = 6
ERRORS = {1: "argument", 2: "cuda", 3: "no device", 4: "self-test", 5: "range", 6: "memory", 7: "state",
          8: "timeout", 9: "cancelled"}
REC_WORDS = 12


class SmbError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("sesmesh_b200 %s error: %s" % (ERRORS.get(code, code), msg))
        self.code = code


class GridRef(C.Structure):
    _fields_ = [("origin", C.c_double * 3), ("cell", C.c_double), ("dims", C.c_uint32 * 3),
                ("starts", C.POINTER(C.c_uint32)), ("items", C.POINTER(C.c_uint32)), ("n_items", C.c_size_t)]


class ArrangementRef(C.Structure):
    _fields_ = [("n_spheres", C.c_size_t), ("center", C.POINTER(C.c_double)), ("expanded", C.POINTER(C.c_double)),
                ("radius", C.POINTER(C.c_double)), ("status", C.POINTER(C.c_uint32)),
                ("nb_off", C.POINTER(C.c_uint32)), ("nb_items", C.POINTER(C.c_uint32)),
                ("n_circles", C.c_size_t), ("circle", C.POINTER(C.c_double)), ("cb_off", C.POINTER(C.c_uint32)),
                ("cb_items", C.POINTER(C.c_uint32)), ("n_vertices", C.c_size_t), ("vertex", C.POINTER(C.c_double)),
                ("sphere_grid", GridRef), ("circle_grid", GridRef), ("vertex_grid", GridRef),
                ("max_expanded", C.c_double), ("rho_max", C.c_double), ("probe", C.c_double), ("kind", C.c_int)]


class LatticeRef(C.Structure):
    _fields_ = [("spacing", C.c_double), ("brick", C.c_uint32), ("frame", C.c_int64 * 3), ("band", C.c_double)]


class BatchTimes(C.Structure):
    _fields_ = [("substates", C.c_double), ("gather", C.c_double), ("sample", C.c_double), ("mc", C.c_double),
                ("total", C.c_double)]


class DeviceInfo(C.Structure):
    _fields_ = [("name", C.c_char * 256), ("major", C.c_int), ("minor", C.c_int), ("multiprocessors", C.c_int),
                ("memory", C.c_size_t)]


class SurfaceParams_(C.Structure):
    _fields_ = [("kind", C.c_int), ("probe_radius", C.c_double), ("spacing", C.c_double), ("brick_size", C.c_uint32),
                ("refine", C.c_int), ("threads", C.c_int)]


STAT_FIELDS = ["spheres", "touched_bricks", "surface_bricks", "samples", "vertices", "triangles", "components"]
TIME_FIELDS = ["t_geometry", "t_upload", "t_classify", "t_substates", "t_gather", "t_sample", "t_mc", "t_device",
               "t_d2h", "t_host_refine", "t_mesh_stage", "t_assemble", "t_measure", "t_total"]


class SurfaceStats_(C.Structure):
    _fields_ = ([(f, C.c_size_t) for f in STAT_FIELDS] + [("area", C.c_double), ("volume", C.c_double),
                                                           ("euler", C.c_int64), ("refine_evaluations", C.c_uint64),
                                                           ("refine_cpu_edges", C.c_uint64)]
                + [(f, C.c_double) for f in TIME_FIELDS] + [("host_threads", C.c_int)]
                + [("arrangement_where", C.c_int), ("finished_on_host", C.c_int), ("upload_bytes", C.c_uint64),
                   ("spacing_used", C.c_double), ("device_bytes_estimate", C.c_uint64)])


class Selection_(C.Structure):
    _fields_ = [("model", C.c_int), ("hydrogens", C.c_int), ("waters", C.c_int), ("hetero", C.c_int)]


PROGRESS_FN = C.CFUNCTYPE(None, C.c_void_p, C.c_int, C.c_uint64, C.c_uint64)


class Control_(C.Structure):
    _fields_ = [("cancel", C.POINTER(C.c_int32)), ("progress", PROGRESS_FN), ("user", C.c_void_p),
                ("max_device_bytes", C.c_uint64), ("auto_coarsen", C.c_int)]


class ArrangementInfo(C.Structure):
    _fields_ = [("n_spheres", C.c_size_t), ("n_contained", C.c_size_t), ("n_circles", C.c_size_t),
                ("n_vertices", C.c_size_t), ("center", C.POINTER(C.c_double)), ("expanded", C.POINTER(C.c_double)),
                ("circle", C.POINTER(C.c_double)), ("vertex", C.POINTER(C.c_double)),
                ("status", C.POINTER(C.c_uint32)), ("orig", C.POINTER(C.c_uint32)),
                ("circle_ij", C.POINTER(C.c_uint32)), ("vertex_atoms", C.POINTER(C.c_uint32)),
                ("nb_off", C.POINTER(C.c_uint32)), ("nb_items", C.POINTER(C.c_uint32)),
                ("cb_off", C.POINTER(C.c_uint32)), ("cb_items", C.POINTER(C.c_uint32)),
                ("max_expanded", C.c_double), ("rho_max", C.c_double), ("band", C.c_double), ("t_min", C.c_double),
                ("frame", C.c_int64 * 3), ("built_on_device", C.c_int)]


class MultiConfig(C.Structure):
    _fields_ = [("brick", C.c_uint32), ("caps_level", C.c_uint32), ("gather_warps", C.c_uint32)]


MULTI_COUNTS = ["structures", "redone", "bricks", "samples"]
MULTI_TIMES = ["t_setup", "t_tune", "t_classify", "t_device", "t_d2h", "t_host", "t_redo", "t_total"]


class MultiTimes(C.Structure):
    _fields_ = [(f, C.c_size_t) for f in MULTI_COUNTS] + [(f, C.c_double) for f in MULTI_TIMES] + \
               [("graph", C.c_int), ("groups", C.c_size_t), ("over_lists", C.c_ulonglong),
                ("over_memory", C.c_ulonglong)]


class BatchInfo(C.Structure):
    _fields_ = [(f, C.c_size_t) for f in ("bricks", "sampled_subblocks", "ids_words", "max_pack_units", "edges",
                                          "triangles", "touched", "resident_bytes")] + \
               [("pack_units", C.c_ulonglong), ("classify_ms", C.c_double), ("exact_block_items", C.c_size_t),
                ("gather_caps", C.c_uint32 * 4), ("gather_warps", C.c_uint32)]


# Every entry point of include/*.h with its ctypes signature.
_vp, _sz, _cp = C.c_void_p, C.c_size_t, C.c_char_p
_u32p, _i32p, _fp = C.POINTER(C.c_uint32), C.POINTER(C.c_int32), C.POINTER(C.c_float)
SIGNATURES = {
    "smb_open": (C.c_int, [C.c_int, C.POINTER(_vp), _cp, _sz]),
    "smb_close": (None, [_vp]),
    "smb_device_info_get": (C.c_int, [_vp, C.POINTER(DeviceInfo)]),
    "smb_self_test": (C.c_int, [_vp, C.c_uint32, _cp, _sz]),
    "smb_resident_new": (C.c_int, [_vp, C.POINTER(ArrangementRef), C.POINTER(LatticeRef), C.POINTER(_vp), _cp, _sz]),
    "smb_resident_free": (None, [_vp]),
    "smb_resident_bytes": (_sz, [_vp]),
    "smb_classify": (C.c_int, [_vp, C.POINTER(_sz), C.POINTER(_sz), _cp, _sz]),
    "smb_resident_bricks": (C.c_int, [_vp, _i32p, _sz]),
    "smb_batch_new": (C.c_int, [_vp, C.POINTER(_vp), _cp, _sz]),
    "smb_batch_free": (None, [_vp]),
    "smb_run": (C.c_int, [_vp, _sz, _sz, _vp, C.POINTER(BatchTimes), _cp, _sz]),
    "smb_batch_bricks": (_sz, [_vp]),
    "smb_batch_records": (C.c_int, [_vp, _u32p]),
    "smb_batch_values": (C.c_int, [_vp, _fp]),
    "smb_batch_ids_words": (_sz, [_vp]),
    "smb_batch_ids": (C.c_int, [_vp, _u32p]),
    "smb_batch_mc_counts": (C.c_int, [_vp, C.POINTER(_sz), C.POINTER(_sz)]),
    "smb_batch_mc": (C.c_int, [_vp, _u32p, _u32p, _fp, _u32p, _u32p]),
    "smb_resident_set_refinement": (C.c_int, [_vp, _cp, _sz]),
    "smb_refine": (C.c_int, [_vp, _vp, C.POINTER(C.c_double), _cp, _sz]),
    "smb_batch_edges": (C.c_int, [_vp, _fp, _u32p, _fp, _u32p]),
    "smb_refine_warm": (C.c_int, [_vp, _vp, _vp, C.POINTER(C.c_double), _cp, _sz]),
    "smb_batch_edge_features": (C.c_int, [_vp, _vp, _fp, C.POINTER(C.c_uint8), _cp, _sz]),
    "smb_batch_record_features": (C.c_int, [_vp, C.c_int]),
    "smb_batch_sample_features": (C.c_int, [_vp, C.POINTER(C.c_uint32)]),
    "smb_resident_set_exact": (C.c_int, [_vp, _u32p, _u32p, _sz, _u32p, _sz, C.c_double, _cp, _sz]),
    "smb_refine_exact": (C.c_int, [_vp, _vp, C.POINTER(C.c_double), _cp, _sz]),
    "smb_batch_vertices": (C.c_int, [_vp, _fp, _fp, _u32p, C.POINTER(C.c_uint8), _fp, _u32p]),
    "smb_batch_set_exact_region": (C.c_int, [_vp, _sz]),
    "smb_batch_set_refine_region": (C.c_int, [_vp, _sz]),
    "smb_batch_set_refine_group": (C.c_int, [_vp, C.c_int]),
    "smb_batch_set_exact_group": (C.c_int, [_vp, C.c_int]),
    "smb_batch_set_exact_hint": (C.c_int, [_vp, C.c_int]),
    "smb_batch_set_sample_region": (C.c_int, [_vp, _sz]),
    "smb_batch_exact_summary": (C.c_int, [_vp, C.POINTER(C.c_ulonglong), C.POINTER(C.c_ulonglong),
                                          C.POINTER(C.c_ulonglong)]),
    "smb_place_fast": (C.c_int, [_vp, _vp, C.POINTER(C.c_double), _cp, _sz]),
    "smb_batch_count_exact_ops": (C.c_int, [_vp, C.POINTER(C.c_ulonglong), _cp, _sz]),
    "smb_batch_count_refine_ops": (C.c_int, [_vp, _vp, C.POINTER(C.c_ulonglong), _cp, _sz]),
    "smb_kernel_launches": (C.c_ulonglong, []),
    "smb_batch_info_get": (C.c_int, [_vp, C.POINTER(BatchInfo)]),
    "smb_batch_count_ops": (C.c_int, [_vp, C.POINTER(C.c_ulonglong), C.POINTER(C.c_ulonglong), _cp, _sz]),
    "smb_engine_batch": (_vp, [_vp]),
    "smb_mlp_new": (C.c_int, [_vp, _fp, C.POINTER(_vp), _cp, _sz]),
    "smb_mlp_free": (None, [_vp]),
    "smb_mlp_set_params": (C.c_int, [_vp, _fp, _cp, _sz]),
    "smb_mlp_get_params": (C.c_int, [_vp, _fp]),
    "smb_compute_surface_with": (C.c_int, [_vp, C.POINTER(C.c_double), _sz, C.POINTER(SurfaceParams_),
                                           C.POINTER(Control_), C.POINTER(_vp), _cp, _sz]),
    "smb_engine_new_with": (C.c_int, [_vp, C.POINTER(C.c_double), _sz, C.POINTER(SurfaceParams_),
                                      C.POINTER(Control_), C.POINTER(_vp), _cp, _sz]),
    "smb_engine_set_control": (C.c_int, [_vp, C.POINTER(Control_)]),
    "smb_multi_set_control": (C.c_int, [_vp, C.POINTER(Control_)]),
    "smb_arrangement_build_with": (C.c_int, [C.POINTER(C.c_double), _sz, C.POINTER(SurfaceParams_),
                                             C.POINTER(Control_), C.POINTER(_vp), _cp, _sz]),
    "smb_device_bytes_estimate": (C.c_uint64, [_sz, C.c_uint32, C.c_double, C.c_double, _sz, C.c_int, C.c_int]),
    "smb_engine_device_bytes": (C.c_uint64, [_vp]),
    "smb_read_structure": (C.c_int, [C.c_char_p, _sz, C.c_int, C.POINTER(Selection_), C.POINTER(C.c_double), _sz,
                                     C.POINTER(_sz), _cp, _sz]),
    "smb_mlp_set_use": (C.c_int, [_vp, C.c_int]),
    "smb_mlp_forward": (C.c_int, [_vp, _fp, _sz, _fp, _cp, _sz]),
    "smb_mlp_gradient": (C.c_int, [_vp, _fp, _fp, _sz, _fp, _fp, _cp, _sz]),
    "smb_mlp_train_epoch": (C.c_int, [_vp, _fp, _fp, _sz, _sz, C.c_float, _fp, _cp, _sz]),
    "smb_mc_noalloc": (C.c_int, [_vp, _vp, _vp, _sz, _vp, _vp, _vp, _sz, _vp, _vp, _sz, C.POINTER(_sz),
                                 C.POINTER(_sz), _cp, _sz]),
    # include/sesmesh_b200_surface.h
    "smb_compute_surface": (C.c_int, [_vp, C.POINTER(C.c_double), _sz, C.POINTER(SurfaceParams_), C.POINTER(_vp),
                                      _cp, _sz]),
    "smb_engine_new": (C.c_int, [_vp, C.POINTER(C.c_double), _sz, C.POINTER(SurfaceParams_), C.POINTER(_vp), _cp,
                                 _sz]),
    "smb_engine_free": (None, [_vp]),
    "smb_engine_run_device": (C.c_int, [_vp, C.POINTER(BatchTimes), _cp, _sz]),
    "smb_engine_bricks": (_sz, [_vp]),
    "smb_engine_mesh": (C.c_int, [_vp, C.POINTER(_vp), _cp, _sz]),
    "smb_engine_set_warm_start": (C.c_int, [_vp, _vp]),
    "smb_engine_set_exact_device": (C.c_int, [_vp, C.c_int]),
    "smb_engine_note": (C.c_char_p, [_vp]),
    "smb_engine_field": (C.c_int, [_vp, C.POINTER(C.c_double), _sz, C.POINTER(C.c_double)]),
    "smb_engine_warm_start_rows": (C.c_int, [_vp, _fp, _fp, _fp, _sz, C.POINTER(_sz), _cp, _sz]),
    "smb_surface_free": (None, [_vp]),
    "smb_surface_arrays": (C.c_int, [_vp] + [C.POINTER(_vp)] * 6),
    "smb_surface_stats_get": (C.c_int, [_vp, C.POINTER(SurfaceStats_)]),
    "smb_surface_mesh": (C.c_int, [_vp, _fp, _fp, _u32p, _u32p, C.POINTER(C.c_uint8), _u32p]),
    "smb_surface_obj": (_sz, [_vp, _cp, _sz]),
    "smb_surface_write_obj": (C.c_int, [_vp, _cp, _cp, _sz]),
    "smb_multi_new": (C.c_int, [_vp, _sz, C.POINTER(C.POINTER(C.c_double)), C.POINTER(_sz),
                                C.POINTER(SurfaceParams_), C.POINTER(MultiConfig), C.POINTER(_vp), _cp, _sz]),
    "smb_multi_free": (None, [_vp]),
    "smb_multi_set_warm_start": (C.c_int, [_vp, _vp]),
    "smb_multi_tune": (C.c_int, [_vp, _cp, _sz]),
    "smb_multi_config_get": (C.c_int, [_vp, C.POINTER(MultiConfig)]),
    "smb_multi_set_device_finish": (C.c_int, [_vp, C.c_int]),
    "smb_multi_run": (C.c_int, [_vp, C.POINTER(MultiTimes), _cp, _sz]),
    "smb_multi_surface": (_vp, [_vp, _sz]),
    "smb_multi_latency": (C.c_int, [_vp, C.POINTER(C.c_double)]),
    "smb_engine_arrangement": (C.c_int, [_vp, C.POINTER(ArrangementInfo)]),
    "smb_set_device_arrangement_min": (None, [_sz]),
    "smb_arrangement_build": (C.c_int, [C.POINTER(C.c_double), _sz, C.POINTER(SurfaceParams_), C.POINTER(_vp), _cp,
                                        _sz]),
}

_LIB = None


def lib():
    """The loaded C-ABI library (raises if it was not built)."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise OSError("libsesmesh_b200.so is not built (run `make -C sesmesh_b200`)")
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in SIGNATURES.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _LIB = L
    return _LIB


def _p(a, t):
    return a.ctypes.data_as(C.POINTER(t))


def _check(rc, err):
    if rc != SMB_OK:
        raise SmbError(rc, err.value.decode(errors="replace"))


class Device:
    """An open CUDA device (smb_open: self-test included)."""

    def __init__(self, index=0):
        err = C.create_string_buffer(1024)
        h = _vp()
        _check(lib().smb_open(index, C.byref(h), err, 1024), err)
        self.h = h
        info = DeviceInfo()
        lib().smb_device_info_get(self.h, C.byref(info))
        self.name = info.name.decode()
        self.capability = (info.major, info.minor)
        self.multiprocessors = info.multiprocessors
        self.memory = info.memory

    def self_test(self, n):
        err = C.create_string_buffer(1024)
        _check(lib().smb_self_test(self.h, n, err, 1024), err)

    def close(self):
        if getattr(self, "h", None):
            lib().smb_close(self.h)
            self.h = None

    def __del__(self):
        self.close()


def _grid(g, keep):
    starts = np.ascontiguousarray(g["starts"], np.uint32)
    items = np.ascontiguousarray(g["items"], np.uint32)
    if len(items) == 0:
        items = np.zeros(1, np.uint32)
        n_items = 0
    else:
        n_items = len(g["items"])
    keep += [starts, items]
    r = GridRef()
    r.origin[:] = [float(v) for v in g["origin"]]
    r.cell = float(g["cell"])
    r.dims[:] = [int(v) for v in g["dims"]]
    r.starts = _p(starts, C.c_uint32)
    r.items = _p(items, C.c_uint32)
    r.n_items = n_items
    return r


class Resident:
    """The arrangement resident on a device (smb_resident_new).

    `arr` holds numpy arrays in internal sphere order: center (n, 3),
    expanded (n,), radius (n,), status (n,), nb_off/nb_items,
    circle (nc, 10), cb_off/cb_items, vertex (nv, 3), grids
    sphere_grid/circle_grid/vertex_grid (dicts of origin, cell, dims, starts,
    items) and max_expanded, rho_max, probe.  `lat` holds spacing, brick,
    frame (3 ints) and band.
    """

    def __init__(self, device, arr, lat):
        self.device = device
        keep = []

        def arrf(x, dt, shape=None):
            a = np.ascontiguousarray(x, dt)
            if a.size == 0:
                a = np.zeros(1, dt)
            keep.append(a)
            return _p(a, C.c_double if dt == np.float64 else C.c_uint32)

        n = len(arr["expanded"])
        ref = ArrangementRef()
        ref.n_spheres = n
        ref.center = arrf(arr["center"], np.float64)
        ref.expanded = arrf(arr["expanded"], np.float64)
        ref.radius = arrf(arr["radius"], np.float64)
        ref.status = arrf(arr["status"], np.uint32)
        ref.nb_off = arrf(arr["nb_off"], np.uint32)
        ref.nb_items = arrf(arr["nb_items"], np.uint32)
        ref.n_circles = len(arr["circle"])
        ref.circle = arrf(arr["circle"], np.float64)
        ref.cb_off = arrf(arr["cb_off"], np.uint32)
        ref.cb_items = arrf(arr["cb_items"], np.uint32)
        ref.n_vertices = len(arr["vertex"])
        ref.vertex = arrf(arr["vertex"], np.float64)
        ref.sphere_grid = _grid(arr["sphere_grid"], keep)
        ref.circle_grid = _grid(arr["circle_grid"], keep)
        ref.vertex_grid = _grid(arr["vertex_grid"], keep)
        ref.max_expanded = float(arr["max_expanded"])
        ref.rho_max = float(arr["rho_max"])
        ref.probe = float(arr["probe"])
        ref.kind = {"ses": 0, "sas": 1, "vdw": 2}[arr.get("kind", "ses")]
        L = LatticeRef()
        L.spacing = float(lat["spacing"])
        L.brick = int(lat["brick"])
        L.frame[:] = [int(v) for v in lat["frame"]]
        L.band = float(lat["band"])
        self.brick = int(lat["brick"])
        err = C.create_string_buffer(1024)
        h = _vp()
        _check(lib().smb_resident_new(device.h, C.byref(ref), C.byref(L), C.byref(h), err, 1024), err)
        self.h = h
        self.n_bricks = 0

    def classify(self):
        err = C.create_string_buffer(1024)
        t, s = _sz(0), _sz(0)
        _check(lib().smb_classify(self.h, C.byref(t), C.byref(s), err, 1024), err)
        self.n_bricks = s.value
        return t.value, s.value

    def bricks(self):
        out = np.zeros((max(self.n_bricks, 1), 3), np.int32)
        rc = lib().smb_resident_bricks(self.h, _p(out, C.c_int32), self.n_bricks)
        if rc != SMB_OK:
            raise SmbError(rc, "smb_resident_bricks")
        return out[:self.n_bricks]

    @property
    def bytes(self):
        return lib().smb_resident_bytes(self.h)

    def close(self):
        if getattr(self, "h", None):
            lib().smb_resident_free(self.h)
            self.h = None

    def __del__(self):
        self.close()


class Batch:
    """Batch buffers (smb_batch_new) and the results of the last run."""

    def __init__(self, resident):
        self.res = resident
        err = C.create_string_buffer(1024)
        h = _vp()
        _check(lib().smb_batch_new(resident.h, C.byref(h), err, 1024), err)
        self.h = h

    def run(self, first=0, count=None):
        if count is None:
            count = self.res.n_bricks - first
        err = C.create_string_buffer(1024)
        t = BatchTimes()
        _check(lib().smb_run(self.res.h, first, count, self.h, C.byref(t), err, 1024), err)
        return dict(substates=t.substates, gather=t.gather, sample=t.sample, mc=t.mc, total=t.total)

    @property
    def n(self):
        return lib().smb_batch_bricks(self.h)

    def records(self):
        out = np.zeros((self.n * 8, REC_WORDS), np.uint32)
        if self.n:
            lib().smb_batch_records(self.h, _p(out, C.c_uint32))
        return out

    def values(self):
        s = self.res.brick + 1
        out = np.zeros((self.n, s * s * s), np.float32)
        if self.n:
            lib().smb_batch_values(self.h, _p(out, C.c_float))
        return out

    def ids(self):
        n = lib().smb_batch_ids_words(self.h)
        out = np.zeros(max(n, 1), np.uint32)
        if n:
            lib().smb_batch_ids(self.h, _p(out, C.c_uint32))
        return out[:n]

    def lists(self, rec, ids):
        """The candidate lists of one sampled sub-block's record."""
        base, n_in, nn, ns, nc, nv, nsb, ncb = (int(rec[k]) for k in (1, 2, 3, 4, 5, 6, 7, 8))
        out = {"n_inside": n_in}
        pos = base
        for key, cnt in (("near", nn), ("s", ns), ("s_off", ns + 1), ("s_blk", nsb), ("c", nc),
                         ("c_off", nc + 1), ("c_blk", ncb), ("v", nv)):
            out[key] = ids[pos:pos + cnt]
            pos += cnt
        return out

    def info(self):
        i = BatchInfo()
        lib().smb_batch_info_get(self.h, C.byref(i))
        return {name: getattr(i, name) for name, _ in i._fields_}

    def count_ops(self):
        err = C.create_string_buffer(1024)
        ops, n = C.c_ulonglong(0), C.c_ulonglong(0)
        _check(lib().smb_batch_count_ops(self.h, C.byref(ops), C.byref(n), err, 1024), err)
        return ops.value, n.value

    def record_features(self, on=True):
        """Later runs' sampling also records each sample's nearest feature
        (the warm start's input; smb_batch_record_features)."""
        _check(lib().smb_batch_record_features(self.h, 1 if on else 0), C.create_string_buffer(8))

    def sample_features(self):
        """The last run's nearest-feature words, (bricks, (b+1)^3) like
        values(); meaningful at samples a sampled sub-block owns."""
        v = np.zeros((self.n, (self.res.brick + 1) ** 3), np.uint32)
        if self.n:
            rc = lib().smb_batch_sample_features(self.h, _p(v, C.c_uint32))
            if rc != SMB_OK:
                raise SmbError(rc, "smb_batch_sample_features")
        return v

    def refine(self, mlp=None, region=None):
        """Fast-mode f32 refinement of the last run's crossing edges on the
        device (smb_refine; smb_refine_warm with an Mlp, which needs a run
        that recorded the features); device ms.  region: per-warp bytes when
        four whole regions do not fit (0: an eighth of the SM's shared
        memory)."""
        err = C.create_string_buffer(1024)
        lib().smb_resident_set_refinement(self.res.h, err, 1024)
        if region is not None:
            if lib().smb_batch_set_refine_region(self.h, int(region)) != SMB_OK:
                raise ValueError("refine region must be 0 or 1 KiB..56 KiB, got %d" % region)
        ms = C.c_double(0)
        if mlp is None:
            _check(lib().smb_refine(self.res.h, self.h, C.byref(ms), err, 1024), err)
        else:
            _check(lib().smb_refine_warm(self.res.h, self.h, mlp.h, C.byref(ms), err, 1024), err)
        return ms.value

    def refine_exact(self, orig, circle_ij, vertex_atoms, t_min, region=None):
        """Exact-mode f64 refinement of the last run's crossing edges on the
        device (smb_resident_set_exact with the attribute tables, then
        smb_refine_exact); device ms."""
        err = C.create_string_buffer(1024)
        orig = np.ascontiguousarray(orig, np.uint32)
        cij = np.ascontiguousarray(circle_ij, np.uint32).reshape(-1)
        va = np.ascontiguousarray(vertex_atoms, np.uint32).reshape(-1)
        _check(lib().smb_resident_set_exact(self.res.h, _p(orig, C.c_uint32), _p(cij, C.c_uint32), len(cij) // 2,
                                            _p(va, C.c_uint32), len(va) // 3, float(t_min), err, 1024), err)
        if region is not None:
            if lib().smb_batch_set_exact_region(self.h, int(region)) != SMB_OK:
                raise ValueError("exact region must be 1 KiB..48 KiB, got %d" % region)
        ms = C.c_double(0)
        _check(lib().smb_refine_exact(self.res.h, self.h, C.byref(ms), err, 1024), err)
        return ms.value

    def vertices(self):
        """Per crossing edge after refine_exact: positions (n, 3), normals
        (n, 3), atoms, patches, t, evaluations (0: left to the host)."""
        ne, nt = _sz(0), _sz(0)
        lib().smb_batch_mc_counts(self.h, C.byref(ne), C.byref(nt))
        n = max(ne.value, 1)
        pos = np.zeros((n, 3), np.float32)
        nrm = np.zeros((n, 3), np.float32)
        atom = np.zeros(n, np.uint32)
        patch = np.zeros(n, np.uint8)
        t = np.zeros(n, np.float32)
        ev = np.zeros(n, np.uint32)
        rc = lib().smb_batch_vertices(self.h, _p(pos, C.c_float), _p(nrm, C.c_float), _p(atom, C.c_uint32),
                                      _p(patch, C.c_uint8), _p(t, C.c_float), _p(ev, C.c_uint32))
        if rc != SMB_OK:
            raise SmbError(rc, "smb_batch_vertices")
        k = ne.value
        return pos[:k], nrm[:k], atom[:k], patch[:k], t[:k], ev[:k]

    def edges(self):
        """Per crossing edge: t, feature, closest point, evaluations (bit 31:
        converged) of the last refinement."""
        ne, nt = _sz(0), _sz(0)
        lib().smb_batch_mc_counts(self.h, C.byref(ne), C.byref(nt))
        n = max(ne.value, 1)
        t = np.zeros(n, np.float32)
        feat = np.zeros(n, np.uint32)
        q = np.zeros((n, 3), np.float32)
        ev = np.zeros(n, np.uint32)
        rc = lib().smb_batch_edges(self.h, _p(t, C.c_float), _p(feat, C.c_uint32), _p(q, C.c_float),
                                   _p(ev, C.c_uint32))
        if rc != SMB_OK:
            raise SmbError(rc, "smb_batch_edges")
        k = ne.value
        return t[:k], feat[:k], q[:k], ev[:k]

    def edge_features(self):
        """Warm-start features (n_edges, 32) and the covered mask."""
        ne, nt = _sz(0), _sz(0)
        lib().smb_batch_mc_counts(self.h, C.byref(ne), C.byref(nt))
        n = max(ne.value, 1)
        x = np.zeros((n, MLP_FEATURES), np.float32)
        cov = np.zeros(n, np.uint8)
        err = C.create_string_buffer(1024)
        lib().smb_resident_set_refinement(self.res.h, err, 1024)
        _check(lib().smb_batch_edge_features(self.res.h, self.h, _p(x, C.c_float), _p(cov, C.c_uint8), err, 1024),
               err)
        return x[:ne.value], cov[:ne.value].astype(bool)

    def mc(self):
        ne, nt = _sz(0), _sz(0)
        lib().smb_batch_mc_counts(self.h, C.byref(ne), C.byref(nt))
        n = self.n
        eo = np.zeros(n + 1, np.uint32)
        to = np.zeros(n + 1, np.uint32)
        edges = np.zeros(max(ne.value, 1), np.uint32)
        vals = np.zeros((max(ne.value, 1), 2), np.float32)
        tris = np.zeros((max(nt.value, 1), 3), np.uint32)
        if n:
            lib().smb_batch_mc(self.h, _p(eo, C.c_uint32), _p(edges, C.c_uint32), _p(vals, C.c_float),
                               _p(to, C.c_uint32), _p(tris, C.c_uint32))
        return dict(edge_off=eo, edges=edges[:ne.value], edge_vals=vals[:ne.value], tri_off=to,
                    tris=tris[:nt.value])

    def close(self):
        if getattr(self, "h", None):
            lib().smb_batch_free(self.h)
            self.h = None

    def __del__(self):
        self.close()


MLP_NPARAM = 6337
MLP_FEATURES = 32


class Mlp:
    """The warm-start MLP on a device (smb_mlp_*)."""

    def __init__(self, device, params):
        self.device = device  # the device must outlive the MLP
        p = np.ascontiguousarray(params, np.float32)
        assert p.size == MLP_NPARAM
        err = C.create_string_buffer(1024)
        h = _vp()
        _check(lib().smb_mlp_new(device.h, _p(p, C.c_float), C.byref(h), err, 1024), err)
        self.h = h

    def set_params(self, params):
        p = np.ascontiguousarray(params, np.float32)
        err = C.create_string_buffer(1024)
        _check(lib().smb_mlp_set_params(self.h, _p(p, C.c_float), err, 1024), err)

    def params(self):
        out = np.zeros(MLP_NPARAM, np.float32)
        lib().smb_mlp_get_params(self.h, _p(out, C.c_float))
        return out

    def set_use(self, use):
        """"gate" (start at t_c where the output is >= 0.5 and both samples
        name t_c's candidate, else the linear guess) or "root" (start at the
        output itself)."""
        if lib().smb_mlp_set_use(self.h, {"gate": 0, "root": 1}[use]) != SMB_OK:
            raise ValueError(use)

    def forward(self, x):
        x = np.ascontiguousarray(x, np.float32).reshape(-1, MLP_FEATURES)
        t = np.zeros(len(x), np.float32)
        err = C.create_string_buffer(1024)
        _check(lib().smb_mlp_forward(self.h, _p(x, C.c_float), len(x), _p(t, C.c_float), err, 1024), err)
        return t

    def gradient(self, x, target):
        x = np.ascontiguousarray(x, np.float32).reshape(-1, MLP_FEATURES)
        y = np.ascontiguousarray(target, np.float32)
        loss = np.zeros(1, np.float32)
        g = np.zeros(MLP_NPARAM, np.float32)
        err = C.create_string_buffer(1024)
        _check(lib().smb_mlp_gradient(self.h, _p(x, C.c_float), _p(y, C.c_float), len(x), _p(loss, C.c_float),
                                      _p(g, C.c_float), err, 1024), err)
        return float(loss[0]), g

    def train_epoch(self, x, target, batch=4096, lr=1e-3):
        x = np.ascontiguousarray(x, np.float32).reshape(-1, MLP_FEATURES)
        y = np.ascontiguousarray(target, np.float32)
        steps = (len(x) + batch - 1) // batch
        losses = np.zeros(steps, np.float32)
        err = C.create_string_buffer(1024)
        _check(lib().smb_mlp_train_epoch(self.h, _p(x, C.c_float), _p(y, C.c_float), len(x), batch, lr,
                                         _p(losses, C.c_float), err, 1024), err)
        return losses

    def close(self):
        if getattr(self, "h", None):
            lib().smb_mlp_free(self.h)
            self.h = None

    def __del__(self):
        self.close()


# ---- seeded synthetic inputs (libsesmesh_synth.so) -------------------------
_SYN = None


def synth():
    global _SYN
    if _SYN is None:
        if not os.path.exists(SYNTH_PATH):
            raise OSError("libsesmesh_synth.so is not built (run `make -C sesmesh_b200`)")
        L = C.CDLL(SYNTH_PATH)
        L.smb_synth_globule.restype = _sz
        L.smb_synth_globule.argtypes = [C.c_uint64, _sz, C.c_double, C.POINTER(C.c_double)]
        L.smb_synth_rings.restype = _sz
        L.smb_synth_rings.argtypes = [C.c_uint64, _sz, C.c_double, C.c_int, C.POINTER(C.c_double),
                                      C.POINTER(C.c_double), C.POINTER(C.c_double), C.POINTER(C.c_double)]
        L.smb_synth_icosahedral.restype = _sz
        L.smb_synth_icosahedral.argtypes = [C.c_uint64, _sz, C.c_double, C.c_double, C.POINTER(C.c_double)]
        _SYN = L
    return _SYN
