"""compute_surface / SurfaceParams / SurfaceEngine over the B200 back end.

The Python face of include/sesmesh_b200_surface.h, shaped like sesmesh's
library API (crates/sesmesh/src/surface.rs:106-241, 599-711) for what the
device path takes: the SES, `refine` exact or fast, `backend` cuda.  Exact
mode gives the CPU back end's mesh and OBJ bytes; fast mode refines edges in
f32 on the device (same triangles, area and volume within 4e-7 relative).
"""
import ctypes as C
from dataclasses import dataclass, replace

import numpy as np

from . import native
from .native import SmbError, _check, _p, lib

REFINE = {"exact": 0, "linear": 1, "fast": 2}
KINDS = {"ses": 0, "sas": 1, "vdw": 2}
QUALITY = {"draft": 1.0, "medium": 0.5, "high": 0.25, "ultra": 0.125}


@dataclass(frozen=True)
class SurfaceParams:
    """SurfaceParams (surface.rs:195-241): surface kind (ses, sas or vdw)
    with probe radius, grid spacing (default Quality::Medium, 0.5 A), refine
    mode, brick edge (default 10), CUDA device, host threads (0 = all)."""
    probe_radius: float = 1.4
    spacing: float = 0.5
    refine: str = "exact"
    brick_size: int = 10
    device: int = 0
    threads: int = 0
    kind: str = "ses"

    @staticmethod
    def ses(probe_radius):
        return SurfaceParams(probe_radius=float(probe_radius))

    @staticmethod
    def sas(probe_radius):
        """SurfaceParams::sas (surface.rs:272-277): the spheres expanded by the probe."""
        return SurfaceParams(probe_radius=float(probe_radius), kind="sas")

    @staticmethod
    def vdw():
        """SurfaceParams::vdw (surface.rs:280-285): the spheres themselves."""
        return SurfaceParams(probe_radius=0.0, kind="vdw")

    def with_spacing(self, h):
        return replace(self, spacing=float(h))

    def with_quality(self, q):
        return replace(self, spacing=QUALITY[q])

    def with_refine(self, mode):
        if mode not in REFINE:
            raise ValueError("refine must be exact, linear or fast")
        return replace(self, refine=mode)

    def with_brick_size(self, b):
        return replace(self, brick_size=int(b))

    def _c(self):
        if self.kind not in KINDS:
            raise SmbError(1, "surface kind must be ses, sas or vdw")
        p = native.SurfaceParams_()
        p.kind = KINDS[self.kind]
        p.probe_radius = float(self.probe_radius)
        p.spacing = float(self.spacing)
        p.brick_size = int(self.brick_size)
        p.refine = REFINE[self.refine]
        p.threads = int(self.threads)
        return p


class _SurfaceHandle:
    """Owns one smb_surface; freed when the output and every array view of
    it are gone."""

    def __init__(self, h, owned):
        self.h = h
        self.owned = owned

    def __del__(self):
        if self.owned and self.h:
            lib().smb_surface_free(self.h)
            self.h = None


class SurfaceOutput:
    """Mesh, statistics (SurfaceStats + stage times in ms) and OBJ text.
    The mesh arrays are read-only views of the library's mesh (no copy) for
    outputs this object owns, copies otherwise."""

    _ARRAYS = (("positions", C.c_float, np.float32, 3), ("normals", C.c_float, np.float32, 3),
               ("triangles", C.c_uint32, np.uint32, 3), ("vertex_atom", C.c_uint32, np.uint32, 0),
               ("vertex_patch", C.c_uint8, np.uint8, 0), ("vertex_component", C.c_uint32, np.uint32, 0))

    def __init__(self, h, owned=True):
        self._keep = _SurfaceHandle(h, owned)
        self._h = h
        self._owned = owned
        st = native.SurfaceStats_()
        lib().smb_surface_stats_get(h, C.byref(st))
        self.stats = {name: getattr(st, name) for name, _ in st._fields_}
        self._arrays = None
        if not owned:
            self._arrays = {k: v.copy() for k, v in self._views().items()}

    def _views(self):
        nv, nt = self.stats["vertices"], self.stats["triangles"]
        ptrs = [C.c_void_p() for _ in self._ARRAYS]
        lib().smb_surface_arrays(self._h, *[C.byref(q) for q in ptrs])
        out = {}
        for (name, ct, dt, width), q in zip(self._ARRAYS, ptrs):
            rows = nt if name == "triangles" else nv
            shape = (rows, width) if width else (rows,)
            n = rows * max(width, 1)
            if not n or not q.value:
                out[name] = np.zeros(shape, dt)
                continue
            buf = (ct * n).from_address(q.value)
            buf.keeper = self._keep  # the mesh lives while any view does
            a = np.frombuffer(buf, dtype=dt).reshape(shape)
            a.flags.writeable = False
            out[name] = a
        return out

    def _array(self, name):
        if self._arrays is None:
            if self._h is None:
                raise ValueError("surface closed")
            self._arrays = self._views()
        return self._arrays[name]

    positions = property(lambda self: self._array("positions"))
    normals = property(lambda self: self._array("normals"))
    triangles = property(lambda self: self._array("triangles"))
    vertex_atom = property(lambda self: self._array("vertex_atom"))
    vertex_patch = property(lambda self: self._array("vertex_patch"))
    vertex_component = property(lambda self: self._array("vertex_component"))

    def obj(self):
        """OBJ bytes with the default options (export/obj.rs:37-73)."""
        n = lib().smb_surface_obj(self._h, None, 0)
        buf = C.create_string_buffer(n)
        lib().smb_surface_obj(self._h, buf, n)
        return buf.raw[:n]

    def write_obj(self, path):
        err = C.create_string_buffer(512)
        _check(lib().smb_surface_write_obj(self._h, path.encode(), err, 512), err)

    def close(self):
        """Drops this object's hold on the mesh (views already taken keep it)."""
        self._h = None
        self._keep = None

    def __del__(self):
        self.close()


STAGES = ("geometry", "classify", "mesh", "assemble", "measure")


class Control:
    """Control (crates/sesmesh/src/control.rs:54-131) plus the device-memory
    guard: cancel() makes a computation under it return SMB_ERR_CANCELLED
    promptly (from any thread); progress(stage, done, total) is called with
    the stage name when a stage starts and ends; max_device_bytes refuses a
    computation whose estimated device bytes exceed it (SMB_ERR_MEMORY), or,
    with auto_coarsen, meshes at the smallest spacing up to 10 A that fits."""

    def __init__(self, progress=None, max_device_bytes=0, auto_coarsen=False):
        self.flag = C.c_int32(0)
        self._user = progress
        self._cb = native.PROGRESS_FN(self._report) if progress else native.PROGRESS_FN()
        self.c = native.Control_()
        self.c.cancel = C.pointer(self.flag)
        self.c.progress = self._cb
        self.c.user = None
        self.c.max_device_bytes = int(max_device_bytes)
        self.c.auto_coarsen = 1 if auto_coarsen else 0

    def _report(self, user, stage, done, total):
        self._user(STAGES[stage] if 0 <= stage < len(STAGES) else stage, int(done), int(total))

    def cancel(self):
        self.flag.value = 1

    def is_cancelled(self):
        return self.flag.value != 0


_DEVICES = {}


def _device(index):
    """Process-wide open devices (backend.rs:163-218 caches them the same way)."""
    if index not in _DEVICES:
        _DEVICES[index] = native.Device(index)
    return _DEVICES[index]


def _spheres(spheres):
    a = np.ascontiguousarray(spheres, np.float64).reshape(-1, 4)
    return a


def compute_surface(spheres, params=SurfaceParams()):
    """compute_surface (surface.rs:599) with Backend::Cuda: spheres as (n, 4)
    rows x, y, z, r."""
    s = _spheres(spheres)
    dev = _device(params.device)
    err = C.create_string_buffer(1024)
    h = C.c_void_p()
    p = params._c()
    _check(lib().smb_compute_surface(dev.h, _p(s, C.c_double), len(s), C.byref(p), C.byref(h), err, 1024), err)
    return SurfaceOutput(h)


def compute_surface_with(spheres, params, control):
    """compute_surface_with (surface.rs:614-631): compute_surface under a
    Control."""
    s = _spheres(spheres)
    dev = _device(params.device)
    err = C.create_string_buffer(1024)
    h = C.c_void_p()
    p = params._c()
    _check(lib().smb_compute_surface_with(dev.h, _p(s, C.c_double), len(s), C.byref(p), C.byref(control.c),
                                          C.byref(h), err, 1024), err)
    return SurfaceOutput(h)


class SurfaceEngine:
    """SurfaceEngine (surface.rs:633-711): arrangement built and uploaded
    once, then meshed (or its device stage run) any number of times."""

    def __init__(self, spheres, params=SurfaceParams(), control=None):
        s = _spheres(spheres)
        self.params = params
        self.dev = _device(params.device)
        self.control = control  # kept alive while the engine uses it
        err = C.create_string_buffer(1024)
        h = C.c_void_p()
        p = params._c()
        _check(lib().smb_engine_new_with(self.dev.h, _p(s, C.c_double), len(s), C.byref(p),
                                         C.byref(control.c) if control is not None else None, C.byref(h), err,
                                         1024), err)
        self.h = h

    def set_control(self, control):
        self.control = control
        lib().smb_engine_set_control(self.h, C.byref(control.c) if control is not None else None)

    def run_device(self):
        """Classification, gather, sampling and marching cubes (and fast-mode
        refinement) on the resident arrangement; device times in ms."""
        err = C.create_string_buffer(1024)
        t = native.BatchTimes()
        _check(lib().smb_engine_run_device(self.h, C.byref(t), err, 1024), err)
        return dict(substates=t.substates, gather=t.gather, sample=t.sample, mc=t.mc, total=t.total)

    @property
    def bricks(self):
        return lib().smb_engine_bricks(self.h)

    def batch_info(self):
        """Sizes and classification time of the last device run."""
        b = lib().smb_engine_batch(self.h)
        i = native.BatchInfo()
        lib().smb_batch_info_get(b, C.byref(i))
        return {name: getattr(i, name) for name, _ in i._fields_}

    def count_exact_ops(self):
        """f64 operations of the last run's exact refinement (its field
        evaluations), counted by re-running it."""
        b = lib().smb_engine_batch(self.h)
        err = C.create_string_buffer(1024)
        ops = C.c_ulonglong(0)
        _check(lib().smb_batch_count_exact_ops(b, C.byref(ops), err, 1024), err)
        return ops.value

    def count_refine_ops(self, mlp=None):
        """f32 operations of the field evaluations of the last run's fast-mode
        refinement (plain, or from the warm start with mlp), counted by
        re-running it."""
        b = lib().smb_engine_batch(self.h)
        err = C.create_string_buffer(1024)
        ops = C.c_ulonglong(0)
        _check(lib().smb_batch_count_refine_ops(b, mlp.h if mlp is not None else None, C.byref(ops), err, 1024),
               err)
        return ops.value

    def count_ops(self):
        """f32 operations and evaluated samples of the last run's sampling pass."""
        b = lib().smb_engine_batch(self.h)
        err = C.create_string_buffer(1024)
        ops, n = C.c_ulonglong(0), C.c_ulonglong(0)
        _check(lib().smb_batch_count_ops(b, C.byref(ops), C.byref(n), err, 1024), err)
        return ops.value, n.value

    def mesh(self):
        err = C.create_string_buffer(1024)
        h = C.c_void_p()
        _check(lib().smb_engine_mesh(self.h, C.byref(h), err, 1024), err)
        return SurfaceOutput(h)

    def field(self, points):
        """The exact f64 SES field at points (n, 3), host threads."""
        p = np.ascontiguousarray(points, np.float64).reshape(-1, 3)
        out = np.zeros(len(p))
        _check(lib().smb_engine_field(self.h, _p(p, C.c_double), len(p), _p(out, C.c_double)),
               C.create_string_buffer(8))
        return out

    def note(self):
        """Why the last mesh was finished on the host ("" when it was not)."""
        return lib().smb_engine_note(self.h).decode()

    def set_exact_on_device(self, on=True):
        """Exact mode: refine vertices in f64 on the device (default) or on
        the host threads (as the reference); the mesh bytes are the same."""
        lib().smb_engine_set_exact_device(self.h, 1 if on else 0)

    def set_warm_start(self, mlp):
        """Start fast-mode refinement from `mlp` (a native.Mlp on this
        engine's device; None: the linear guess)."""
        self.warm = mlp  # kept alive while the engine uses it
        lib().smb_engine_set_warm_start(self.h, mlp.h if mlp is not None else None)

    def warm_start_rows(self):
        """(features (n, 32), exact root parameters (n,), plain f32 root
        parameters (n,), NaN where plain refinement did not converge) for
        every edge the device refines, from a fresh device run."""
        err = C.create_string_buffer(1024)
        n = C.c_size_t(0)
        _check(lib().smb_engine_warm_start_rows(self.h, None, None, None, 0, C.byref(n), err, 1024), err)
        x = np.zeros((max(n.value, 1), native.MLP_FEATURES), np.float32)
        t = np.zeros(max(n.value, 1), np.float32)
        tp = np.zeros(max(n.value, 1), np.float32)
        _check(lib().smb_engine_warm_start_rows(self.h, _p(x, C.c_float), _p(t, C.c_float), _p(tp, C.c_float), len(t),
                                                C.byref(n), err, 1024), err)
        return x[:n.value], t[:n.value], tp[:n.value]

    def close(self):
        self.warm = None
        if getattr(self, "h", None):
            lib().smb_engine_free(self.h)
            self.h = None

    def __del__(self):
        self.close()


def _arrangement_arrays(h):
    info = native.ArrangementInfo()
    lib().smb_engine_arrangement(h, C.byref(info))
    n, nc, nv = info.n_spheres, info.n_circles, info.n_vertices

    def arr(ptr, count, dt):
        if count == 0:
            return np.zeros(0, dt)
        return np.ctypeslib.as_array(ptr, shape=(count,)).astype(dt).copy()

    out = dict(center=arr(info.center, 3 * n, np.float64).reshape(-1, 3),
               expanded=arr(info.expanded, n, np.float64), status=arr(info.status, n, np.uint32),
               orig=arr(info.orig, n, np.uint32), circle=arr(info.circle, 10 * nc, np.float64).reshape(-1, 10),
               circle_ij=arr(info.circle_ij, 2 * nc, np.uint32).reshape(-1, 2),
               vertex=arr(info.vertex, 3 * nv, np.float64).reshape(-1, 3),
               vertex_atoms=arr(info.vertex_atoms, 3 * nv, np.uint32).reshape(-1, 3),
               nb_off=arr(info.nb_off, n + 1, np.uint32), cb_off=arr(info.cb_off, nc + 1, np.uint32),
               n_contained=info.n_contained, max_expanded=info.max_expanded, rho_max=info.rho_max,
               built_on_device=bool(info.built_on_device))
    out["nb_items"] = arr(info.nb_items, int(out["nb_off"][-1]), np.uint32)
    out["cb_items"] = arr(info.cb_items, int(out["cb_off"][-1]), np.uint32)
    return out


def host_arrangement(spheres, params=SurfaceParams(), control=None):
    """The host-built arrangement (no device), as numpy copies."""
    s = _spheres(spheres)
    err = C.create_string_buffer(1024)
    h = C.c_void_p()
    p = params._c()
    _check(lib().smb_arrangement_build_with(_p(s, C.c_double), len(s), C.byref(p),
                                            C.byref(control.c) if control is not None else None, C.byref(h), err,
                                            1024), err)
    try:
        return _arrangement_arrays(h)
    finally:
        lib().smb_engine_free(h)


def set_device_arrangement_min(n):
    """Inputs of at least n spheres get their arrangement built on the
    device (process-wide; 0 = always, None = never)."""
    lib().smb_set_device_arrangement_min(C.c_size_t(2 ** 64 - 1 if n is None else int(n)))


def engine_arrangement(engine):
    """An engine's arrangement (copied from the device when the device built
    it), as numpy copies; built_on_device tells which."""
    return _arrangement_arrays(engine.h)


class MultiBatch:
    """Many structures meshed in one device pass (smb_multi_*): fast mode,
    optionally with the learned warm start, the autotuned brick edge,
    candidate caps and gather block shape unless `config` fixes them.

    `structures` is a list of (spheres, SurfaceParams) pairs."""

    def __init__(self, structures, config=None, warm=None, device=0):
        self.dev = _device(device)
        self._keep = [_spheres(sp) for sp, _ in structures]
        n = len(self._keep)
        ptrs = (C.POINTER(C.c_double) * n)(*[_p(a, C.c_double) for a in self._keep])
        counts = (C.c_size_t * n)(*[len(a) for a in self._keep])
        params = (native.SurfaceParams_ * n)(*[p.with_refine("fast")._c() for _, p in structures])
        cfg = native.MultiConfig(*(config or (0, 0, 0)))
        err = C.create_string_buffer(2048)
        h = C.c_void_p()
        _check(lib().smb_multi_new(self.dev.h, n, ptrs, counts, params, C.byref(cfg), C.byref(h), err, 2048), err)
        self.h = h
        self.n = n
        self.warm = None
        if warm is not None:
            self.set_warm_start(warm)

    def set_warm_start(self, mlp):
        self.warm = mlp  # kept alive while the batch uses it
        lib().smb_multi_set_warm_start(self.h, mlp.h if mlp is not None else None)

    def set_control(self, control):
        """Cancel flag and progress (structures finished) of the runs."""
        self.control = control
        lib().smb_multi_set_control(self.h, C.byref(control.c) if control is not None else None)

    def set_device_finish(self, on=True):
        """Finish each structure on the device (default) or on the host threads."""
        lib().smb_multi_set_device_finish(self.h, 1 if on else 0)

    def tune(self):
        err = C.create_string_buffer(1024)
        _check(lib().smb_multi_tune(self.h, err, 1024), err)
        return self.config()

    def config(self):
        c = native.MultiConfig()
        lib().smb_multi_config_get(self.h, C.byref(c))
        return dict(brick=c.brick, caps_level=c.caps_level, gather_warps=c.gather_warps)

    def run(self):
        """Meshes every structure; returns the run's counts and times (ms)."""
        t = native.MultiTimes()
        err = C.create_string_buffer(2048)
        _check(lib().smb_multi_run(self.h, C.byref(t), err, 2048), err)
        return {name: getattr(t, name) for name, _ in t._fields_}

    def surface(self, i):
        """Structure i's mesh of the last run (valid until the next run)."""
        h = lib().smb_multi_surface(self.h, i)
        if not h:
            raise IndexError(i)
        return SurfaceOutput(C.c_void_p(h), owned=False)

    def latency(self):
        out = np.zeros(self.n, np.float64)
        lib().smb_multi_latency(self.h, _p(out, C.c_double))
        return out

    def close(self):
        if getattr(self, "h", None):
            lib().smb_multi_free(self.h)
            self.h = None
        self.warm = None

    def __del__(self):
        self.close()
