"""ctypes binding of libfold3dpmm.so (the C-ABI declared in include/fold3dpmm.h).

This is the Python host side of the library: it mirrors the C entry points
one to one and adds nothing to the numerics.  Every solve runs in the CUDA
kernels of libfold3dpmm.so; if the library has not been built, loading it
raises instead of falling back to anything else.

Fields are numpy (host) or torch (device) float64 arrays of shape
(nz+2, ny+2, nx+2) in C order, i.e. flat index i + (nx+2)*(j + (ny+2)*k), the
reference's layout (Stencil-OpenACC/AN_ISO_1_OpenACC.c:195).
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
# FOLD3D_LIBRARY may name another build of the same library.
LIB_PATH = os.environ.get("FOLD3D_LIBRARY") or os.path.join(HERE, "libfold3dpmm.so")

OK, ERR_INVALID, ERR_NOMEM, ERR_CUDA, ERR_TIMEOUT, ERR_UNSUPPORTED = range(6)
MAXT = 10e15 * 1.0
X_DOWN, X_UP, K_UP, K_DOWN, Y_UP, Y_DOWN = range(6)
ENGINE_AUTO, ENGINE_PLANES, ENGINE_WAVEFRONT = range(3)

# The reference medium (Stencil-OpenACC/Fold3dPMM.h:49-52).
REF_F = 1.1
REF_A = (-0.35, 0.4, 0.7)

# Every exported symbol of include/fold3dpmm.h and include/fold3d_acc.h.
EXPORTED = (
    "fold3d_last_error", "fold3d_version", "fold3d_default_opts", "fold3d_create", "fold3d_destroy",
    "fold3d_solve", "fold3d_solve_host", "fold3d_plane", "fold3d_init_implicit", "fold3d_init_point",
    "fold3d_exact_time", "fold3d_compat_set_grid", "fold3d_solve_noalloc", "fold3d_compat_plane",
    "fold3d_selftest_wait_timeout", "fold3d_ellip_metric", "fold3d_solve_ellip", "fold3d_solve_batch",
    "fold3d_adjoint_batch", "fold3d_init_implicit_device", "fold3d_write_text", "fold3d_write_vtk",
    "fold3d_write_raw", "fold3d_solve_ellip_f32", "fold3d_solve_ellip_record_f32", "fold3d_adjoint_ellip_f32",
    "fold3d_solve_batch_f32", "fold3d_adjoint_batch_f32",
    "fold3d_solve_ellip_record", "fold3d_adjoint_ellip",
    "fold3d_solve_tti", "fold3d_solve_tti_record", "fold3d_adjoint_tti", "fold3d_solve_batch_tti",
    "fold3d_adjoint_batch_tti", "fold3d_batch_set_config", "fold3d_batch_get_config",
    "InitFoldFromPoint", "ImpSurfF", "ImplicitInitialiser", "InitNode", "updateVoxel", "x", "y", "z",
    "function_x_down", "function_x_up", "function_y_up", "function_y_down", "function_k_up",
    "function_k_down",
    "acc_malloc", "acc_free", "acc_memcpy_to_device", "acc_memcpy_from_device",
)


class Fold3dError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__("fold3d error %d: %s" % (code, msg))
        self.code = code


class Grid(C.Structure):
    _fields_ = [("nx", C.c_int), ("ny", C.c_int), ("nz", C.c_int),
                ("dx", C.c_double), ("dy", C.c_double), ("dz", C.c_double)]


class Medium(C.Structure):
    _fields_ = [("F", C.c_double), ("ax", C.c_double), ("ay", C.c_double), ("az", C.c_double)]


class Ellip(C.Structure):
    _fields_ = [(n, C.c_void_p) for n in ("mxx", "mxy", "mxz", "myy", "myz", "mzz")]


class Instance(C.Structure):
    _fields_ = [("grid", Grid), ("medium", Ellip), ("T", C.c_void_p), ("winners", C.c_void_p)]


class AdjInstance(C.Structure):
    _fields_ = [("grid", Grid), ("medium", Ellip), ("T", C.c_void_p), ("winners", C.c_void_p),
                ("dLdT", C.c_void_p), ("lambda_", C.c_void_p), ("dLdM", C.c_void_p)]


class Tti(C.Structure):
    """fold3d_tti: the FP64 parameter arrays (s, eps, nx, ny) of a tilted
    elliptical medium."""
    _fields_ = [(n, C.c_void_p) for n in ("s", "eps", "nx", "ny")]


class TtiInstance(C.Structure):
    _fields_ = [("grid", Grid), ("medium", Tti), ("T", C.c_void_p), ("winners", C.c_void_p)]


class TtiAdjInstance(C.Structure):
    _fields_ = [("grid", Grid), ("medium", Tti), ("T", C.c_void_p), ("winners", C.c_void_p),
                ("dLdT", C.c_void_p), ("lambda_", C.c_void_p), ("dLdP", C.c_void_p)]


class Opts(C.Structure):
    _fields_ = [("max_sweeps", C.c_int), ("fixed", C.c_int), ("tol", C.c_double),
                ("engine", C.c_int), ("skip", C.c_int), ("variant", C.c_int)]


VARIANT_FAST, VARIANT_LITERAL, VARIANT_COMPACT = 0, 1, 2


class Report(C.Structure):
    _fields_ = [("sweeps", C.c_int), ("max_delta", C.c_double), ("elapsed_ms", C.c_double),
                ("nominal_updates", C.c_uint64), ("evaluated_updates", C.c_uint64),
                ("engine", C.c_int)]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


_lib = None


def lib() -> C.CDLL:
    """Load libfold3dpmm.so (raises if it has not been built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError("libfold3dpmm.so is not built (run __graft_entry__.build() or "
                           "python fgcs-openacc-advanced_b200/build.py)")
    L = C.CDLL(LIB_PATH)
    vp, i, d = C.c_void_p, C.c_int, C.c_double
    P = C.POINTER
    L.fold3d_last_error.restype = C.c_char_p
    L.fold3d_version.restype = C.c_char_p
    L.fold3d_default_opts.argtypes = [P(Opts)]
    L.fold3d_create.argtypes = [P(vp), i]
    L.fold3d_destroy.argtypes = [vp]
    L.fold3d_solve.argtypes = [vp, P(Grid), P(Medium), vp, P(Opts), vp, P(Report)]
    L.fold3d_solve_host.argtypes = [vp, P(Grid), P(Medium), vp, vp, P(Opts), vp, P(Report)]
    L.fold3d_plane.argtypes = [P(Grid), P(Medium), vp, i, i, vp]
    L.fold3d_solve_noalloc.argtypes = [P(Grid), P(Medium), vp, P(Opts), vp, P(Report)]
    L.fold3d_init_implicit.argtypes = [vp, P(Grid), P(Medium)]
    L.fold3d_init_point.argtypes = [vp, P(Grid), i, i, i]
    L.fold3d_exact_time.argtypes = [P(Medium), d, d, d]
    L.fold3d_exact_time.restype = d
    L.fold3d_compat_set_grid.argtypes = [i, i, i]
    L.fold3d_compat_plane.argtypes = [i, vp, i] + [d] * 10
    L.fold3d_selftest_wait_timeout.argtypes = [vp, d]
    L.fold3d_ellip_metric.argtypes = [d, d, d, d, d, C.POINTER(C.c_float)]
    L.fold3d_solve_ellip.argtypes = [vp, P(Grid), P(Ellip), vp, P(Opts), vp, P(Report)]
    L.fold3d_solve_batch.argtypes = [vp, i, P(Instance), P(Opts), vp, P(Report)]
    L.fold3d_adjoint_batch.argtypes = [vp, i, P(AdjInstance), i, d, i, vp, P(Report)]
    L.fold3d_init_implicit_device.argtypes = [vp, P(Grid), P(Medium), vp, vp]
    for name in ("fold3d_write_text", "fold3d_write_raw"):
        getattr(L, name).argtypes = [C.c_char_p, vp, P(Grid)]
    L.fold3d_write_vtk.argtypes = [C.c_char_p, vp, P(Grid), i]
    L.fold3d_solve_ellip_record.argtypes = [vp, P(Grid), P(Ellip), vp, vp, P(Opts), vp, P(Report)]
    L.fold3d_adjoint_ellip.argtypes = [vp, P(Grid), P(Ellip), vp, vp, vp, vp, vp, i, C.c_double, vp, P(Report)]
    L.InitFoldFromPoint.argtypes = [d] * 7
    L.InitFoldFromPoint.restype = d
    L.ImpSurfF.argtypes = [d] * 3
    L.ImpSurfF.restype = d
    L.ImplicitInitialiser.argtypes = [vp, i, i, i, d, d, d]
    L.InitNode.argtypes = [d, d, d, i, i, i, vp]
    L.updateVoxel.argtypes = [vp, i, i, i, d, d, d, d, d, d]
    for n in ("x", "y", "z"):
        getattr(L, n).argtypes = [i, d]
        getattr(L, n).restype = d
    for n in ("function_x_down", "function_x_up", "function_y_up", "function_y_down",
              "function_k_up", "function_k_down"):
        getattr(L, n).argtypes = [vp, i] + [d] * 10
    L.acc_malloc.argtypes = [C.c_size_t]
    L.acc_malloc.restype = vp
    L.acc_free.argtypes = [vp]
    L.acc_memcpy_to_device.argtypes = [vp, vp, C.c_size_t]
    L.acc_memcpy_from_device.argtypes = [vp, vp, C.c_size_t]
    L.fold3d_batch_set_config.argtypes = [vp, i, i]
    L.fold3d_batch_get_config.argtypes = [vp, P(i), P(i)]
    L.fold3d_solve_tti.argtypes = [vp, P(Grid), P(Tti), vp, P(Opts), vp, P(Report)]
    L.fold3d_solve_tti_record.argtypes = [vp, P(Grid), P(Tti), vp, vp, P(Opts), vp, P(Report)]
    L.fold3d_adjoint_tti.argtypes = [vp, P(Grid), P(Tti), vp, vp, vp, vp, vp, i, C.c_double, vp, P(Report)]
    L.fold3d_solve_batch_tti.argtypes = [vp, i, P(TtiInstance), P(Opts), vp, P(Report)]
    L.fold3d_adjoint_batch_tti.argtypes = [vp, i, P(TtiAdjInstance), i, d, i, vp, P(Report)]
    # the float32 build takes the same arguments (float fields)
    L.fold3d_solve_ellip_f32.argtypes = list(L.fold3d_solve_ellip.argtypes)
    L.fold3d_solve_ellip_record_f32.argtypes = list(L.fold3d_solve_ellip_record.argtypes)
    L.fold3d_adjoint_ellip_f32.argtypes = list(L.fold3d_adjoint_ellip.argtypes)
    L.fold3d_solve_batch_f32.argtypes = list(L.fold3d_solve_batch.argtypes)
    L.fold3d_adjoint_batch_f32.argtypes = list(L.fold3d_adjoint_batch.argtypes)
    _lib = L
    return L


def last_error() -> str:
    return lib().fold3d_last_error().decode()


def _check(rc: int):
    if rc != OK:
        raise Fold3dError(rc, last_error())


def version() -> str:
    return lib().fold3d_version().decode()


def grid(nx, ny, nz, h) -> Grid:
    if not hasattr(h, "__len__"):
        h = (h, h, h)
    return Grid(int(nx), int(ny), int(nz), float(h[0]), float(h[1]), float(h[2]))


def medium(F=REF_F, a=REF_A) -> Medium:
    return Medium(float(F), float(a[0]), float(a[1]), float(a[2]))


def opts(max_sweeps=1000, fixed=False, tol=0.0, engine=ENGINE_AUTO, skip=True, variant=VARIANT_FAST) -> Opts:
    o = Opts()
    lib().fold3d_default_opts(C.byref(o))
    o.max_sweeps, o.fixed, o.tol, o.engine, o.skip = int(max_sweeps), int(bool(fixed)), float(tol), \
        int(engine), int(bool(skip))
    o.variant = int(variant)
    return o


def grid_of(T) -> tuple:
    nz, ny, nx = (int(s) - 2 for s in T.shape)
    return nx, ny, nz


def _host_ptr(a: np.ndarray):
    if a.dtype != np.float64 or not a.flags.c_contiguous:
        raise ValueError("field must be a C-contiguous float64 array")
    return a.ctypes.data_as(C.c_void_p)


def _any_host_ptr(a):
    if isinstance(a, np.ndarray):
        return _host_ptr(a)
    import torch

    if a.dtype != torch.float64 or not a.is_contiguous() or a.is_cuda:
        raise ValueError("host field must be a contiguous float64 CPU tensor")
    return C.c_void_p(a.data_ptr())


def _dev_ptr(t):
    import torch

    if t.dtype != torch.float64 or not t.is_contiguous() or not t.is_cuda:
        raise ValueError("device field must be a contiguous float64 CUDA tensor")
    return C.c_void_p(t.data_ptr())


def init_implicit(nx, ny, nz, h, med: Medium | None = None, out: np.ndarray | None = None) -> np.ndarray:
    """Host field initialised from the reference's implicit surface (into
    `out`, a float64 array of the field's shape, when given)."""
    if out is not None and out.shape != (nz + 2, ny + 2, nx + 2):
        raise ValueError("out must have the field's shape")
    T = np.empty((nz + 2, ny + 2, nx + 2), dtype=np.float64) if out is None else out
    _check(lib().fold3d_init_implicit(_host_ptr(T), C.byref(grid(nx, ny, nz, h)),
                                      C.byref(med or medium())))
    return T


def init_implicit_device(ctx: "Context", T, h, med: Medium | None = None, stream=None):
    """fold3d_init_implicit_device: the implicit-surface initialiser into the
    device field T (float64 CUDA tensor, field layout)."""
    nx, ny, nz = grid_of(T)
    _on_context(ctx, T)
    _check(lib().fold3d_init_implicit_device(ctx._h, C.byref(grid(nx, ny, nz, h)), C.byref(med or medium()),
                                             _dev_ptr(T), C.c_void_p(stream) if stream else None))


def write_text(path, T: np.ndarray, h):
    """fold3d_write_text: the reference's %f dump of a host field."""
    nx, ny, nz = grid_of(T)
    _check(lib().fold3d_write_text(os.fsencode(path), _host_ptr(T), C.byref(grid(nx, ny, nz, h))))


def write_vtk(path, T: np.ndarray, h, ghosts=False):
    """fold3d_write_vtk: legacy VTK structured points (binary)."""
    nx, ny, nz = grid_of(T)
    _check(lib().fold3d_write_vtk(os.fsencode(path), _host_ptr(T), C.byref(grid(nx, ny, nz, h)), int(bool(ghosts))))


def write_raw(path, T: np.ndarray, h):
    """fold3d_write_raw: 64-byte header and the whole field."""
    nx, ny, nz = grid_of(T)
    _check(lib().fold3d_write_raw(os.fsencode(path), _host_ptr(T), C.byref(grid(nx, ny, nz, h))))


def read_raw(path):
    """A file of fold3d_write_raw: (field, (dx, dy, dz))."""
    with open(path, "rb") as f:
        head = f.read(64)
        if head[:8] != b"FOLD3DRW":
            raise ValueError("not a fold3d raw file")
        ver, nx, ny, nz = np.frombuffer(head[8:24], dtype="<i4")
        h = tuple(float(v) for v in np.frombuffer(head[24:48], dtype="<f8"))
        T = np.fromfile(f, dtype="<f8").reshape(nz + 2, ny + 2, nx + 2)
    return T, h


def init_point(nx, ny, nz, src) -> np.ndarray:
    T = np.empty((nz + 2, ny + 2, nx + 2), dtype=np.float64)
    _check(lib().fold3d_init_point(_host_ptr(T), C.byref(grid(nx, ny, nz, 1.0)), *map(int, src)))
    return T


def exact_time(med: Medium, x, y, z) -> float:
    return lib().fold3d_exact_time(C.byref(med), float(x), float(y), float(z))


class Context:
    """A fold3d_ctx on one device."""

    def __init__(self, device: int = 0):
        self._h = C.c_void_p()
        self.device = int(device)
        _check(lib().fold3d_create(C.byref(self._h), self.device))

    def close(self):
        if self._h:
            lib().fold3d_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def solve(self, T, h, med: Medium | None = None, o: Opts | None = None, stream=None,
              out=None) -> Report:
        """Solve in place.  T: float64 CUDA tensor (device path), or a host
        array -- numpy, or a (pinned) CPU torch tensor -- for the host path,
        which copies in and out inside the call; `out` then receives the
        result (default: T itself)."""
        nx, ny, nz = grid_of(T)
        g = grid(nx, ny, nz, h)
        rep = Report()
        o = o or opts()
        med = med or medium()
        s = C.c_void_p(stream) if stream else None
        if isinstance(T, np.ndarray) or not T.is_cuda:
            src = _any_host_ptr(T)
            if out is not None and tuple(out.shape) != tuple(T.shape):  # the library writes a whole field
                raise ValueError("out must have the field's shape %s, got %s" % (tuple(T.shape), tuple(out.shape)))
            dst = _any_host_ptr(out) if out is not None else src
            _check(lib().fold3d_solve_host(self._h, C.byref(g), C.byref(med), src, dst, C.byref(o), s,
                                           C.byref(rep)))
        else:
            _on_context(self, T)
            _check(lib().fold3d_solve(self._h, C.byref(g), C.byref(med), _dev_ptr(T), C.byref(o), s,
                                      C.byref(rep)))
        return rep


def ellip_metric(vz, eps, axis):
    """The six float metric entries (xx, xy, xz, yy, yz, zz) of a tilted
    elliptical cell (fold3d_ellip_metric)."""
    out = (C.c_float * 6)()
    lib().fold3d_ellip_metric(float(vz), float(eps), float(axis[0]), float(axis[1]), float(axis[2]), out)
    return list(out)


def ellip(M, like=None):
    """fold3d_ellip from six contiguous float32 CUDA tensors (xx xy xz yy yz
    zz).  like: the field they go with; every array must then have its shape
    and device, since the kernels read the metric at the field's indices and
    the library cannot check the size behind a pointer."""
    import torch

    if len(M) != 6:
        raise ValueError("a metric is six arrays (xx xy xz yy yz zz), got %d" % len(M))
    for m in M:
        if like is not None and (tuple(m.shape) != tuple(like.shape) or m.device != like.device):
            raise ValueError("metric arrays must have the field's shape %s and device %s, got %s on %s"
                             % (tuple(like.shape), like.device, tuple(m.shape), m.device))
        if m.dtype != torch.float32 or not m.is_cuda or not m.is_contiguous():
            raise ValueError("metric arrays must be contiguous float32 CUDA tensors")
    return Ellip(*(C.c_void_p(m.data_ptr()) for m in M))


def tti(P, like=None):
    """fold3d_tti from four contiguous float64 CUDA tensors (slowness,
    epsilon, axis x and y components), each shaped like the field `like`."""
    import torch

    if len(P) != 4:
        raise ValueError("a parameter medium is four arrays (s, eps, nx, ny), got %d" % len(P))
    for m in P:
        if like is not None and (tuple(m.shape) != tuple(like.shape) or m.device != like.device):
            raise ValueError("medium arrays must have the field's shape %s and device %s, got %s on %s"
                             % (tuple(like.shape), like.device, tuple(m.shape), m.device))
        if m.dtype != torch.float64 or not m.is_cuda or not m.is_contiguous():
            raise ValueError("parameter arrays must be contiguous float64 CUDA tensors")
    return Tti(*(C.c_void_p(m.data_ptr()) for m in P))


def is_tti(M) -> bool:
    """A medium given as four FP64 parameter arrays (else six float32 metric
    arrays)."""
    return len(M) == 4


def _medium_arg(M, T):
    """(struct, entry-point suffix, gradient arrays) of a medium: the six
    float32 metric arrays (fold3d_*_ellip) or the four FP64 parameter arrays
    (fold3d_*_tti, float64 fields only: the library cannot see a field's type
    behind its pointer)."""
    if is_tti(M):
        import torch

        if T.dtype != torch.float64:
            raise ValueError("the FP64 parameter medium needs a float64 field")
        return tti(M, T), "tti", 4
    return ellip(M, T), "ellip", 6


def _on_context(ctx, T, name="field"):
    """T must live on the context's device."""
    if getattr(T, "is_cuda", False) and T.device.index != ctx.device:
        raise ValueError("%s is on %s but the context is on cuda:%d" % (name, T.device, ctx.device))


def _same_length(**lists):
    n = {k: len(v) for k, v in lists.items()}
    if len(set(n.values())) > 1:
        raise ValueError("batch lists differ in length: %s" % n)


NOALLOC_MAX_SWEEPS = 4096


def solve_noalloc(T, h, med: Medium | None = None, o: Opts | None = None, stream=None) -> Report:
    """fold3d_solve_noalloc on a float64 CUDA tensor, in place: the solve
    entry point that allocates no memory (see include/fold3dpmm.h)."""
    nx, ny, nz = grid_of(T)
    rep = Report()
    _check(lib().fold3d_solve_noalloc(C.byref(grid(nx, ny, nz, h)), C.byref(med or medium()), _dev_ptr(T),
                                      C.byref(o or opts()), C.c_void_p(stream) if stream else None,
                                      C.byref(rep)))
    return rep


def _field_ptr(t):
    """A float64 or float32 device field: (pointer, float32?)."""
    import torch

    if t.dtype not in (torch.float64, torch.float32) or not t.is_contiguous() or not t.is_cuda:
        raise ValueError("device field must be a contiguous float64 or float32 CUDA tensor")
    return C.c_void_p(t.data_ptr()), t.dtype == torch.float32


def _entry(name, f32):
    return getattr(lib(), name + ("_f32" if f32 else ""))


def solve_ellip(ctx: "Context", T, h, M, o: Opts | None = None, stream=None) -> Report:
    """Solve in place on a float64 (or float32: the float32 build) CUDA
    tensor with an elliptical medium M: six float32 CUDA metric tensors in
    the field layout (fold3d_solve_ellip), or four float64 parameter tensors
    s, eps, nx, ny (fold3d_solve_tti, float64 fields only)."""
    nx, ny, nz = grid_of(T)
    rep = Report()
    e, kind, _ = _medium_arg(M, T)
    ptr, f32 = _field_ptr(T)
    _on_context(ctx, T)
    fn = lib().fold3d_solve_tti if kind == "tti" else _entry("fold3d_solve_ellip", f32)
    _check(fn(ctx._h, C.byref(grid(nx, ny, nz, h)), C.byref(e), ptr, C.byref(o or opts()),
              C.c_void_p(stream) if stream else None, C.byref(rep)))
    return rep


def _check_like(name, X, T, itemsize=None, lead=()):
    """X must be a contiguous CUDA tensor of shape lead + T.shape with
    itemsize-byte elements (the library writes that many bytes); itemsize
    None: of T's dtype (a field-typed array)."""
    ok = X.is_cuda and X.is_contiguous() and tuple(X.shape) == tuple(lead) + tuple(T.shape)
    ok = ok and (X.dtype == T.dtype if itemsize is None else X.element_size() == itemsize)
    if not ok:
        raise ValueError("%s: need a contiguous CUDA tensor of shape %s and %s" % (
            name, tuple(lead) + tuple(T.shape), T.dtype if itemsize is None else "%d-byte elements" % itemsize))


def solve_ellip_record(ctx: "Context", T, h, M, W, o: Opts | None = None, stream=None) -> Report:
    """solve_ellip that also fills W (a uint8 CUDA tensor shaped like T) with
    each cell's winner record (the adjoint's checkpoint): direction * 33 +
    candidate id, 0xff where no candidate set the cell's time."""
    _check_like("W", W, T, 1)
    nx, ny, nz = grid_of(T)
    rep = Report()
    ptr, f32 = _field_ptr(T)
    _on_context(ctx, T)
    e, kind, _ = _medium_arg(M, T)
    fn = lib().fold3d_solve_tti_record if kind == "tti" else _entry("fold3d_solve_ellip_record", f32)
    _check(fn(ctx._h, C.byref(grid(nx, ny, nz, h)), C.byref(e), ptr, C.c_void_p(W.data_ptr()), C.byref(o or opts()),
              C.c_void_p(stream) if stream else None, C.byref(rep)))
    return rep


def adjoint_ellip(ctx: "Context", T, h, M, W, dLdT, lam, dLdM, max_sweeps=1000, tol=0.0, stream=None) -> Report:
    """fold3d_adjoint_ellip(_f32): lam <- dL/dT (total), dLdM (shape
    (6,)+T.shape) <- dL/dM, from the converged T, its winner record W and
    dLdT (all of T's dtype).  With a parameter medium (four arrays,
    fold3d_adjoint_tti) dLdM has shape (4,)+T.shape and receives dL/ds,
    dL/deps, dL/dnx and dL/dny.  Backward sweeps stop once one pushes at most
    tol times the first sweep's largest push (tol 0: once one pushes
    nothing)."""
    _check_like("W", W, T, 1)
    _check_like("dLdT", dLdT, T)
    _check_like("lam", lam, T)
    e, kind, ng = _medium_arg(M, T)
    _check_like("dLdM", dLdM, T, lead=(ng,))
    nx, ny, nz = grid_of(T)
    rep = Report()
    ptr, f32 = _field_ptr(T)
    _on_context(ctx, T)
    fn = lib().fold3d_adjoint_tti if kind == "tti" else _entry("fold3d_adjoint_ellip", f32)
    _check(fn(ctx._h, C.byref(grid(nx, ny, nz, h)), C.byref(e), ptr, C.c_void_p(W.data_ptr()),
              C.c_void_p(dLdT.data_ptr()), C.c_void_p(lam.data_ptr()), C.c_void_p(dLdM.data_ptr()), int(max_sweeps),
              float(tol), C.c_void_p(stream) if stream else None, C.byref(rep)))
    return rep


def solve_batch(ctx: "Context", fields, hs, media, o: Opts | None = None, stream=None, winners=None) -> list:
    """fold3d_solve_batch: fields[i] (float64 CUDA tensors, in place), hs[i]
    spacings, media[i] six float32 CUDA metric tensors, winners[i] (optional)
    uint8 winner records shaped like fields[i].  Returns the per-instance
    reports."""
    n = len(fields)
    _same_length(fields=fields, hs=hs, media=media, **({} if winners is None else {"winners": winners}))
    tti_batch = n > 0 and is_tti(media[0])
    if any(is_tti(M) != tti_batch for M in media):
        raise ValueError("a batch's media are all metric arrays or all parameter arrays")
    arr = ((TtiInstance if tti_batch else Instance) * n)()
    kinds = set()
    for i, (T, h, M) in enumerate(zip(fields, hs, media)):
        nx, ny, nz = grid_of(T)
        arr[i].grid = grid(nx, ny, nz, h)
        arr[i].medium = _medium_arg(M, T)[0]
        arr[i].T, f32 = _field_ptr(T)
        _on_context(ctx, T, "fields[%d]" % i)
        kinds.add(f32)
        if winners is not None and winners[i] is not None:
            _check_like("winners[%d]" % i, winners[i], T, 1)
            arr[i].winners = winners[i].data_ptr()
    if len(kinds) > 1:
        raise ValueError("a batch is all float64 or all float32")
    reps = (Report * n)()
    fn = lib().fold3d_solve_batch_tti if tti_batch else _entry("fold3d_solve_batch", kinds.pop())
    _check(fn(ctx._h, n, arr, C.byref(o or opts()), C.c_void_p(stream) if stream else None, reps))
    return list(reps)


def adjoint_batch(ctx: "Context", fields, hs, media, winners, dLdT, lam, dLdM, max_sweeps=1000, tol=0.0,
                  accumulate=False, stream=None) -> list:
    """fold3d_adjoint_batch: per instance i the arguments of adjoint_ellip
    (fields[i] converged, winners[i] its record, dLdT[i], lam[i], dLdM[i]).
    accumulate: dLdM[i] += the gradient (instances may share one dLdM).
    Returns the per-instance reports."""
    n = len(fields)
    _same_length(fields=fields, hs=hs, media=media, winners=winners, dLdT=dLdT, lam=lam, dLdM=dLdM)
    tti_batch = n > 0 and is_tti(media[0])
    if any(is_tti(M) != tti_batch for M in media):
        raise ValueError("a batch's media are all metric arrays or all parameter arrays")
    arr = ((TtiAdjInstance if tti_batch else AdjInstance) * n)()
    kinds = set()
    for i, (T, h, M) in enumerate(zip(fields, hs, media)):
        _check_like("winners[%d]" % i, winners[i], T, 1)
        _check_like("dLdT[%d]" % i, dLdT[i], T)
        _check_like("lam[%d]" % i, lam[i], T)
        _check_like("dLdM[%d]" % i, dLdM[i], T, lead=(4 if tti_batch else 6,))
        nx, ny, nz = grid_of(T)
        arr[i].grid = grid(nx, ny, nz, h)
        arr[i].medium = _medium_arg(M, T)[0]
        arr[i].T, f32 = _field_ptr(T)
        _on_context(ctx, T, "fields[%d]" % i)
        kinds.add(f32)
        arr[i].winners = winners[i].data_ptr()
        arr[i].dLdT = dLdT[i].data_ptr()
        arr[i].lambda_ = lam[i].data_ptr()
        if tti_batch:
            arr[i].dLdP = dLdM[i].data_ptr()
        else:
            arr[i].dLdM = dLdM[i].data_ptr()
    if len(kinds) > 1:
        raise ValueError("a batch is all float64 or all float32")
    reps = (Report * n)()
    fn = lib().fold3d_adjoint_batch_tti if tti_batch else _entry("fold3d_adjoint_batch", kinds.pop())
    _check(fn(ctx._h, n, arr, int(max_sweeps), float(tol), int(bool(accumulate)),
              C.c_void_p(stream) if stream else None, reps))
    return list(reps)


def batch_set_config(ctx: "Context", tile_rows=0, ctas_per_sm=0):
    """fold3d_batch_set_config: fix the batched solves' tile height (2, 4 or
    8 rows) and resident CTAs per SM, or 0 to let the autotuner choose."""
    _check(lib().fold3d_batch_set_config(ctx._h, int(tile_rows), int(ctas_per_sm)))


def batch_get_config(ctx: "Context"):
    """(tile rows, CTAs per SM) of the last batched solve on ctx."""
    a, b = C.c_int(), C.c_int()
    _check(lib().fold3d_batch_get_config(ctx._h, C.byref(a), C.byref(b)))
    return a.value, b.value


def plane(T, h, dir_, src, med: Medium | None = None, stream=None):
    """One plane step on a device field (asynchronous on stream)."""
    nx, ny, nz = grid_of(T)
    _check(lib().fold3d_plane(C.byref(grid(nx, ny, nz, h)), C.byref(med or medium()), _dev_ptr(T),
                              int(dir_), int(src), C.c_void_p(stream) if stream else None))
