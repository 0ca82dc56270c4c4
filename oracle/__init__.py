"""CPU oracle for the Fold3dPMM plane sweep -- TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py`` (its
``cpu_baseline`` leg and ``--impl reference``) may import this package, and
only to check results or as the timed CPU baseline; the product library
never does.

Two oracles live here:

* :class:`Oracle` wraps ``liboracle.so``, this repository's plain-C
  restatement of the reference's single-device path (run-time sizes,
  non-cubic grids, run-time medium).
* :class:`RefLib` wraps ``_ref/n<N>/libref[_omp].so``, the reference's own
  ``AN_ISO_1_OpenACC.c`` + ``Fold3dPMM.c`` compiled for the host at a fixed
  cubic size N, driven plane by plane in the order and with the arguments of
  the reference's ``main`` (``Stencil-OpenACC/AN_ISO_1_OpenACC.c:1195-1236``).

Arrays are numpy float64 of shape (nz+2, ny+2, nx+2) in C order, so the flat
index is ``i + (nx+2)*(j + (ny+2)*k)`` as in the reference.
"""
from __future__ import annotations

import ctypes as C
import math
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

# Reference medium and source constants (Fold3dPMM.h:6, :49-52).
MAXT = 10e15 * 1.0
REF_F = 1.1
REF_A = (-0.35, 0.4, 0.7)

_dbl = C.c_double
_int = C.c_int
_ptr = C.c_void_p


def ref_spacing(n: int) -> float:
    """Grid spacing of the reference driver, h = (10 - 0) / (n - 1.0)
    (AN_ISO_1_OpenACC.c:1154-1156)."""
    return (10.0 - 0.0) / (n - 1.0)


def empty_field(nx: int, ny: int, nz: int) -> np.ndarray:
    return np.empty((nz + 2, ny + 2, nx + 2), dtype=np.float64)


def _p(a: np.ndarray):
    assert a.dtype == np.float64 and a.flags.c_contiguous
    return a.ctypes.data_as(_ptr)


class Oracle:
    """ctypes wrapper of liboracle.so (oracle/fold3d_oracle.c)."""

    def __init__(self, path: str | None = None):
        if path is None:
            path = os.path.join(HERE, "liboracle.so")
            if not os.path.exists(path):
                from . import build

                build.build_oracle()
        L = C.CDLL(path)
        L.orc_plane.argtypes = [_ptr, _int, _int, _int, _dbl, _dbl, _dbl, _dbl, _dbl, _dbl, _dbl, _int, _int]
        L.orc_pass.argtypes = [_ptr, _int, _int, _int, _dbl, _dbl, _dbl, _dbl, _dbl, _dbl, _dbl, _int]
        L.orc_solve.argtypes = [_ptr, _int, _int, _int, _dbl, _dbl, _dbl, _dbl, _dbl, _dbl, _dbl, _int, _dbl,
                                C.POINTER(_dbl)]
        L.orc_solve.restype = _int
        L.orc_init_implicit.argtypes = [_ptr, _int, _int, _int, _dbl, _dbl, _dbl, _dbl, _dbl, _dbl, _dbl]
        L.orc_init_implicit.restype = _int
        L.orc_init_point.argtypes = [_ptr, _int, _int, _int, _int, _int, _int]
        L.orc_fold_from_point.argtypes = [_dbl] * 7
        L.orc_fold_from_point.restype = _dbl
        L.orc_surface.argtypes = [_dbl] * 3
        L.orc_surface.restype = _dbl
        L.orc_last_overfull.restype = C.c_long
        L.orc_ell_solve.argtypes = [_ptr, C.POINTER(C.c_void_p), _int, _int, _int, _dbl, _dbl, _dbl, _int, _dbl,
                                    C.POINTER(_dbl)]
        L.orc_ell_solve.restype = _int
        L.orc_ell_plane.argtypes = [_ptr, C.POINTER(C.c_void_p), _int, _int, _int, _dbl, _dbl, _dbl, _int, _int]
        L.orc_ell_solve_rec.argtypes = [_ptr, C.POINTER(C.c_void_p), _ptr, _int, _int, _int, _dbl, _dbl, _dbl, _int,
                                        _dbl, C.POINTER(_dbl)]
        L.orc_ell_solve_rec.restype = _int
        L.orc_ellf_solve_rec.argtypes = list(L.orc_ell_solve_rec.argtypes)
        L.orc_ellf_solve_rec.restype = _int
        L.orc_ellf_plane_rec.argtypes = [_ptr, C.POINTER(C.c_void_p), _ptr, _int, _int, _int, _dbl, _dbl, _dbl, _int,
                                         _int]
        L.orc_ell_adjoint_rec.argtypes = [_ptr, C.POINTER(C.c_void_p), _ptr, _int, _int, _int, _dbl, _dbl, _dbl, _ptr,
                                          _ptr, _ptr]
        L.orc_ell_adjoint_rec.restype = C.c_long
        L.orc_tti_metric.argtypes = [_ptr, _ptr, _ptr, _ptr, C.c_int64, C.POINTER(C.c_void_p)]
        L.orc_ell_plane_d.argtypes = list(L.orc_ell_plane.argtypes)
        L.orc_ell_solve_rec_d.argtypes = list(L.orc_ell_solve_rec.argtypes)
        L.orc_ell_solve_rec_d.restype = _int
        L.orc_ell_adjoint_rec_d.argtypes = list(L.orc_ell_adjoint_rec.argtypes)
        L.orc_ell_adjoint_rec_d.restype = C.c_long
        self.L = L

    @staticmethod
    def _dims(T):
        nz, ny, nx = (s - 2 for s in T.shape)
        return nx, ny, nz

    def init_implicit(self, nx, ny, nz, h, F=REF_F, a=REF_A) -> np.ndarray:
        T = empty_field(nx, ny, nz)
        rc = self.L.orc_init_implicit(_p(T), nx, ny, nz, h[0], h[1], h[2], F, *a)
        if rc != 0:
            raise MemoryError("orc_init_implicit failed")
        return T

    def init_point(self, nx, ny, nz, src) -> np.ndarray:
        T = empty_field(nx, ny, nz)
        self.L.orc_init_point(_p(T), nx, ny, nz, *src)
        return T

    def plane(self, T, h, dir_, src, F=REF_F, a=REF_A):
        self.L.orc_plane(_p(T), *self._dims(T), h[0], h[1], h[2], F, *a, dir_, src)

    def pass_(self, T, h, dir_, F=REF_F, a=REF_A):
        self.L.orc_pass(_p(T), *self._dims(T), h[0], h[1], h[2], F, *a, dir_)

    def solve(self, T, h, nsweeps, tol=-1.0, F=REF_F, a=REF_A):
        """In place.  Returns (sweeps_run, max|dT| of the last sweep)."""
        d = _dbl(0.0)
        s = self.L.orc_solve(_p(T), *self._dims(T), h[0], h[1], h[2], F, *a, nsweeps, tol, C.byref(d))
        if s < 0:
            raise MemoryError("orc_solve failed")
        return s, d.value

    @staticmethod
    def _metric(M):
        arrs = [np.ascontiguousarray(m, dtype=np.float32) for m in M]
        ptrs = (C.c_void_p * 6)(*(a.ctypes.data for a in arrs))
        return arrs, ptrs

    def ell_solve(self, T, M, h, nsweeps, tol=-1.0):
        """Elliptical medium (six float32 metric arrays, field layout), in
        place.  Returns (sweeps_run, max|dT| of the last sweep)."""
        arrs, ptrs = self._metric(M)
        d = _dbl(0.0)
        s = self.L.orc_ell_solve(_p(T), ptrs, *self._dims(T), h[0], h[1], h[2], nsweeps, tol, C.byref(d))
        if s < 0:
            raise MemoryError("orc_ell_solve failed")
        return s, d.value

    def ell_solve_rec(self, T, M, h, nsweeps, tol=-1.0):
        """ell_solve that also returns the winner record (uint8, field layout:
        direction * 33 + candidate id, 0xff where no candidate set the value)."""
        arrs, ptrs = self._metric(M)
        W = np.full(T.shape, 0xFF, dtype=np.uint8)
        d = _dbl(0.0)
        s = self.L.orc_ell_solve_rec(_p(T), ptrs, W.ctypes.data_as(_ptr), *self._dims(T), h[0], h[1], h[2], nsweeps,
                                     tol, C.byref(d))
        return s, d.value, W

    def ellf_solve_rec(self, T, M, h, nsweeps, tol=-1.0):
        """The float32 build (T: float32 field, in place): (sweeps, last
        change, winner record)."""
        if T.dtype != np.float32 or not T.flags.c_contiguous:
            raise ValueError("need a contiguous float32 field")
        arrs, ptrs = self._metric(M)
        W = np.full(T.shape, 0xFF, dtype=np.uint8)
        d = _dbl(0.0)
        s = self.L.orc_ellf_solve_rec(T.ctypes.data_as(_ptr), ptrs, W.ctypes.data_as(_ptr), *self._dims(T), h[0], h[1],
                                      h[2], nsweeps, tol, C.byref(d))
        return s, d.value, W

    def ell_adjoint(self, T, M, h, W, r):
        """FP64 adjoint from the winner record: (lambda, dL/dM (6, ...),
        number of non-causal weights)."""
        arrs, ptrs = self._metric(M)
        lam = np.zeros_like(T)
        g = np.zeros((6,) + T.shape)
        r = np.ascontiguousarray(r, dtype=np.float64)
        Wc = np.ascontiguousarray(W, dtype=np.uint8)
        nc = self.L.orc_ell_adjoint_rec(_p(T), ptrs, Wc.ctypes.data_as(_ptr), *self._dims(T), h[0], h[1], h[2],
                                        r.ctypes.data_as(_ptr), lam.ctypes.data_as(_ptr), g.ctypes.data_as(_ptr))
        return lam, g, nc

    def tti_metric(self, P):
        """The six float64 metric arrays (xx xy xz yy yz zz) of the FP64
        parameter medium P = (s, eps, nx, ny), formed as the GPU kernels do."""
        P = [np.ascontiguousarray(a, dtype=np.float64) for a in P]
        out = [np.empty_like(P[0]) for _ in range(6)]
        ptrs = (C.c_void_p * 6)(*(a.ctypes.data for a in out))
        self.L.orc_tti_metric(*(_p(a) for a in P), P[0].size, ptrs)
        return out

    def tti_solve_rec(self, T, P, h, nsweeps, tol=-1.0):
        """The FP64 parameter medium P = (s, eps, nx, ny) (field layout), in
        place: (sweeps, last change, winner record)."""
        Md = self.tti_metric(P)
        ptrs = (C.c_void_p * 6)(*(a.ctypes.data for a in Md))
        W = np.full(T.shape, 0xFF, dtype=np.uint8)
        d = _dbl(0.0)
        s = self.L.orc_ell_solve_rec_d(_p(T), ptrs, W.ctypes.data_as(_ptr), *self._dims(T), h[0], h[1], h[2],
                                       nsweeps, tol, C.byref(d))
        if s < 0:
            raise MemoryError("orc_ell_solve_rec_d failed")
        return s, d.value, W

    def tti_adjoint(self, T, P, h, W, r):
        """FP64 adjoint of the parameter medium: (lambda, dL/dP (4, ...) with
        respect to s, eps, nx, ny, number of non-causal weights).  The chain
        from the metric entries to the parameters is the one the GPU gradient
        kernel applies."""
        Md = self.tti_metric(P)
        ptrs = (C.c_void_p * 6)(*(a.ctypes.data for a in Md))
        lam = np.zeros_like(T)
        g = np.zeros((6,) + T.shape)
        r = np.ascontiguousarray(r, dtype=np.float64)
        Wc = np.ascontiguousarray(W, dtype=np.uint8)
        nc = self.L.orc_ell_adjoint_rec_d(_p(T), ptrs, Wc.ctypes.data_as(_ptr), *self._dims(T), h[0], h[1], h[2],
                                          r.ctypes.data_as(_ptr), lam.ctypes.data_as(_ptr), g.ctypes.data_as(_ptr))
        return lam, tti_param_gradient(P, g), nc

    def fold_from_point(self, F, ax, ay, az, x, y, z) -> float:
        return self.L.orc_fold_from_point(F, ax, ay, az, x, y, z)

    def overfull_voxels(self) -> int:
        return self.L.orc_last_overfull()


def tti_param_gradient(P, gM):
    """dL/d(s, eps, nx, ny) from dL/dM (six entries xx xy xz yy yz zz) for
    M = a I + b n n^T, a = s^2/(1+2 eps), b = s^2 - a, nz = sqrt(1 - nx^2 -
    ny^2) following nx and ny (where nz = 0 only the direct terms)."""
    s, eps, nx, ny = (np.asarray(a, dtype=np.float64) for a in P)
    s2, den = s * s, 1.0 + 2.0 * eps
    a = s2 / den
    b = s2 - a
    nz = np.sqrt(np.maximum((1.0 - nx * nx) - ny * ny, 0.0))
    g = gM
    ga = g[0] + g[3] + g[5]
    gb = g[0] * nx * nx + g[3] * ny * ny + g[5] * nz * nz + g[1] * nx * ny + g[2] * nx * nz + g[4] * ny * nz
    gnx = 2.0 * b * nx * g[0] + b * ny * g[1] + b * nz * g[2]
    gny = 2.0 * b * ny * g[3] + b * nx * g[1] + b * nz * g[4]
    gnz = 2.0 * b * nz * g[5] + b * nx * g[2] + b * ny * g[4]
    with np.errstate(divide="ignore", invalid="ignore"):
        gnx = np.where(nz > 0, gnx - gnz * nx / nz, gnx)
        gny = np.where(nz > 0, gny - gnz * ny / nz, gny)
    da_ds, da_de = 2.0 * s / den, -2.0 * s2 / (den * den)
    return np.stack([ga * da_ds + gb * (2.0 * s - da_ds), ga * da_de - gb * da_de, gnx, gny])


# The reference driver's sweep order and argument permutations
# (AN_ISO_1_OpenACC.c:1195-1236).  Each entry: symbol, plane range kind,
# spacing permutation, drift arguments (ay, ax, az) as passed.
_REF_CALLS = (
    ("function_x_down", "up", ("DX", "dz", "dy", "DYZP", "DXZP", "DXYP"), (+1, "y"), (+1, "z"), (+1, "x")),
    ("function_x_up", "down", ("DX", "dz", "dy", "DYZP", "DXZP", "DXYP"), (-1, "y"), (-1, "z"), (-1, "x")),
    ("function_k_up", "up", ("dz", "dy", "DX", "DXYP", "DYZP", "DXZP"), (+1, "x"), (+1, "y"), (+1, "z")),
    ("function_k_down", "down", ("dz", "dy", "DX", "DXYP", "DYZP", "DXZP"), (-1, "x"), (-1, "y"), (-1, "z")),
    ("function_y_up", "down", ("dy", "DX", "dz", "DXZP", "DXYP", "DYZP"), (-1, "z"), (-1, "x"), (-1, "y")),
    ("function_y_down", "up", ("dy", "DX", "dz", "DXZP", "DXYP", "DYZP"), (+1, "z"), (+1, "x"), (+1, "y")),
)


class RefLib:
    """The reference's own code built for the host at size n (oracle/_ref)."""

    def __init__(self, n: int, omp: bool = False):
        from . import build

        path = build.ref_lib_path(n, omp)
        if not os.path.exists(path):
            build.build_ref(n)
        self.n = n
        L = C.CDLL(path)
        L.ImplicitInitialiser.argtypes = [_ptr, _int, _int, _int, _dbl, _dbl, _dbl]
        L.InitFoldFromPoint.argtypes = [_dbl] * 7
        L.InitFoldFromPoint.restype = _dbl
        L.ImpSurfF.argtypes = [_dbl] * 3
        L.ImpSurfF.restype = _dbl
        for name, *_ in _REF_CALLS:
            getattr(L, name).argtypes = [_ptr, _int] + [_dbl] * 10
        self.L = L
        DX = dy = dz = ref_spacing(n)
        self.sp = {
            "DX": DX, "dy": dy, "dz": dz,
            "DXYP": math.sqrt(DX * DX + dy * dy),
            "DXZP": math.sqrt(DX * DX + dz * dz),
            "DYZP": math.sqrt(dy * dy + dz * dz),
        }
        self.const = {"x": REF_A[0], "y": REF_A[1], "z": REF_A[2]}

    def init_implicit(self) -> np.ndarray:
        n = self.n
        T = empty_field(n, n, n)
        self.L.ImplicitInitialiser(_p(T), n, n, n, self.sp["DX"], self.sp["dy"], self.sp["dz"])
        return T

    def _args(self, entry):
        _, _, sp, *drift = entry
        s = [self.sp[k] for k in sp]
        d = [sg * self.const[c] for sg, c in drift]
        return s + [REF_F] + d

    def plane(self, T, dir_, src):
        entry = _REF_CALLS[dir_]
        getattr(self.L, entry[0])(_p(T), src, *self._args(entry))

    def pass_(self, T, dir_):
        n = self.n
        entry = _REF_CALLS[dir_]
        fn = getattr(self.L, entry[0])
        args = self._args(entry)
        planes = range(1, n) if entry[1] == "up" else range(n, 1, -1)
        for s in planes:
            fn(_p(T), s, *args)

    def sweeps(self, T, nsweeps):
        for _ in range(nsweeps):
            for d in range(6):
                self.pass_(T, d)
