"""The kernels' arithmetic core without a GPU: the library's point update
(csrc/fold3d_fast.cuh) and direction tables (csrc/fold3d_tables.cpp), built
for the host by tests/fast_solver_host.cu, swept over whole fields and
compared bit for bit with the oracle's statement of the reference
(Stencil-OpenACC/AN_ISO_1_OpenACC.c:59-326).  Both IEEE double builds round
every operation on its own, so equal bits here are the bits the kernels
compute: the folded constants, the division by constants without a divide
instruction, the slot loops and the skipping of solver bodies that cannot
lower the time (csrc/fold3d_fast.cuh, 3. and 4.), over media and spacings
the GPU tests do not reach, drifts close to F among them."""
import ctypes as C
import hashlib
import math
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT, assert_bitwise
from oracle import REF_A, REF_F, ref_spacing

_dbl, _int, _ptr = C.c_double, C.c_int, C.c_void_p


@pytest.fixture(scope="module")
def host(tmp_path_factory):
    import build as pkg_build  # fgcs-openacc-advanced_b200/build.py

    out = str(tmp_path_factory.mktemp("fast_host") / "libfast_host.so")
    cmd = [pkg_build.NVCC, "-O2", "-std=c++17", *pkg_build.ARCH, "--fmad=false", "-shared",
           "-Xcompiler", "-fPIC,-ffp-contract=off,-fno-fast-math", "-I", pkg_build.INCLUDE, "-I", pkg_build.CSRC,
           os.path.join(ROOT, "tests", "fast_solver_host.cu"), os.path.join(pkg_build.CSRC, "fold3d_tables.cpp"),
           "-o", out]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    L = C.CDLL(out)
    L.fast_host_sweeps.argtypes = [_ptr, _int, _int, _int, _dbl, _dbl, _dbl, _dbl, _dbl, _dbl, _dbl, _int, _int]
    L.fast_host_sweeps.restype = _int
    L.fast_host_bounds.argtypes = [_dbl, _dbl, _dbl, _dbl, _dbl, _dbl, _dbl, _ptr]
    L.fast_host_bounds.restype = None
    return L


def _host_sweeps(host, T, h, F, a, sweeps, skip=1):
    nz, ny, nx = (s - 2 for s in T.shape)
    host.fast_host_sweeps(T.ctypes.data, nx, ny, nz, *h, F, *a, sweeps, int(skip))


# (dims, spacings, F, drift, source): the reference's medium and others, with
# drifts from zero to 0.98 F (the skip is off above 0.95 F)
CASES = [
    ((37, 37, 37), None, REF_F, REF_A, "implicit"),
    ((29, 21, 25), (0.7, 0.9, 1.1), REF_F, REF_A, "implicit"),
    ((24, 17, 30), (0.41, 0.33, 0.5), 1.0, (0.0, 0.0, 0.0), "point"),
    ((33, 35, 18), (1.0, 0.6, 0.8), 1.3, (0.2, -0.5, 0.3), "point"),
    ((26, 26, 26), (0.5, 0.5, 0.5), 1.0, (0.55, -0.55, 0.55), "point"),
    ((20, 31, 22), (0.3, 0.45, 0.4), 2.0, (-1.1, 0.6, -1.2), "implicit"),
    ((21, 19, 23), (0.5, 0.5, 0.5), 1.0, (0.6, 0.5, 0.6), "point"),
    ((40, 30, 50), (0.2, 0.05, 0.3), 1.0, (0.0, 0.0, 0.0), "point"),
    ((24, 28, 20), (0.25, 0.3, 0.2), 1.5, (1.3, -0.3, 0.4), "implicit"),
]


@pytest.mark.parametrize("case", CASES, ids=lambda c: "x".join(map(str, c[0])) + c[4])
def test_host_build_of_the_point_update_matches_oracle(orc, host, case):
    dims, h, F, a, src = case
    nx, ny, nz = dims
    if h is None:
        h = (ref_spacing(nx),) * 3
    if src == "implicit":
        T0 = orc.init_implicit(nx, ny, nz, h, F=F, a=a)
    else:
        T0 = orc.init_point(nx, ny, nz, (nx // 3 + 1, ny // 2 + 1, nz - 2))
    ref = T0.copy()
    orc.solve(ref, h, 8, F=F, a=a)
    for skip in (1, 2, 0):  # searched bounds, closed-form bounds (the no-alloc solve's), none
        T = T0.copy()
        _host_sweeps(host, T, h, F, a, 8, skip)
        assert_bitwise(T, ref, "host build of the point update, skip mode %d" % skip)


@pytest.mark.parametrize("n", [37, 99])
@pytest.mark.parametrize("name,src", [("corner_point", lambda n: (2, 1, 2)),
                                      ("face_point", lambda n: (n, n // 3 + 1, 2 * n // 3 + 1))])
def test_host_build_matches_reference_off_centre_sources(orc, host, digests, n, name, src):
    """The reference's own 8-sweep results for point sources next to a
    corner and on a face, through the host build of the kernels' code."""
    h = (ref_spacing(n),) * 3
    P = orc.init_point(n, n, n, src(n))
    _host_sweeps(host, P, h, REF_F, REF_A, 8)
    assert hashlib.sha256(np.ascontiguousarray(P).tobytes()).hexdigest() == digests["n%d_%s_s8" % (n, name)]


def test_host_build_matches_reference_digest_99(host, digests):
    """The reference's own 8-sweep result at 99^3 (partial tiles on every
    axis), through the host build."""
    from oracle import Oracle

    n = 99
    h = (ref_spacing(n),) * 3
    T = Oracle().init_implicit(n, n, n, h)
    _host_sweeps(host, T, h, REF_F, REF_A, 8)
    assert hashlib.sha256(np.ascontiguousarray(T).tobytes()).hexdigest() == digests["n99_s8"]


# the reference's direction table (AN_ISO_1_OpenACC.c:1195-1236): normal axis,
# sign, local x axis and sign, local y axis and sign
_DIRS = [(0, +1, 2, +1, 1, +1), (0, -1, 2, -1, 1, -1), (2, +1, 1, +1, 0, +1),
         (2, -1, 1, -1, 0, -1), (1, -1, 0, -1, 2, -1), (1, +1, 0, +1, 2, +1)]


def _edge_bound(F, ax, ay, az, dzz):
    """fold3d_fast.cuh 4., restated: the FoldEdge2Points skip bound."""
    Fp2 = F * F - ay * ay
    ga = Fp2 - az * az
    if not (F * F >= 1.1 * (ax * ax + ay * ay + az * az) and ga > 0):
        return 0.0
    Fp, a2 = math.sqrt(Fp2), math.hypot(ax, az)
    if not (abs(ax) < 0.95 * math.sqrt(ga) and a2 < 0.95 * Fp):
        return 0.0
    if not ((F >= 1 and az >= 0) or (F <= 1 and az <= 0)):
        return 0.0
    P = 1 - Fp * (1 - 1 / F) / (Fp - a2) if F >= 1 else 1.0
    W = Fp / F + az
    return dzz * P / W * (1 - 1e-3) if P > 0 and W > 0 else 0.0


def _edge_sampled_inf(F, ax, ay, az, hx, hz, n=200001):
    """Smallest increment over min(s0, s1) that a FoldEdge2Points call with
    these arguments accepts (AN_ISO_1_OpenACC.c:71-95), over n values of
    d = (s1 - s0)/dxx spanning the interval where its square root is real;
    an upper estimate of the true infimum.  None when that interval is not
    bounded, inf when no sample is accepted."""
    g = F * F - ay * ay
    ga = g - az * az
    if not (ga > 0 and abs(ax) < math.sqrt(ga)):
        return None
    lo, hi = 1 / (ax - math.sqrt(ga)), 1 / (ax + math.sqrt(ga))
    if ax > 0:
        hi = 0.0
    d = np.linspace(lo, hi, n)[1:-1]
    c0 = 1 - d * ax
    Q = g * (c0 * c0 - d * d * ga)
    ok = Q > 0
    c = (-az * c0 + np.sqrt(np.where(ok, Q, 0))) / ga
    mn = np.minimum(0, d * hx)
    G = np.sqrt((d * d + c * c) * F * F / g)
    with np.errstate(divide="ignore", invalid="ignore"):
        xe = -hz * (d + ax * G) / (c + az * G)
    acc = ok & (hz * c > mn) & (xe > 0) & (xe < hx)
    return float((hz * c - mn)[acc].min()) if acc.any() else math.inf


def _surf_sampled_inf(F, ax, ay, az, hx, hy, hz, n=601):
    """Smallest increment over min(s0, s1, s2) that a FoldSurf3Points call
    with these arguments accepts (AN_ISO_1_OpenACC.c:131-165), over an n x n
    grid of the gradients (dx, dy) covering the disc where its square root
    is real; an upper estimate of the true infimum (inf when no sample is
    accepted, None when the disc is not bounded)."""
    g = F * F - az * az
    ain = math.hypot(ax, ay)
    if not (g > 0 and ain < math.sqrt(g)):
        return None
    R = 1 / (math.sqrt(g) - ain)
    xs = np.linspace(-R, 0.0 if ax > 0 else R, n)
    ys = np.linspace(-R, 0.0 if ay > 0 else R, n)
    dx, dy = np.meshgrid(xs, ys)
    dd = dx * dx + dy * dy
    al = 1 - ax * dx - ay * dy
    q = al * al - dd * g
    ok = q > 0
    al2 = (-az * al + F * np.sqrt(np.where(ok, q, 0))) / g
    mn = np.minimum(0, np.minimum(dx * hx, dx * hx + dy * hy))
    inc = hz * al2 - mn
    r = np.sqrt(dd + al2 * al2)
    with np.errstate(divide="ignore", invalid="ignore"):
        d2 = -hz / (F * al2 + az * r)
        xe, ye = d2 * (F * dx + ax * r), d2 * (F * dy + ay * r)
        acc = ok & (inc > 0) & (np.minimum(xe, ye) >= 0) & (ye * hx <= xe * hy) & (xe <= hx)
    return float(inc[acc].min()) if acc.any() else math.inf


@pytest.mark.parametrize("F,a,h", [(REF_F, REF_A, (0.7, 0.9, 1.1)), (REF_F, REF_A, (1.0, 1.0, 1.0)),
                                   (1.3, (0.2, -0.5, 0.3), (1.0, 0.6, 0.8)), (0.8, (0.3, -0.2, -0.4), (0.5, 0.5, 0.5)),
                                   (1.0, (0.6, 0.5, 0.6), (0.5, 0.5, 0.5))])
def test_skip_bounds_are_proved_lower_bounds(host, F, a, h):
    """Every FoldSurf3Points call's B (AN_ISO_1_OpenACC.c:233-240) is at
    least the physical bound dzz / (F + az) (1 - 1e-3), az the drift along
    the normal towards the target (negated on the negative side); every
    FoldEdge2Points call's B (:242-253, and the nested calls :172-173, with
    each call's own arguments) is at least the analytic bound of
    fold3d_fast.cuh 4.  Each is at most the smallest accepted increment found
    by dense sampling, and all are 0 where F^2 < 1.1 |a|^2.  In the
    reference's medium the searches bring the edge bounds within 2% of the
    sampled infimum and the triangle bounds within 10%."""
    out = np.zeros(6 * 2 * 24)
    host.fast_host_bounds(*h, F, *a, out.ctypes.data)
    out = out.reshape(6, 2, 24)
    strong = F * F < 1.1 * sum(x * x for x in a)
    tight, tight_s = [], []
    for d, (nrm, sg, xa, xs, ya, ys) in enumerate(_DIRS):
        for side in (0, 1):
            s = -1 if side else 1
            ax, ay, az = s * xs * a[xa], s * ys * a[ya], s * sg * a[nrm]
            hx, hy, hz = h[xa], h[ya], h[nrm]
            hxy, hxz, hyz = math.hypot(hx, hy), math.hypot(hx, hz), math.hypot(hy, hz)
            edges = [(ax, ay, az, hx, hz), ((ax * hx + ay * hy) / hxy, (-ax * hy + ay * hx) / hxy, az, hxy, hz),
                     (ay, ax, az, hy, hz), (-(ax * hx - ay * hy) / hxy, (ax * hy + ay * hx) / hxy, az, hxy, hz),
                     (-ax, ay, az, hx, hz), (-(ax * hx + ay * hy) / hxy, (-ax * hy + ay * hx) / hxy, az, hxy, hz),
                     (-ay, ax, az, hy, hz), ((ax * hx - ay * hy) / hxy, (ax * hy + ay * hx) / hxy, az, hxy, hz)]
            surfs = [(ax, ay, hx, hy, hxz), (ax, -ay, hx, hy, hxz), (-ax, -ay, hx, hy, hxz), (-ax, ay, hx, hy, hxz),
                     (-ay, -ax, hy, hx, hyz), (-ay, ax, hy, hx, hyz), (ay, ax, hy, hx, hyz), (ay, -ax, hy, hx, hyz)]
            nests = [(say, (sax * hz + az * shx) / shxz, (-sax * shx + az * hz) / shxz, shy, shxz)
                     for sax, say, shx, shy, shxz in surfs]
            for k, (sax, say, shx, shy, _) in enumerate(surfs):
                B = out[d, side, k]
                if strong:
                    assert B == 0.0
                    continue
                assert B >= hz / (F + az) * (1 - 1e-3) * (1 - 1e-12)
                inf = _surf_sampled_inf(F, sax, say, az, shx, shy, hz)
                if inf is not None and inf < math.inf:
                    assert B <= inf
                    tight_s.append(B / inf)
            for k, (cax, cay, caz, chx, chz) in enumerate(edges + nests):
                B = out[d, side, 8 + k]
                if strong:
                    assert B == 0.0
                    continue
                assert B >= _edge_bound(F, cax, cay, caz, chz) * (1 - 1e-12)
                inf = _edge_sampled_inf(F, cax, cay, caz, chx, chz)
                if inf is None:
                    assert B == _edge_bound(F, cax, cay, caz, chz)
                elif inf < math.inf:
                    assert B <= inf
                    tight.append(B / inf)
    if F == REF_F:
        assert min(tight) > 0.98 and min(tight_s) > 0.9
    if not strong:
        assert (out[:, :, :8] > 0).all() and (out[:, :, 8:] > 0).any()


@pytest.fixture(scope="module")
def ellip_host(tmp_path_factory):
    import build as pkg_build  # fgcs-openacc-advanced_b200/build.py

    out = str(tmp_path_factory.mktemp("ellip_host") / "libellip_host.so")
    cmd = [pkg_build.NVCC, "-O2", "-std=c++17", *pkg_build.ARCH, "--fmad=false", "-shared",
           "-Xcompiler", "-fPIC,-ffp-contract=off,-fno-fast-math", "-I", pkg_build.INCLUDE, "-I", pkg_build.CSRC,
           os.path.join(ROOT, "tests", "ellip_solver_host.cu"), "-o", out]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    L = C.CDLL(out)
    L.ellip_host_sweeps.argtypes = [_ptr, _ptr, _ptr, _int, _int, _int, _dbl, _dbl, _dbl, _int, _int]
    L.ellip_host_sweeps.restype = _int
    L.ellip_host_bound.argtypes = [_dbl] * 6
    L.ellip_host_bound.restype = _dbl
    return L


def _tti(kind, dims):
    import media

    nx, ny, nz = dims
    if kind == "c1":  # the tilted ellipse of the 128^3 configuration: Vz 2000, Vx=Vy 2400, tilt 30, azimuth 45
        M = media.homogeneous_ellip(nx, ny, nz, 2000.0, 0.22, 30.0, 45.0)
    elif kind == "strong":  # eps 0.25 with the axis tilted 70 degrees
        M = media.homogeneous_ellip(nx, ny, nz, 1800.0, 0.25, 70.0, 200.0)
    elif kind == "extreme":  # eps 2 (speeds differ by sqrt(5)), axis tilted 45 degrees
        M = media.homogeneous_ellip(nx, ny, nz, 1500.0, 2.0, 45.0, 30.0)
    else:
        M = media.heterogeneous_tti(nx, ny, nz, 10.0, seed=int(kind[-1]))
    return [np.ascontiguousarray(m.numpy(), dtype=np.float32) for m in M]


# (medium, dims, spacings, source)
ELLIP_CASES = [
    ("c1", (24, 24, 24), (10.0, 10.0, 10.0), (13, 13, 13)),
    ("strong", (21, 26, 19), (8.0, 12.0, 10.0), (4, 20, 10)),
    ("seed0", (30, 22, 27), (10.0, 10.0, 10.0), (15, 11, 4)),
    ("seed1", (25, 31, 20), (6.0, 9.0, 14.0), (20, 5, 18)),
    ("extreme", (23, 20, 25), (12.0, 5.0, 8.0), (2, 19, 24)),
]


@pytest.mark.parametrize("f32", [False, True], ids=["f64", "f32"])
@pytest.mark.parametrize("case", ELLIP_CASES, ids=lambda c: c[0])
def test_host_build_of_the_elliptical_update_matches_oracle(orc, ellip_host, case, f32):
    """Fields and winner records after 6 sweeps, bit for bit, against
    orc_ell_solve_rec / orc_ellf_solve_rec (which skip nothing)."""
    kind, dims, h, src = case
    nx, ny, nz = dims
    M = _tti(kind, dims)
    dt = np.float32 if f32 else np.float64
    T0 = np.full((nz + 2, ny + 2, nx + 2), 1e16, dtype=dt)
    T0[src[2], src[1], src[0]] = 0.0
    ref = T0.copy()
    _, _, Wref = (orc.ellf_solve_rec if f32 else orc.ell_solve_rec)(ref, M, h, 6, tol=-1.0)
    T = T0.copy()
    W = np.full(T.shape, 0xFF, dtype=np.uint8)
    ptrs = (C.c_void_p * 6)(*(m.ctypes.data for m in M))
    ellip_host.ellip_host_sweeps(T.ctypes.data, W.ctypes.data, ptrs, nx, ny, nz, *h, 6, int(f32))
    assert np.array_equal(T.view(np.uint32 if f32 else np.uint64), ref.view(np.uint32 if f32 else np.uint64))
    assert np.array_equal(W, Wref)
    assert (np.abs(T[1:-1, 1:-1, 1:-1]) < 1e15).all()  # every interior cell reached


def test_elliptical_skip_bound_is_the_plane_distance(ellip_host):
    """ell_skip_bound = 0.999 min over the source plane of ||X - p||_M, i.e.
    0.999 / sqrt((A^-1)_zz) for the scaled local metric A, X = (0, 0, 1)."""
    rng = np.random.default_rng(3)
    for _ in range(200):
        G = rng.normal(size=(3, 3))
        A = G @ G.T + 0.05 * np.eye(3)
        got = ellip_host.ellip_host_bound(A[0, 0], A[1, 1], A[2, 2], A[0, 1], A[0, 2], A[1, 2])
        assert got == pytest.approx(0.999 / math.sqrt(np.linalg.inv(A)[2, 2]), rel=1e-9)
    assert ellip_host.ellip_host_bound(1.0, 1.0, 1.0, 1.0, 0.0, 0.0) == 0.0  # singular in-plane block


def test_tables_are_the_same_from_concurrent_threads(host):
    """build_dir_table keeps a per-thread memo and its searches use only local
    state: tables built for several media from four threads at once (ctypes
    releases the GIL) equal the ones built one after the other."""
    import threading

    media_ = [(REF_F, REF_A, (0.7, 0.9, 1.1)), (1.3, (0.2, -0.5, 0.3), (1.0, 0.6, 0.8)),
              (0.8, (0.1, -0.2, -0.3), (0.5, 0.5, 0.5)), (1.1, (0.3, 0.3, -0.5), (1.0, 1.0, 1.0))]

    def bounds(F, a, h):
        out = np.zeros(288)
        host.fast_host_bounds(*h, F, *a, out.ctypes.data)
        return out

    want = [bounds(*m) for m in media_]
    got = [[None] * len(media_) for _ in range(4)]

    def work(t):
        for q in range(len(media_)):
            m = media_[(q + t) % len(media_)]
            got[t][(q + t) % len(media_)] = bounds(*m)

    threads = [threading.Thread(target=work, args=(t,)) for t in range(4)]
    for th in threads:
        th.start()
    for th in threads:
        th.join()
    for t in range(4):
        for q in range(len(media_)):
            assert np.array_equal(got[t][q], want[q])


def test_host_build_matches_oracle_in_random_media(orc, host):
    """64 seeded random media (F in [0.5, 3], drift up to 0.95 F in any
    direction, anisotropic spacings, point and implicit sources, 6-21 points
    per axis): the host build of the kernels' update with its searched skip
    bounds equals the oracle bit for bit after 8 sweeps."""
    rng = np.random.default_rng(20261204)
    for it in range(64):
        F = rng.uniform(0.5, 3.0)
        d = rng.normal(size=3)
        a = tuple(float(x) for x in d / np.linalg.norm(d) * rng.uniform(0.0, 0.95) * F)
        nx, ny, nz = (int(x) for x in rng.integers(6, 22, size=3))
        h = tuple(float(x) for x in rng.uniform(0.1, 1.0, size=3))
        if it % 2 == 0:
            src = tuple(int(rng.integers(1, m + 1)) for m in (nx, ny, nz))
            T0 = orc.init_point(nx, ny, nz, src)
        else:
            T0 = orc.init_implicit(nx, ny, nz, h, F=F, a=a)
        ref = T0.copy()
        orc.solve(ref, h, 8, F=F, a=a)
        T = T0.copy()
        _host_sweeps(host, T, h, F, a, 8)
        assert_bitwise(T, ref, "random medium %d (F=%g, a=%s, h=%s)" % (it, F, a, h))


@pytest.mark.parametrize("f32", [False, True], ids=["f64", "f32"])
def test_host_build_of_the_elliptical_update_in_random_media(orc, ellip_host, f32):
    """16 seeded random tilted ellipses (Vz 1000-4000, eps 0-0.4, any axis;
    6-20 points per axis, spacings 3-15, a random point source): fields and
    winner records after 6 sweeps equal the oracle's bit for bit."""
    import media

    rng = np.random.default_rng(1204 + int(f32))
    dt = np.float32 if f32 else np.float64
    for it in range(16):
        nx, ny, nz = (int(x) for x in rng.integers(6, 21, size=3))
        h = tuple(float(x) for x in rng.uniform(3.0, 15.0, size=3))
        M = media.homogeneous_ellip(nx, ny, nz, float(rng.uniform(1000.0, 4000.0)), float(rng.uniform(0.0, 0.4)),
                                    float(rng.uniform(0.0, 90.0)), float(rng.uniform(0.0, 360.0)))
        M = [np.ascontiguousarray(m.numpy(), dtype=np.float32) for m in M]
        src = tuple(int(rng.integers(1, m + 1)) for m in (nx, ny, nz))
        T0 = np.full((nz + 2, ny + 2, nx + 2), 1e16, dtype=dt)
        T0[src[2], src[1], src[0]] = 0.0
        ref = T0.copy()
        _, _, Wref = (orc.ellf_solve_rec if f32 else orc.ell_solve_rec)(ref, M, h, 6, tol=-1.0)
        T = T0.copy()
        W = np.full(T.shape, 0xFF, dtype=np.uint8)
        ptrs = (C.c_void_p * 6)(*(m.ctypes.data for m in M))
        ellip_host.ellip_host_sweeps(T.ctypes.data, W.ctypes.data, ptrs, nx, ny, nz, *h, 6, int(f32))
        bits = np.uint32 if f32 else np.uint64
        assert np.array_equal(T.view(bits), ref.view(bits)), (it, nx, ny, nz, h, src)
        assert np.array_equal(W, Wref), it
