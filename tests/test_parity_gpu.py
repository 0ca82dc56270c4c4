"""GPU parity: the CUDA sweep against the reference's own outputs (golden
fixtures and digests) and against the oracle, bit for bit.

The bar is bit-exact equality of the float64 fields: every kernel follows
the reference's operand order and is compiled without FMA contraction.
"""
import ctypes as C
import hashlib

import numpy as np
import pytest

from conftest import assert_bitwise

from oracle import MAXT, REF_A, REF_F, ref_spacing

pytestmark = pytest.mark.gpu

ENGINES = ["planes", "planes-literal", "planes-compact", "wavefront", "wavefront-skip"]


def engine_opts(f3d, name):
    """'<engine>[-literal|-compact|-skip]': engine, solver variant, skipping."""
    eng, _, var = name.partition("-")
    return ({"planes": f3d.ENGINE_PLANES, "wavefront": f3d.ENGINE_WAVEFRONT}[eng],
            {"literal": f3d.VARIANT_LITERAL, "compact": f3d.VARIANT_COMPACT}.get(var, f3d.VARIANT_FAST),
            var == "skip")


def gpu_solve(f3d, ctx, cuda, T, h, sweeps, *, fixed=True, tol=0.0, engine="planes", med=None):
    d = cuda.from_numpy(T.copy()).cuda()
    eng, var, skip = engine_opts(f3d, engine)
    rep = ctx.solve(d, h, med, f3d.opts(max_sweeps=sweeps, fixed=fixed, tol=tol, engine=eng, skip=skip,
                                         variant=var))
    return d.cpu().numpy(), rep


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


@pytest.mark.parametrize("engine", ENGINES)
@pytest.mark.parametrize("n", [8, 16])
def test_golden_implicit_surface(f3d, ctx, cuda, golden, n, engine):
    h = (ref_spacing(n),) * 3
    g = golden[n]
    for k, key in ((1, "s1"), (2, "s2"), (8, "s8")):
        out, rep = gpu_solve(f3d, ctx, cuda, g["init"], h, k, engine=engine)
        assert rep.sweeps == k
        assert_bitwise(out, g[key], "%s n=%d after %d sweeps" % (engine, n, k))


@pytest.mark.parametrize("engine", ENGINES)
@pytest.mark.parametrize("n", [8, 16])
def test_golden_point_source(f3d, ctx, cuda, golden, n, engine):
    h = (ref_spacing(n),) * 3
    c = n // 2 + 1
    T = f3d.init_point(n, n, n, (c, c, c))
    out, _ = gpu_solve(f3d, ctx, cuda, T, h, 8, engine=engine)
    assert_bitwise(out, golden[n]["point_s8"], "point source")


@pytest.mark.parametrize("engine", ENGINES)
def test_digests_64(f3d, ctx, cuda, digests, engine):
    n = 64
    h = (ref_spacing(n),) * 3
    T = f3d.init_implicit(n, n, n, h[0])
    assert sha(T) == digests["n64_init"]
    out, _ = gpu_solve(f3d, ctx, cuda, T, h, 8, engine=engine)
    assert sha(out) == digests["n64_s8"]
    c = n // 2 + 1
    P = f3d.init_point(n, n, n, (c, c, c))
    out, _ = gpu_solve(f3d, ctx, cuda, P, h, 8, engine=engine)
    assert sha(out) == digests["n64_point_s8"]


@pytest.mark.parametrize("engine", ["wavefront", "planes"])
@pytest.mark.parametrize("n", [37, 99])
@pytest.mark.parametrize("name,src", [("corner_point", lambda n: (2, 1, 2)),
                                      ("face_point", lambda n: (n, n // 3 + 1, 2 * n // 3 + 1))])
def test_digests_off_centre_point_sources(f3d, ctx, cuda, digests, n, name, src, engine):
    """The reference's own 8-sweep results for point sources next to a
    corner and on a face, at sizes that leave partial tiles on every axis."""
    h = (ref_spacing(n),) * 3
    P = f3d.init_point(n, n, n, src(n))
    out, _ = gpu_solve(f3d, ctx, cuda, P, h, 8, engine=engine)
    assert sha(out) == digests["n%d_%s_s8" % (n, name)]


CASES = [
    # dims, spacing, F, drift, source
    ((13, 9, 11), (0.7, 0.9, 1.1), 1.3, (0.2, -0.5, 0.3), "implicit"),
    ((24, 17, 30), (0.41, 0.33, 0.5), 1.0, (0.0, 0.0, 0.0), "point"),
    ((31, 40, 19), (0.25, 0.3, 0.35), 2.0, (-0.9, 0.4, 1.1), "point"),
    ((33, 20, 27), (0.3, 0.3, 0.3), 1.1, REF_A, "implicit"),
    ((2, 5, 3), (1.0, 1.0, 1.0), 1.1, REF_A, "point"),
]


def make_case(f3d, orc, dims, h, F, a, src):
    if src == "implicit":
        return orc.init_implicit(*dims, h, F=F, a=a)
    rng = np.random.default_rng(sum(dims))
    s = tuple(int(rng.integers(1, d + 1)) for d in dims)
    return orc.init_point(*dims, s)


@pytest.mark.parametrize("engine", ENGINES)
@pytest.mark.parametrize("case", CASES, ids=lambda c: "x".join(map(str, c[0])) + c[4])
def test_oracle_fixed_sweeps(f3d, orc, ctx, cuda, case, engine):
    dims, h, F, a, src = case
    T0 = make_case(f3d, orc, dims, h, F, a, src)
    for k in (1, 3):
        ref = T0.copy()
        orc.solve(ref, h, k, F=F, a=a)
        out, rep = gpu_solve(f3d, ctx, cuda, T0, h, k, engine=engine, med=f3d.medium(F, a))
        assert_bitwise(out, ref, "%s %s %d sweeps" % (engine, dims, k))
        assert rep.nominal_updates == k * 2 * ((dims[0] - 1) * dims[1] * dims[2] +
                                               (dims[1] - 1) * dims[0] * dims[2] +
                                               (dims[2] - 1) * dims[0] * dims[1])


@pytest.mark.parametrize("engine", ENGINES)
@pytest.mark.parametrize("case", CASES[:4], ids=lambda c: "x".join(map(str, c[0])) + c[4])
def test_oracle_convergence(f3d, orc, ctx, cuda, case, engine):
    """Run both to max|dT| == 0: same number of sweeps, same field."""
    dims, h, F, a, src = case
    T0 = make_case(f3d, orc, dims, h, F, a, src)
    ref = T0.copy()
    s_ref, d_ref = orc.solve(ref, h, 300, tol=0.0, F=F, a=a)
    out, rep = gpu_solve(f3d, ctx, cuda, T0, h, 300, fixed=False, tol=0.0, engine=engine,
                         med=f3d.medium(F, a))
    assert d_ref == 0.0 and rep.max_delta == 0.0
    assert rep.sweeps == s_ref
    assert_bitwise(out, ref, "converged")


def test_tolerance_stop_matches_oracle(f3d, orc, ctx, cuda):
    n = 20
    h = (ref_spacing(n),) * 3
    T0 = orc.init_implicit(n, n, n, h)
    ref = T0.copy()
    s_ref, d_ref = orc.solve(ref, h, 300, tol=1e-3)
    out, rep = gpu_solve(f3d, ctx, cuda, T0, h, 300, fixed=False, tol=1e-3)
    assert rep.sweeps == s_ref and rep.max_delta == d_ref
    assert_bitwise(out, ref, "tol stop")


def test_host_path_equals_device_path(f3d, orc, ctx, cuda):
    n = 24
    h = (ref_spacing(n),) * 3
    T0 = orc.init_implicit(n, n, n, h)
    dev, _ = gpu_solve(f3d, ctx, cuda, T0, h, 4)
    host = T0.copy()
    rep = ctx.solve(host, h, None, f3d.opts(max_sweeps=4, fixed=True))
    assert rep.sweeps == 4
    assert_bitwise(host, dev, "host vs device")


def test_plane_entry_point_matches_oracle(f3d, orc, cuda):
    dims, h = (21, 14, 17), (0.5, 0.6, 0.7)
    T0 = orc.init_implicit(*dims, h)
    d = cuda.from_numpy(T0.copy()).cuda()
    ref = T0.copy()
    for dir_, src in ((0, 1), (0, 2), (1, 21), (2, 1), (3, 17), (4, 14), (5, 1), (5, 7)):
        f3d.plane(d, h, dir_, src)
        orc.plane(ref, h, dir_, src)
    cuda.cuda.synchronize()
    assert_bitwise(d.cpu().numpy(), ref, "plane steps")


def test_reference_compatible_entry_points(f3d, golden, cuda):
    """Drive the six function_* exactly as the reference's main does, on a
    field allocated with the library's acc_malloc (which records the grid
    size), and compare with the reference's own 8-sweep result."""
    from oracle import _REF_CALLS, RefLib

    n = 16
    L = f3d.lib()
    r = RefLib(n)  # only for the argument lists of the reference driver
    T = golden[n]["init"].copy()
    nbytes = T.nbytes
    d = L.acc_malloc(nbytes)
    assert d
    try:
        L.acc_memcpy_to_device(C.c_void_p(d), T.ctypes.data_as(C.c_void_p), nbytes)
        for _ in range(8):
            for entry in _REF_CALLS:
                fn = getattr(L, entry[0])
                args = r._args(entry)
                planes = range(1, n) if entry[1] == "up" else range(n, 1, -1)
                for p in planes:
                    fn(C.c_void_p(d), p, *args)
                assert f3d.last_error() == ""
        out = np.empty_like(T)
        L.acc_memcpy_from_device(out.ctypes.data_as(C.c_void_p), C.c_void_p(d), nbytes)
    finally:
        L.acc_free(C.c_void_p(d))
    assert_bitwise(out, golden[n]["s8"], "function_* path")


def test_compat_rejects_unknown_grid(f3d, cuda):
    L = f3d.lib()
    t = cuda.zeros(10 * 10 * 10, dtype=cuda.float64, device="cuda")
    L.function_x_down(C.c_void_p(t.data_ptr()), 1, *([1.0] * 6), 1.1, 0.4, 0.7, -0.35)
    assert "grid size unknown" in f3d.last_error()
    assert L.fold3d_compat_set_grid(8, 8, 8) == f3d.OK
    try:
        L.function_x_down(C.c_void_p(t.data_ptr()), 1, *([1.0] * 6), 1.1, 0.4, 0.7, -0.35)
        assert f3d.last_error() == ""
        L.function_x_down(C.c_void_p(t.data_ptr()), 8, *([1.0] * 6), 1.1, 0.4, 0.7, -0.35)
        assert "out of range" in f3d.last_error()
    finally:
        L.fold3d_compat_set_grid(0, 0, 0)


def test_compat_rejects_pointer_inside_acc_block(f3d, cuda):
    """A sweep call given a pointer into the middle of an acc_malloc block
    (no grid size set) is rejected: the grid cannot be inferred from the
    block, and a field placed there would run past the block's end.  With a
    grid set, the field must fit between the pointer and the block's end.
    Nothing is launched in the rejected calls."""
    L = f3d.lib()
    nbytes = 10 * 10 * 10 * 8
    d = L.acc_malloc(nbytes)
    assert d
    try:
        L.function_x_down(C.c_void_p(d + 8 * 100), 1, *([1.0] * 6), 1.1, 0.4, 0.7, -0.35)
        assert "not at its start" in f3d.last_error()
        assert L.fold3d_compat_set_grid(8, 8, 8) == f3d.OK
        L.function_x_down(C.c_void_p(d + 8 * 100), 1, *([1.0] * 6), 1.1, 0.4, 0.7, -0.35)
        assert "does not fit" in f3d.last_error()
        L.function_x_down(C.c_void_p(d), 1, *([1.0] * 6), 1.1, 0.4, 0.7, -0.35)
        assert f3d.last_error() == ""
    finally:
        L.fold3d_compat_set_grid(0, 0, 0)
        L.acc_free(C.c_void_p(d))


@pytest.mark.parametrize("bad", ["inf_spacing", "inf_F"])
def test_solve_rejects_infinite_grid_or_medium(f3d, ctx, cuda, bad):
    """fold3d_solve and fold3d_solve_noalloc reject an infinite spacing or
    medium constant with the same code."""
    T = cuda.from_numpy(f3d.init_point(8, 8, 8, (4, 4, 4))).cuda()
    L = f3d.lib()
    inf = float("inf")
    g = f3d.Grid(8, 8, 8, 1.0, inf, 1.0) if bad == "inf_spacing" else f3d.grid(8, 8, 8, 1.0)
    m = f3d.Medium(inf, 0, 0, 0) if bad == "inf_F" else f3d.medium()
    o = f3d.opts(max_sweeps=2, fixed=True)
    assert L.fold3d_solve(ctx._h, C.byref(g), C.byref(m), C.c_void_p(T.data_ptr()), C.byref(o), None,
                          None) == f3d.ERR_INVALID
    assert L.fold3d_solve_noalloc(C.byref(g), C.byref(m), C.c_void_p(T.data_ptr()), C.byref(o), None,
                                  None) == f3d.ERR_INVALID


def test_full_size_planes_512(f3d, orc, ctx, cuda):
    """At the benchmark size (512^3, reference medium and source), the first
    planes of every direction match the oracle bit for bit."""
    n = 512
    h = (ref_spacing(n),) * 3
    T0 = f3d.init_implicit(n, n, n, h[0])
    d = cuda.from_numpy(T0).cuda()
    ref = T0.copy()
    for dir_ in range(6):
        first = 1 if dir_ in (0, 2, 5) else n
        step = 1 if dir_ in (0, 2, 5) else -1
        for p in range(3):
            f3d.plane(d, h, dir_, first + step * p)
            orc.plane(ref, h, dir_, first + step * p)
    cuda.cuda.synchronize()
    assert_bitwise(d.cpu().numpy(), ref, "512^3 planes")


def test_full_size_properties_512(f3d, ctx, cuda):
    """Size-independent properties at 512^3: deterministic (two runs equal
    bit for bit), magnitudes never increase, signs never change."""
    n = 512
    h = (ref_spacing(n),) * 3
    T0 = f3d.init_implicit(n, n, n, h[0])
    a = cuda.from_numpy(T0).cuda()
    b = a.clone()
    o = f3d.opts(max_sweeps=2, fixed=True, engine=f3d.ENGINE_PLANES, skip=False)
    ctx.solve(a, h, None, o)
    ctx.solve(b, h, None, o)
    assert cuda.equal(a.view(cuda.int64), b.view(cuda.int64))
    t0 = cuda.from_numpy(T0).cuda()
    assert bool((a.abs() <= t0.abs()).all())
    assert bool(((a > 0) == (t0 > 0)).all())


def test_variants_agree_full_size_512(f3d, ctx, cuda):
    """At the benchmark size (512^3, 8 sweeps) the folded-constant solver and
    the literal reference-expression solver give the same field bit for bit
    (the literal one is pinned to the oracle by the tests above)."""
    n = 512
    h = (ref_spacing(n),) * 3
    T0 = f3d.init_implicit(n, n, n, h[0])
    a = cuda.from_numpy(T0).cuda()
    b = a.clone()
    ra = ctx.solve(a, h, None, f3d.opts(max_sweeps=8, fixed=True, engine=f3d.ENGINE_PLANES,
                                        variant=f3d.VARIANT_FAST))
    rb = ctx.solve(b, h, None, f3d.opts(max_sweeps=8, fixed=True, engine=f3d.ENGINE_PLANES,
                                        variant=f3d.VARIANT_LITERAL))
    assert ra.max_delta == rb.max_delta
    assert cuda.equal(a.view(cuda.int64), b.view(cuda.int64))
    c = cuda.from_numpy(T0).cuda()
    rc = ctx.solve(c, h, None, f3d.opts(max_sweeps=8, fixed=True, engine=f3d.ENGINE_PLANES,
                                        variant=f3d.VARIANT_COMPACT))
    assert rc.max_delta == ra.max_delta
    assert cuda.equal(a.view(cuda.int64), c.view(cuda.int64))


def test_division_by_constant_matches_ieee(f3d, cuda):
    """div_by_const (Markstein's method, fold3d_fast.cuh) against CUDA's IEEE
    division, bit for bit: the divisors of every solver table of several
    media and grids, and random divisors, over quotient operands spanning
    the safe range, zeros and out-of-range values."""
    import os
    import subprocess

    from conftest import PKG, ROOT

    so = os.path.join(ROOT, "tests", "_build", "libdivcheck.so")
    src = os.path.join(ROOT, "tests", "csrc", "divcheck.cu")
    if not os.path.exists(so) or os.path.getmtime(so) < os.path.getmtime(src):
        os.makedirs(os.path.dirname(so), exist_ok=True)
        subprocess.run(["nvcc", "-O3", "-std=c++17", "-gencode", "arch=compute_100a,code=sm_100a", "--fmad=false",
                        "-Xcompiler", "-fPIC", "-shared", "-I", os.path.join(PKG, "csrc"), "-I",
                        os.path.join(ROOT, "include"), "-o", so, src], check=True)
    L = C.CDLL(so)
    L.divcheck.argtypes = [C.c_void_p] * 3 + [C.c_longlong, C.c_int, C.c_void_p, C.c_void_p]
    rng = np.random.default_rng(11)
    cs = [0.0196, 0.00391389432485323, 10.0 / 511, 1.21 - 0.16, 1.21 - 0.49, 0.5649, 1.0, 3.0, 0.7, 2.5e-7,
          1e5, 1.0 / 3.0, np.sqrt(2.0) * 0.0196]
    cs += list(rng.uniform(0.01, 10.0, 40)) + list(-rng.uniform(0.01, 10.0, 8))
    cs += list(2.0 ** rng.uniform(-390, 390, 16))
    c = np.array(cs, dtype=np.float64)
    r = 1.0 / c
    n = 1 << 25
    mant = rng.uniform(1.0, 2.0, n)
    ex = rng.integers(-60, 61, n)
    x = np.ldexp(mant, ex) * rng.choice([-1.0, 1.0], n)
    x[: n // 8] = np.ldexp(mant[: n // 8], rng.integers(-420, 421, n // 8))  # edges of the safe range
    x[::997] = 0.0
    x[1::1009] = 1e16 - x[1::1009]
    dx = cuda.from_numpy(x).cuda()
    dc = cuda.from_numpy(c).cuda()
    dr = cuda.from_numpy(r).cuda()
    mm = cuda.zeros(1, dtype=cuda.int64, device="cuda")
    first = cuda.zeros(1, dtype=cuda.int64, device="cuda")
    assert L.divcheck(dx.data_ptr(), dc.data_ptr(), dr.data_ptr(), n, len(c), mm.data_ptr(),
                      first.data_ptr()) == 0
    i = int(first.item())
    assert int(mm.item()) == 0, "x=%r c=%r" % (x[i], c[i % len(c)])


def test_reference_program_runs_on_library(f3d, digests, cuda, tmp_path):
    """The reference's unmodified single-GPU program (its own main,
    AN_ISO_1_OpenACC.c:1150-1295) linked against libfold3dpmm: 8 sweeps at
    128^3 through this library's ImplicitInitialiser, acc_* runtime and sweep
    kernels write the reference's own output file, identical byte for byte
    (md5 of an_iso_1_openacc.txt)."""
    import os
    import subprocess

    from oracle import build

    exe = build.dropin_path(128)
    if not os.path.exists(exe):
        pytest.skip("drop-in program not built (needs the reference sources at build time)")
    r = subprocess.run([exe], cwd=tmp_path, capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    assert "Time taken for the 1 GPU" in r.stdout
    data = (tmp_path / "an_iso_1_openacc.txt").read_bytes()
    assert hashlib.md5(data).hexdigest() == digests["n128_s8_text_md5"]


def test_wavefront_skip_matches_planes_full_size_512(f3d, ctx, cuda):
    """512^3, 8 sweeps: the wavefront engine with tile skipping gives the
    per-plane engine's field bit for bit, evaluating fewer points."""
    n = 512
    h = (ref_spacing(n),) * 3
    T0 = f3d.init_implicit(n, n, n, h[0])
    a = cuda.from_numpy(T0).cuda()
    b = a.clone()
    ra = ctx.solve(a, h, None, f3d.opts(max_sweeps=8, fixed=True, engine=f3d.ENGINE_PLANES))
    rb = ctx.solve(b, h, None, f3d.opts(max_sweeps=8, fixed=True, engine=f3d.ENGINE_WAVEFRONT, skip=True))
    assert rb.max_delta == ra.max_delta
    assert cuda.equal(a.view(cuda.int64), b.view(cuda.int64))
    assert rb.nominal_updates == ra.nominal_updates
    assert 0 < rb.evaluated_updates <= rb.nominal_updates


def test_wavefront_skip_converges_like_planes(f3d, ctx, cuda):
    """Run to max|dT| == 0 at 96^3 (implicit surface and point source): same
    sweep count and field as the per-plane engine; skipping evaluates far
    fewer points once most of the field has settled."""
    n = 96
    h = (ref_spacing(n),) * 3
    for T0 in (f3d.init_implicit(n, n, n, h[0]), f3d.init_point(n, n, n, (30, 50, 70))):
        a = cuda.from_numpy(T0.copy()).cuda()
        b = a.clone()
        ra = ctx.solve(a, h, None, f3d.opts(max_sweeps=500, tol=0.0, engine=f3d.ENGINE_PLANES))
        rb = ctx.solve(b, h, None, f3d.opts(max_sweeps=500, tol=0.0, engine=f3d.ENGINE_WAVEFRONT, skip=True))
        assert ra.max_delta == 0.0 and rb.max_delta == 0.0
        assert rb.sweeps == ra.sweeps
        assert cuda.equal(a.view(cuda.int64), b.view(cuda.int64))
        assert rb.evaluated_updates < 0.8 * rb.nominal_updates


def test_wavefront_bounded_wait_times_out_cleanly(f3d, ctx, cuda, golden):
    """A dependency wait that can never be satisfied gives up after its limit
    and reports FOLD3D_ERR_TIMEOUT; the context keeps working afterwards."""
    L = f3d.lib()
    rc = L.fold3d_selftest_wait_timeout(ctx._h, 1.0)
    assert rc == f3d.ERR_TIMEOUT, f3d.last_error()
    n = 16
    out, _ = gpu_solve(f3d, ctx, cuda, golden[n]["init"], (ref_spacing(n),) * 3, 8, engine="wavefront-skip")
    assert_bitwise(out, golden[n]["s8"], "after the timeout")


# -- elliptical (tilted) medium ----------------------------------------------

def _ell_case(kind, dims, h, seed=0):
    import media

    nx, ny, nz = dims
    if kind == "homog":
        eps = ((2400.0 / 2000.0) ** 2 - 1.0) / 2.0
        return media.homogeneous_ellip(nx, ny, nz, 2000.0, eps, 30.0, 45.0)
    return media.heterogeneous_tti(nx, ny, nz, h, seed=seed)


@pytest.mark.parametrize("kind,dims,src", [("homog", (40, 40, 40), (21, 21, 21)),
                                           ("tti", (37, 29, 33), (5, 20, 9)),
                                           ("tti", (64, 64, 64), (33, 33, 9))])
@pytest.mark.parametrize("skip", [False, True])
def test_ellip_matches_oracle(f3d, orc, ctx, cuda, kind, dims, src, skip):
    """The elliptical solver on the GPU (wavefront engine) equals the FP64 CPU
    statement bit for bit, after 3 fixed sweeps and when run to
    max|dT| <= 1e-10."""
    h = (10.0, 10.0, 10.0)
    M = _ell_case(kind, dims, h[0])
    Md = [m.cuda() for m in M]
    Mh = [m.numpy() for m in M]
    T0 = orc.init_point(*dims, src)
    for fixed, sweeps, tol in ((True, 3, 0.0), (False, 300, 1e-10)):
        ref = T0.copy()
        s_ref, d_ref = orc.ell_solve(ref, Mh, h, sweeps, tol=(-1.0 if fixed else tol))
        d = cuda.from_numpy(T0.copy()).cuda()
        rep = f3d.solve_ellip(ctx, d, h, Md, f3d.opts(max_sweeps=sweeps, fixed=fixed, tol=tol, skip=skip))
        assert rep.sweeps == s_ref
        assert rep.max_delta == d_ref
        assert_bitwise(d.cpu().numpy(), ref, "%s %s fixed=%s" % (kind, dims, fixed))


def test_c1_tilted_ellipse_128(f3d, orc, ctx, cuda):
    """The 128^3 configuration: h = 10 m, source at the grid centre, a
    homogeneous tilted ellipse (Vz 2000, Vx = Vy = 2400 m/s, tilt 30,
    azimuth 45 degrees), solved to max|dT| <= 1e-10.  GPU = FP64 CPU
    statement bit for bit; against the closed form t = sqrt(x^T M x) the
    first-order solver is within 5% (max) and 1.5% (mean) away from the source
    (cells farther than 5 h)."""
    import media

    n, h = 128, 10.0
    eps = ((2400.0 / 2000.0) ** 2 - 1.0) / 2.0
    M = media.homogeneous_ellip(n, n, n, 2000.0, eps, 30.0, 45.0)
    c = n // 2 + 1
    T0 = orc.init_point(n, n, n, (c, c, c))
    ref = T0.copy()
    s_ref, d_ref = orc.ell_solve(ref, [m.numpy() for m in M], (h,) * 3, 100, tol=1e-10)
    d = cuda.from_numpy(T0.copy()).cuda()
    rep = f3d.solve_ellip(ctx, d, h, [m.cuda() for m in M], f3d.opts(max_sweeps=100, tol=1e-10))
    assert rep.sweeps == s_ref and rep.max_delta <= 1e-10
    out = d.cpu().numpy()
    assert_bitwise(out, ref, "C1 128^3")
    M6 = [float(m[c, c, c]) for m in M]
    k, j, i = np.meshgrid(*(np.arange(1, n + 1, 4),) * 3, indexing="ij")
    x, y, z = (i - c) * h, (j - c) * h, (k - c) * h
    xx, xy, xz, yy, yz, zz = M6
    ex = np.sqrt(xx * x * x + yy * y * y + zz * z * z + 2 * (xy * x * y + xz * x * z + yz * y * z))
    far = np.sqrt(x * x + y * y + z * z) > 5 * h
    err = np.abs(np.abs(out[k, j, i]) - ex)[far] / ex[far]
    assert err.max() < 0.05 and err.mean() < 0.015, (err.max(), err.mean())


def test_ellip_full_size_skip_exact_512(f3d, ctx, cuda):
    """512^3 heterogeneous TTI medium (seed 0), source at depth 64: the run to
    max|dT| <= 1e-10 with tile skipping equals the run without, bit for bit,
    and skipping evaluates fewer points."""
    import media

    n = 512
    M = [m.cuda() for m in media.heterogeneous_tti(n, n, n, 10.0, seed=0, device="cuda")]
    T0 = torch_point(cuda, n, (257, 257, 65))
    a, b = T0.clone(), T0
    o = dict(max_sweeps=200, fixed=False, tol=1e-10)
    ra = f3d.solve_ellip(ctx, a, 10.0, M, f3d.opts(skip=False, **o))
    rb = f3d.solve_ellip(ctx, b, 10.0, M, f3d.opts(skip=True, **o))
    assert ra.sweeps == rb.sweeps and ra.max_delta == rb.max_delta <= 1e-10
    assert cuda.equal(a.view(cuda.int64), b.view(cuda.int64))
    assert rb.evaluated_updates < ra.evaluated_updates


def torch_point(cuda, n, src):
    T = cuda.full((n + 2,) * 3, 10e15 * 1.0, dtype=cuda.float64, device="cuda")
    T[src[2], src[1], src[0]] = 0.0
    return T


# -- batched solves -----------------------------------------------------------

def _batch_instances(cuda, count, lo, hi, seed):
    import media

    rng = np.random.default_rng(seed)
    inst = []
    for i in range(count):
        dims = tuple(int(v) for v in rng.integers(lo, hi + 1, 3))
        M = [m.cuda() for m in media.heterogeneous_tti(*dims, 10.0, seed=100 + i)]
        src = tuple(int(rng.integers(1, d + 1)) for d in dims)
        T = torch_point_dims(cuda, dims, src)
        inst.append((T, M))
    return inst


def torch_point_dims(cuda, dims, src):
    nx, ny, nz = dims
    T = cuda.full((nz + 2, ny + 2, nx + 2), 10e15 * 1.0, dtype=cuda.float64, device="cuda")
    T[src[2], src[1], src[0]] = 0.0
    return T


@pytest.mark.parametrize("fixed", [True, False])
def test_batch_equals_one_by_one(f3d, ctx, cuda, fixed):
    """A batch of instances with different (non-cubic) grids, media and
    sources gives each instance exactly the field and sweep count of its own
    fold3d_solve_ellip (3 fixed sweeps, or per-instance convergence to
    max|dT| <= 1e-10 with instances stopping at different sweeps)."""
    inst = _batch_instances(cuda, 7, 9, 41, seed=5)
    o = f3d.opts(max_sweeps=3, fixed=True) if fixed else f3d.opts(max_sweeps=300, tol=1e-10)
    alone = []
    for T, M in inst:
        t = T.clone()
        r = f3d.solve_ellip(ctx, t, 10.0, M, o)
        alone.append((t, r))
    fields = [T.clone() for T, _ in inst]
    reps = f3d.solve_batch(ctx, fields, [10.0] * len(inst), [M for _, M in inst], o)
    sweeps = set()
    for (t, r), f, rb in zip(alone, fields, reps):
        assert rb.sweeps == r.sweeps and rb.max_delta == r.max_delta
        assert rb.nominal_updates == r.nominal_updates
        assert cuda.equal(t.view(cuda.int64), f.view(cuda.int64))
        sweeps.add(r.sweeps)
    if not fixed:
        assert len(sweeps) > 1  # instances did stop at different sweeps


def test_batch_c4_subset_equals_one_by_one(f3d, ctx, cuda):
    """The batched configuration's size mix: 16 instances with dims drawn per
    axis from [96, 320] (seed 1), each its own seeded heterogeneous medium
    and source, converged to max|dT| <= 1e-10 in one batched call (the sweep
    loop on the device, the configuration chosen by the autotuner).  Every
    field, sweep count and last change equals the instance's own solve, bit
    for bit."""
    import media

    rng = np.random.default_rng(1)
    o = f3d.opts(max_sweeps=300, tol=1e-10)
    fields, media_, alone = [], [], []
    for i in range(16):
        dims = tuple(int(v) for v in rng.integers(96, 321, 3))
        src = tuple(int(rng.integers(1, d + 1)) for d in dims)
        M = media.heterogeneous_tti(*dims, 10.0, seed=1000 + i, device="cuda")
        T = torch_point_dims(cuda, dims, src)
        t = T.clone()
        alone.append((t, f3d.solve_ellip(ctx, t, 10.0, M, o)))
        fields.append(T)
        media_.append(M)
    reps = f3d.solve_batch(ctx, fields, [10.0] * len(fields), media_, o)
    for (t, r), f, rb in zip(alone, fields, reps):
        assert rb.sweeps == r.sweeps and rb.max_delta == r.max_delta
        assert cuda.equal(t.view(cuda.int64), f.view(cuda.int64))


@pytest.mark.parametrize("rows,ctas", [(2, 0), (4, 0), (8, 0), (4, 3), (8, 1)])
def test_batch_configurations_agree(f3d, ctx, cuda, rows, ctas):
    """Every tile height and CTA count the autotuner may pick gives the
    one-by-one results bit for bit (here forced with
    fold3d_batch_set_config)."""
    inst = _batch_instances(cuda, 9, 9, 45, seed=8)
    o = f3d.opts(max_sweeps=300, tol=1e-10)
    alone = []
    for T, M in inst:
        t = T.clone()
        alone.append((t, f3d.solve_ellip(ctx, t, 10.0, M, o)))
    fields = [T.clone() for T, _ in inst]
    f3d.batch_set_config(ctx, rows, ctas)
    try:
        reps = f3d.solve_batch(ctx, fields, [10.0] * len(inst), [M for _, M in inst], o)
        got_rows, got_ctas = f3d.batch_get_config(ctx)
    finally:
        f3d.batch_set_config(ctx, 0, 0)
    assert got_rows == rows and got_ctas >= 1 and (ctas == 0 or got_ctas <= ctas)
    for (t, r), f, rb in zip(alone, fields, reps):
        assert rb.sweeps == r.sweeps and rb.max_delta == r.max_delta
        assert cuda.equal(t.view(cuda.int64), f.view(cuda.int64))


def test_batch_autotuner_picks_a_candidate(f3d, ctx, cuda):
    """With 8 or more instances the autotuner runs once per size mix, on
    copies (the caller's fields are solved once, with the chosen
    configuration) and reports one of its candidates."""
    inst = _batch_instances(cuda, 10, 20, 48, seed=12)
    o = f3d.opts(max_sweeps=300, tol=1e-10)
    fields = [T.clone() for T, _ in inst]
    f3d.solve_batch(ctx, fields, [10.0] * len(inst), [M for _, M in inst], o)
    rows, ctas = f3d.batch_get_config(ctx)
    assert rows in (2, 4, 8) and ctas >= 1
    for (T, M), f in zip(inst, fields):
        t = T.clone()
        f3d.solve_ellip(ctx, t, 10.0, M, o)
        assert cuda.equal(t.view(cuda.int64), f.view(cuda.int64))


def test_batch_rejects_bad_input(f3d, ctx, cuda):
    L = f3d.lib()
    assert L.fold3d_solve_batch(ctx._h, 0, None, C.byref(f3d.opts()), None, None) == f3d.ERR_INVALID


# -- adjoint of the elliptical solver ----------------------------------------

_DIAG_OF = {0: (0, 0), 1: (0, 3), 2: (0, 5), 3: (3, 3), 4: (3, 5), 5: (5, 5)}


def _fd_pair(base, comp, k, j, i, rel=1e-6):
    """Metric component comp of cell (k, j, i) moved up and down by rel times
    the cell's metric scale sqrt(M_ii M_jj) (the entry itself for diagonal
    entries; off-diagonal entries can be many orders smaller than the
    metric, so a step relative to them alone drowns in rounding of the loss).
    Returns the two float64 metrics and the float32 difference applied."""
    a, b = _DIAG_OF[comp]
    scale = (float(base[a][k, j, i]) * float(base[b][k, j, i])) ** 0.5
    v = float(base[comp][k, j, i])
    up, dn = base[comp].clone(), base[comp].clone()
    up[k, j, i] = v + rel * scale
    dn[k, j, i] = v - rel * scale
    dv = float(up[k, j, i]) - float(dn[k, j, i])
    Mu = [x.double() if c != comp else up.double() for c, x in enumerate(base)]
    Md = [x.double() if c != comp else dn.double() for c, x in enumerate(base)]
    return Mu, Md, dv

def _adj_case(cuda, dims=(23, 19, 27), seed=4, src=(12, 9, 5)):
    import media

    M = media.heterogeneous_tti(*dims, 10.0, seed=seed)
    T0 = torch_point_dims(cuda, dims, src)
    rec = (slice(1, 2), slice(1, -1, 2), slice(1, -1, 2))  # receivers on the k = 1 face
    return M, T0, rec


def test_winner_record_matches_oracle(f3d, orc, ctx, cuda):
    M, T0, _ = _adj_case(cuda)
    Md = [m.cuda() for m in M]
    T = T0.clone()
    W = cuda.empty(T.shape, dtype=cuda.uint8, device="cuda")
    rep = f3d.solve_ellip_record(ctx, T, 10.0, Md, W, f3d.opts(max_sweeps=300, tol=0.0))
    ref = T0.cpu().numpy()
    s, d, Wref = orc.ell_solve_rec(ref, [m.numpy() for m in M], (10.0,) * 3, 300, tol=0.0)
    assert rep.sweeps == s
    assert_bitwise(T.cpu().numpy(), ref, "field")
    assert np.array_equal(W.cpu().numpy(), Wref)
    assert (Wref != 0xFF).sum() > 0.9 * Wref[1:-1, 1:-1, 1:-1].size


def test_adjoint_matches_cpu_adjoint(f3d, orc, ctx, cuda):
    """lambda and dL/dM of the GPU adjoint against the FP64 CPU adjoint (which
    processes cells by decreasing time and finds the winner graph causal)."""
    M, T0, rec = _adj_case(cuda)
    Md = [m.cuda() for m in M]
    T = T0.clone()
    W = cuda.empty(T.shape, dtype=cuda.uint8, device="cuda")
    f3d.solve_ellip_record(ctx, T, 10.0, Md, W, f3d.opts(max_sweeps=300, tol=0.0))
    r = cuda.zeros_like(T)
    r[rec] = T[rec] * 0.01 + 1.0
    lam = cuda.full_like(T, float("nan"))
    g = cuda.full((6,) + tuple(T.shape), float("nan"), dtype=cuda.float64, device="cuda")  # every cell is written
    rep = f3d.adjoint_ellip(ctx, T, 10.0, Md, W, r, lam, g)
    assert rep.max_delta == 0.0 and rep.sweeps >= 2
    lr, gr, nc = orc.ell_adjoint(T.cpu().numpy(), [m.numpy() for m in M], (10.0,) * 3,
                                 W.cpu().numpy(), r.cpu().numpy())
    assert nc == 0
    np.testing.assert_allclose(lam.cpu().numpy(), lr, rtol=1e-9, atol=1e-12)
    np.testing.assert_allclose(g.cpu().numpy(), gr, rtol=1e-9, atol=1e-12 * np.abs(gr).max())


def test_adjoint_matches_finite_differences(f3d, ctx, cuda):
    """dL/dM from the adjoint against central differences of the loss
    L = 1/2 sum over receivers (T - t_obs)^2, step 1e-6 relative (of the
    cell's metric scale) on the solver's own float32 metric entries, divided
    by the float32 difference actually applied, at 32 random cells."""
    import tomo

    M, T0, rec = _adj_case(cuda)
    Md = [m.double().cuda().requires_grad_(True) for m in M]
    T = tomo.solve(T0, 10.0, Md)
    tobs = (T[rec] * 0.97).detach()
    L = 0.5 * ((T[rec] - tobs) ** 2).sum()
    L.backward()
    G = [m.grad for m in Md]

    def loss(Mx):
        with cuda.no_grad():
            Tx = tomo.solve(T0, 10.0, Mx)
            return float(0.5 * ((Tx[rec] - tobs) ** 2).sum())

    rng = np.random.default_rng(7)
    base = [m.detach().float().cuda() for m in Md]
    cand = cuda.nonzero(G[0].abs() > 0).cpu().numpy()
    errs = []
    for q in rng.choice(len(cand), 32, replace=False):
        k, j, i = (int(v) for v in cand[q])
        comp = int(rng.integers(0, 6))
        Mu, Md, dv = _fd_pair(base, comp, k, j, i)
        fd = (loss(Mu) - loss(Md)) / dv
        ad = float(G[comp][k, j, i])
        errs.append(abs(fd - ad) / max(abs(ad), abs(fd), 1e-300))
    assert np.median(errs) < 1e-6 and max(errs) < 1e-4, (np.median(errs), max(errs))


def test_adjoint_chain_to_slowness_and_epsilon(cuda):
    """Through torch's chain rule, gradients with respect to per-cell
    slowness and epsilon agree with central differences (relative step 1e-3:
    the metric is stored as float32, so smaller steps in these parameters are
    lost to rounding)."""
    import math

    import media
    import tomo

    dims, h = (21, 17, 19), 10.0
    nx, ny, nz = dims
    shape = (nz + 2, ny + 2, nx + 2)
    gen = cuda.Generator(device="cpu").manual_seed(3)
    s0 = (1.0 / (1800.0 + 400.0 * cuda.rand(shape, generator=gen, dtype=cuda.float64))).cuda()
    e0 = (0.2 * cuda.rand(shape, generator=gen, dtype=cuda.float64)).cuda()
    th, ph = math.radians(25.0), math.radians(60.0)
    axis = tuple(cuda.full(shape, v, dtype=cuda.float64, device="cuda")
                 for v in (math.sin(th) * math.cos(ph), math.sin(th) * math.sin(ph), math.cos(th)))
    T0 = torch_point_dims(cuda, dims, (11, 9, 3))
    rec = (slice(1, 2), slice(1, -1, 2), slice(1, -1, 2))

    def metric(s, e):
        return [m.double() for m in media.metric_from(1.0 / s, e, axis)]

    s = s0.clone().requires_grad_(True)
    e = e0.clone().requires_grad_(True)
    T = tomo.solve(T0, h, metric(s, e))
    tobs = (T[rec] * 0.98).detach()
    (0.5 * ((T[rec] - tobs) ** 2).sum()).backward()

    def loss(sv, ev):
        with cuda.no_grad():
            Tx = tomo.solve(T0, h, metric(sv, ev))
            return float(0.5 * ((Tx[rec] - tobs) ** 2).sum())

    rng = np.random.default_rng(1)
    cells = cuda.nonzero(s.grad.abs() > 1e-3 * s.grad.abs().max()).cpu().numpy()
    for q in rng.choice(len(cells), 8, replace=False):
        k, j, i = (int(v) for v in cells[q])
        for var, g, base in (("s", s.grad, s0), ("eps", e.grad, e0)):
            step = 1e-3 * float(base[k, j, i]) if float(base[k, j, i]) != 0 else 1e-4
            up, dn = base.clone(), base.clone()
            up[k, j, i] += step
            dn[k, j, i] -= step
            fd = (loss(up, e0) - loss(dn, e0)) / (2 * step) if var == "s" else \
                (loss(s0, up) - loss(s0, dn)) / (2 * step)
            ad = float(g[k, j, i])
            assert abs(fd - ad) <= 2e-2 * max(abs(ad), abs(fd)) + 1e-9 * float(g.abs().max()), (var, fd, ad)


def test_adjoint_finite_differences_256(f3d, cuda):
    """Full tomography size: 256^3 seeded heterogeneous TTI medium (seed 2),
    one source 10 cells below the top face, 4096 receivers on the top face.
    dL/dM from the adjoint against central differences (1e-6 relative to
    the cell's metric scale, float32-exact, on the solver's metric entries)
    at 32 random cells among those whose gradient is at least 1e-3 of the
    largest.  Median relative error below 1e-6; every sample below 1e-5 (the
    rounding of a loss summed over 4096 receivers is a few 1e-16 of it,
    against differences of about 1e-10 of it)."""
    import media
    import tomo

    n, h = 256, 10.0
    M = [m.double().requires_grad_(True) for m in media.heterogeneous_tti(n, n, n, h, seed=2, device="cuda")]
    T0 = cuda.full((n + 2,) * 3, MAXT, dtype=cuda.float64, device="cuda")
    T0[11, 100, 140] = 0.0
    ridx = cuda.arange(3, n + 1, 4, device="cuda")
    rec = (1, ridx.view(-1, 1), ridx.view(1, -1))
    T = tomo.solve(T0, h, M)
    tobs = (T[rec] * 0.97).detach()
    (0.5 * ((T[rec] - tobs) ** 2).sum()).backward()
    G = [m.grad for m in M]

    def loss(Mx):
        with cuda.no_grad():
            Tx = tomo.solve(T0, h, Mx)
            return float(0.5 * ((Tx[rec] - tobs) ** 2).sum())

    base = [m.detach().float() for m in M]
    gmax = max(float(g.abs().max()) for g in G)
    rng = np.random.default_rng(11)
    errs = []
    for q in range(32):
        comp = int(rng.integers(0, 6))
        cand = cuda.nonzero(G[comp].abs() >= 1e-3 * gmax)
        k, j, i = (int(v) for v in cand[int(rng.integers(0, len(cand)))].tolist())
        Mu, Md, dv = _fd_pair(base, comp, k, j, i)
        fd = (loss(Mu) - loss(Md)) / dv
        ad = float(G[comp][k, j, i])
        errs.append(abs(fd - ad) / max(abs(ad), abs(fd)))
    assert np.median(errs) < 1e-6 and max(errs) < 1e-5, (np.median(errs), max(errs))


def test_adjoint_tolerance_stops_early(f3d, ctx, cuda):
    """A relative tolerance ends the backward sweeps early with the gradient
    still within ~1e-9 of the exact (tol 0) one."""
    M, T0, rec = _adj_case(cuda, dims=(40, 36, 44), seed=9, src=(20, 18, 6))
    Md = [m.cuda() for m in M]
    T = T0.clone()
    W = cuda.empty(T.shape, dtype=cuda.uint8, device="cuda")
    f3d.solve_ellip_record(ctx, T, 10.0, Md, W, f3d.opts(max_sweeps=300, tol=0.0))
    r = cuda.zeros_like(T)
    r[rec] = 1.0
    out = {}
    for tol in (0.0, 1e-12):
        lam = cuda.empty_like(T)
        g = cuda.empty((6,) + tuple(T.shape), dtype=cuda.float64, device="cuda")
        out[tol] = (f3d.adjoint_ellip(ctx, T, 10.0, Md, W, r, lam, g, tol=tol), g)
    assert out[1e-12][0].sweeps <= out[0.0][0].sweeps
    assert out[0.0][0].max_delta == 0.0
    err = float((out[1e-12][1] - out[0.0][1]).norm() / out[0.0][1].norm())
    assert err < 1e-9, err


def _batch_sources(cuda, dims, srcs, seed):
    import media

    M = [m.cuda() for m in media.heterogeneous_tti(*dims, 10.0, seed=seed)]
    nx, ny, nz = dims
    T0 = cuda.full((len(srcs), nz + 2, ny + 2, nx + 2), MAXT, dtype=cuda.float64, device="cuda")
    for s, (i, j, k) in enumerate(srcs):
        T0[s, k, j, i] = 0.0
    return M, T0


def test_batch_records_equal_single_records(f3d, ctx, cuda):
    """Batched recording solves of grids of different sizes: fields and winner
    records equal those of one-by-one recording solves, bit for bit."""
    import media

    cases = [((30, 22, 26), (7, 9, 4), 11), ((19, 33, 24), (15, 3, 20), 12), ((41, 17, 20), (30, 9, 10), 13)]
    Ms, Ts, Ws = [], [], []
    for dims, src, seed in cases:
        M = [m.cuda() for m in media.heterogeneous_tti(*dims, 10.0, seed=seed)]
        nx, ny, nz = dims
        T = cuda.full((nz + 2, ny + 2, nx + 2), MAXT, dtype=cuda.float64, device="cuda")
        T[src[2], src[1], src[0]] = 0.0
        Ms.append(M)
        Ts.append(T)
        Ws.append(cuda.empty(T.shape, dtype=cuda.uint8, device="cuda"))
    o = f3d.opts(max_sweeps=300, tol=1e-10)
    Tb = [t.clone() for t in Ts]
    f3d.solve_batch(ctx, Tb, [10.0] * 3, Ms, o, winners=Ws)
    for T, M, Tbat, Wbat in zip(Ts, Ms, Tb, Ws):
        W1 = cuda.empty(T.shape, dtype=cuda.uint8, device="cuda")
        T1 = T.clone()
        f3d.solve_ellip_record(ctx, T1, 10.0, M, W1, o)
        assert_bitwise(Tbat.cpu().numpy(), T1.cpu().numpy(), "batched field")
        assert cuda.equal(Wbat, W1)


def test_batch_adjoint_grouped_x_passes_match_single_adjoints(f3d, ctx, cuda):
    """Eight sources in one medium whose x-normal planes are large (300^2
    cells): the batched adjoint runs its x-normal backward passes over groups
    of instances (one launch per group, sized to share L2), and every
    source's lambda and dL/dM still equal its own adjoint's to rounding."""
    dims = (30, 300, 296)
    rng = np.random.default_rng(4)
    srcs = [(int(rng.integers(1, 31)), int(rng.integers(1, 301)), int(rng.integers(1, 297))) for _ in range(8)]
    import media

    M = media.heterogeneous_tti(*dims, 10.0, seed=23, device="cuda")  # built on the GPU (a flat grid)
    nx, ny, nz = dims
    T0 = cuda.full((len(srcs), nz + 2, ny + 2, nx + 2), MAXT, dtype=cuda.float64, device="cuda")
    for q, (i, j, k) in enumerate(srcs):
        T0[q, k, j, i] = 0.0
    S = len(srcs)
    T = T0.clone()
    W = cuda.empty(T.shape, dtype=cuda.uint8, device="cuda")
    f3d.solve_batch(ctx, [T[s] for s in range(S)], [10.0] * S, [M] * S, f3d.opts(max_sweeps=300, tol=0.0),
                    winners=[W[s] for s in range(S)])
    r = cuda.zeros_like(T)
    r[:, 1, 1:-1:7, 1:-1:7] = T[:, 1, 1:-1:7, 1:-1:7] * 0.01
    shape = tuple(T.shape[1:])
    lamb = cuda.full_like(T, float("nan"))
    gb = cuda.full((S, 6) + shape, float("nan"), dtype=cuda.float64, device="cuda")
    f3d.adjoint_batch(ctx, [T[s] for s in range(S)], [10.0] * S, [M] * S, [W[s] for s in range(S)],
                      [r[s] for s in range(S)], [lamb[s] for s in range(S)], [gb[s] for s in range(S)])
    for s in range(S):
        lam = cuda.empty(shape, dtype=cuda.float64, device="cuda")
        g = cuda.empty((6,) + shape, dtype=cuda.float64, device="cuda")
        f3d.adjoint_ellip(ctx, T[s], 10.0, M, W[s], r[s].contiguous(), lam, g)
        assert cuda.allclose(lamb[s], lam, rtol=1e-12, atol=0), s
        assert cuda.allclose(gb[s], g, rtol=1e-12, atol=1e-12 * float(g.abs().max())), s


def test_batch_adjoint_matches_single_adjoints(f3d, ctx, cuda):
    """fold3d_adjoint_batch equals fold3d_adjoint_ellip per source (to the
    rounding of the atomic sums), and with accumulate its shared dL/dM is the
    sum over sources."""
    dims = (28, 24, 30)
    srcs = [(5, 6, 4), (20, 12, 4), (14, 20, 8), (9, 3, 25)]
    M, T0 = _batch_sources(cuda, dims, srcs, seed=21)
    S = len(srcs)
    T = T0.clone()
    W = cuda.empty(T.shape, dtype=cuda.uint8, device="cuda")
    f3d.solve_batch(ctx, [T[s] for s in range(S)], [10.0] * S, [M] * S, f3d.opts(max_sweeps=300, tol=0.0),
                    winners=[W[s] for s in range(S)])
    r = cuda.zeros_like(T)
    r[:, 1, 1:-1:2, 1:-1:2] = T[:, 1, 1:-1:2, 1:-1:2] * 0.01
    shape = tuple(T.shape[1:])
    lam1, g1 = [], []
    for s in range(S):
        lam = cuda.empty(shape, dtype=cuda.float64, device="cuda")
        g = cuda.empty((6,) + shape, dtype=cuda.float64, device="cuda")
        f3d.adjoint_ellip(ctx, T[s], 10.0, M, W[s], r[s].contiguous(), lam, g)
        lam1.append(lam)
        g1.append(g)
    lamb = cuda.full_like(T, float("nan"))
    gb = cuda.full((S, 6) + shape, float("nan"), dtype=cuda.float64, device="cuda")
    reps = f3d.adjoint_batch(ctx, [T[s] for s in range(S)], [10.0] * S, [M] * S, [W[s] for s in range(S)],
                             [r[s] for s in range(S)], [lamb[s] for s in range(S)], [gb[s] for s in range(S)])
    assert all(rep.max_delta == 0.0 for rep in reps)
    for s in range(S):
        assert cuda.allclose(lamb[s], lam1[s], rtol=1e-12, atol=0), s
        assert cuda.allclose(gb[s], g1[s], rtol=1e-12, atol=1e-12 * float(g1[s].abs().max())), s
    acc = cuda.zeros((6,) + shape, dtype=cuda.float64, device="cuda")
    f3d.adjoint_batch(ctx, [T[s] for s in range(S)], [10.0] * S, [M] * S, [W[s] for s in range(S)],
                      [r[s] for s in range(S)], [lamb[s] for s in range(S)], [acc] * S, accumulate=True)
    total = sum(g1)
    assert cuda.allclose(acc, total, rtol=1e-12, atol=1e-12 * float(total.abs().max()))


def test_batched_autograd_matches_per_source(cuda):
    """tomo.solve_batch (batched forward and adjoint) gives the fields and the
    gradient of the per-source tomo.solve calls."""
    import tomo

    dims = (26, 22, 24)
    srcs = [(4, 5, 3), (20, 17, 3), (13, 11, 6)]
    M, T0 = _batch_sources(cuda, dims, srcs, seed=31)
    rec = (slice(None), 1, slice(1, -1, 2), slice(1, -1, 2))
    Mb = [m.double().requires_grad_(True) for m in M]
    Tb = tomo.solve_batch(T0, 10.0, Mb)
    (0.5 * (Tb[rec] * 0.03) ** 2).sum().backward()
    Ms = [m.double().requires_grad_(True) for m in M]
    loss = 0
    for s in range(len(srcs)):
        Ts = tomo.solve(T0[s].contiguous(), 10.0, Ms)
        assert_bitwise(Tb[s].detach().cpu().numpy(), Ts.detach().cpu().numpy(), "source %d" % s)
        loss = loss + (0.5 * (Ts[rec[1:]] * 0.03) ** 2).sum()
    loss.backward()
    for a, b in zip(Mb, Ms):
        assert cuda.allclose(a.grad, b.grad, rtol=1e-11, atol=1e-12 * float(b.grad.abs().max()))


@pytest.mark.parametrize("dims,h,med", [((16, 16, 16), None, None),
                                        ((20, 13, 17), (0.5, 0.8, 0.6), (1.3, (0.2, -0.5, 0.3))),
                                        ((400, 400, 400), None, None)],
                         ids=["16-golden", "20x13x17", "400-three-slabs"])
def test_device_initialiser_matches_host(f3d, ctx, cuda, golden, dims, h, med):
    """fold3d_init_implicit_device equals the host initialiser (and so the
    reference's ImplicitInitialiser) bit for bit, ghosts included; at 400^3
    the surface reaches the device in three slabs."""
    n = dims[0]
    if h is None:
        h = (ref_spacing(n),) * 3
    m = f3d.medium(*med) if med else f3d.medium()
    ref = f3d.init_implicit(*dims, h, m)
    if dims == (16, 16, 16):
        assert_bitwise(ref, golden[16]["init"], "host init")
    T = cuda.empty(ref.shape, dtype=cuda.float64, device="cuda")
    f3d.init_implicit_device(ctx, T, h, m)
    assert_bitwise(T.cpu().numpy(), ref, "device init")


# -- float32 build of the elliptical solver -----------------------------------

@pytest.mark.parametrize("kind,dims,src", [("homog", (40, 40, 40), (21, 21, 21)),
                                           ("tti", (37, 29, 33), (5, 20, 9))])
def test_ellip_f32_matches_float_oracle(f3d, orc, ctx, cuda, kind, dims, src):
    """The float32 build on the GPU equals the oracle's float statement bit
    for bit (fields and winner records), after 3 fixed sweeps and when run
    until nothing changes."""
    h = (10.0, 10.0, 10.0)
    M = _ell_case(kind, dims, h[0])
    Md = [m.cuda() for m in M]
    Mh = [m.numpy() for m in M]
    T0 = orc.init_point(*dims, src).astype(np.float32)
    for fixed, sweeps, tol in ((True, 3, 0.0), (False, 300, 0.0)):
        ref = T0.copy()
        s_ref, d_ref, W_ref = orc.ellf_solve_rec(ref, Mh, h, sweeps, tol=(-1.0 if fixed else tol))
        d = cuda.from_numpy(T0.copy()).cuda()
        W = cuda.empty(d.shape, dtype=cuda.uint8, device="cuda")
        rep = f3d.solve_ellip_record(ctx, d, h, Md, W, f3d.opts(max_sweeps=sweeps, fixed=fixed, tol=tol))
        assert rep.sweeps == s_ref
        out = d.cpu().numpy()
        assert np.array_equal(out.view(np.uint32), ref.view(np.uint32)), \
            "%d cells differ" % int((out.view(np.uint32) != ref.view(np.uint32)).sum())
        assert np.array_equal(W.cpu().numpy(), W_ref)


def test_adjoint_f32_matches_cpu_adjoint(f3d, orc, ctx, cuda):
    """The float32 adjoint against the FP64 CPU adjoint of the same (float)
    field and winner record, within float rounding."""
    M, T0, rec = _adj_case(cuda)
    Md = [m.cuda() for m in M]
    T = T0.float().clone()
    W = cuda.empty(T.shape, dtype=cuda.uint8, device="cuda")
    f3d.solve_ellip_record(ctx, T, 10.0, Md, W, f3d.opts(max_sweeps=300, tol=0.0))
    r = cuda.zeros_like(T)
    r[rec] = T[rec] * 0.01 + 1.0
    lam = cuda.empty_like(T)
    g = cuda.empty((6,) + tuple(T.shape), dtype=cuda.float32, device="cuda")
    rep = f3d.adjoint_ellip(ctx, T, 10.0, Md, W, r, lam, g)
    assert rep.max_delta == 0.0
    lr, gr, nc = orc.ell_adjoint(T.double().cpu().numpy(), [m.numpy() for m in M], (10.0,) * 3,
                                 W.cpu().numpy(), r.double().cpu().numpy())
    assert nc == 0
    lam_h, g_h = lam.double().cpu().numpy(), g.double().cpu().numpy()
    assert np.abs(lam_h - lr).max() <= 1e-4 * np.abs(lr).max()
    assert np.linalg.norm(g_h - gr) <= 1e-4 * np.linalg.norm(gr)


def test_batch_f32_equals_one_by_one(f3d, ctx, cuda):
    import media

    cases = [((30, 22, 26), (7, 9, 4), 41), ((19, 33, 24), (15, 3, 20), 42)]
    Ms, Ts = [], []
    for dims, src, seed in cases:
        Ms.append([m.cuda() for m in media.heterogeneous_tti(*dims, 10.0, seed=seed)])
        nx, ny, nz = dims
        T = cuda.full((nz + 2, ny + 2, nx + 2), MAXT, dtype=cuda.float32, device="cuda")
        T[src[2], src[1], src[0]] = 0.0
        Ts.append(T)
    o = f3d.opts(max_sweeps=300, tol=0.0)
    Tb = [t.clone() for t in Ts]
    f3d.solve_batch(ctx, Tb, [10.0] * 2, Ms, o)
    for T, M, Tbat in zip(Ts, Ms, Tb):
        T1 = T.clone()
        f3d.solve_ellip(ctx, T1, 10.0, M, o)
        assert cuda.equal(Tbat.view(cuda.int32), T1.view(cuda.int32))


def test_batched_autograd_f32_close_to_f64(cuda):
    """The float32 build through tomo.solve_batch: fields within float
    rounding of the float64 build, gradients close (winners can differ where
    candidates tie within float rounding)."""
    import tomo

    dims = (26, 22, 24)
    srcs = [(4, 5, 3), (20, 17, 3)]
    M, T0 = _batch_sources(cuda, dims, srcs, seed=51)
    rec = (slice(None), 1, slice(1, -1, 2), slice(1, -1, 2))
    out = {}
    for dt in (cuda.float64, cuda.float32):
        Mx = [m.double().requires_grad_(True) for m in M]
        T = tomo.solve_batch(T0.to(dt), 10.0, Mx)
        (0.5 * (T[rec].double() * 0.03) ** 2).sum().backward()
        out[dt] = (T.detach().double(), [m.grad for m in Mx])
    (T64, g64), (T32, g32) = out[cuda.float64], out[cuda.float32]
    I = (slice(None), slice(1, -1), slice(1, -1), slice(1, -1))
    assert float(((T32 - T64)[I]).abs().max() / T64[I].abs().max()) < 1e-6
    num = sum(float((a - b).norm()) ** 2 for a, b in zip(g32, g64)) ** 0.5
    den = sum(float(b.norm()) ** 2 for b in g64) ** 0.5
    assert num <= 2e-2 * den, num / den


# -- the variants compiled for large planes -----------------------------------

def test_large_plane_variant_drift_matches_planes(f3d, ctx, cuda):
    """Planes of >= 8192 tiles (here the k-planes of 1024 x 1040) run the
    kernel variant compiled for large planes; 8 sweeps equal the PLANES
    engine bit for bit."""
    dims = (1024, 1040, 5)
    h = (0.01, 0.011, 0.012)
    T0 = f3d.init_point(*dims, (500, 600, 3))
    out = {}
    for eng in ("planes", "wavefront"):
        d = cuda.from_numpy(T0.copy()).cuda()
        e = f3d.ENGINE_PLANES if eng == "planes" else f3d.ENGINE_WAVEFRONT
        ctx.solve(d, h, None, f3d.opts(max_sweeps=8, fixed=True, engine=e))
        out[eng] = d.cpu().numpy()
    assert_bitwise(out["wavefront"], out["planes"], "large-plane variant")


@pytest.mark.parametrize("dtype", ["f64", "f32"])
def test_large_plane_variant_ellip_matches_oracle(f3d, orc, ctx, cuda, dtype):
    """The elliptical solver's large-plane variants (float64 and float32)
    against the CPU statements, 3 sweeps.  The medium is built on the GPU:
    torch's CPU irfftn crashes on such flat shapes (4 or 6 planes of
    1040 x 1024)."""
    import media

    dims = (1024, 1040, 4)
    h = (10.0, 10.0, 10.0)
    Md = media.heterogeneous_tti(*dims, 10.0, seed=61, device="cuda")
    Mh = [m.cpu().numpy() for m in Md]
    T0 = orc.init_point(*dims, (300, 700, 2))
    if dtype == "f32":
        T0 = T0.astype(np.float32)
        ref = T0.copy()
        orc.ellf_solve_rec(ref, Mh, h, 3, tol=-1.0)
    else:
        ref = T0.copy()
        orc.ell_solve(ref, Mh, h, 3, tol=-1.0)
    d = cuda.from_numpy(T0.copy()).cuda()
    f3d.solve_ellip(ctx, d, h, Md, f3d.opts(max_sweeps=3, fixed=True))
    out = d.cpu().numpy()
    w = np.uint32 if dtype == "f32" else np.uint64
    assert np.array_equal(out.view(w), ref.view(w)), int((out.view(w) != ref.view(w)).sum())
