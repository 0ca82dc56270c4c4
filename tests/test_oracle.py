"""CPU tests: the oracle pinned against the reference's own outputs, and the
product's host-side initialiser checked against both."""
import hashlib
import os

import numpy as np
import pytest

from conftest import assert_bitwise

from oracle import MAXT, REF_A, REF_F, ref_spacing


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


@pytest.mark.parametrize("n", [8, 16])
def test_oracle_init_matches_reference(orc, golden, n):
    h = ref_spacing(n)
    T = orc.init_implicit(n, n, n, (h, h, h))
    assert_bitwise(T, golden[n]["init"], "init n=%d" % n)
    assert orc.overfull_voxels() == 0


@pytest.mark.parametrize("n", [8, 16])
def test_oracle_sweeps_match_reference(orc, golden, n):
    h = (ref_spacing(n),) * 3
    T = golden[n]["init"].copy()
    orc.solve(T, h, 1)
    assert_bitwise(T, golden[n]["s1"], "1 sweep")
    orc.solve(T, h, 1)
    assert_bitwise(T, golden[n]["s2"], "2 sweeps")
    orc.solve(T, h, 6)
    assert_bitwise(T, golden[n]["s8"], "8 sweeps")


@pytest.mark.parametrize("n", [8, 16])
def test_oracle_point_source_matches_reference(orc, golden, n):
    h = (ref_spacing(n),) * 3
    c = n // 2 + 1
    T = orc.init_point(n, n, n, (c, c, c))
    orc.solve(T, h, 8)
    assert_bitwise(T, golden[n]["point_s8"], "point source")


@pytest.mark.parametrize("n", [32, 37, 64, 99])
def test_oracle_digests_match_reference(orc, digests, n):
    h = (ref_spacing(n),) * 3
    T = orc.init_implicit(n, n, n, h)
    assert sha(T) == digests["n%d_init" % n]
    orc.solve(T, h, 8)
    assert sha(T) == digests["n%d_s8" % n]
    c = n // 2 + 1
    P = orc.init_point(n, n, n, (c, c, c))
    orc.solve(P, h, 8)
    assert sha(P) == digests["n%d_point_s8" % n]


@pytest.mark.parametrize("n", [37, 99])
@pytest.mark.parametrize("name,src", [("corner_point", lambda n: (2, 1, 2)),
                                      ("face_point", lambda n: (n, n // 3 + 1, 2 * n // 3 + 1))])
def test_oracle_off_centre_point_sources_match_reference(orc, digests, n, name, src):
    """Point sources next to a corner and on a face (the reference's own
    sweeps from the same field, tests/golden/make_golden.py), 8 sweeps."""
    h = (ref_spacing(n),) * 3
    P = orc.init_point(n, n, n, src(n))
    orc.solve(P, h, 8)
    assert sha(P) == digests["n%d_%s_s8" % (n, name)]


def test_oracle_reproduces_reference_text_dump_128(orc, digests):
    """The reference program's own output file at 128^3 after 8 sweeps
    (AN_ISO_1_OpenACC.c:1244-1260: '%f' per value, i outermost, k innermost)."""
    n = 128
    h = (ref_spacing(n),) * 3
    T = orc.init_implicit(n, n, n, h)
    orc.solve(T, h, 8)
    vals = T.transpose(2, 1, 0).reshape(-1)  # i outer, j, k inner
    text = ("%f\n" * vals.size) % tuple(vals.tolist())
    assert hashlib.md5(text.encode()).hexdigest() == digests["n128_s8_text_md5"]


def test_oracle_exact_time_and_convergence(orc):
    """Closed form (Fold3dPMM.c:9-26) agrees with a PMM point-source solve to
    discretisation accuracy, and the convergence test stops the solve."""
    n = 24
    h = (10.0 / (n - 1),) * 3
    c = n // 2 + 1
    T = orc.init_point(n, n, n, (c, c, c))
    sweeps, delta = orc.solve(T, h, 200, tol=0.0)
    assert delta == 0.0 and sweeps < 200
    k, j, i = np.meshgrid(*(np.arange(n + 2),) * 3, indexing="ij")
    errs = []
    for (kk, jj, ii) in [(c + 5, c - 3, c + 2), (c - 6, c + 4, c - 7), (c + 8, c + 8, c - 8)]:
        x, y, z = (ii - c) * h[0], (jj - c) * h[1], (kk - c) * h[2]
        exact = orc.fold_from_point(REF_F, *REF_A, x, y, z)
        errs.append(abs(abs(T[kk, jj, ii]) - exact) / exact)
    assert max(errs) < 0.15


def test_oracle_noncubic_runs(orc):
    nx, ny, nz = 9, 6, 7
    h = (0.7, 0.9, 1.1)
    T = orc.init_implicit(nx, ny, nz, h)
    s, d = orc.solve(T, h, 50, tol=0.0)
    assert d == 0.0
    assert np.all(np.isfinite(T))


# -- the product's host-side initialiser ------------------------------------

@pytest.mark.parametrize("n", [8, 16])
def test_product_init_matches_reference(f3d, golden, n):
    h = ref_spacing(n)
    T = f3d.init_implicit(n, n, n, h)
    assert_bitwise(T, golden[n]["init"], "product init n=%d" % n)


@pytest.mark.parametrize("n", [37, 64, 99])
def test_product_init_digest(f3d, digests, n):
    T = f3d.init_implicit(n, n, n, ref_spacing(n))
    assert sha(T) == digests["n%d_init" % n]


@pytest.mark.parametrize("dims,h", [((9, 6, 7), (0.7, 0.9, 1.1)), ((20, 13, 17), (0.5, 0.8, 0.6)),
                                    ((24, 17, 19), (0.5, 0.25, 0.75))])  # the last: few distinct x + y
def test_product_init_noncubic_matches_oracle(f3d, orc, dims, h):
    med = f3d.medium(1.3, (0.2, -0.5, 0.3))
    T = f3d.init_implicit(*dims, h, med)
    R = orc.init_implicit(*dims, h, F=1.3, a=(0.2, -0.5, 0.3))
    assert_bitwise(T, R, "non-cubic init")


def test_product_init_thread_count_invariant(f3d, monkeypatch):
    n = 30
    monkeypatch.setenv("FOLD3D_HOST_THREADS", "1")
    A = f3d.init_implicit(n, n, n, ref_spacing(n))
    monkeypatch.setenv("FOLD3D_HOST_THREADS", "7")
    B = f3d.init_implicit(n, n, n, ref_spacing(n))
    assert_bitwise(A, B, "threads")


def test_product_scalar_helpers_match_reference(f3d):
    from oracle import RefLib

    r = RefLib(8)
    L = f3d.lib()
    rng = np.random.default_rng(3)
    for _ in range(200):
        x, y, z = rng.uniform(-6, 12, 3)
        assert L.ImpSurfF(x, y, z) == r.L.ImpSurfF(x, y, z)
        a = rng.uniform(-0.6, 0.6, 3)
        assert L.InitFoldFromPoint(1.1, *a, x, y, z) == r.L.InitFoldFromPoint(1.1, *a, x, y, z)
    assert L.InitFoldFromPoint(1.1, *REF_A, 0.0, 0.0, 0.0) == MAXT


def test_product_node_helpers_match_reference(f3d):
    """InitNode and updateVoxel (Fold3dPMM.c:35-112) and the coordinate
    helpers x, y, z (:115-126) against the reference's own build at 8^3,
    bit for bit, on fields of both signs; the pitch comes from
    fold3d_compat_set_grid, then from the last ImplicitInitialiser call."""
    import ctypes as C

    from oracle import RefLib

    n = 8
    r = RefLib(n)
    L = f3d.lib()
    rng = np.random.default_rng(11)
    h = ref_spacing(n)
    try:
        for how in ("set_grid", "initialiser"):
            if how == "set_grid":
                assert L.fold3d_compat_set_grid(n, n, n) == 0
            else:
                assert L.fold3d_compat_set_grid(0, 0, 0) == 0
                scratch = np.empty((n + 2,) * 3)
                L.ImplicitInitialiser(scratch.ctypes.data_as(C.c_void_p), n, n, n, h, h, h)
            A = np.where(rng.random((n + 2,) * 3) < 0.5, -MAXT, MAXT)
            B = A.copy()
            pa, pb = A.ctypes.data_as(C.c_void_p), B.ctypes.data_as(C.c_void_p)
            for _ in range(40):
                i, j, k = (int(v) for v in rng.integers(2, n - 1, 3))
                xp, yp, zp = rng.uniform(-1.5, 1.5, 3) * h
                L.InitNode(xp, yp, zp, i, j, k, pa)
                r.L.InitNode.argtypes = L.InitNode.argtypes
                r.L.InitNode(xp, yp, zp, i, j, k, pb)
                hh = rng.uniform(0.5, 2.0, 3) * h
                L.updateVoxel(pa, i, j, k, xp, yp, zp, *hh)
                r.L.updateVoxel.argtypes = L.updateVoxel.argtypes
                r.L.updateVoxel(pb, i, j, k, xp, yp, zp, *hh)
            assert_bitwise(A, B, how)
            assert np.abs(A).min() < MAXT
    finally:
        L.fold3d_compat_set_grid(0, 0, 0)
    for name in ("x", "y", "z"):
        fr = getattr(r.L, name)
        fr.argtypes, fr.restype = [C.c_int, C.c_double], C.c_double
        for q in range(-1, n + 3):
            assert getattr(L, name)(q, 0.37) == fr(q, 0.37)


def test_reference_header_program_links_to_library_alone(f3d, tmp_path):
    """A C program written against the reference's own Fold3dPMM.h, calling
    all of its host functions (tests/csrc/ref_helpers.c), links against
    libfold3dpmm.so alone and prints the same bits as when it is linked
    against the reference's own build."""
    import subprocess

    from oracle import build

    if not build.reference_available():
        pytest.skip("the reference's header is not available")
    build.build_ref(8)
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    src = os.path.join(root, "tests", "csrc", "ref_helpers.c")
    inc = ["-DREF_HEADER", "-I", build.REF_DIR]
    libdir = os.path.dirname(f3d.LIB_PATH)
    ours = tmp_path / "ours"
    subprocess.run(["gcc", "-Wall", *inc, src, "-o", str(ours), "-L", libdir, "-lfold3dpmm",
                    "-Wl,-rpath," + libdir], check=True, capture_output=True)
    refdir = os.path.dirname(build.ref_lib_path(8))
    theirs = tmp_path / "theirs"
    subprocess.run(["gcc", "-Wall", *inc, src, "-o", str(theirs), "-L", refdir, "-lref",
                    "-Wl,-rpath," + refdir, "-lm"], check=True, capture_output=True)
    ldd = subprocess.run(["ldd", str(ours)], capture_output=True, text=True).stdout
    assert "libfold3dpmm.so" in ldd and "libref" not in ldd
    a = subprocess.run([str(ours)], capture_output=True, text=True, check=True).stdout
    b = subprocess.run([str(theirs)], capture_output=True, text=True, check=True).stdout
    assert len(a.splitlines()) == 7 and a == b
    # and against this library's own header
    own = tmp_path / "own"
    subprocess.run(["gcc", "-Wall", "-Werror", "-I", os.path.join(root, "include"), src, "-o", str(own), "-L",
                    libdir, "-lfold3dpmm", "-Wl,-rpath," + libdir], check=True, capture_output=True)
    assert subprocess.run([str(own)], capture_output=True, text=True, check=True).stdout == a


def test_product_point_init(f3d):
    T = f3d.init_point(5, 4, 3, (2, 3, 1))
    assert T[1, 3, 2] == 0.0
    T[1, 3, 2] = MAXT
    assert np.all(T == MAXT)


# -- elliptical (tilted) medium: the project's own solver -------------------

def _ellip_errors(T, M6, c, n, h, rmin):
    import media

    errs = []
    for kk in range(1, n + 1, 3):
        for jj in range(1, n + 1, 3):
            for ii in range(1, n + 1, 3):
                ex = media.exact_time(M6, (ii - c) * h, (jj - c) * h, (kk - c) * h)
                if ex > rmin:
                    errs.append(abs(abs(T[kk, jj, ii]) - ex) / ex)
    return max(errs), float(np.mean(errs))


def test_oracle_ellip_matches_closed_form():
    """Point source in the tilted ellipse of the 128^3 configuration (Vz 2000,
    Vx = Vy = 2400 m/s, tilt 30, azimuth 45 degrees; here 40^3, h = 10 m):
    the converged solve agrees with t = sqrt(x^T M x) to first-order accuracy
    (reported: max and mean relative error away from the source)."""
    import media
    from oracle import Oracle

    o = Oracle()
    n, h = 40, 10.0
    eps = ((2400.0 / 2000.0) ** 2 - 1.0) / 2.0
    M = [m.numpy() for m in media.homogeneous_ellip(n, n, n, 2000.0, eps, 30.0, 45.0)]
    c = n // 2 + 1
    T = o.init_point(n, n, n, (c, c, c))
    s, d = o.ell_solve(T, M, (h, h, h), 100, tol=1e-10)
    assert d <= 1e-10 and s < 10
    mx, mean = _ellip_errors(T, [M[k][c, c, c] for k in range(6)], c, n, h, 0.05)
    assert mx < 0.05 and mean < 0.02, (mx, mean)


def test_oracle_ellip_isotropic_symmetry():
    """Isotropic metric: the converged field is symmetric under the grid's
    reflections (the sweep order is not, so this checks the solver)."""
    import media
    from oracle import Oracle

    o = Oracle()
    n = 21
    M = [m.numpy() for m in media.homogeneous_ellip(n, n, n, 1500.0, 0.0, 0.0, 0.0)]
    T = o.init_point(n, n, n, (11, 11, 11))
    o.ell_solve(T, M, (5.0, 5.0, 5.0), 100, tol=0.0)
    inner = T[1:-1, 1:-1, 1:-1]
    for ax in range(3):
        assert np.allclose(inner, np.flip(inner, axis=ax), rtol=1e-12, atol=0)
    assert np.allclose(inner, inner.transpose(2, 1, 0), rtol=1e-12, atol=0)


def test_ellip_metric_helper_matches_generator(f3d):
    import math

    import media
    import torch

    th, ph = math.radians(30.0), math.radians(45.0)
    ref = media.metric_from(torch.tensor(2000.0, dtype=torch.float64), torch.tensor(0.22, dtype=torch.float64),
                            tuple(torch.tensor(v, dtype=torch.float64) for v in
                                  (math.sin(th) * math.cos(ph), math.sin(th) * math.sin(ph), math.cos(th))))
    got = f3d.ellip_metric(2000.0, 0.22, (math.sin(th) * math.cos(ph), math.sin(th) * math.sin(ph), math.cos(th)))
    assert [float(r) for r in ref] == got


def test_heterogeneous_tti_generator_is_seeded_and_spd():
    import media
    import torch

    a = media.heterogeneous_tti(24, 20, 28, 10.0, seed=0)
    b = media.heterogeneous_tti(24, 20, 28, 10.0, seed=0)
    c = media.heterogeneous_tti(24, 20, 28, 10.0, seed=1)
    assert all(torch.equal(x, y) for x, y in zip(a, b))
    assert not torch.equal(a[0], c[0])
    xx, xy, xz, yy, yz, zz = (m.double() for m in a)
    det = xx * (yy * zz - yz * yz) - xy * (xy * zz - yz * xz) + xz * (xy * yz - yy * xz)
    assert bool((xx > 0).all()) and bool((xx * yy - xy * xy > 0).all()) and bool((det > 0).all())


def test_oracle_adjoint_matches_finite_differences():
    """The FP64 CPU adjoint (winner records from the CPU solve, cells pushed
    by decreasing time) against central differences of the CPU solve: step
    1e-6 of the cell's metric scale on the float32 metric entries, divided by
    the float32 difference applied."""
    import media
    from oracle import Oracle

    o = Oracle()
    dims, h = (14, 12, 16), (10.0,) * 3
    M = [m.numpy() for m in media.heterogeneous_tti(*dims, 10.0, seed=5)]
    nx, ny, nz = dims
    T0 = o.init_point(nx, ny, nz, (7, 6, 3))
    T = T0.copy()
    s, d, W = o.ell_solve_rec(T, M, h, 300, tol=0.0)
    inner = W[1:-1, 1:-1, 1:-1]
    assert d == 0.0 and W.dtype == np.uint8
    assert (inner == 0xFF).sum() == 1 and W[3, 6, 7] == 0xFF  # only the source has no winner
    assert int(inner[inner != 0xFF].max()) < 6 * 33
    rec = (1, slice(1, -1, 2), slice(1, -1, 2))
    tobs = T[rec] * 0.97
    r = np.zeros_like(T)
    r[rec] = T[rec] - tobs
    lam, G, nc = o.ell_adjoint(T, M, h, W, r)
    assert nc == 0

    def loss(Mx):
        Tx = T0.copy()
        o.ell_solve(Tx, Mx, h, 300, tol=0.0)
        return 0.5 * float(((Tx[rec] - tobs) ** 2).sum())

    diag = {0: (0, 0), 1: (0, 3), 2: (0, 5), 3: (3, 3), 4: (3, 5), 5: (5, 5)}
    rng = np.random.default_rng(2)
    errs = []
    for _ in range(12):
        comp = int(rng.integers(0, 6))
        cand = np.argwhere(np.abs(G[comp]) >= 1e-3 * np.abs(G).max())
        k, j, i = cand[int(rng.integers(0, len(cand)))]
        a, b = diag[comp]
        step = 1e-6 * float(np.sqrt(M[a][k, j, i] * M[b][k, j, i]))
        up = [m.copy() for m in M]
        dn = [m.copy() for m in M]
        up[comp][k, j, i] = np.float32(M[comp][k, j, i] + step)
        dn[comp][k, j, i] = np.float32(M[comp][k, j, i] - step)
        dv = float(up[comp][k, j, i]) - float(dn[comp][k, j, i])
        fd = (loss(up) - loss(dn)) / dv
        errs.append(abs(fd - G[comp][k, j, i]) / max(abs(fd), abs(G[comp][k, j, i])))
    assert np.median(errs) < 1e-6 and max(errs) < 1e-4, (np.median(errs), max(errs))


# -- output files ------------------------------------------------------------

def test_text_dump_matches_reference_program_128(f3d, orc, digests, tmp_path):
    """fold3d_write_text gives the bytes of the reference program's own 128^3
    output file (md5 from the reference's run)."""
    n = 128
    h = (ref_spacing(n),) * 3
    T = orc.init_implicit(n, n, n, h)
    orc.solve(T, h, 8)
    p = tmp_path / "t.txt"
    f3d.write_text(str(p), T, h[0])
    assert hashlib.md5(p.read_bytes()).hexdigest() == digests["n128_s8_text_md5"]


def test_vtk_and_raw_round_trip(f3d, tmp_path):
    nx, ny, nz = 7, 5, 6
    h = (0.5, 0.25, 0.75)
    rng = np.random.default_rng(0)
    T = rng.standard_normal((nz + 2, ny + 2, nx + 2))
    for ghosts in (False, True):
        p = tmp_path / ("t%d.vtk" % ghosts)
        f3d.write_vtk(str(p), T, h, ghosts=ghosts)
        raw = p.read_bytes()
        head, _, data = raw.partition(b"LOOKUP_TABLE default\n")
        lines = head.decode().splitlines()
        e = 0 if ghosts else 1
        dims = (nx + 2 - 2 * e, ny + 2 - 2 * e, nz + 2 - 2 * e)
        assert lines[2] == "BINARY" and lines[3] == "DATASET STRUCTURED_POINTS"
        assert lines[4] == "DIMENSIONS %d %d %d" % dims
        assert [float(v) for v in lines[6].split()[1:]] == list(h)
        vals = np.frombuffer(data[:8 * int(np.prod(dims))], dtype=">f8").reshape(dims[::-1])
        inner = T[e:T.shape[0] - e, e:T.shape[1] - e, e:T.shape[2] - e]
        assert np.array_equal(vals, inner)
    p = tmp_path / "t.raw"
    f3d.write_raw(str(p), T, h)
    R, hr = f3d.read_raw(str(p))
    assert hr == h and np.array_equal(R.view(np.uint64), T.view(np.uint64))


def test_writers_reject_bad_paths(f3d, tmp_path):
    T = np.zeros((5, 5, 5))
    with pytest.raises(RuntimeError):
        f3d.write_raw(str(tmp_path / "no" / "such" / "dir" / "t.raw"), T, 1.0)


def test_heterogeneous_tti_float32_construction_close_to_float64():
    """The float32 construction (used for grids too large for float64
    temporaries) gives a positive-definite metric within float rounding of
    the float64 construction."""
    import media
    import torch

    a = media.heterogeneous_tti(30, 26, 34, 5.0, seed=3)
    b = media.heterogeneous_tti(30, 26, 34, 5.0, seed=3, dtype=torch.float32)
    for x, y in zip(a, b):
        assert float((x.double() - y.double()).abs().max()) <= 1e-5 * float(x.double().abs().max())
    xx, xy, xz, yy, yz, zz = (m.double() for m in b)
    det = xx * (yy * zz - yz * yz) - xy * (xy * zz - yz * xz) + xz * (xy * yz - yy * xz)
    assert bool((xx > 0).all()) and bool((xx * yy - xy * xy > 0).all()) and bool((det > 0).all())


def test_oracle_float_statement_close_to_double():
    """The oracle's float32 statement of the elliptical solver (the float32
    build's checker) converges and agrees with the FP64 statement to float
    precision; its winner codes are valid."""
    import media
    from oracle import Oracle

    o = Oracle()
    dims = (20, 18, 22)
    M = [m.numpy() for m in media.heterogeneous_tti(*dims, 10.0, seed=3)]
    T0 = o.init_point(*dims, (10, 9, 5))
    Tf, Td = T0.astype(np.float32), T0.copy()
    sf, df, Wf = o.ellf_solve_rec(Tf, M, (10.0,) * 3, 300, tol=0.0)
    sd, dd, Wd = o.ell_solve_rec(Td, M, (10.0,) * 3, 300, tol=0.0)
    assert df == 0.0 and dd == 0.0
    I = (slice(1, -1),) * 3
    assert np.abs(Tf[I] - Td[I]).max() <= 4e-7 * np.abs(Td[I]).max()
    inner = Wf[I]
    assert (inner == 0xFF).sum() == 1 and int(inner[inner != 0xFF].max()) < 6 * 33
    assert (Wf[I] != Wd[I]).mean() < 0.05  # winners differ only where candidates tie within float rounding


def test_oracle_tti_metric_matches_float64_formula():
    """orc_tti_metric (the FP64 parameter medium's metric, in the kernels'
    operation order) against the same formula evaluated by numpy, and the
    parameter form of a seeded medium against its six-array form."""
    import torch

    import media
    from oracle import Oracle

    o = Oracle()
    dims = (9, 7, 8)
    vz, eps, axis = media.tti_params(*dims, 10.0, seed=6, pad=True)
    P = [p.numpy() for p in media.params_from(vz, eps, axis)]
    Md = o.tti_metric(P)
    s, e, nx, ny = P
    s2 = s * s
    a = s2 / (1.0 + 2.0 * e)
    b = s2 - a
    nz = np.sqrt(np.maximum((1.0 - nx * nx) - ny * ny, 0.0))
    want = [a + b * nx * nx, b * nx * ny, b * nx * nz, a + b * ny * ny, b * ny * nz, a + b * nz * nz]
    for k in range(6):
        np.testing.assert_allclose(Md[k], want[k], rtol=1e-15, atol=1e-15 * np.abs(want[k]).max())
    M32 = media.metric_from(vz, eps, axis)
    for k in range(6):
        np.testing.assert_allclose(Md[k], M32[k].double().numpy(), rtol=2e-6,
                                   atol=2e-6 * float(torch.max(torch.abs(M32[k]))))


def test_oracle_tti_adjoint_matches_finite_differences():
    """The FP64 CPU adjoint of the parameter medium, chained to (s, eps, nx,
    ny), against central differences of the oracle's own solve (relative step
    1e-6) on a small seeded case: the chain rule the GPU gradient kernel
    applies, checked without a GPU."""
    import media
    from oracle import Oracle

    o = Oracle()
    dims, h = (11, 9, 10), (10.0,) * 3
    vz, eps, axis = media.tti_params(*dims, 10.0, seed=8, pad=True)
    P = [p.numpy().copy() for p in media.params_from(vz, eps, axis)]
    T0 = o.init_point(*dims, (6, 5, 2))
    rec = (slice(1, 2), slice(1, -1), slice(1, -1))

    def solve(Px):
        T = T0.copy()
        s, d, W = o.tti_solve_rec(T, Px, h, 200, tol=0.0)
        return T, W

    T, W = solve(P)
    tobs = T[rec] * 0.97
    r = np.zeros_like(T)
    r[rec] = T[rec] - tobs
    lam, g, nc = o.tti_adjoint(T, P, h, W, r)
    assert nc == 0

    def loss(Px):
        Tx, _ = solve(Px)
        return 0.5 * float(((Tx[rec] - tobs) ** 2).sum())

    rng = np.random.default_rng(2)
    errs = []
    for v in range(4):
        cand = np.argwhere(np.abs(g[v]) >= 1e-3 * np.abs(g[v]).max())
        for q in rng.choice(len(cand), 4, replace=False):
            k, j, i = cand[q]
            base = P[v][k, j, i]
            step = 1e-6 * max(abs(base), 1e-3)
            up = [p.copy() for p in P]
            dn = [p.copy() for p in P]
            up[v][k, j, i] = base + step
            dn[v][k, j, i] = base - step
            fd = (loss(up) - loss(dn)) / (up[v][k, j, i] - dn[v][k, j, i])
            errs.append(abs(fd - g[v][k, j, i]) / max(abs(fd), abs(g[v][k, j, i])))
    assert np.median(errs) < 1e-6 and max(errs) < 1e-4, (np.median(errs), max(errs))
