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


@pytest.mark.parametrize("n", [32, 64])
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


def test_product_init_digest_64(f3d, digests):
    n = 64
    T = f3d.init_implicit(n, n, n, ref_spacing(n))
    assert sha(T) == digests["n64_init"]


@pytest.mark.parametrize("dims,h", [((9, 6, 7), (0.7, 0.9, 1.1)), ((20, 13, 17), (0.5, 0.8, 0.6))])
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


def test_product_point_init(f3d):
    T = f3d.init_point(5, 4, 3, (2, 3, 1))
    assert T[1, 3, 2] == 0.0
    T[1, 3, 2] = MAXT
    assert np.all(T == MAXT)
