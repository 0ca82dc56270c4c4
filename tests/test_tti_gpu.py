"""GPU tests of the FP64 parameter medium (fold3d_*_tti): the tilted
elliptical medium given by slowness, Thomsen epsilon and the symmetry axis in
float64, from which the kernels form the metric per cell.

* fields and winner records against the oracle's FP64 statement
  (orc_tti_metric + orc_ell_solve_rec_d), bit for bit;
* the adjoint's parameter gradients against the FP64 CPU adjoint with the
  same chain rule;
* gradients with respect to slowness and epsilon against central finite
  differences with a relative step of 1e-6 (median relative error at most
  1e-6), at a small size and at the tomography configuration's 256^3;
* batches against one-by-one solves and adjoints, bit for bit.
"""
import numpy as np
import pytest

from conftest import assert_bitwise

pytestmark = pytest.mark.gpu

MAXT = 10e15 * 1.0


def point_field(cuda, dims, src):
    nx, ny, nz = dims
    T = cuda.full((nz + 2, ny + 2, nx + 2), MAXT, dtype=cuda.float64, device="cuda")
    T[src[2], src[1], src[0]] = 0.0
    return T


def hetero(dims, seed, h=10.0):
    import media

    return [p.cuda() for p in media.heterogeneous_tti_params(*dims, h, seed=seed)]


CASES = [
    ("homog", (40, 40, 40), (21, 21, 21), None),
    ("hetero", (37, 29, 33), (12, 20, 6), 3),
    ("hetero", (64, 64, 64), (33, 20, 11), 0),
]


@pytest.mark.parametrize("kind,dims,src,seed", CASES, ids=["homog40", "hetero37x29x33", "hetero64"])
def test_tti_matches_oracle(f3d, orc, ctx, cuda, kind, dims, src, seed):
    import media

    if kind == "homog":
        P = [p.cuda() for p in media.homogeneous_tti(*dims, 2000.0, 0.2, 30.0, 45.0)]
    else:
        P = hetero(dims, seed)
    T0 = point_field(cuda, dims, src)
    T = T0.clone()
    W = cuda.empty(T.shape, dtype=cuda.uint8, device="cuda")
    rep = f3d.solve_ellip_record(ctx, T, 10.0, P, W, f3d.opts(max_sweeps=300, tol=1e-10))
    ref = T0.cpu().numpy()
    s, d, Wref = orc.tti_solve_rec(ref, [p.cpu().numpy() for p in P], (10.0,) * 3, 300, tol=1e-10)
    assert rep.sweeps == s and rep.max_delta == d
    assert_bitwise(T.cpu().numpy(), ref, "field")
    assert np.array_equal(W.cpu().numpy(), Wref)
    if kind == "homog":
        # closed form sqrt(x^T M x) from the source: the first-order scheme's error, stated
        Md = orc.tti_metric([p.cpu().numpy() for p in P])
        M6 = [m[1, 1, 1] for m in Md]
        t = T.cpu().numpy()
        errs = []
        for (k, j, i) in [(21, 21, 40), (40, 21, 21), (21, 40, 21), (40, 40, 40), (2, 30, 9)]:
            d3 = ((i - src[0]) * 10.0, (j - src[1]) * 10.0, (k - src[2]) * 10.0)
            exact = media.exact_time(M6, *d3)
            errs.append(abs(t[k, j, i] - exact) / exact)
        assert max(errs) < 0.05, errs


def test_tti_solve_without_record_equals_record(f3d, ctx, cuda):
    dims, src = (37, 29, 33), (12, 20, 6)
    P = hetero(dims, 3)
    A = point_field(cuda, dims, src)
    B = A.clone()
    W = cuda.empty(A.shape, dtype=cuda.uint8, device="cuda")
    ra = f3d.solve_ellip(ctx, A, 10.0, P, f3d.opts(max_sweeps=300, tol=1e-10))
    rb = f3d.solve_ellip_record(ctx, B, 10.0, P, W, f3d.opts(max_sweeps=300, tol=1e-10))
    assert ra.sweeps == rb.sweeps
    assert_bitwise(A.cpu().numpy(), B.cpu().numpy(), "record on/off")


def test_tti_adjoint_matches_cpu_adjoint(f3d, orc, ctx, cuda):
    """lambda and dL/d(s, eps, nx, ny) of the GPU adjoint against the FP64 CPU
    adjoint (cells by decreasing time) with the same chain rule."""
    dims, src = (23, 19, 27), (12, 9, 5)
    P = hetero(dims, 4)
    T = point_field(cuda, dims, src)
    W = cuda.empty(T.shape, dtype=cuda.uint8, device="cuda")
    f3d.solve_ellip_record(ctx, T, 10.0, P, W, f3d.opts(max_sweeps=300, tol=0.0))
    rec = (slice(1, 2), slice(1, -1, 2), slice(1, -1, 2))
    r = cuda.zeros_like(T)
    r[rec] = T[rec] * 0.01 + 1.0
    lam = cuda.full_like(T, float("nan"))
    g = cuda.full((4,) + tuple(T.shape), float("nan"), dtype=cuda.float64, device="cuda")  # every cell written
    rep = f3d.adjoint_ellip(ctx, T, 10.0, P, W, r, lam, g)
    assert rep.max_delta == 0.0
    lr, gr, nc = orc.tti_adjoint(T.cpu().numpy(), [p.cpu().numpy() for p in P], (10.0,) * 3, W.cpu().numpy(),
                                 r.cpu().numpy())
    assert nc == 0
    np.testing.assert_allclose(lam.cpu().numpy(), lr, rtol=1e-9, atol=1e-12)
    gg = g.cpu().numpy()
    for m in range(4):
        np.testing.assert_allclose(gg[m], gr[m], rtol=1e-9, atol=1e-12 * np.abs(gr[m]).max())


def _fd_check(cuda, P, T0, h, rec, ncells, rng_seed, floor=1e-3):
    """Relative errors of dL/ds and dL/deps from the adjoint against central
    differences with step 1e-6 of the parameter, at ncells cells (each
    variable) among those whose gradient is at least `floor` of its
    largest."""
    import tomo

    Pg = [p.clone().requires_grad_(True) for p in P]
    T = tomo.solve(T0, h, Pg)
    tobs = (T[rec] * 0.97).detach()
    (0.5 * ((T[rec] - tobs) ** 2).sum()).backward()

    def loss(Px):
        with cuda.no_grad():
            Tx = tomo.solve(T0, h, Px)
            return float(0.5 * ((Tx[rec] - tobs) ** 2).sum())

    rng = np.random.default_rng(rng_seed)
    errs = {"s": [], "eps": []}
    for var, v in (("s", 0), ("eps", 1)):
        G = Pg[v].grad
        cand = cuda.nonzero(G.abs() >= floor * G.abs().max()).cpu().numpy()
        for q in rng.choice(len(cand), min(ncells, len(cand)), replace=False):
            k, j, i = (int(x) for x in cand[q])
            base = float(P[v][k, j, i])
            step = 1e-6 * abs(base) if base != 0.0 else 1e-8
            up = [p.clone() for p in P]
            dn = [p.clone() for p in P]
            up[v][k, j, i] = base + step
            dn[v][k, j, i] = base - step
            dv = float(up[v][k, j, i]) - float(dn[v][k, j, i])
            fd = (loss(up) - loss(dn)) / dv
            ad = float(G[k, j, i])
            errs[var].append(abs(fd - ad) / max(abs(ad), abs(fd), 1e-300))
    return errs


def test_tti_gradient_slowness_epsilon_finite_differences(cuda):
    """dL/ds and dL/deps with respect to the FP64 parameters against central
    differences with a 1e-6 relative step: median relative error at most
    1e-6 (nothing is rounded to float32 on the way)."""
    dims, h = (21, 17, 19), 10.0
    P = hetero(dims, 5)
    T0 = point_field(cuda, dims, (11, 9, 3))
    rec = (slice(1, 2), slice(1, -1, 2), slice(1, -1, 2))
    errs = _fd_check(cuda, P, T0, h, rec, 12, 1)
    for var, e in errs.items():
        assert np.median(e) <= 1e-6 and max(e) < 1e-4, (var, np.median(e), max(e))


def test_tti_gradient_finite_differences_256(cuda):
    """The tomography configuration's size: 256^3 seeded heterogeneous medium
    (seed 2) as FP64 parameters, one source 10 cells below the top face,
    4096 receivers on the top face; dL/ds and dL/deps against central
    differences (1e-6 relative step) at 16 cells each, among those whose
    gradient is at least 1e-2 of the largest.  Median relative error at most
    1e-6, every sample below 1e-5.  (Below that floor a cell moves the
    receivers' times by so little that the difference quotient is dominated
    by the solves' rounding, a few ulps of each time: about 1e-10 relative
    divided by the cell's sensitivity.)"""
    n, h = 256, 10.0
    P = hetero((n, n, n), 2)
    T0 = cuda.full((n + 2,) * 3, MAXT, dtype=cuda.float64, device="cuda")
    T0[11, 100, 140] = 0.0
    ridx = cuda.arange(3, n + 1, 4, device="cuda")
    rec = (1, ridx.view(-1, 1), ridx.view(1, -1))
    errs = _fd_check(cuda, P, T0, h, rec, 16, 11, floor=1e-2)
    for var, e in errs.items():
        assert np.median(e) <= 1e-6 and max(e) < 1e-5, (var, np.median(e), max(e))


def test_tti_batch_equals_one_by_one(f3d, ctx, cuda):
    """A batch of parameter-medium instances (non-cubic grids, own media and
    sources) gives each one its own solve's field, record and sweep count,
    bit for bit; the batched adjoint equals the single adjoints to rounding
    (relative 1e-12)."""
    rng = np.random.default_rng(9)
    inst = []
    for q in range(5):
        dims = tuple(int(v) for v in rng.integers(9, 33, 3))
        src = tuple(int(rng.integers(1, d + 1)) for d in dims)
        inst.append((dims, hetero(dims, 20 + q), point_field(cuda, dims, src)))
    o = f3d.opts(max_sweeps=300, tol=1e-10)
    fields = [T0.clone() for _, _, T0 in inst]
    Ws = [cuda.empty(T.shape, dtype=cuda.uint8, device="cuda") for T in fields]
    reps = f3d.solve_batch(ctx, fields, [10.0] * len(inst), [P for _, P, _ in inst], o, winners=Ws)
    for (dims, P, T0), T, W, r in zip(inst, fields, Ws, reps):
        A = T0.clone()
        WA = cuda.empty(A.shape, dtype=cuda.uint8, device="cuda")
        ra = f3d.solve_ellip_record(ctx, A, 10.0, P, WA, o)
        assert ra.sweeps == r.sweeps
        assert_bitwise(T.cpu().numpy(), A.cpu().numpy(), "batch field %s" % (dims,))
        assert cuda.equal(W, WA)
    dL = [cuda.zeros_like(T) for T in fields]
    for d in dL:
        d[1, 1:-1:2, 1:-1:2] = 1.0
    lam = [cuda.empty_like(T) for T in fields]
    g = [cuda.empty((4,) + tuple(T.shape), dtype=cuda.float64, device="cuda") for T in fields]
    f3d.adjoint_batch(ctx, fields, [10.0] * len(inst), [P for _, P, _ in inst], Ws, dL, lam, g)
    for (dims, P, _), T, W, d, la, gb in zip(inst, fields, Ws, dL, lam, g):
        l1 = cuda.empty_like(T)
        g1 = cuda.empty_like(gb)
        f3d.adjoint_ellip(ctx, T, 10.0, P, W, d, l1, g1)
        # lambda is pushed with atomic adds, whose order differs between launches: equal to rounding
        assert cuda.allclose(la, l1, rtol=1e-12, atol=0), dims
        assert cuda.allclose(gb, g1, rtol=1e-12, atol=1e-12 * float(g1.abs().max())), dims


def test_tti_rejects_float32_fields(f3d, ctx, cuda):
    dims = (8, 8, 8)
    P = hetero(dims, 1)
    T = point_field(cuda, dims, (4, 4, 4)).float()
    with pytest.raises(ValueError, match="float64 field"):
        f3d.solve_ellip(ctx, T, 10.0, P)
