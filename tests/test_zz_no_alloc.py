"""fold3d_solve_noalloc: the solve entry point that allocates nothing.

Some callers cannot let this library allocate device memory for them: a host
program whose device buffers all come from another runtime (an OpenACC driver
using acc_malloc, a framework whose caching allocator already holds the GPU's
memory), or a plugin host that lends buffers to its plugins and budgets every
byte.  fold3d_solve_noalloc runs the same kernels as fold3d_solve with a
static per-sweep scratch array instead of allocations.

These tests call it through the C-ABI twice in a row, on two different
problems, and compare each result with fold3d_solve's bit for bit (the
tolerance of every parity test here), then check the limit of its scratch.
The file is named to be collected last, and passes alone in a fresh process
as well as after the other tests.
"""
import ctypes as C

import pytest

from conftest import assert_bitwise

from oracle import ref_spacing

pytestmark = pytest.mark.gpu


def test_noalloc_matches_solve_on_two_calls_in_a_row(f3d, ctx, cuda):
    # call 1: the reference's implicit-surface source at 24^3, 5 fixed sweeps
    n = 24
    h = (ref_spacing(n),) * 3
    T0 = f3d.init_implicit(n, n, n, h[0])
    want = cuda.from_numpy(T0.copy()).cuda()
    rw = ctx.solve(want, h, None, f3d.opts(max_sweeps=5, fixed=True))
    got = cuda.from_numpy(T0.copy()).cuda()
    rg = f3d.solve_noalloc(got, h, None, f3d.opts(max_sweeps=5, fixed=True))
    assert rg.sweeps == rw.sweeps == 5
    assert rg.max_delta == rw.max_delta
    assert_bitwise(got.cpu().numpy(), want.cpu().numpy(), "first call")

    # call 2: a non-cubic point source in another medium, run to convergence
    # (a different number of sweeps, so stale scratch slots would show)
    dims, h2 = (19, 13, 16), (0.5, 0.6, 0.7)
    med = f3d.medium(1.3, (0.2, -0.4, 0.3))
    P0 = f3d.init_point(*dims, (5, 7, 9))
    want = cuda.from_numpy(P0.copy()).cuda()
    rw = ctx.solve(want, h2, med, f3d.opts(max_sweeps=f3d.NOALLOC_MAX_SWEEPS, tol=0.0))
    got = cuda.from_numpy(P0.copy()).cuda()
    rg = f3d.solve_noalloc(got, h2, med, f3d.opts(max_sweeps=f3d.NOALLOC_MAX_SWEEPS, tol=0.0))
    assert rw.max_delta == 0.0 and rg.max_delta == 0.0
    assert rg.sweeps == rw.sweeps
    assert_bitwise(got.cpu().numpy(), want.cpu().numpy(), "second call")


def test_noalloc_rejects_more_sweeps_than_its_scratch(f3d, cuda):
    n = 8
    T = cuda.from_numpy(f3d.init_point(n, n, n, (4, 4, 4))).cuda()
    with pytest.raises(f3d.Fold3dError) as e:
        f3d.solve_noalloc(T, 1.0, None, f3d.opts(max_sweeps=f3d.NOALLOC_MAX_SWEEPS + 1, fixed=True))
    assert e.value.code == f3d.ERR_INVALID
    assert "FOLD3D_NOALLOC_MAX_SWEEPS" in str(e.value)
    L = f3d.lib()
    rc = L.fold3d_solve_noalloc(None, None, C.c_void_p(T.data_ptr()), None, None, None)
    assert rc == f3d.ERR_INVALID
