"""GPU parity at the benchmarked sizes: the default solve path (WAVEFRONT
engine, tile skipping on, the fast solver with its proved body skips) against
sha256 digests of the reference's own results at 512^3 and 1280^3
(tests/golden/digests_large.json, written by tests/golden/make_golden.py
--large from the reference's AN_ISO_1_OpenACC.c and Fold3dPMM.c built for
the host).  Bit-exact: a digest matches only if every cell does.

The 1280^3 tests hold a 16.9 GB field on the device and one copy on the
host.
"""
import hashlib
import json
import os

import numpy as np
import pytest

from conftest import GOLDEN

from oracle import ref_spacing

pytestmark = pytest.mark.gpu

# point source of the 512^3 digest (1-based i, j, k), as in make_golden.py
POINT_512 = (65, 257, 257)


@pytest.fixture(scope="module")
def large():
    with open(os.path.join(GOLDEN, "digests_large.json")) as fh:
        return json.load(fh)


def sha_dev(T):
    """sha256 of a device field's float64 bytes (one host copy, no more)."""
    a = T.cpu().numpy()
    return hashlib.sha256(memoryview(np.ascontiguousarray(a)).cast("B")).hexdigest()


def default_opts(f3d, sweeps):
    # the bench's configuration: AUTO engine (WAVEFRONT for the fast solver), skipping on
    return f3d.opts(max_sweeps=sweeps, fixed=True)


def test_reference_digest_512_implicit_surface(f3d, ctx, cuda, large):
    n = 512
    h = ref_spacing(n)
    T = cuda.empty((n + 2,) * 3, dtype=cuda.float64, device="cuda")
    f3d.init_implicit_device(ctx, T, h)
    assert sha_dev(T) == large["n512_init"], "device initialiser"
    T0 = T.clone()
    rep = ctx.solve(T, h, None, default_opts(f3d, 8))
    assert rep.sweeps == 8 and rep.engine == f3d.ENGINE_WAVEFRONT
    assert rep.evaluated_updates < rep.nominal_updates  # tile skipping was active
    assert sha_dev(T) == large["n512_s8"], "WAVEFRONT, skipping, fast solver"
    # the per-plane engine on the same input
    T.copy_(T0)
    ctx.solve(T, h, None, f3d.opts(max_sweeps=8, fixed=True, engine=f3d.ENGINE_PLANES))
    assert sha_dev(T) == large["n512_s8"], "PLANES engine"


def test_reference_digest_512_point_source(f3d, ctx, cuda, large):
    n = 512
    T = cuda.from_numpy(f3d.init_point(n, n, n, POINT_512)).cuda()
    rep = ctx.solve(T, ref_spacing(n), None, default_opts(f3d, 8))
    assert rep.sweeps == 8
    assert sha_dev(T) == large["n512_point_s8"]


def test_reference_digest_1280(f3d, ctx, cuda, large):
    """1280^3 (the headline size): the device initialiser, one sweep of the
    default solve, and the longest solve the reference digests cover."""
    n = 1280
    if "n1280_s1" not in large:
        pytest.skip("no 1280^3 reference digest")
    free, _ = cuda.cuda.mem_get_info()
    if free < 20e9:
        pytest.skip("needs 20 GB of free device memory")
    h = ref_spacing(n)
    T = cuda.empty((n + 2,) * 3, dtype=cuda.float64, device="cuda")
    f3d.init_implicit_device(ctx, T, h)
    assert sha_dev(T) == large["n1280_init"], "device initialiser"
    last = max(int(k[len("n1280_s"):]) for k in large if k.startswith("n1280_s"))
    T0 = T.clone()
    ctx.solve(T, h, None, default_opts(f3d, 1))
    assert sha_dev(T) == large["n1280_s1"], "after 1 sweep"
    if last > 1:
        # the whole solve in one call, tile skipping active from its second sweep
        T.copy_(T0)
        rep = ctx.solve(T, h, None, default_opts(f3d, last))
        assert rep.sweeps == last and rep.evaluated_updates < rep.nominal_updates
        assert sha_dev(T) == large["n1280_s%d" % last], "after %d sweeps" % last
    del T, T0
