"""Shared fixtures.  Tests marked `gpu` need a CUDA device (a B200); all
others run on the CPU.  Parity tests compare bit patterns, not values."""
import os
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "fgcs-openacc-advanced_b200")
GOLDEN = os.path.join(ROOT, "tests", "golden")
for p in (ROOT, PKG):
    if p not in sys.path:
        sys.path.insert(0, p)


@pytest.hookimpl(tryfirst=True)
def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (runs on the B200 box)")
    # temporary files of the tests stay inside the checkout (git-ignored)
    if not config.option.basetemp:
        config.option.basetemp = os.path.join(ROOT, ".pytest_tmp")


def bits(a):
    return np.ascontiguousarray(a).view(np.uint64)


def assert_bitwise(a, b, what=""):
    a = np.ascontiguousarray(a)
    b = np.ascontiguousarray(b)
    assert a.shape == b.shape, what
    ne = bits(a) != bits(b)
    if ne.any():
        idx = np.argwhere(ne)
        k = tuple(idx[0])
        raise AssertionError("%s: %d cells differ; first at (k,j,i)=%s: %r vs %r"
                             % (what, int(ne.sum()), k, a[k], b[k]))


@pytest.fixture(scope="session")
def orc():
    from oracle import Oracle

    return Oracle()


@pytest.fixture(scope="session")
def f3d():
    import fold3dpmm

    if not os.path.exists(fold3dpmm.LIB_PATH):
        import build as pkg_build  # fgcs-openacc-advanced_b200/build.py

        pkg_build.build()
    fold3dpmm.lib()
    return fold3dpmm


@pytest.fixture(scope="session")
def golden():
    out = {}
    for n in (8, 16):
        with np.load(os.path.join(GOLDEN, "ref_n%d.npz" % n)) as z:
            out[n] = {k: z[k] for k in z.files}
    return out


@pytest.fixture(scope="session")
def digests():
    import json

    with open(os.path.join(GOLDEN, "digests.json")) as fh:
        return json.load(fh)


@pytest.fixture(scope="session")
def cuda():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


@pytest.fixture(scope="session")
def ctx(f3d, cuda):
    c = f3d.Context(0)
    yield c
    c.close()
