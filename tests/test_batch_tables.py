"""CPU test of the batched solver's item tables (batch_tables, run on the
device by the restage kernel after every sweep): for random batches and
random sets of converged instances, the tables list exactly the active
instances' (step, tile) items, step-major, in the direction's order, and
every global item maps back to the right instance and step."""
import ctypes as C
import os
import subprocess

import numpy as np
import pytest

from conftest import ROOT


@pytest.fixture(scope="module")
def lib(tmp_path_factory):
    import build as pkg_build  # fgcs-openacc-advanced_b200/build.py

    out = str(tmp_path_factory.mktemp("tables") / "libtables.so")
    cmd = ["g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-I", pkg_build.INCLUDE, "-I", pkg_build.CSRC,
           "-I", "/usr/local/cuda/include", os.path.join(ROOT, "tests", "csrc", "batch_tables_host.cpp"), "-o", out]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    L = C.CDLL(out)
    L.host_batch_tables.restype = C.c_uint
    return L


@pytest.mark.parametrize("seed", range(6))
def test_batch_tables_list_the_active_items(lib, seed):
    rng = np.random.default_rng(seed)
    n = int(rng.integers(1, 40))
    steps = np.sort(rng.integers(1, 60, n))[::-1].astype(np.int32)  # a direction's order: steps descending
    order = rng.permutation(n).astype(np.int32)
    tiles = rng.integers(1, 50, n).astype(np.int64)
    active = (rng.random(n) < 0.6).astype(np.int32)
    max_steps = int(steps.max())
    act = np.full(n, -1, np.int32)
    tile_pre = np.zeros(n + 1, np.int64)
    step_k = np.zeros(max_steps, np.int32)
    step_off = np.zeros(max_steps + 1, np.int64)
    p = lambda a: a.ctypes.data_as(C.c_void_p)
    total = lib.host_batch_tables(p(order), p(steps), p(tiles), p(active), n, max_steps, p(act), p(tile_pre),
                                  p(step_k), p(step_off))
    # the active positions, in order
    want = [q for q in range(n) if active[order[q]]]
    k = len(want)
    assert list(act[:k]) == want
    assert total == sum(int(tiles[q]) * int(steps[q]) for q in want)
    # every global item, step-major: step p holds the tiles of every active position with more than p steps
    items = []
    for s in range(max_steps):
        for slot, q in enumerate(want):
            if steps[q] > s:
                items += [(slot, s, t) for t in range(tiles[q])]
    assert len(items) == total
    for g in rng.integers(0, max(total, 1), min(200, total)):
        slot, s, t = items[g]
        # the kernel's lookup: the step by step_off, the slot by tile_pre
        ps = int(np.searchsorted(step_off, g, side="right") - 1)
        r = g - step_off[ps]
        sl = int(np.searchsorted(tile_pre[:step_k[ps] + 1], r, side="right") - 1)
        assert (sl, ps, r - tile_pre[sl]) == (slot, s, t)
