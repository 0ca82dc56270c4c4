"""Multi-process plumbing of bench.py on the CPU: world size 2 over gloo
(127.0.0.1).  The GPU runs use the same helpers with NCCL."""
import os
import socket
import subprocess
import sys

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank_main(rank, world, port, out_dir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    import bench

    dist = bench.init_ranks(rank, backend="gloo")
    v = bench.max_over_ranks(1.5 + rank, dist, device="cpu")
    dist.barrier()
    dist.destroy_process_group()
    with open(os.path.join(out_dir, "rank%d" % rank), "w") as f:
        f.write(repr(v))


def test_max_over_ranks_world_2(tmp_path):
    """Each rank times a different value; every rank ends with the largest."""
    import torch.multiprocessing as mp

    mp.start_processes(_rank_main, args=(2, _free_port(), str(tmp_path)), nprocs=2, start_method="spawn")
    assert [float((tmp_path / ("rank%d" % r)).read_text()) for r in range(2)] == [2.5, 2.5]


def test_single_process_needs_no_group(monkeypatch):
    monkeypatch.delenv("WORLD_SIZE", raising=False)
    sys.path.insert(0, ROOT)
    import bench

    assert bench.init_ranks(0) is None
    assert bench.max_over_ranks(3.25, None) == 3.25


def test_reference_arm_runs_on_rank_0_only():
    """Under torchrun the reference arm's other ranks exit 0 without work."""
    env = dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1")
    p = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference"], env=env,
                       capture_output=True, text=True, timeout=300)
    assert p.returncode == 0, p.stderr
    assert p.stdout.strip() == ""


def test_reference_arm_line_on_a_small_grid():
    """The reference arm's JSON line at 64^3: the OpenMP transform's rate as
    the value, the unmodified one-thread build's rate beside it."""
    import json

    env = dict(os.environ)
    for k in ("RANK", "WORLD_SIZE", "LOCAL_RANK"):
        env.pop(k, None)
    p = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--size", "64",
                        "--steps", "1", "--warmup", "0", "--ref-seconds", "0.5"], env=env,
                       capture_output=True, text=True, timeout=300)
    assert p.returncode == 0, p.stderr
    line = json.loads(p.stdout.strip().splitlines()[-1])
    if "unavailable" in line:
        pytest.skip(line["unavailable"])
    assert line["impl"] == "reference" and line["value"] > 0
    cb = line["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["value"] == line["value"]
    assert cb["single_thread_value"] > 0 and "unmodified" in cb["single_thread_sample"]
    assert line["e2e"]["h2d_bytes_per_step"] == 0


def test_oracle_sample_times_the_elliptical_statement():
    """bench.py's CPU sample of the elliptical statement: runs the first
    sweep of small instances (float64 and float32) and counts their updates."""
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "fgcs-openacc-advanced_b200"))
    import numpy as np

    import bench
    import media
    from oracle import Oracle

    o = Oracle()
    dims = [(9, 7, 8), (6, 10, 5)]
    for f32 in (False, True):
        fields = [o.init_point(*d, (2, 3, 2)) for d in dims]
        if f32:
            fields = [f.astype(np.float32) for f in fields]
        Ms = [[m.numpy() for m in media.heterogeneous_tti(*d, 10.0, seed=1)] for d in dims]
        rate, done, upd = bench.oracle_ellip_sample(fields, Ms, [10.0, 10.0], 60.0, f32=f32)
        assert done == 2 and rate > 0
        assert upd == sum(2 * ((nx - 1) * ny * nz + (ny - 1) * nx * nz + (nz - 1) * nx * ny) for nx, ny, nz in dims)
        assert all(np.isfinite(f[1:-1, 1:-1, 1:-1]).all() and (f[1:-1, 1:-1, 1:-1] < 1e15).any() for f in fields)


def test_oracle_adjoint_sample_times_forward_and_adjoint():
    """bench.py's CPU sample of one source's gradient: one recording forward
    sweep from the initial field (left untouched) plus the whole FP64 adjoint
    from the converged field's winner record; the estimate adds the sweep
    time times the forward sweep count to the adjoint time."""
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "fgcs-openacc-advanced_b200"))
    import numpy as np

    import bench
    import media
    from oracle import Oracle

    o = Oracle()
    d = (9, 7, 8)
    T0 = o.init_point(*d, (2, 3, 2))
    M = [m.numpy() for m in media.heterogeneous_tti(*d, 10.0, seed=1)]
    T = T0.copy()
    s, _, W = o.ell_solve_rec(T, M, (10.0,) * 3, 100, tol=0.0)
    r = np.zeros_like(T)
    r[1, 1:-1, 1:-1] = 1.0
    before = T0.copy()
    per_src, sweep_s, adj_s = bench.oracle_adjoint_sample(T0, T, M, 10.0, W, r, s)
    assert np.array_equal(T0.view(np.uint64), before.view(np.uint64))
    assert sweep_s > 0 and adj_s > 0
    assert per_src == sweep_s * s + adj_s


def test_partition_splits_every_item_once_and_balances():
    """shard.partition: greedy longest-processing-time split; every item in
    exactly one part, parts ascending, the largest part at most the mean plus
    the largest item, the same split on every call, equal costs dealt round
    robin, one part = everything in order."""
    sys.path.insert(0, os.path.join(ROOT, "fgcs-openacc-advanced_b200"))
    import numpy as np

    import shard

    rng = np.random.default_rng(5)
    for count, parts in ((256, 8), (256, 3), (17, 4), (5, 5), (3, 7), (0, 2)):
        costs = [int(c) for c in rng.integers(98, 323, count) ** 3]
        split = shard.partition(costs, parts)
        assert len(split) == parts
        assert sorted(i for p in split for i in p) == list(range(count))
        assert all(p == sorted(p) for p in split)
        if count:
            loads = [sum(costs[i] for i in p) for p in split]
            assert max(loads) <= sum(costs) / parts + max(costs)
        assert split == shard.partition(costs, parts)
    assert shard.partition([1] * 10, 3) == [[0, 3, 6, 9], [1, 4, 7], [2, 5, 8]]
    assert shard.partition([4, 1, 9], 1) == [[0, 1, 2]]
    assert shard.partition([3, 3, 2, 2, 2], 2) == [[0, 2, 4], [1, 3]]
    for bad in (([1, 2], 0), ([1, -1], 2)):
        with pytest.raises(ValueError):
            shard.partition(*bad)


def _oracle_source_grad(src, n, M):
    """One source's misfit and dL/dM by the oracle (converged recording
    solve, then the FP64 adjoint), with t_obs = 0 at every top-face cell."""
    import numpy as np

    from oracle import Oracle

    o = Oracle()
    T = np.full((n + 2,) * 3, 1e16)
    T[src[2], src[1], src[0]] = 0.0
    _, _, W = o.ell_solve_rec(T, M, (10.0,) * 3, 200, tol=0.0)
    r = np.zeros_like(T)
    r[1, 1:-1, 1:-1] = T[1, 1:-1, 1:-1]
    _, g, nc = o.ell_adjoint(T, M, (10.0,) * 3, W, r)
    assert nc == 0
    return 0.5 * float((T[1, 1:-1, 1:-1] ** 2).sum()), g


_SHOTS = dict(n=10, srcs=[(2, 3, 2), (8, 8, 2), (5, 2, 3), (3, 9, 2), (7, 4, 2)])


def _survey_rank_main(rank, world, port, out_dir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank),
                      WORLD_SIZE=str(world), LOCAL_RANK=str(rank))
    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "fgcs-openacc-advanced_b200"))
    import numpy as np
    import torch

    import bench
    import media
    import shard

    dist = bench.init_ranks(rank, backend="gloo")
    n, srcs = _SHOTS["n"], _SHOTS["srcs"]
    M = [m.numpy() for m in media.heterogeneous_tti(n, n, n, 10.0, seed=1)]
    mine = shard.partition([1] * len(srcs), world)[rank]
    loss = torch.zeros(1, dtype=torch.float64)
    G = torch.zeros((6,) + (n + 2,) * 3, dtype=torch.float64)
    for q in mine:
        l_, g = _oracle_source_grad(srcs[q], n, M)
        loss += l_
        G += torch.from_numpy(g)
    shard.sum_over_ranks_([loss, G], dist)
    stats = bench.over_ranks([len(mine), rank, -rank], dist, "sum", device="cpu") + \
        bench.over_ranks([rank + 1.5], dist, "min", device="cpu") + \
        bench.over_ranks([rank + 1.5], dist, "max", device="cpu")
    dist.barrier()
    dist.destroy_process_group()
    np.save(os.path.join(out_dir, "G%d.npy" % rank), G.numpy())
    with open(os.path.join(out_dir, "rank%d" % rank), "w") as f:
        f.write(repr((float(loss), stats, mine)))


def test_survey_gradient_split_over_two_ranks(tmp_path):
    """A tomography step split over two gloo ranks (sources dealt by
    shard.partition, each rank's gradient summed by sum_over_ranks_) gives
    every rank the whole survey's loss and dL/dM, equal to one process
    summing all sources (to rounding: the sums are grouped differently).  The
    per-source gradient is the oracle's, standing in for the library."""
    import ast

    import numpy as np
    import torch.multiprocessing as mp

    sys.path.insert(0, ROOT)
    sys.path.insert(0, os.path.join(ROOT, "fgcs-openacc-advanced_b200"))
    import media

    mp.start_processes(_survey_rank_main, args=(2, _free_port(), str(tmp_path)), nprocs=2, start_method="spawn")
    n, srcs = _SHOTS["n"], _SHOTS["srcs"]
    M = [m.numpy() for m in media.heterogeneous_tti(n, n, n, 10.0, seed=1)]
    loss1, G1 = 0.0, np.zeros((6,) + (n + 2,) * 3)
    for sp_ in srcs:
        l_, g = _oracle_source_grad(sp_, n, M)
        loss1 += l_
        G1 += g
    assert np.abs(G1).max() > 0
    got = [ast.literal_eval((tmp_path / ("rank%d" % r)).read_text()) for r in range(2)]
    assert [g[2] for g in got] == [[0, 2, 4], [1, 3]]
    for r, (loss, stats, _) in enumerate(got):
        assert stats == [5.0, 1.0, -1.0, 1.5, 2.5]
        assert loss == pytest.approx(loss1, rel=1e-13)
        np.testing.assert_allclose(np.load(tmp_path / ("G%d.npy" % r)), G1, rtol=1e-12, atol=1e-12 * np.abs(G1).max())
    assert np.array_equal(np.load(tmp_path / "G0.npy"), np.load(tmp_path / "G1.npy"))
