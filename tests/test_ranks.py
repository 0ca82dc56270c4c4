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
