"""Benchmark of the Fold3dPMM sweep on B200.

Workload (one "step"): a full reference-model solve -- the reference's drift
medium (F = 1.1, a = (-0.35, 0.4, 0.7)), its implicit-surface source, a 1280^3
grid (h = 10/1279; --size picks another), 8 sweeps of the six directional
passes, exactly the reference driver's loop
(Stencil-OpenACC/AN_ISO_1_OpenACC.c:1187-1237).  The published single-GPU
A100 figures for this workload are 35.163471 s at 1280^3 and 3.037851 s at
512^3 (plots/perfect-2-gpu.py:24), i.e. 2.86 and 2.12 Gcell-updates/s.  The
initial field is built on the device (fold3d_init_implicit_device) and its
sha256, and that of the solve's result, are compared with the reference's own
(tests/golden/digests_large.json) and reported in the line's "parity".

Metric: Gcell-updates/s = nominal point updates / time, nominal updates per
sweep = 2 * [(nx-1)ny nz + (ny-1)nx nz + (nz-1)nx ny].

  value : device-resident throughput -- each step copies the pristine initial
          field (already in HBM) into the working field and solves; timed
          with CUDA events on the solve stream.  The field (16.9 GB at
          1280^3, 1.09 GB at 512^3) is larger than L2, so no flush is needed
          between steps.
  e2e   : the same solve through the C-ABI host entry point
          (fold3d_solve_host) from pinned host memory: H2D copy of the field,
          solve, D2H copy of the result, all inside the timed region.

N > 1 GPUs: a single solve does not shard (every plane depends on the whole
previous plane), so each rank solves its own replica (weak scaling, no
collective on the data path); value = all ranks' updates / max-over-ranks
time.

--impl reference: the reference's own CPU implementation (oracle/_ref:
AN_ISO_1_OpenACC.c built for the host; its OpenMP transform on all host
cores), each step a bounded sample of the same workload (the first planes of
each of the six passes of sweep 1, from the same initial field).
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "fgcs-openacc-advanced_b200")
for _p in (ROOT, PKG):
    if _p not in sys.path:
        sys.path.insert(0, _p)

PUBLISHED_S = {512: 3.037851, 1280: 35.163471}  # plots/perfect-2-gpu.py:24 (V2, A100, 8 sweeps)
REF_F, REF_A = 1.1, (-0.35, 0.4, 0.7)
BYTES_PER_UPDATE = 16  # read old target + write new target, FP64; medium is constant (m = 0)
# DRAM bytes (read + write) per update of wave_pass_kernel<drift>, from an ncu
# capture of the x_down, x_up and k_up passes of one sweep at 512^3 without
# tile skipping: 4.1662 GB over 3 x 511 x 512^2 updates
WAVE_DRAM_BYTES_PER_UPDATE = 4166210304 / (3 * 511 * 512 * 512)


def load_large_digests():
    """sha256 digests of the reference's own fields at the benchmarked sizes
    (tests/golden/digests_large.json, from tests/golden/make_golden.py)."""
    try:
        with open(os.path.join(ROOT, "tests", "golden", "digests_large.json")) as fh:
            return json.load(fh)
    except (OSError, ValueError):
        return {}


def sha256_of(a):
    """sha256 of an array's bytes, without another copy of it."""
    import hashlib

    import numpy as np

    return hashlib.sha256(memoryview(np.ascontiguousarray(a)).cast("B")).hexdigest()


def nominal_updates(n, sweeps):
    return sweeps * 6 * (n - 1) * n * n


def published_rate(n, sweeps=8):
    s = PUBLISHED_S.get(n)
    return None if s is None else nominal_updates(n, sweeps) / s / 1e9


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            p = json.load(f)
        return float(p["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clock/throttle sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), "--query-gpu=" + self.Q, "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        self.out = ""
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.out, _ = self.proc.communicate(timeout=5)
            except Exception:
                self.proc.kill()
                self.out = ""

    def summary(self):
        rows = []
        for ln in (self.out or "").splitlines():
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                rows.append((float(f[1]), float(f[2]), f[5:9]))
            except ValueError:
                continue
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for _, _, flags in rows:
            for nm, fl in zip(names, flags):
                if fl.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(r[0] for r in rows), "sm_max_mhz": max(r[1] for r in rows),
                "reasons": sorted(reasons), "samples": len(rows)}


def host_threads():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


def init_ranks(local, backend="nccl"):
    """One process per GPU under torchrun: join the process group (short
    timeout, so ranks that wait for a missing peer end with an error).
    Returns torch.distributed, or None for a single process."""
    if int(os.environ.get("WORLD_SIZE", "1")) <= 1:
        return None
    import datetime

    import torch
    import torch.distributed as dist

    kw = {"device_id": torch.device("cuda", local)} if backend == "nccl" else {}
    dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300), **kw)
    return dist


def max_over_ranks(ms, dist, device="cuda"):
    """The largest of every rank's ms (identity for a single process)."""
    if dist is None:
        return ms
    import torch

    t = torch.tensor([ms], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def over_ranks(vals, dist, op, device="cuda"):
    """Element-wise "sum" | "min" | "max" of every rank's list of numbers
    (float64, exact for integers below 2^53); the list itself for a single
    process."""
    if dist is None:
        return [float(v) for v in vals]
    import torch

    t = torch.tensor([float(v) for v in vals], device=device, dtype=torch.float64)
    dist.all_reduce(t, op={"sum": dist.ReduceOp.SUM, "min": dist.ReduceOp.MIN, "max": dist.ReduceOp.MAX}[op])
    return t.tolist()


def reference_cpu_sample(T0, n, seconds=None, planes=None, threads=None, omp=True):
    """Time the reference's own sweep functions (oracle/_ref: the OpenMP
    transform on `threads` cores, or with omp=False the unmodified build,
    whose OpenACC regions run on one host thread) on the first planes of each
    of the six passes of sweep 1, starting from T0.  Returns (updates/s,
    info)."""
    import numpy as np

    from oracle import RefLib, build

    if threads and omp:
        os.environ["OMP_NUM_THREADS"] = str(threads)
    path = build.ref_lib_path(n, omp=omp)
    kind = "reference"
    if not os.path.exists(path):
        raise RuntimeError("reference host build missing: %s" % path)
    r = RefLib(n, omp=omp)
    if planes is None:  # calibrate: one plane of x_down
        T = np.array(T0, copy=True)
        t = time.perf_counter()
        r.plane(T, 0, 1)
        per_plane = max(time.perf_counter() - t, 1e-4)
        planes = max(1, min(n - 1, int((seconds or 10.0) / (6 * per_plane))))
        del T
    T = np.array(T0, copy=True)
    t = time.perf_counter()
    for d in range(6):
        first, step = (1, 1) if d in (0, 2, 5) else (n, -1)
        for p in range(planes):
            r.plane(T, d, first + step * p)
    dt = time.perf_counter() - t
    upd = 6 * planes * n * n
    info = {"kind": kind, "cores": int(os.environ.get("OMP_NUM_THREADS", host_threads())) if omp else 1,
            "sample": "%d planes of each of the 6 passes of sweep 1 at %d^3 (%d updates), reference "
                      "AN_ISO_1_OpenACC.c host build, %s" % (
                          planes, n, upd, "OpenMP transform" if omp else "unmodified (one thread)"),
            "seconds": dt, "planes": planes}
    return upd / dt, info


def single_thread_reference(T0, n, seconds=3.0):
    """The unmodified reference build's rate on one host thread, over a short
    sample, for the line's cpu_baseline ({} if unavailable)."""
    try:
        rate, info = reference_cpu_sample(T0, n, seconds=seconds, omp=False)
        return {"single_thread_value": rate / 1e9, "single_thread_sample": info["sample"]}
    except Exception as e:
        return {"single_thread_value": None, "single_thread_sample": "unavailable: %s" % str(e).splitlines()[0]}


def run_reference(args):
    """--impl reference: rank 0 only."""
    import numpy as np

    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    n = args.size
    from oracle import RefLib, build, ref_spacing

    try:
        if not os.path.exists(build.ref_lib_path(n, omp=True)):
            if build.reference_available():
                build.build_ref(n)
            else:
                raise RuntimeError("no host build of the reference at %d^3" % n)
        threads = host_threads()
        os.environ["OMP_NUM_THREADS"] = str(threads)
        r = RefLib(n, omp=True)
        if n <= 640:
            T0 = r.init_implicit()  # the reference's own ImplicitInitialiser
            setup = "starting field from the reference's own ImplicitInitialiser"
        else:
            # The reference's initialiser is single-threaded and takes minutes at
            # this size; the starting field (untimed) comes from this library's
            # host initialiser, whose result equals the reference's bit for bit
            # (sha256 n1280_init in tests/golden/digests_large.json).
            import fold3dpmm as f3d

            T0 = f3d.init_implicit(n, n, n, ref_spacing(n))
            setup = ("starting field (untimed) from fold3d_init_implicit, bit-identical to the reference's "
                     "ImplicitInitialiser; only the reference's sweep functions are timed")
    except Exception as e:
        print(json.dumps({"impl": "reference", "unavailable": str(e).splitlines()[0]}))
        return
    rates = []
    info = None
    planes = None
    for it in range(args.warmup + args.steps):
        rate, info = reference_cpu_sample(T0, n, seconds=args.ref_seconds, planes=planes, threads=threads)
        planes = info["planes"]
        if it >= args.warmup:
            rates.append(rate)
    value = statistics.mean(rates) / 1e9
    upd_per_step = 6 * planes * n * n
    out = {
        "impl": "reference", "metric": "Gcell-updates/s", "value": value, "unit": "Gcell-updates/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": upd_per_step / (value * 1e9) * 1e3, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic: reference implicit-surface source",
        "config": workload_config(args),
        "cpu_baseline": {"value": value, "unit": "Gcell-updates/s", "cores": info["cores"], "kind": "reference",
                         "sample": info["sample"] + "; " + setup} | single_thread_reference(T0, n),
        "e2e": {"value": value, "unit": "Gcell-updates/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(out))


# Directions in the solve's order (x_down, x_up, k_up, k_down, y_up, y_down):
# normal axis (0 x, 1 y, 2 z) and step sign.
_DIR_NRM = (0, 0, 2, 2, 1, 1)
_DIR_SG = (1, -1, 1, -1, -1, 1)


def oracle_ellip_sample(fields, media_h, hs, seconds, f32=False):
    """The oracle's CPU statement of the elliptical solver (OpenMP) timed on a
    bounded sample: the six passes of a first sweep of each instance in turn
    (host fields, float64 or float32, and float32 metrics), until `seconds`
    have passed.  Returns (cell updates per second, instances done,
    updates)."""
    import ctypes as C

    from oracle import Oracle

    orc = Oracle()
    upd, done = 0, 0
    t1 = time.perf_counter()
    for T, M, h in zip(fields, media_h, hs):
        nz, ny, nx = (int(v) - 2 for v in T.shape)
        n = (nx, ny, nz)
        arrs, ptrs = orc._metric(M)
        Tp = T.ctypes.data_as(C.c_void_p)
        for d in range(6):
            nn = n[_DIR_NRM[d]]
            planes = range(1, nn) if _DIR_SG[d] > 0 else range(nn, 1, -1)
            for p in planes:
                if f32:
                    orc.L.orc_ellf_plane_rec(Tp, ptrs, None, nx, ny, nz, h, h, h, d, p)
                else:
                    orc.L.orc_ell_plane(Tp, ptrs, nx, ny, nz, h, h, h, d, p)
            upd += (nn - 1) * (nx * ny * nz // nn)
        done += 1
        if time.perf_counter() - t1 >= seconds:
            break
    return upd / (time.perf_counter() - t1), done, upd


def oracle_adjoint_sample(T0, T, M, h, W, r, fwd_sweeps):
    """The oracle's CPU statement of one source's gradient, timed in two
    parts: one recording forward sweep (six passes, OpenMP) from the initial
    field T0, and the whole FP64 adjoint (winner weights, cells by decreasing
    time, dL/dM) from the converged field T, its winner record W and
    r = dL/dT.  Host arrays; M as six float32 metric arrays, or four FP64
    parameter arrays (the FP64 statement with the metric formed from them,
    and the chain rule to the parameters).  Returns (seconds per
    source-gradient = sweep time x fwd_sweeps + adjoint time, sweep seconds,
    adjoint seconds)."""
    from oracle import Oracle

    orc = Oracle()
    t1 = time.perf_counter()
    if len(M) == 4:
        orc.tti_solve_rec(T0.copy(), M, (h,) * 3, 1, tol=0.0)
    else:
        orc.ell_solve_rec(T0.copy(), M, (h,) * 3, 1, tol=0.0)
    sweep_s = time.perf_counter() - t1
    t1 = time.perf_counter()
    if len(M) == 4:
        orc.tti_adjoint(T, M, (h,) * 3, W, r)
    else:
        orc.ell_adjoint(T, M, (h,) * 3, W, r)
    adj_s = time.perf_counter() - t1
    return sweep_s * fwd_sweeps + adj_s, sweep_s, adj_s


def run_tti(args):
    """--medium tti: the 512^3 heterogeneous tilted-elliptical configuration
    (seeded medium, point source at depth index 64 of the centre column), each
    step a solve run to max|dT| <= 1e-10.  The medium is the FP64 parameter
    form (slowness, eps, axis; fold3d_solve_tti) with float64 fields, or the
    six float32 metric arrays (--tti-medium metric, and the float32 build).
    Bytes per update: 16 for the field plus 32 for the four FP64 parameter
    words of the target (24 for six float32 metric words)."""
    import numpy as np
    import torch

    import fold3dpmm as f3d
    import media

    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    torch.cuda.set_device(local)
    dist = init_ranks(local)
    n, h = args.size, args.spacing
    # grids above 768^3 are built in float32 (float64 temporaries would not fit)
    gen_dtype = torch.float64 if n <= 768 else torch.float32
    param = args.tti_medium == "param" and args.field_dtype == "f64"
    t0 = time.perf_counter()
    if param:
        M = media.heterogeneous_tti_params(n, n, n, h, seed=0, device="cuda", dtype=gen_dtype)
    else:
        M = media.heterogeneous_tti(n, n, n, h, seed=0, device="cuda", dtype=gen_dtype)
    torch.cuda.synchronize()
    gen_s = time.perf_counter() - t0
    gen_peak_gb = torch.cuda.max_memory_allocated() / 1e9
    torch.cuda.empty_cache()
    if args.source == "top":
        src = (n // 2 + 1, n // 2 + 1, 1)  # (i, j, k): top-face centre
    else:
        src = (n // 2 + 1, n // 2 + 1, n // 8 + 1)  # centre column, depth index n/8
    fdt = torch.float32 if args.field_dtype == "f32" else torch.float64
    T0 = torch.full((n + 2,) * 3, 10e15 * 1.0, dtype=fdt, device="cuda")
    T0[src[2], src[1], src[0]] = 0.0
    T = torch.empty_like(T0)
    ctx = f3d.Context(local)
    stream = torch.cuda.current_stream()
    sp = stream.cuda_stream
    o = f3d.opts(max_sweeps=2000, fixed=False, tol=1e-10, skip=bool(args.skip))
    rep = None
    for _ in range(args.warmup):
        T.copy_(T0)
        rep = f3d.solve_ellip(ctx, T, h, M, o, stream=sp)
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    solve_ms = 0.0
    with ClockSampler(local) as clk:
        ev0.record(stream)
        for _ in range(args.steps):
            T.copy_(T0)
            rep = f3d.solve_ellip(ctx, T, h, M, o, stream=sp)
            solve_ms += rep.elapsed_ms
        ev1.record(stream)
        torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1)
    ms = max_over_ranks(ms, dist)
    upd = rep.nominal_updates
    value = world * upd * args.steps / (ms / 1e3) / 1e9
    e2e = None
    if not args.no_e2e and n <= 768:  # larger: the pinned copies of field and medium would not fit the host
        hT0 = T0.cpu().pin_memory()
        hM = [m.cpu().pin_memory() for m in M]
        hout = torch.empty_like(hT0).pin_memory()
        dM = M  # the medium is uploaded into its own device arrays every step (the same values)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            T.copy_(hT0, non_blocking=True)
            for d_, h_ in zip(dM, hM):
                d_.copy_(h_, non_blocking=True)
            f3d.solve_ellip(ctx, T, h, dM, o, stream=sp)
            hout.copy_(T, non_blocking=True)
        e1.record(stream)
        torch.cuda.synchronize()
        ems = e0.elapsed_time(e1)
        nb_in = hT0.numel() * hT0.element_size() + sum(m.numel() * m.element_size() for m in hM)
        e2e = {"value": world * upd * args.steps / (ems / 1e3) / 1e9, "unit": "Gcell-updates/s",
               "h2d_bytes_per_step": nb_in, "d2h_bytes_per_step": hT0.numel() * hT0.element_size(),
               "ms_per_step": ems / args.steps}
    peak, peak_kind = load_peaks()
    per_ms = solve_ms / args.steps
    # field read + write, and the target's medium: four FP64 parameters or six float32 metric words
    bpu = (16.0 if fdt == torch.float64 else 8.0) + (32.0 if param else 24.0)
    achieved = bpu * upd / (per_ms / 1e3) / 1e9
    launches = rep.sweeps * 6
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        try:
            from oracle import Oracle

            if param and n > 640:
                raise RuntimeError("the CPU statement's double metric for %d^3 would need %.0f GB of host memory"
                                   % (n, 6 * (n + 2) ** 3 * 8 / 1e9))
            orc = Oracle()
            Th = T0.cpu().numpy()
            import ctypes as C

            if param:  # the metric formed from the FP64 parameters, as the kernels form it
                Md = orc.tti_metric([m.cpu().numpy() for m in M])
                ptrs = (C.c_void_p * 6)(*(a.ctypes.data for a in Md))
            else:
                Mh = [m.cpu().numpy() for m in M]
                arrs, ptrs = orc._metric(Mh)

            planes, upd_cpu = 0, 0
            t1 = time.perf_counter()
            while time.perf_counter() - t1 < args.cpu_seconds and planes < n - 1:
                for d in range(6):
                    first, step = (1, 1) if d in (0, 2, 5) else (n, -1)
                    if fdt == torch.float32:
                        orc.L.orc_ellf_plane_rec(Th.ctypes.data_as(C.c_void_p), ptrs, None, n, n, n, h, h, h, d,
                                                 first + step * planes)
                    elif param:
                        orc.L.orc_ell_plane_d(Th.ctypes.data_as(C.c_void_p), ptrs, n, n, n, h, h, h, d,
                                              first + step * planes)
                    else:
                        orc.L.orc_ell_plane(Th.ctypes.data_as(C.c_void_p), ptrs, n, n, n, h, h, h, d,
                                            first + step * planes)
                planes += 1
                upd_cpu += 6 * n * n
            dt = time.perf_counter() - t1
            cpu = {"value": upd_cpu / dt / 1e9, "unit": "Gcell-updates/s", "cores": host_threads(), "kind": "port",
                   "sample": "%d planes of each of the 6 passes of sweep 1 at %d^3 (%d updates), this "
                             "repository's %s CPU statement of the elliptical solver (no reference "
                             "implementation exists), OpenMP" % (planes, n, upd_cpu, args.field_dtype.upper())}
        except Exception as e:
            cpu = {"value": None, "unit": "Gcell-updates/s", "cores": 0, "kind": "port",
                   "sample": "unavailable: %s" % str(e).splitlines()[0]}
    out = {
        "metric": "Gcell-updates/s", "value": value, "unit": "Gcell-updates/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": args.field_dtype,
        "data": "synthetic: seeded heterogeneous tilted-elliptical medium (seed 0), point source",
        "config": {"workload": "TTI %d^3 h=%g m heterogeneous (seed 0), source (i,j,k)=%s, run to max|dT|<=1e-10"
                               % (n, h, src), "grid": n, "sweeps": rep.sweeps, "engine": "wavefront",
                   "medium_construction": str(gen_dtype).replace("torch.", ""),
                   "skip": bool(args.skip),
                   "medium": "4 FP64 parameter words per cell (slowness, eps, axis x, y); metric formed in the "
                             "kernel" if param else "6 float32 metric words per cell",
                   "l2": "field + medium %.1f GB > 126 MB L2" % ((n + 2) ** 3 * bpu / 2 / 1e9),
                   "parallelism": "replicas" if world > 1 else "single"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": None, "peak_kind": peak_kind, "kernel": "wave_pass_kernel<ellip>",
                     "alg_bytes_per_update": bpu, "note": "ALU bound"},
        "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches * args.steps, "clocks": clk.summary(),
        "solve_ms": per_ms, "evaluated_updates_per_step": rep.evaluated_updates, "medium_gen_s": gen_s,
        "medium_gen_peak_gb": gen_peak_gb,
    }
    if rank == 0:
        print(json.dumps(out))
    ctx.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def run_batch(args):
    """--medium batch: args.batch instances, grid sizes per axis uniform in
    [96, 320] (seed 1), each with its own seeded heterogeneous TTI medium
    (seed 1000 + i) and a uniformly placed point source, each run to
    max|dT| <= 1e-10.  One step = one batched solve of all instances.  The
    same fields are also solved one after the other (fold3d_solve_ellip) to
    give the batched launch's speed-up over sequential solves.  Under
    torchrun the instances are split over the ranks, greedily by cell count
    (shard.partition); each rank solves its part in one batch, with no
    exchange, and the step time is the slowest rank's."""
    import numpy as np
    import torch

    import fold3dpmm as f3d
    import media
    import shard

    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    if args.batch < world:
        raise SystemExit("--batch %d is smaller than the %d ranks" % (args.batch, world))
    torch.cuda.set_device(local)
    dist = init_ranks(local)
    rng = np.random.default_rng(1)
    lo, hi = args.batch_dims
    dims = [tuple(int(v) for v in rng.integers(lo, hi + 1, 3)) for _ in range(args.batch)]
    srcs = [tuple(int(rng.integers(1, d + 1)) for d in dd) for dd in dims]
    parts = shard.partition([(d[0] + 2) * (d[1] + 2) * (d[2] + 2) for d in dims], world)
    mine = parts[rank]
    t0 = time.perf_counter()
    M, T0 = [], []
    for i in mine:
        dd, sp_ = dims[i], srcs[i]
        M.append(media.heterogeneous_tti(*dd, 10.0, seed=1000 + i, device="cuda"))
        nx, ny, nz = dd
        t = torch.full((nz + 2, ny + 2, nx + 2), 10e15 * 1.0,
                       dtype=torch.float32 if args.field_dtype == "f32" else torch.float64, device="cuda")
        t[sp_[2], sp_[1], sp_[0]] = 0.0
        T0.append(t)
    torch.cuda.synchronize()
    gen_s = time.perf_counter() - t0
    T = [t.clone() for t in T0]
    ctx = f3d.Context(local)
    f3d.batch_set_config(ctx, *args.batch_config)
    stream = torch.cuda.current_stream()
    sp = stream.cuda_stream
    o = f3d.opts(max_sweeps=2000, fixed=False, tol=1e-10, skip=bool(args.skip))
    hs = [10.0] * len(mine)

    def restore():
        for a, b in zip(T, T0):
            a.copy_(b)

    def sync_all():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    reps = None
    for _ in range(args.warmup):
        restore()
        reps = f3d.solve_batch(ctx, T, hs, M, o, stream=sp)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    batch_ms = 0.0
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            restore()
            sync_all()
            ev0.record(stream)
            reps = f3d.solve_batch(ctx, T, hs, M, o, stream=sp)
            ev1.record(stream)
            sync_all()
            batch_ms += ev0.elapsed_time(ev1)
    batch_ms = max_over_ranks(batch_ms / args.steps, dist)
    batched = [t.clone() for t in T]
    # the same solves one after the other
    restore()
    seq_reps = []
    sync_all()
    ev0.record(stream)
    for q in range(len(mine)):
        seq_reps.append(f3d.solve_ellip(ctx, T[q], 10.0, M[q], o, stream=sp))
    ev1.record(stream)
    sync_all()
    seq_ms = max_over_ranks(ev0.elapsed_time(ev1), dist)
    ibits = lambda t: t.view(torch.int64 if t.element_size() == 8 else torch.int32)
    same = all(torch.equal(ibits(a), ibits(b)) for a, b in zip(batched, T))
    tuned_rows, tuned_ctas = f3d.batch_get_config(ctx)
    # one graph per batched solve: the prologue's table kernel, then per sweep six passes and the restage kernel
    nominal, evald, nsame, launches = over_ranks(
        [sum(r.nominal_updates for r in reps), sum(r.evaluated_updates for r in reps), int(same),
         (7 * max(r.sweeps for r in reps) + 1) * args.steps], dist, "sum")
    smin, = over_ranks([min(r.sweeps for r in reps)], dist, "min")
    smax, = over_ranks([max(r.sweeps for r in reps)], dist, "max")
    cells = sum((d[0] + 2) * (d[1] + 2) * (d[2] + 2) for d in dims)
    peak, peak_kind = load_peaks()
    # per GPU: each rank's kernels move 40 B per update of its own instances
    achieved = 40.0 * nominal / world / (batch_ms / 1e3) / 1e9
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:  # the first 16 instances, a first sweep each, within --cpu-seconds
        try:
            k = min(16, args.batch)
            f32 = args.field_dtype == "f32"
            rate, done, upd_cpu = oracle_ellip_sample([t.cpu().numpy() for t in T0[:k]],
                                                      [[m.cpu().numpy() for m in Mi] for Mi in M[:k]],
                                                      hs[:k], args.cpu_seconds, f32=f32)
            cpu = {"value": rate / 1e9, "unit": "Gcell-updates/s", "cores": host_threads(), "kind": "port",
                   "sample": "first sweep of %d of the first %d instances (%d updates), this repository's %s CPU "
                             "statement of the elliptical solver (no reference implementation exists), OpenMP"
                             % (done, k, upd_cpu, "F32" if f32 else "F64")}
        except Exception as e:
            cpu = {"value": None, "unit": "Gcell-updates/s", "cores": 0, "kind": "port",
                   "sample": "unavailable: %s" % str(e).splitlines()[0]}
    out = {
        "metric": "Gcell-updates/s", "value": nominal / (batch_ms / 1e3) / 1e9, "unit": "Gcell-updates/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": batch_ms,
        "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": args.field_dtype,
        "data": "synthetic: %d seeded heterogeneous TTI media and point sources" % args.batch,
        "config": {"workload": "batch of %d solves, dims per axis U[%d,%d] (seed 1), h=10 m, each run to "
                               "max|dT|<=1e-10" % (args.batch, lo, hi), "cells": cells,
                   "sweeps_min_max": [int(smin), int(smax)],
                   "engine": "wavefront batch, sweep loop on the device (one CUDA graph)", "skip": bool(args.skip),
                   "autotuned": {"tile_rows": tuned_rows, "threads_per_cta": 32 * tuned_rows,
                                 "ctas_per_sm": tuned_ctas},
                   "parallelism": "instances split over %d ranks by cells, no exchange" % world
                   if world > 1 else "single",
                   "instances_per_rank": [len(q) for q in parts]},
        "sequential_ms": seq_ms, "speedup_vs_sequential": seq_ms / batch_ms,
        "batched_equals_sequential": nsame == world,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "traffic": None, "peak_kind": peak_kind, "kernel": "batch_pass_kernel",
                     "alg_bytes_per_update": 40},
        "evaluated_updates_per_step": evald, "clocks": clk.summary(), "medium_gen_s": gen_s,
        "cpu_baseline": cpu,
        "gpu_launches": int(launches),
    }
    if rank == 0:
        print(json.dumps(out))
    ctx.close()
    if dist is not None:
        dist.destroy_process_group()


def run_adjoint(args):
    """--medium adjoint: traveltime tomography at --adj-size^3 (256), h=10 m.
    True medium: the seeded heterogeneous TTI construction (seed 2); starting
    medium: its slowness, eps and axis smoothed by a Gaussian of 16 cells.
    64 sources on a jittered 8 x 8 grid 10 cells below the top face (k = 11),
    4096 receivers on a 64 x 64 grid on the top face (k = 1).  Observed times
    come from solves in the true medium (untimed).  One step = the loss
    1/2 sum (t - t_obs)^2 over all sources and receivers and its gradient with
    respect to per-cell slowness and eps: per source a recording forward solve
    (to max|dT| <= 1e-10) and the adjoint, through tomo.EllipSolve (torch
    autograd over the C-ABI), then torch's chain rule from the metric to
    slowness and eps.  The forward and adjoint library calls are also timed
    on their own (CUDA events inside the library).  Under torchrun the
    sources are split over the ranks (shard.partition); each rank solves its
    own sources in the whole medium, and the step ends with one sum over the
    ranks of the loss and of the two gradient fields (NCCL all-reduce), so
    every rank holds the survey's full gradient."""
    import numpy as np
    import torch

    import media
    import shard
    import tomo

    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    torch.cuda.set_device(local)
    dist = init_ranks(local)
    n, h = args.adj_size, 10.0
    nsrc_side, nrec_side = 8, 64
    t0 = time.perf_counter()
    vz_t, eps_t, ax_t = media.tti_params(n, n, n, h, seed=2, device="cuda", pad=True)
    # FP64 fields: the FP64 parameter medium (fold3d_*_tti), gradients straight to slowness and eps;
    # the float32 build: six metric arrays and torch's chain rule from them
    param = args.field_dtype == "f64" and args.tti_medium == "param"
    M_true = media.params_from(vz_t, eps_t, ax_t) if param else \
        [m.double() for m in media.metric_from(vz_t, eps_t, ax_t)]
    vz0, eps0, ax0 = media.smooth_params(vz_t, eps_t, ax_t, 16.0)
    axis0 = media.params_from(vz0, eps0, ax0)[2:] if param else None
    del vz_t, eps_t, ax_t
    rng = np.random.default_rng(2)
    cell = n / nsrc_side
    srcs = []
    for b in range(nsrc_side):
        for a in range(nsrc_side):
            i = int((a + 0.5) * cell + rng.uniform(-cell / 4, cell / 4)) + 1
            j = int((b + 0.5) * cell + rng.uniform(-cell / 4, cell / 4)) + 1
            srcs.append((min(max(i, 1), n), min(max(j, 1), n), 11))
    nsrc = len(srcs)
    if nsrc < world:
        raise SystemExit("%d sources for %d ranks" % (nsrc, world))
    parts = shard.partition([1] * nsrc, world)
    srcs = [srcs[q] for q in parts[rank]]  # this rank's sources
    ridx = torch.tensor([1 + (n // nrec_side) // 2 + (n // nrec_side) * q for q in range(nrec_side)],
                        device="cuda")
    rec = (1, ridx.view(-1, 1), ridx.view(1, -1))  # (k, j, i): top face

    fdt = torch.float32 if args.field_dtype == "f32" else torch.float64

    def t0_of(sp_):
        t = torch.full((n + 2,) * 3, 10e15 * 1.0, dtype=fdt, device="cuda")
        t[sp_[2], sp_[1], sp_[0]] = 0.0
        return t

    tol = 1e-10
    tobs = []
    with torch.no_grad():
        for sp_ in srcs:
            tobs.append(tomo.solve(t0_of(sp_), h, M_true, tol=tol)[rec].clone())
    del M_true
    torch.cuda.synchronize()
    setup_s = time.perf_counter() - t0
    reps = []
    tomo.collect_reports(reps)

    B = max(1, min(args.adj_batch, len(srcs)))
    if B > 1:
        T0s = torch.stack([t0_of(sp_) for sp_ in srcs])
        tobs_s = torch.stack(tobs)
        brec = (slice(None),) + rec

    def step():
        s = (1.0 / vz0).requires_grad_(True)
        e = eps0.clone().requires_grad_(True)
        if param:
            Mg = None
            Ml = [s, e] + list(axis0)
        else:
            Mg = [m.double() for m in media.metric_from(1.0 / s, e, ax0)]
            Ml = [m.detach().requires_grad_(True) for m in Mg]
        loss = torch.zeros((1,), dtype=torch.float64, device="cuda")
        if B > 1:  # B sources per batched forward solve and batched adjoint
            for c0 in range(0, len(srcs), B):
                T = tomo.solve_batch(T0s[c0:c0 + B], h, Ml, tol=tol, adj_tol=args.adj_tol)
                Ls = 0.5 * ((T[brec].double() - tobs_s[c0:c0 + B].double()) ** 2).sum()
                Ls.backward()
                loss += Ls.detach()
        else:
            for sp_, to in zip(srcs, tobs):
                T = tomo.solve(t0_of(sp_), h, Ml, tol=tol, adj_tol=args.adj_tol)
                Ls = 0.5 * ((T[rec].double() - to.double()) ** 2).sum()
                Ls.backward()
                loss += Ls.detach()
        if Mg is not None:
            torch.autograd.backward(Mg, [m.grad for m in Ml])
        shard.sum_over_ranks_([loss, s.grad, e.grad], dist)  # the survey's loss and gradient on every rank
        return float(loss), s.grad, e.grad

    def sync_all():
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    for _ in range(args.warmup):
        step()
    reps.clear()
    stream = torch.cuda.current_stream()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    sync_all()
    with ClockSampler(local) as clk:
        ev0.record(stream)
        for _ in range(args.steps):
            loss, gs, ge = step()
        ev1.record(stream)
        sync_all()
    tomo.collect_reports(None)
    ms = max_over_ranks(ev0.elapsed_time(ev1) / args.steps, dist)
    if B > 1:
        fr = [r for k, r in reps if k == "forward_batch"]
        ar = [r for k, r in reps if k == "adjoint_batch"]
        # a batch's reports share its elapsed time; count it once per batch
        per_batch = lambda rs: [rs[q:q + B] for q in range(0, len(rs), B)]
        fwd = sum(g[0].elapsed_ms for g in per_batch(fr)) / len(fr)
        adj = sum(g[0].elapsed_ms for g in per_batch(ar)) / len(ar)
        # forward: one graph per batch (its table kernel, then per sweep six passes and the restage
        # kernel); adjoint: one launch per direction pass of the slowest instance, plus one gradient
        # launch per source
        launches = sum(7 * max(r.sweeps for r in g) + 1 for g in per_batch(fr)) + \
            sum(6 * max(r.sweeps for r in g) + len(g) for g in per_batch(ar))
    else:
        fr = [r for k, r in reps if k == "forward"]
        ar = [r for k, r in reps if k == "adjoint"]
        fwd = sum(r.elapsed_ms for r in fr) / len(fr)
        adj = sum(r.elapsed_ms for r in ar) / len(ar)
        # one launch per direction pass (forward and backward), plus the gradient
        launches = sum(6 * r.sweeps for r in fr) + sum(6 * r.sweeps + 1 for r in ar)
    launches = int(over_ranks([launches], dist, "sum")[0])
    cpu = None  # timed on a single process only
    if world == 1 and not args.no_cpu and (n + 2) ** 3 > 322 ** 3:
        cpu = {"value": None, "unit": "source-gradients/s", "cores": 0, "kind": "port",
               "sample": "skipped: grids above 320^3 (the CPU adjoint's per-cell records need ~110 B a cell)"}
    elif world == 1 and not args.no_cpu:
        # source 0 in the starting medium, its field and winner record from one more (untimed) solve
        try:
            import fold3dpmm as f3d

            M32 = [(1.0 / vz0).contiguous(), eps0.contiguous()] + list(axis0) if param else \
                [m.double().float().contiguous() for m in media.metric_from(1.0 / (1.0 / vz0), eps0, ax0)]
            Tc = t0_of(srcs[0]).double()
            T0h = Tc.cpu().numpy()
            Wc = torch.empty(Tc.shape, dtype=torch.uint8, device="cuda")
            f3d.solve_ellip_record(tomo.context(), Tc, h, M32, Wc, f3d.opts(max_sweeps=1000, fixed=False, tol=tol))
            rh = torch.zeros_like(Tc)
            rh[rec] = Tc[rec] - tobs[0].double()
            Th, Wh, rh = Tc.cpu().numpy(), Wc.cpu().numpy(), rh.cpu().numpy()
            Mh = [m.cpu().numpy() for m in M32]
            del Tc, Wc, M32
            sw = sum(r.sweeps for r in fr) / len(fr)
            per_src, sweep_s, adj_s = oracle_adjoint_sample(T0h, Th, Mh, h, Wh, rh, sw)
            cpu = {"value": 1.0 / per_src, "unit": "source-gradients/s", "cores": host_threads(), "kind": "port",
                   "sample": "source 0: one recording forward sweep (%.2f s) x the GPU's mean %.1f forward sweeps "
                             "+ the whole FP64 adjoint from its winner record (%.2f s); this repository's CPU "
                             "statement (no reference implementation exists), OpenMP" % (sweep_s, sw, adj_s)}
        except Exception as e:
            cpu = {"value": None, "unit": "source-gradients/s", "cores": 0, "kind": "port",
                   "sample": "unavailable: %s" % str(e).splitlines()[0]}
    out = {
        "metric": "source-gradients/s", "value": nsrc / (ms / 1e3), "unit": "source-gradients/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
        "scaling": "strong", "vs_baseline": None, "dtype": args.field_dtype,
        "data": "synthetic: seeded heterogeneous TTI true medium (seed 2), smoothed starting medium",
        "config": {"workload": "tomography gradient %d^3 h=10 m, %d sources (jittered %dx%d, k=11), %d receivers "
                               "(%dx%d, k=1), loss 1/2 sum (t-t_obs)^2, solves to max|dT|<=1e-10"
                               % (n, nsrc, nsrc_side, nsrc_side, nrec_side ** 2, nrec_side, nrec_side),
                   "grid": n, "sources": nsrc, "receivers": nrec_side ** 2,
                   "gradient": "slowness and eps (torch autograd over the C-ABI)", "adjoint_tol": args.adj_tol,
                   "medium": "4 FP64 parameter words per cell (slowness, eps, axis x, y); gradients with respect "
                             "to them from the library" if param else "6 float32 metric words per cell; torch's "
                             "chain rule from dL/dM",
                   "sources_per_batch": B,
                   "parallelism": "sources split over %d ranks, gradient summed by all-reduce" % world
                   if world > 1 else "single",
                   "sources_per_rank": [len(q) for q in parts]},
        "forward_ms_per_source": fwd, "adjoint_ms_per_source": adj, "adjoint_over_forward": adj / fwd,
        "forward_sweeps": [min(r.sweeps for r in fr), max(r.sweeps for r in fr)],
        "adjoint_sweeps": [min(r.sweeps for r in ar), max(r.sweeps for r in ar)],
        "harness_ms_per_source": ms / nsrc - fwd - adj, "loss": loss,
        "grad_norms": {"slowness": float(gs.norm()), "eps": float(ge.norm())},
        "clocks": clk.summary(), "setup_s": setup_s, "gpu_launches": launches, "cpu_baseline": cpu,
    }
    if rank == 0:
        print(json.dumps(out))
    if dist is not None:
        dist.destroy_process_group()


def workload_config(args):
    what = "run to max|dT| = 0" if getattr(args, "converge", False) else "%d sweeps" % args.sweeps
    return {"workload": "fold-ref %d^3 implicit-surface source, %s" % (args.size, what),
            "grid": args.size, "sweeps": args.sweeps, "medium": "F=1.1 a=(-0.35,0.4,0.7)",
            "spacing": "h=10/(n-1)", "engine": args.engine, "skip": bool(args.skip), "variant": args.variant,
            "l2": "field %.2f GB > 126 MB L2; no flush needed" % ((args.size + 2) ** 3 * 8 / 1e9),
            "parallelism": "replicas" if args.gpus > 1 else "single"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--size", type=int, default=1280)
    ap.add_argument("--sweeps", type=int, default=8)
    ap.add_argument("--engine", choices=["planes", "wavefront", "auto"], default="auto")
    ap.add_argument("--skip", type=int, default=1,
                    help="1: skip tiles whose inputs did not change (result identical bit for bit; the "
                         "JSON line reports evaluated updates beside nominal ones); 0: evaluate all")
    ap.add_argument("--variant", choices=["fast", "literal", "compact"], default="fast",
                    help="local-solver form (identical results)")
    ap.add_argument("--batch", type=int, default=256, help="instances of --medium batch")
    ap.add_argument("--batch-dims", type=int, nargs=2, default=(96, 320), help="grid size range per axis")
    ap.add_argument("--batch-config", type=int, nargs=2, default=(0, 0), metavar=("ROWS", "CTAS"),
                    help="--medium batch: tile rows (2, 4, 8) and CTAs per SM of the batched kernel; 0 0: the "
                         "library's autotuner (default)")
    ap.add_argument("--adj-size", type=int, default=256, help="grid of --medium adjoint")
    ap.add_argument("--spacing", type=float, default=10.0, help="--medium tti: grid spacing h (m)")
    ap.add_argument("--source", choices=["depth", "top"], default="depth",
                    help="--medium tti: point source in the centre column at depth index n/8, or at the "
                         "top-face centre")
    ap.add_argument("--field-dtype", choices=["f64", "f32"], default="f64",
                    help="--medium tti/batch/adjoint: float64 fields, or the float32 build of the elliptical "
                         "solver (and adjoint)")
    ap.add_argument("--adj-batch", type=int, default=64,
                    help="--medium adjoint: sources per batched forward solve and adjoint (1: one by one)")
    ap.add_argument("--adj-tol", type=float, default=1e-12,
                    help="--medium adjoint: backward sweeps stop once one pushes at most this fraction of the "
                         "first sweep's largest push (0: until nothing is pushed)")
    ap.add_argument("--tti-medium", choices=["param", "metric"], default="param",
                    help="--medium tti: the FP64 parameter medium (slowness, eps, axis; float64 fields) or six "
                         "float32 metric arrays")
    ap.add_argument("--medium", choices=["fold", "tti", "batch", "adjoint"], default="fold",
                    help="fold: the reference's drift medium and source (default); tti: the "
                         "heterogeneous tilted-elliptical configuration")
    ap.add_argument("--converge", action="store_true",
                    help="run each solve until max|dT| == 0 instead of a fixed sweep count")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--ref-seconds", type=float, default=4.0)
    ap.add_argument("--cpu-seconds", type=float, default=10.0)
    ap.add_argument("--prof-nz", type=int, default=0,
                    help="with --prof-sweep: planes along z (the grid is size x size x prof-nz), to profile the "
                         "kernels of large z-normal planes on a small field")
    ap.add_argument("--prof-sweep", type=int, default=0,
                    help="profiling aid: run sweeps 1..S-1, then sweep S inside a CUDA profiler range "
                         "(for ncu --profile-from-start off), then exit")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)
    if args.medium == "tti":
        return run_tti(args)
    if args.medium == "adjoint":
        return run_adjoint(args)
    if args.medium == "batch":
        return run_batch(args)

    import numpy as np
    import torch

    import fold3dpmm as f3d

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = init_ranks(local)

    n, sweeps = args.size, args.sweeps
    h = 10.0 / (n - 1.0)
    engine = {"planes": f3d.ENGINE_PLANES, "wavefront": f3d.ENGINE_WAVEFRONT, "auto": f3d.ENGINE_AUTO}[args.engine]
    variant = {"fast": f3d.VARIANT_FAST, "literal": f3d.VARIANT_LITERAL, "compact": f3d.VARIANT_COMPACT}[args.variant]
    opts = f3d.opts(max_sweeps=sweeps, fixed=True, engine=engine, skip=bool(args.skip), variant=variant)
    if args.converge:
        opts = f3d.opts(max_sweeps=2000, fixed=False, tol=0.0, engine=engine, skip=bool(args.skip),
                        variant=variant)

    ctx = f3d.Context(local)
    stream = torch.cuda.current_stream()
    sp = stream.cuda_stream
    nz = args.prof_nz if (args.prof_sweep > 0 and args.prof_nz > 0) else n
    shape = (nz + 2, n + 2, n + 2)
    large = load_large_digests() if nz == n else {}
    parity = {}

    # the initial field: the reference's ImplicitInitialiser built on the
    # device (fold3d_init_implicit_device), kept in HBM and in pinned memory
    T0_dev = torch.empty(shape, dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    f3d.init_implicit_device(ctx, T0_dev, h, stream=sp)
    torch.cuda.synchronize()
    init_dev_s = time.perf_counter() - t0
    T0_pin = torch.empty(shape, dtype=torch.float64).pin_memory()
    T0_pin.copy_(T0_dev)
    T0_host = T0_pin.numpy()
    init_s = None
    if ("n%d_init" % n) in large:
        parity["init_reference_digest"] = "match" if sha256_of(T0_host) == large["n%d_init" % n] else "MISMATCH"
    elif n <= 640 and nz == n:  # against the host initialiser (pinned to the reference by the tests)
        t0 = time.perf_counter()
        Th = f3d.init_implicit(n, n, n, h)
        init_s = time.perf_counter() - t0
        parity["init_host"] = "match" if np.array_equal(Th.view(np.uint64), T0_host.view(np.uint64)) else "MISMATCH"
        del Th
    if "MISMATCH" in parity.values():
        raise RuntimeError("device initialiser differs from the reference: %s" % parity)
    out_pin = torch.empty(shape, dtype=torch.float64).pin_memory()
    T_dev = torch.empty_like(T0_dev)

    def step():
        T_dev.copy_(T0_dev)
        return ctx.solve(T_dev, h, None, opts, stream=sp)

    if args.prof_sweep > 0:
        if args.prof_sweep > 1:
            T_dev.copy_(T0_dev)
            ctx.solve(T_dev, h, None, f3d.opts(max_sweeps=args.prof_sweep - 1, fixed=True, engine=engine,
                                               skip=bool(args.skip), variant=variant), stream=sp)
        else:
            T_dev.copy_(T0_dev)
        torch.cuda.synchronize()
        torch.cuda.profiler.start()
        r1 = ctx.solve(T_dev, h, None, f3d.opts(max_sweeps=1, fixed=True, engine=engine, skip=bool(args.skip),
                                                variant=variant), stream=sp)
        torch.cuda.synchronize()
        torch.cuda.profiler.stop()
        print(json.dumps({"prof_sweep": args.prof_sweep, "sweep_ms": r1.elapsed_ms,
                          "updates": r1.nominal_updates, "evaluated": r1.evaluated_updates}))
        ctx.close()
        return

    rep = None
    for _ in range(args.warmup):
        rep = step()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    kernel_ms = 0.0
    evaluated = 0
    with ClockSampler(local) as clk:
        ev0.record(stream)
        for _ in range(args.steps):
            rep = step()
            kernel_ms += rep.elapsed_ms
            evaluated += rep.evaluated_updates
        ev1.record(stream)
        torch.cuda.synchronize()
    ms = ev0.elapsed_time(ev1)
    ms = max_over_ranks(ms, dist)
    clocks = clk.summary()
    if args.converge:
        sweeps = rep.sweeps
    upd = nominal_updates(n, sweeps)
    value = world * upd * args.steps / (ms / 1e3) / 1e9
    engine_ran = {1: "planes", 2: "wavefront"}.get(rep.engine, str(rep.engine))
    launches_per_step = sweeps * 6 * (n - 1) if rep.engine == f3d.ENGINE_PLANES else sweeps * 6

    # end to end through the host entry point (pinned in, pinned out)
    e2e = None
    if not args.no_e2e:
        ctx.solve(T0_pin, h, None, opts, stream=sp, out=out_pin)  # warm: allocates the context buffer
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(args.steps):
            ctx.solve(T0_pin, h, None, opts, stream=sp, out=out_pin)
        e1.record(stream)
        torch.cuda.synchronize()
        ems = e0.elapsed_time(e1)
        ems = max_over_ranks(ems, dist)
        nb = T0_pin.numel() * 8
        e2e = {"value": world * upd * args.steps / (ems / 1e3) / 1e9, "unit": "Gcell-updates/s",
               "h2d_bytes_per_step": nb, "d2h_bytes_per_step": nb, "ms_per_step": ems / args.steps}
        T0_dev.copy_(out_pin)  # the initial field is not needed any more: compare on the device
        if not torch.equal(T0_dev.view(torch.int64), T_dev.view(torch.int64)):
            raise RuntimeError("host-path result differs from the device-path result")
        del T0_dev
    # the solve's result against the reference's own (sha256 of its field)
    key = "n%d_s%d" % (n, sweeps)
    if not args.converge and key in large:
        res = out_pin.numpy() if e2e is not None else T_dev.cpu().numpy()
        parity["result_reference_digest"] = "match" if sha256_of(res) == large[key] else "MISMATCH"
        if parity["result_reference_digest"] != "match":
            print("bench: the result differs from the reference's (%s)" % key, file=sys.stderr)
    elif not args.converge:
        parity["result_reference_digest"] = "no reference digest for %s" % key

    peak, peak_kind = load_peaks()
    solve_ms = kernel_ms / args.steps
    alg_bytes = BYTES_PER_UPDATE * upd
    launches = launches_per_step * args.steps
    achieved = alg_bytes / (solve_ms / 1e3) / 1e9
    # DRAM bytes per launch: the bytes per update that ncu measured for this
    # kernel (profiles/wave_pass_kernel_fold512_full.md) times this launch's
    # updates, and the FP64 pipe's share of the active cycles from the capture
    # of the same code path (512^2 planes: CTA items; 1280^2 planes: warp
    # items, profiles/wave_pass_kernel_fold1280_planes.md)
    wave = rep.engine == f3d.ENGINE_WAVEFRONT
    upd_launch = upd / launches_per_step
    traffic = WAVE_DRAM_BYTES_PER_UPDATE * upd_launch if wave else None
    large_planes = n * n >= 8192 * 128
    fp64 = None
    if wave:
        fp64 = ({"pct_of_active_cycles": 35.0, "issue_active_pct": 71.9,
                 "capture": "k_up pass over 1280^2 planes (1280x1280x16 grid, sweep 2) of the kernel built for 8 CTAs "
                            "per SM (64 registers); the kernel timed here is built for 7 (72 registers)"} if large_planes else
                {"pct_of_active_cycles": 30.5, "issue_active_pct": 50.9,
                 "capture": "x_down, x_up, k_up passes of sweep 3 at 512^3 (mean)"})
    roofline = {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "traffic": traffic, "peak_kind": peak_kind,
                "kernel": "plane_kernel" if rep.engine == f3d.ENGINE_PLANES else "wave_pass_kernel<drift>",
                "alg_bytes_per_launch": alg_bytes / launches_per_step,
                "avg_launch_us": solve_ms * 1e3 / launches_per_step,
                "note": "FP64 latency bound, not HBM bound: ~100 dependent FP64 operations per 16 B",
                "fp64_pipe": fp64,
                "traffic_note": ("ncu's %.2f DRAM bytes per update (512^3, three passes of a sweep without tile "
                                 "skipping) x %.4g updates per launch; each target is read once, the source "
                                 "plane comes from L2" % (WAVE_DRAM_BYTES_PER_UPDATE, upd_launch)) if wave else None}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        try:
            rate, info = reference_cpu_sample(T0_pin.numpy(), n, seconds=args.cpu_seconds, threads=host_threads())
            cpu = {"value": rate / 1e9, "unit": "Gcell-updates/s", "cores": info["cores"], "kind": info["kind"],
                   "sample": info["sample"]} | single_thread_reference(T0_pin.numpy(), n)
        except Exception as e:
            cpu = {"value": None, "unit": "Gcell-updates/s", "cores": 0, "kind": "reference",
                   "sample": "unavailable: %s" % str(e).splitlines()[0]}

    pub = published_rate(n, sweeps) if (sweeps == 8 and not args.converge) else None
    out = {
        "metric": "Gcell-updates/s", "value": value, "unit": "Gcell-updates/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": (value / pub) if pub else None, "dtype": "f64",
        "data": "synthetic: reference implicit-surface source and drift medium (no dataset)",
        "config": workload_config(args) | {"engine": engine_ran},
        "roofline": roofline, "cpu_baseline": cpu, "e2e": e2e, "gpu_launches": launches,
        "clocks": clocks, "solve_ms": solve_ms, "evaluated_updates_per_step": evaluated / args.steps,
        "init_s": init_s, "init_device_s": init_dev_s, "host_threads": host_threads(), "parity": parity,
    }
    if rank == 0:
        print(json.dumps(out))
    ctx.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
