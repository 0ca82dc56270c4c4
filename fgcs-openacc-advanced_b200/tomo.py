"""Traveltime-tomography harness: the elliptical solver as a differentiable
torch operation.  torch is used here only as the harness; the forward solve
and its adjoint run in libfold3dpmm (fold3d_solve_ellip_record,
fold3d_adjoint_ellip).

EllipSolve.apply(T0, h, max_sweeps, tol, adj_tol, *M) returns the converged
field for the initial field T0 (a point source; float64, or float32 for the
float32 build) and a medium M in the field layout: either six CUDA tensors of
the metric, xx xy xz yy yz zz (the solver stores them as float32), or four
float64 CUDA tensors of the FP64 parameter medium, slowness, eps and the
axis's x and y components (fold3d_*_tti; gradients with respect to them).  tol stops the forward sweeps (max |dT| <= tol), adj_tol the
backward ones (fold3d_adjoint_ellip's tol).
Its backward pass returns dL/dM in float64, so torch carries the gradient on
to whatever produced M (slowness, epsilon and axis through
media.metric_from).
"""
from __future__ import annotations

import torch

import fold3dpmm as f3d

_ctx = {}
_reports = None


def collect_reports(lst):
    """Append (kind, fold3d_report) of every later library call to lst, kind
    "forward" | "adjoint" | "forward_batch" | "adjoint_batch" (one report per
    instance of a batch); None stops collecting."""
    global _reports
    _reports = lst


def _note(kind, rep):
    if _reports is not None:
        _reports.append((kind, rep))
    return rep


def context(device=None) -> f3d.Context:
    """The library context of a device (default: the current one), created
    once per process."""
    dev = torch.cuda.current_device() if device is None else device
    if dev not in _ctx:
        _ctx[dev] = f3d.Context(dev)
    return _ctx[dev]


def _stored(M):
    """The medium as the library reads it: four FP64 parameter arrays (s,
    eps, nx, ny; fold3d_*_tti) as they are, or six metric arrays rounded to
    float32 (fold3d_*_ellip)."""
    if f3d.is_tti(M):
        return [m.detach().to(torch.float64).contiguous() for m in M]
    return [m.detach().to(torch.float32).contiguous() for m in M]


class EllipSolve(torch.autograd.Function):
    @staticmethod
    def forward(ctx, T0, h, max_sweeps, tol, adj_tol, *M):
        M32 = _stored(M)
        T = T0.detach().clone()
        W = torch.empty(T.shape, dtype=torch.uint8, device=T.device)
        ctx.mdtypes = [m.dtype for m in M]
        rep = _note("forward", f3d.solve_ellip_record(context(T.device.index), T, h, M32, W,
                                                      f3d.opts(max_sweeps=max_sweeps, fixed=False, tol=tol)))
        ctx.save_for_backward(T, W, *M32)
        ctx.h = h
        ctx.sweeps = rep.sweeps
        ctx.adj_tol = adj_tol
        return T

    @staticmethod
    def backward(ctx, gT):
        T, W, *M32 = ctx.saved_tensors
        lam = torch.empty_like(T)
        ng = len(M32)
        dLdM = torch.empty((ng,) + tuple(T.shape), dtype=T.dtype, device=T.device)
        _note("adjoint", f3d.adjoint_ellip(context(T.device.index), T, ctx.h, M32, W, gT.to(T.dtype).contiguous(),
                                           lam, dLdM, tol=ctx.adj_tol))
        return (None, None, None, None, None) + tuple(dLdM[m].to(ctx.mdtypes[m]) for m in range(ng))


def solve(T0, h, M, max_sweeps=1000, tol=0.0, adj_tol=0.0):
    return EllipSolve.apply(T0, h, max_sweeps, tol, adj_tol, *M)


class EllipSolveBatch(torch.autograd.Function):
    """Many sources in one medium: T0s (S, nz+2, ny+2, nx+2) initial fields,
    one per source.  The forward solves all S at once (fold3d_solve_batch
    with winner records), the backward runs their adjoints at once
    (fold3d_adjoint_batch) and sums the S gradients into one dL/dM."""

    @staticmethod
    def forward(ctx, T0s, h, max_sweeps, tol, adj_tol, *M):
        M32 = _stored(M)
        T = T0s.detach().clone().contiguous()
        W = torch.empty(T.shape, dtype=torch.uint8, device=T.device)
        S = T.shape[0]
        ctx.mdtypes = [m.dtype for m in M]
        reps = f3d.solve_batch(context(T.device.index), [T[s] for s in range(S)], [h] * S, [M32] * S,
                               f3d.opts(max_sweeps=max_sweeps, fixed=False, tol=tol),
                               winners=[W[s] for s in range(S)])
        for r in reps:
            _note("forward_batch", r)
        ctx.save_for_backward(T, W, *M32)
        ctx.h = h
        ctx.adj_tol = adj_tol
        return T

    @staticmethod
    def backward(ctx, gT):
        T, W, *M32 = ctx.saved_tensors
        S = T.shape[0]
        gT = gT.to(T.dtype).contiguous()
        lam = torch.empty_like(T)
        ng = len(M32)
        dLdM = torch.zeros((ng,) + tuple(T.shape[1:]), dtype=T.dtype, device=T.device)
        reps = f3d.adjoint_batch(context(T.device.index), [T[s] for s in range(S)], [ctx.h] * S, [M32] * S,
                                 [W[s] for s in range(S)], [gT[s] for s in range(S)], [lam[s] for s in range(S)],
                                 [dLdM] * S, tol=ctx.adj_tol, accumulate=True)
        for r in reps:
            _note("adjoint_batch", r)
        return (None, None, None, None, None) + tuple(dLdM[m].to(ctx.mdtypes[m]) for m in range(ng))


def solve_batch(T0s, h, M, max_sweeps=1000, tol=0.0, adj_tol=0.0):
    """Fields of all sources (S, ...) in medium M, differentiable in M."""
    return EllipSolveBatch.apply(T0s, h, max_sweeps, tol, adj_tol, *M)
