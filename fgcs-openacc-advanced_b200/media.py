"""Seeded synthetic media for the elliptical (tilted transversely isotropic)
solver.

The benchmark configurations name no public model, so media are generated
here from a seed.  A medium is the per-cell metric M = a I + b n n^T of a
tilted elliptical cell (a = 1/(Vz^2 (1 + 2 eps)), b = 1/Vz^2 - a, n the
symmetry axis), returned as six float32 arrays (xx, xy, xz, yy, yz, zz in the
i, j, k axes) in the field layout, shape (nz+2, ny+2, nx+2), ghost layer
copied from the nearest interior cell; or as the FP64 parameter medium
(slowness, eps and the axis's x and y components, four float64 arrays) from
which the solver forms M per cell (params_from, heterogeneous_tti_params).

heterogeneous_tti() follows the construction of the 512^3 configuration:
Vz = 1500 + 0.8 * depth (m), times 1 + the sum of 16 Gaussian anomalies of
+-15 % (sigma 20-60 cells at 512^3, centres uniform); eps uniform in
[0, 0.25] smoothed by a Gaussian of sigma 8 cells; tilt uniform in
[0, 45] degrees and azimuth uniform in [0, 360) degrees, smoothed likewise
through their unit vectors (no wrap-around).  Lengths in cells scale with
n / 512.  k is the depth axis.  Smoothing is an FFT convolution with a
periodic Gaussian, in float64.
"""
from __future__ import annotations

import math

import torch


def metric_from(vz, eps, n_axis):
    """M = a I + b n n^T (float64 tensors) -> six float32 tensors."""
    nx, ny, nz = n_axis
    nn = torch.sqrt(nx * nx + ny * ny + nz * nz)
    nx, ny, nz = nx / nn, ny / nn, nz / nn
    a = 1.0 / (vz * vz * (1.0 + 2.0 * eps))
    b = 1.0 / (vz * vz) - a
    comps = (a + b * nx * nx, b * nx * ny, b * nx * nz, a + b * ny * ny, b * ny * nz, a + b * nz * nz)
    return [c.to(torch.float32) for c in comps]


def params_from(vz, eps, n_axis):
    """The FP64 parameter medium (fold3d_tti) of a tilted elliptical cell:
    slowness s = 1/vz, eps, and the x, y components of the unit axis, the
    axis flipped where needed so that its z component is >= 0 (n and -n are
    the same axis).  Four float64 tensors."""
    nx, ny, nz = (a.to(torch.float64) for a in n_axis)
    nn = torch.sqrt(nx * nx + ny * ny + nz * nz)
    sg = torch.where(nz < 0, -1.0, 1.0).to(torch.float64)
    return [(1.0 / vz.to(torch.float64)).contiguous(), eps.to(torch.float64).contiguous(),
            (sg * nx / nn).contiguous(), (sg * ny / nn).contiguous()]


def homogeneous_tti(nx, ny, nz, vz, eps, tilt_deg, azimuth_deg, device="cpu"):
    """homogeneous_ellip() as the FP64 parameter medium (four arrays)."""
    th, ph = math.radians(tilt_deg), math.radians(azimuth_deg)
    shape = (nz + 2, ny + 2, nx + 2)
    f = lambda v: torch.full(shape, float(v), dtype=torch.float64, device=device)
    return params_from(f(vz), f(eps), (f(math.sin(th) * math.cos(ph)), f(math.sin(th) * math.sin(ph)),
                                       f(math.cos(th))))


def heterogeneous_tti_params(nx, ny, nz, h, seed=0, device="cpu", anomalies=16, dtype=torch.float64):
    """The seeded heterogeneous medium of heterogeneous_tti() as the FP64
    parameter medium (four float64 arrays, field layout, ghosts copied).
    dtype: working precision of the construction (float64 by default;
    float32 for grids too large for float64 temporaries, the parameters then
    being float32 values held in float64).  Each parameter array is padded as
    soon as it is formed."""
    vz, eps, (ax, ay, az) = tti_params(nx, ny, nz, h, seed, device, anomalies, dtype=dtype)
    # one parameter at a time, each padded as soon as it is formed and its
    # inputs freed: the peak stays near the construction's own (params_from's
    # arithmetic, in the working precision, then float64)
    s = _pad((1.0 / vz).to(torch.float64))
    del vz
    e = _pad(eps.to(torch.float64))
    del eps
    nn = torch.sqrt(ax * ax + ay * ay + az * az)
    sg = torch.where(az < 0, -1.0, 1.0).to(nn.dtype)
    del az
    nn.reciprocal_().mul_(sg)
    del sg
    ax.mul_(nn)
    ay.mul_(nn)
    del nn
    nx_ = _pad(ax.to(torch.float64))
    del ax
    ny_ = _pad(ay.to(torch.float64))
    del ay
    return [s, e, nx_, ny_]


def _pad(t):
    """(nz, ny, nx) interior -> (nz+2, ny+2, nx+2), ghosts copied from the nearest interior cell."""
    return torch.nn.functional.pad(t[None, None], (1, 1, 1, 1, 1, 1), mode="replicate")[0, 0].contiguous()


def homogeneous_ellip(nx, ny, nz, vz, eps, tilt_deg, azimuth_deg, device="cpu"):
    th, ph = math.radians(tilt_deg), math.radians(azimuth_deg)
    shape = (nz + 2, ny + 2, nx + 2)
    f = lambda v: torch.full(shape, float(v), dtype=torch.float64, device=device)
    return metric_from(f(vz), f(eps), (f(math.sin(th) * math.cos(ph)), f(math.sin(th) * math.sin(ph)),
                                       f(math.cos(th))))


def _smooth(x, sigma):
    """Periodic Gaussian smoothing of a (nz, ny, nx) tensor (float64 or
    float32; the result has its type).  The kernel is built from broadcast
    1-D frequency axes and applied in place, to keep the temporaries to the
    spectrum and one kernel array."""
    if sigma <= 0:
        return x
    spec = torch.fft.rfftn(x)
    ft = x.dtype
    k = [torch.fft.fftfreq(n, device=x.device, dtype=ft) for n in x.shape[:2]]
    k.append(torch.fft.rfftfreq(x.shape[2], device=x.device, dtype=ft))
    kz, ky, kx = k[0].view(-1, 1, 1), k[1].view(1, -1, 1), k[2].view(1, 1, -1)
    g = kx * kx + ky * ky + kz * kz
    g.mul_(-2.0 * (math.pi * sigma) ** 2).exp_()
    spec.mul_(g)
    del g
    return torch.fft.irfftn(spec, s=x.shape)


def heterogeneous_tti(nx, ny, nz, h, seed=0, device="cpu", anomalies=16, dtype=torch.float64):
    """Six float32 metric arrays of the seeded heterogeneous TTI medium.
    dtype: working precision of the construction (float32 for grids too large
    for float64 temporaries, e.g. 1280^3 on one GPU)."""
    vz, eps, axis = tti_params(nx, ny, nz, h, seed, device, anomalies, dtype=dtype)
    M = metric_slabs(vz, eps, axis)
    del vz, eps, axis
    for k in range(6):
        M[k] = _pad(M[k])
    return M


def tti_params(nx, ny, nz, h, seed=0, device="cpu", anomalies=16, pad=False, dtype=torch.float64):
    """The parameters of heterogeneous_tti(): (vz, eps, (ax, ay, az)) on the
    interior (nz, ny, nx), or in the field layout with pad=True.  dtype is the
    working precision: float64 (the default) or float32 for grids too large
    for float64 temporaries (the random numbers are drawn in float64 either
    way, from the same seeded stream).  Anomalies are accumulated from
    broadcast 1-D coordinates and arrays are freed as soon as they are used,
    so the peak is about twelve arrays of the grid's size."""
    gen = torch.Generator(device="cpu").manual_seed(seed)
    scale = max(nx, ny, nz) / 512.0
    shape = (nz, ny, nx)
    dev = torch.device(device)
    kz = torch.arange(nz, dtype=dtype, device=dev).view(nz, 1, 1)
    ky = torch.arange(ny, dtype=dtype, device=dev).view(1, ny, 1)
    kx = torch.arange(nx, dtype=dtype, device=dev).view(1, 1, nx)
    vz = (1500.0 + 0.8 * (kz * h)).expand(shape).clone()
    pert = torch.zeros(shape, dtype=dtype, device=dev)
    for _ in range(anomalies):
        c = torch.rand(3, generator=gen, dtype=torch.float64) * torch.tensor([nz, ny, nx], dtype=torch.float64)
        sig = (20.0 + 40.0 * torch.rand(1, generator=gen, dtype=torch.float64).item()) * scale
        amp = 0.15 if torch.rand(1, generator=gen).item() < 0.5 else -0.15
        r2 = (kz - c[0].item()) ** 2 + (ky - c[1].item()) ** 2 + (kx - c[2].item()) ** 2
        r2.neg_().div_(2.0 * sig * sig).exp_().mul_(amp)
        pert.add_(r2)
        del r2
    pert.add_(1.0)
    vz.mul_(pert)
    del pert
    sig = 8.0 * scale
    eps = _smooth((0.25 * torch.rand(shape, generator=gen, dtype=torch.float64)).to(dev, dtype), sig)
    th = torch.deg2rad(45.0 * torch.rand(shape, generator=gen, dtype=torch.float64)).to(dev, dtype)
    ph = torch.deg2rad(360.0 * torch.rand(shape, generator=gen, dtype=torch.float64)).to(dev, dtype)
    st = torch.sin(th)
    ax = st * torch.cos(ph)
    ay = st * torch.sin(ph)
    del st
    az = torch.cos(th)
    del th, ph
    ax, ay, az = _smooth(ax, sig), _smooth(ay, sig), _smooth(az, sig)
    eps = eps.clamp_(0.0, 0.25)
    if pad:
        return _pad(vz), _pad(eps), (_pad(ax), _pad(ay), _pad(az))
    return vz, eps, (ax, ay, az)


def metric_slabs(vz, eps, n_axis, planes=64):
    """metric_from() one block of z-planes at a time (the same values; the
    temporaries are a block's, not the volume's)."""
    nz = vz.shape[0]
    out = [torch.empty(vz.shape, dtype=torch.float32, device=vz.device) for _ in range(6)]
    for k0 in range(0, nz, planes):
        sl = slice(k0, min(nz, k0 + planes))
        for o, m in zip(out, metric_from(vz[sl], eps[sl], tuple(a[sl] for a in n_axis))):
            o[sl] = m
    return out


def _smooth_edges(x, sigma):
    """Gaussian smoothing without wrap-around: the (nz, ny, nx) tensor is
    extended by 3 sigma of edge copies on every side, smoothed periodically
    and cropped."""
    p = int(math.ceil(3.0 * sigma))
    big = torch.nn.functional.pad(x[None, None], (p,) * 6, mode="replicate")[0, 0]
    return _smooth(big, sigma)[p:-p, p:-p, p:-p].contiguous()


def smooth_params(vz, eps, axis, sigma):
    """Gaussian smoothing (sigma in cells, no wrap-around) of padded
    parameters: slowness and eps are smoothed, the axis through its
    components; ghosts re-copied."""
    inner = lambda t: t[1:-1, 1:-1, 1:-1]
    s = _smooth_edges(inner(1.0 / vz), sigma)
    return (_pad(1.0 / s), _pad(_smooth_edges(inner(eps), sigma)),
            tuple(_pad(_smooth_edges(inner(a), sigma)) for a in axis))


def exact_time(M6, dx, dy, dz):
    """sqrt(d^T M d) for one homogeneous metric (six floats) and offset d."""
    xx, xy, xz, yy, yz, zz = (float(m) for m in M6)
    q = xx * dx * dx + yy * dy * dy + zz * dz * dz + 2 * (xy * dx * dy + xz * dx * dz + yz * dy * dz)
    return math.sqrt(q)
