"""Seeded synthetic inputs for benchmarks and examples (torch, on the GPU).

* ``foam_volume``: a 3-D foam -- random spheres of density 1 in a cylinder
  of density 0.2 -- the full-volume MBIR workload's phantom.
* ``ellipse_slices``: random-ellipse phantoms, one per slice.
* ``transmission_noise``: Poisson counting noise on line integrals,
  y = -ln(Poisson(I0 exp(-mu p)) / I0) / mu.
"""
from __future__ import annotations

import math

import torch


def foam_volume(S: int, n: int, n_spheres: int = 2000, rmin: float = 5.0, rmax: float = 60.0,
                matrix: float = 0.2, seed: int = 0, device="cuda", total: int = 0,
                first: int = 0) -> torch.Tensor:
    """Slices [first, first + S) of a foam volume of `total` slices (default S):
    the spheres are drawn for the whole volume, so a sub-volume equals the
    same slices of the whole one."""
    total = total if total > 0 else S
    if first < 0 or first + S > total:
        raise ValueError("slices [first, first + S) must lie inside the volume")
    g = torch.Generator(device="cpu").manual_seed(seed)
    vol = torch.zeros((S, n, n), dtype=torch.float32, device=device)
    yy = torch.arange(n, device=device, dtype=torch.float32) - (n - 1) / 2
    rad2 = yy[:, None] ** 2 + yy[None, :] ** 2
    R = 0.95 * n / 2
    vol += (rad2 <= R * R).to(torch.float32)[None] * matrix
    rs = rmin + (rmax - rmin) * torch.rand(n_spheres, generator=g)
    # centres inside the cylinder, any slice
    ang = 2 * math.pi * torch.rand(n_spheres, generator=g)
    rho = torch.sqrt(torch.rand(n_spheres, generator=g)) * (R - rs).clamp(min=0)
    cz = torch.rand(n_spheres, generator=g) * total - first
    cy = (n - 1) / 2 + rho * torch.sin(ang)
    cx = (n - 1) / 2 + rho * torch.cos(ang)
    for k in range(n_spheres):
        r = float(rs[k])
        z0, z1 = max(0, int(cz[k] - r)), min(S, int(cz[k] + r) + 1)
        y0, y1 = max(0, int(cy[k] - r)), min(n, int(cy[k] + r) + 1)
        x0, x1 = max(0, int(cx[k] - r)), min(n, int(cx[k] + r) + 1)
        if z0 >= z1 or y0 >= y1 or x0 >= x1:
            continue
        z = torch.arange(z0, z1, device=device, dtype=torch.float32) - float(cz[k])
        y = torch.arange(y0, y1, device=device, dtype=torch.float32) - float(cy[k])
        x = torch.arange(x0, x1, device=device, dtype=torch.float32) - float(cx[k])
        d2 = z[:, None, None] ** 2 + y[None, :, None] ** 2 + x[None, None, :] ** 2
        vol[z0:z1, y0:y1, x0:x1].masked_fill_(d2 <= r * r, 1.0)
    return vol


def ellipse_slices(S: int, n: int, n_ellipses: int = 10, seed: int = 0, device="cuda",
                   lo: float = 0.1, hi: float = 1.0) -> torch.Tensor:
    g = torch.Generator(device="cpu").manual_seed(seed)
    c = (torch.arange(n, device=device, dtype=torch.float32) - (n - 1) / 2) / (n / 2)
    yy, xx = c[:, None], c[None, :]
    out = torch.zeros((S, n, n), dtype=torch.float32, device=device)
    for s in range(S):
        for _ in range(n_ellipses):
            cx, cy = (torch.rand(2, generator=g) - 0.5).tolist()
            ax, ay = (0.08 + 0.32 * torch.rand(2, generator=g)).tolist()
            th = float(torch.rand(1, generator=g)) * math.pi
            rho = lo + (hi - lo) * float(torch.rand(1, generator=g))
            xr = (xx - cx) * math.cos(th) + (yy - cy) * math.sin(th)
            yr = -(xx - cx) * math.sin(th) + (yy - cy) * math.cos(th)
            out[s] += ((xr / ax) ** 2 + (yr / ay) ** 2 <= 1.0).to(torch.float32) * rho
    return out


def transmission_noise(p: torch.Tensor, I0: float = 1e4, max_atten: float = 3.0,
                       seed: int = 0) -> torch.Tensor:
    """Poisson noise at I0 counts; p is scaled so its maximum attenuates by max_atten."""
    mu = max_atten / float(p.max().clamp(min=1e-30))
    gen = torch.Generator(device=p.device).manual_seed(seed)
    counts = torch.poisson(I0 * torch.exp(-mu * p), generator=gen).clamp_(min=1.0)
    return -torch.log(counts / I0) / mu
