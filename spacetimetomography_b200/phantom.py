"""Seeded synthetic inputs for the benchmark configurations.

The reference ships no dataset (its KAUST scans are external), so these
generators stand in for measured data:

* random ellipsoid phantoms: centres uniform in the inner 80% of the volume,
  semi-axes uniform in [lo, hi] voxels, a uniformly random orientation,
  additive densities uniform in [0.1, 1];
* an optional porous background of uniform-random spheres (radius 2-6 voxels)
  of density 0.5;
* the smooth deformation u(x, t) = A sin(2 pi t / T + phi) (sin kx, sin ky, sin kz)
  applied to the ellipsoid centres of each frame;
* additive Gaussian noise of a given fraction of the sinogram's RMS.

Random streams come from numpy's PCG64 seeded by the caller; volumes are
rasterised with torch on whatever device is given (CPU in tests, the GPU in
the benchmark), float32, layout (nz, ny, nx).
"""
from __future__ import annotations

import math

import numpy as np


def _rand_rotation(rng: np.random.Generator) -> np.ndarray:
    q = rng.normal(size=4)
    q /= np.linalg.norm(q)
    w, x, y, z = q
    return np.array([[1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
                     [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
                     [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])


def ellipsoid_params(n: int, dims, seed: int, semi=(5.0, 40.0), density=(0.1, 1.0)):
    """List of (centre[3], semi-axes[3], rotation[3x3], density), centres in voxel (x,y,z)."""
    rng = np.random.default_rng(seed)
    d = np.asarray(dims, np.float64)
    out = []
    for _ in range(n):
        c = rng.uniform(0.1 * (d - 1), 0.9 * (d - 1))
        a = rng.uniform(semi[0], semi[1], 3)
        R = _rand_rotation(rng)
        rho = rng.uniform(density[0], density[1])
        out.append((c, a, R, rho))
    return out


def rasterize(params, dims, device="cpu", background=None):
    """Sum of ellipsoid indicator functions (and optional background) at voxel centres."""
    import torch

    nx, ny, nz = dims
    vol = torch.zeros((nz, ny, nx), dtype=torch.float32, device=device)
    if background is not None:
        vol += background.to(device)
    zs = torch.arange(nz, device=device, dtype=torch.float32)
    ys = torch.arange(ny, device=device, dtype=torch.float32)
    xs = torch.arange(nx, device=device, dtype=torch.float32)
    for c, a, R, rho in params:
        r = float(np.max(a)) + 1.0
        lo = [max(0, int(math.floor(c[k] - r))) for k in range(3)]
        hi = [min(dims[k], int(math.ceil(c[k] + r)) + 1) for k in range(3)]
        if any(hi[k] <= lo[k] for k in range(3)):
            continue
        Z, Y, X = torch.meshgrid(zs[lo[2]:hi[2]] - c[2], ys[lo[1]:hi[1]] - c[1], xs[lo[0]:hi[0]] - c[0],
                                 indexing="ij")
        Rt = torch.tensor(R.T, dtype=torch.float32, device=device)  # body coords = R^T (p - c)
        u = Rt[0, 0] * X + Rt[0, 1] * Y + Rt[0, 2] * Z
        v = Rt[1, 0] * X + Rt[1, 1] * Y + Rt[1, 2] * Z
        w = Rt[2, 0] * X + Rt[2, 1] * Y + Rt[2, 2] * Z
        inside = (u / a[0]) ** 2 + (v / a[1]) ** 2 + (w / a[2]) ** 2 <= 1.0
        vol[lo[2]:hi[2], lo[1]:hi[1], lo[0]:hi[0]] += inside.to(torch.float32) * float(rho)
    return vol


def porous_background(dims, seed: int, count: int, radius=(2.0, 6.0), density=0.5, device="cpu",
                      chunk: int = 4096):
    """Uniform-random spheres of the given density (the 512^3 workload's
    background): `count` centres uniform over the volume, radii uniform in
    `radius`; a voxel whose centre lies in any sphere gets `density`.  The
    spheres are rasterised `chunk` at a time over their bounding boxes."""
    import torch

    rng = np.random.default_rng(seed)
    nx, ny, nz = dims
    centres = rng.uniform([0, 0, 0], [nx - 1, ny - 1, nz - 1], (count, 3))
    radii = rng.uniform(radius[0], radius[1], count)
    bg = torch.zeros(nz * ny * nx, dtype=torch.float32, device=device)
    rmax = int(math.ceil(radius[1])) + 1
    o = torch.arange(-rmax, rmax + 1, device=device, dtype=torch.float32)
    oz, oy, ox = torch.meshgrid(o, o, o, indexing="ij")
    offs = torch.stack([ox.reshape(-1), oy.reshape(-1), oz.reshape(-1)], 1)  # (K, 3) integer offsets
    lim = torch.tensor([nx - 1, ny - 1, nz - 1], device=device, dtype=torch.float32)
    for s in range(0, count, chunk):
        c = torch.as_tensor(centres[s:s + chunk], device=device, dtype=torch.float32)
        r = torch.as_tensor(radii[s:s + chunk], device=device, dtype=torch.float32)
        p = torch.floor(c)[:, None, :] + offs[None]  # (m, K, 3) voxel centres around each sphere
        inside = (((p - c[:, None, :]) ** 2).sum(-1) <= (r * r)[:, None]) & (p >= 0).all(-1) & (p <= lim).all(-1)
        q = p[inside].long()
        bg[q[:, 0] + nx * (q[:, 1] + ny * q[:, 2])] = density
    return bg.view(nz, ny, nx)


def ellipsoid_phantom(dims, n: int, seed: int, semi=(5.0, 40.0), device="cpu"):
    return rasterize(ellipsoid_params(n, dims, seed, semi), dims, device)


def displaced_params(params, t: float, period: float, amplitude: float = 4.0,
                     k: float = 2 * math.pi / 256, phase: float = 0.0):
    """Centres moved by u(c, t) = A sin(2 pi t/T + phi) (sin k cx, sin k cy, sin k cz)."""
    s = amplitude * math.sin(2 * math.pi * t / period + phase)
    out = []
    for c, a, R, rho in params:
        u = s * np.sin(k * np.asarray(c))
        out.append((np.asarray(c) + u, a, R, rho))
    return out


def deformation_flow(dims, t0: float, t1: float, period: float, amplitude: float = 4.0,
                     k: float = 2 * math.pi / 256, phase: float = 0.0, device="cpu"):
    """u(x, t1) - u(x, t0) as a (3, nz, ny, nx) field (the true inter-frame motion)."""
    import torch

    nx, ny, nz = dims
    s = amplitude * (math.sin(2 * math.pi * t1 / period + phase) - math.sin(2 * math.pi * t0 / period + phase))
    fx = torch.sin(k * torch.arange(nx, device=device, dtype=torch.float32)) * s
    fy = torch.sin(k * torch.arange(ny, device=device, dtype=torch.float32)) * s
    fz = torch.sin(k * torch.arange(nz, device=device, dtype=torch.float32)) * s
    # sin(k x) vanishes exactly at the nodes x = 0, pi/k, ...; float rounding
    # leaves ~1e-16 there, which the semi-Lagrangian trace would resolve
    # differently in FP32 and FP64 (the clamped tricubic sampler is
    # discontinuous across cell boundaries), so the exact zeros are restored.
    fx, fy, fz = (torch.where(v.abs() < 1e-6 * max(abs(s), 1e-30), torch.zeros_like(v), v) for v in (fx, fy, fz))
    flow = torch.empty((3, nz, ny, nx), dtype=torch.float32, device=device)
    flow[0] = fx.view(1, 1, nx).expand(nz, ny, nx)
    flow[1] = fy.view(1, ny, 1).expand(nz, ny, nx)
    flow[2] = fz.view(nz, 1, 1).expand(nz, ny, nx)
    return flow


def add_noise(proj, rel: float, seed: int):
    """proj + N(0, (rel * rms(proj))^2), seeded (torch generator on proj's device)."""
    import torch

    if rel <= 0:
        return proj.clone()
    rms = torch.sqrt(torch.mean(proj.double() ** 2)).item()
    g = torch.Generator(device=proj.device)
    g.manual_seed(seed)
    return proj + torch.randn(proj.shape, generator=g, device=proj.device, dtype=proj.dtype) * (rel * rms)


def golden_angle_views(n: int, start: float = 0.0) -> np.ndarray:
    """n angles (rad) stepping by the golden angle pi*(3 - sqrt 5)."""
    return (start + np.arange(n) * math.pi * (3.0 - math.sqrt(5.0))) % (2 * math.pi)


def equispaced_views(n: int, span: float = 2 * math.pi) -> np.ndarray:
    return np.arange(n, dtype=np.float64) * (span / n)
