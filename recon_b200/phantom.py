"""Seeded synthetic phantoms and noisy projection data.

A phantom is a background cylinder of 0.02 /mm (radius 0.45 of the volume's
x-y extent, full height) plus random ellipsoids (uniform semi-axes, a rotation
drawn from the uniform quaternion distribution, additive attenuation),
voxelised at voxel centres.  Semi-axis ranges are 2-12 mm for a 32 mm
volume and scale with the volume's extent.  Optional high-attenuation inserts
(0.2 /mm spheres of 1-3 mm radius, scaled likewise) are placed inside the
cylinder.  Measured data follow ``counts = max(Poisson(I0 * exp(-p)), 1)`` and
``g = ln(I0 / counts)`` for line integrals ``p``.
"""
from __future__ import annotations

import numpy as np


def _random_rotation(rng: np.random.Generator) -> np.ndarray:
    q = rng.normal(size=4)
    q /= np.linalg.norm(q)
    w, x, y, z = q
    return np.array([
        [1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
        [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
        [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)],
    ])


def _centers(n: int, vox: float) -> np.ndarray:
    return (-(n - 1) / 2.0 + np.arange(n)) * vox


def phantom(cfg: dict, seed: int | None = None, n_ellipsoids: int | None = None,
            n_inserts: int | None = None, device=None):
    """Attenuation volume (float32, shape (Zdim, Ydim, Xdim)) for a preset dict.

    With ``device`` (a torch device) the voxelisation runs there and a torch
    tensor is returned; the random draws are the same numpy ones, so only the
    arithmetic's platform differs."""
    seed = cfg.get("seed", 0) if seed is None else seed
    n_ell = cfg.get("n_ellipsoids", 10) if n_ellipsoids is None else n_ellipsoids
    n_ins = cfg.get("n_inserts", 0) if n_inserts is None else n_inserts
    X, Y, Z = int(cfg["Xdim"]), int(cfg["Ydim"]), int(cfg["Zdim"])
    vx, vy, vz = float(cfg["XVoxSize"]), float(cfg["YVoxSize"]), float(cfg["ZVoxSize"])
    rng = np.random.default_rng(seed)
    xs, ys, zs = _centers(X, vx), _centers(Y, vy), _centers(Z, vz)
    if device is not None:
        return _phantom_torch(rng, xs, ys, zs, X, Y, Z, vx, vy, vz, n_ell, n_ins, device)
    ext_xy = min(X * vx, Y * vy)
    scale = max(X * vx, Y * vy, Z * vz) / 32.0
    rcyl = 0.45 * ext_xy
    vol = np.zeros((Z, Y, X), np.float32)
    inside = (xs[None, :] ** 2 + ys[:, None] ** 2) <= rcyl * rcyl
    vol[:, inside] = 0.02
    zhalf = Z * vz / 2.0

    def add_blob(center, axes, rot, value):
        # inside <=> p^T A p <= 1 with A = R diag(1/a^2) R^T, p = voxel centre - centre
        r = float(np.max(axes))
        lo = [np.searchsorted(c, center[k] - r) for k, c in enumerate((xs, ys, zs))]
        hi = [np.searchsorted(c, center[k] + r, side="right") for k, c in enumerate((xs, ys, zs))]
        if any(h <= l for l, h in zip(lo, hi)):
            return
        A = rot @ np.diag(1.0 / np.asarray(axes, np.float64) ** 2) @ rot.T
        px = (xs[lo[0]:hi[0]] - center[0])[None, None, :]
        py = (ys[lo[1]:hi[1]] - center[1])[None, :, None]
        pz = (zs[lo[2]:hi[2]] - center[2])[:, None, None]
        q = (A[0, 0] * px * px + A[1, 1] * py * py + A[2, 2] * pz * pz +
             2.0 * (A[0, 1] * px * py + A[0, 2] * px * pz + A[1, 2] * py * pz))
        vol[lo[2]:hi[2], lo[1]:hi[1], lo[0]:hi[0]] += np.float32(value) * (q <= 1.0)

    for _ in range(n_ell):
        axes = rng.uniform(2.0, 12.0, size=3) * scale
        rho = rcyl * np.sqrt(rng.uniform())
        phi = rng.uniform(0.0, 2 * np.pi)
        center = np.array([rho * np.cos(phi), rho * np.sin(phi), rng.uniform(-0.8, 0.8) * zhalf])
        add_blob(center, axes, _random_rotation(rng), rng.uniform(0.01, 0.05))
    for _ in range(n_ins):
        rad = rng.uniform(1.0, 3.0) * scale
        rho = (rcyl - rad) * np.sqrt(rng.uniform())
        phi = rng.uniform(0.0, 2 * np.pi)
        center = np.array([rho * np.cos(phi), rho * np.sin(phi), rng.uniform(-0.6, 0.6) * zhalf])
        add_blob(center, np.array([rad, rad, rad]), np.eye(3), 0.2)
    return vol


def _phantom_torch(rng, xs, ys, zs, X, Y, Z, vx, vy, vz, n_ell, n_ins, device):
    """phantom() voxelised with torch on `device` (same draws, same rule)."""
    import torch

    tx, ty, tz = (torch.as_tensor(c, dtype=torch.float64, device=device) for c in (xs, ys, zs))
    ext_xy = min(X * vx, Y * vy)
    scale = max(X * vx, Y * vy, Z * vz) / 32.0
    rcyl = 0.45 * ext_xy
    vol = torch.zeros((Z, Y, X), dtype=torch.float32, device=device)
    inside = (tx[None, :] ** 2 + ty[:, None] ** 2) <= rcyl * rcyl
    vol[:, inside] = 0.02
    zhalf = Z * vz / 2.0

    def add_blob(center, axes, rot, value):
        r = float(np.max(axes))
        lo = [int(np.searchsorted(c, center[k] - r)) for k, c in enumerate((xs, ys, zs))]
        hi = [int(np.searchsorted(c, center[k] + r, side="right")) for k, c in enumerate((xs, ys, zs))]
        if any(h <= l for l, h in zip(lo, hi)):
            return
        A = rot @ np.diag(1.0 / np.asarray(axes, np.float64) ** 2) @ rot.T
        px = (tx[lo[0]:hi[0]] - center[0])[None, None, :]
        py = (ty[lo[1]:hi[1]] - center[1])[None, :, None]
        pz = (tz[lo[2]:hi[2]] - center[2])[:, None, None]
        q = (A[0, 0] * px * px + A[1, 1] * py * py + A[2, 2] * pz * pz +
             2.0 * (A[0, 1] * px * py + A[0, 2] * px * pz + A[1, 2] * py * pz))
        vol[lo[2]:hi[2], lo[1]:hi[1], lo[0]:hi[0]] += float(np.float32(value)) * (q <= 1.0).to(torch.float32)

    for _ in range(n_ell):
        axes = rng.uniform(2.0, 12.0, size=3) * scale
        rho = rcyl * np.sqrt(rng.uniform())
        phi = rng.uniform(0.0, 2 * np.pi)
        center = np.array([rho * np.cos(phi), rho * np.sin(phi), rng.uniform(-0.8, 0.8) * zhalf])
        add_blob(center, axes, _random_rotation(rng), rng.uniform(0.01, 0.05))
    for _ in range(n_ins):
        rad = rng.uniform(1.0, 3.0) * scale
        rho = (rcyl - rad) * np.sqrt(rng.uniform())
        phi = rng.uniform(0.0, 2 * np.pi)
        center = np.array([rho * np.cos(phi), rho * np.sin(phi), rng.uniform(-0.6, 0.6) * zhalf])
        add_blob(center, np.array([rad, rad, rad]), np.eye(3), 0.2)
    return vol


def noisy(p, I0: float, seed: int, clip: bool = True):
    """g = ln(I0 / max(Poisson(I0 * exp(-p)), 1)) for line integrals p
    (numpy array, or torch tensor -- then sampled on its device).

    With ``clip`` (the default) negative values -- rays through air whose
    photon count exceeds I0 -- are set to 0.  Line integrals are non-negative,
    and MLEM's multiplicative update keeps the image non-negative only for
    non-negative data: with the raw values MLEM goes negative at air voxels
    and becomes chaotic (in FP64, a 1e-7 relative data perturbation grows to
    a 0.26 relative image difference by iteration 10 on a 48x48x40, 45-view
    case), so no FP32 result can track an FP64 one there."""
    try:
        import torch

        if isinstance(p, torch.Tensor):
            gen = torch.Generator(device=p.device)
            gen.manual_seed(int(seed))
            lam = float(I0) * torch.exp(-p.double())
            counts = torch.poisson(lam, generator=gen).clamp_min(1.0)
            g = torch.log(float(I0) / counts)
            if clip:
                g = g.clamp_min(0.0)
            return g.to(torch.float32)
    except ImportError:
        pass
    rng = np.random.default_rng(seed)
    lam = float(I0) * np.exp(-np.asarray(p, np.float64))
    counts = np.maximum(rng.poisson(lam), 1).astype(np.float64)
    g = np.log(float(I0) / counts)
    if clip:
        g = np.maximum(g, 0.0)
    return g.astype(np.float32)


def noisy_views(p, I0: float, seed: int, clip: bool = True):
    """noisy() view by view on the host: view n of p ([view][v][u], numpy array
    or torch tensor) is drawn from the seed ``seed * 100000 + n``, so that any
    subset of views can be reproduced without the others.  Returns the type
    (and device) of p."""
    try:
        import torch

        if isinstance(p, torch.Tensor):
            host = p.detach().cpu().numpy()
            out = np.stack([noisy(host[n], I0, seed * 100000 + n, clip) for n in range(host.shape[0])])
            return torch.from_numpy(out).to(p.device)
    except ImportError:
        pass
    p = np.asarray(p)
    return np.stack([noisy(p[n], I0, seed * 100000 + n, clip) for n in range(p.shape[0])])


def workload(cfg: dict, device, host_phantom: bool = True):
    """The measured workload of a preset: its phantom (voxelised on the host
    with numpy, or on `device` when host_phantom is False), forward projected
    by the EXACT projector of a default plan on `device`, with Poisson noise
    view by view (noisy_views).  Returns (volume, sinogram) as device tensors."""
    import torch

    from .api import Plan

    dev = torch.device(device)
    vol = torch.from_numpy(phantom(cfg)).to(dev) if host_phantom else phantom(cfg, device=dev)
    p = Plan(cfg).fp_views(vol)
    g = noisy_views(p, cfg["I0"], cfg["seed"])
    del p
    return vol, g
