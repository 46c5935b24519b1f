"""Scanner / volume presets for the five measured workloads.

Keys are the reference configuration-file keys (CT_Recon/MasterParameterFile.origin
and CT_Recon/CTSystemElements_HF.h:13-151).  Common geometry: circular cone
beam, source to isocentre ``Rf`` = 500 mm, source to detector ``R = Ry``,
magnification ``M`` = 1, no detector misalignment, views uniform over 360
degrees (``DeltaAng = 360 / NumProj``).  Where the workload description leaves a
value open, the choice made here is noted next to it.
"""
from __future__ import annotations

import copy

_COMMON = dict(R=800.0, Rf=500.0, Ry=800.0, Dx=0.0, Dz=0.0, xangle=0.0, yangle=0.0, zangle=0.0, M=1.0)


def _cfg(vol, vox, det, pitch, nproj, iters, **extra):
    X, Y, Z = vol
    Nu, Nv = det
    d = dict(_COMMON)
    d.update(
        Xdim=X, Ydim=Y, Zdim=Z, XVoxSize=vox, YVoxSize=vox, ZVoxSize=vox,
        AxPixels=Nu, TAxPixels=Nv, AxPixDim=pitch, TAxPixDim=pitch,
        NumProj=nproj, DeltaAng=360.0 / nproj, N_iteration=iters,
    )
    d.update(extra)
    return d


# 1 -- plain MLEM, small: 64^3 x 0.5 mm, 128^2 x 1 mm detector, 90 views, 10 iterations.
CPU_SMALL = _cfg((64, 64, 64), 0.5, (128, 128), 1.0, 90, 10, n_ellipsoids=10, I0=1e5, seed=1)
# 2 -- plain GPU drop-in: 256^3 x 0.25 mm, 512^2 x 0.5 mm detector, 360 views, 20 iterations.
PLAIN_GPU = _cfg((256, 256, 256), 0.25, (512, 512), 0.5, 360, 20, n_ellipsoids=40, I0=1e5, seed=2)
# 3 -- differentiable projector: 128^3, 180 views, 256^2 detector.  Pitches are
#      not given; 0.5 mm voxels and 1 mm pixels are used.
DIFFERENTIABLE = _cfg((128, 128, 128), 0.5, (256, 256), 1.0, 180, 10, n_ellipsoids=10, I0=1e5, seed=3)
# 5 -- large: 512^3 x 0.125 mm, detector 1024 (Ax) x 768 (TAx); pixel pitch not
#      given, 0.25 mm is used.  720 views, 10 iterations.
LARGE = _cfg((512, 512, 512), 0.125, (1024, 768), 0.25, 720, 10, n_ellipsoids=100, n_inserts=5,
             I0=1e5, seed=5)

PRESETS = {"cpu_small": CPU_SMALL, "plain_gpu": PLAIN_GPU, "differentiable": DIFFERENTIABLE, "large": LARGE}


def geom_dict(cfg: dict) -> dict:
    """The CalibrationParam / Detector / VoxVolParam fields of a preset."""
    return dict(
        R=cfg["R"], Rf=cfg["Rf"], Ry=cfg["Ry"], Dx=cfg["Dx"], Dz=cfg["Dz"], xangle=cfg["xangle"],
        yangle=cfg["yangle"], zangle=cfg["zangle"], M=cfg["M"],
        NumTAxPixels=cfg["TAxPixels"], NumAxPixels=cfg["AxPixels"],
        TAxPixDimMm=cfg["TAxPixDim"], AxPixDimMm=cfg["AxPixDim"],
        Xdim=cfg["Xdim"], Ydim=cfg["Ydim"], Zdim=cfg["Zdim"],
        XVoxSize=cfg["XVoxSize"], YVoxSize=cfg["YVoxSize"], ZVoxSize=cfg["ZVoxSize"],
    )


def scaled(cfg: dict, **overrides) -> dict:
    c = copy.deepcopy(cfg)
    c.update(overrides)
    if "NumProj" in overrides and "DeltaAng" not in overrides:
        c["DeltaAng"] = 360.0 / c["NumProj"]
    return c


def batched_problems(n: int = 48, seed: int = 4, iters: int = 20) -> list[dict]:
    """The batched workload: ``n`` problems drawn from ``seed``.

    Volumes 32..192 per axis (independent, so non-cubic), 60..360 views,
    square detectors 64..384, source-detector distance 600..1000 mm, I0 in
    1e4..1e6 (log-uniform).  Every dimension is a multiple of 4 (the reference
    launches 4-wide blocks with no bounds checks).  Rf = 500 mm.  Voxel size:
    the largest volume axis spans 0.8 of the field of view at isocentre,
    ``vox = 0.8 * (Nu * pitch * Rf / SDD) / max(X, Y, Z)``, with a 1 mm pitch,
    reduced where needed so that the volume's bounding sphere stays within
    0.9 of the isocentre-to-detector distance (SDD - Rf): the detector must
    not cut through the object.
    """
    import numpy as np

    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        X, Y, Z = (int(rng.integers(8, 49)) * 4 for _ in range(3))
        nproj = int(rng.integers(15, 91)) * 4
        Nu = int(rng.integers(16, 97)) * 4
        sdd = float(rng.uniform(600.0, 1000.0))
        I0 = float(10.0 ** rng.uniform(4.0, 6.0))
        pitch = 1.0
        vox = 0.8 * (Nu * pitch * 500.0 / sdd) / max(X, Y, Z)
        half_diag = 0.5 * float(np.sqrt(X * X + Y * Y + Z * Z))
        vox = min(vox, 0.9 * min(500.0, sdd - 500.0) / half_diag)
        vox = float(np.float32(round(vox, 4)))
        c = _cfg((X, Y, Z), vox, (Nu, Nu), pitch, nproj, iters, n_ellipsoids=10, I0=I0, seed=1000 + i)
        c["R"] = c["Ry"] = float(np.float32(round(sdd, 2)))
        out.append(c)
    return out
