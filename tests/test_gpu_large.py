"""The large workload in both precision modes, checked against FP64 on a 64-slice sub-volume.

512^3 FP32 volume of 0.125 mm voxels, 720 views of a 1024 (u) x 768 (v)
detector of 0.25 mm pixels, 100 ellipsoids + 5 inserts of 0.2 /mm, Poisson
noise at I0 = 1e5, 10 MLEM iterations (recon_b200.configs.LARGE).  For each
sinogram storage mode (FP32 with Kahan ray sums; BF16 with FP32 accumulation)
the GPU's image after iteration 9 is updated once more on the GPU and, for the
central 64 slices, in FP64 on the host (oracle orc_x_slab_update: full-length
line integrals of every ray crossing the slab, the slab's back projection and
sensitivity).  Reported: seconds per iteration, the forward and back halves of
iteration 10, the designs the plan picked, relative L2 and max-abs error of
iteration 10 on the slab, and each projector's count of (ray, voxel) pairs,
which must equal the ray walk's.  Bounds: 1e-5 relative L2 for FP32 (the
per-iteration tolerance), 2e-2 for BF16 sinograms.

Runs only with RECON_LARGE=1 (several GB of device memory, a few minutes of
host FP64 work); the summary is printed as one JSON line.
"""
import json
import os
import time

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

if os.environ.get("RECON_LARGE") != "1":
    pytest.skip("large workload: set RECON_LARGE=1", allow_module_level=True)

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

from oracle import oracle as O  # noqa: E402
from recon_b200 import PROJECTOR_BACK, PROJECTOR_FORWARD, SINO_BF16, SINO_F32, Options, Plan  # noqa: E402
from recon_b200.configs import LARGE, geom_dict  # noqa: E402
from recon_b200.phantom import noisy, phantom  # noqa: E402

ITERS = 10
Z0, Z1 = 224, 288  # central 64 slices


def _run(cfg, g, sino_mode):
    P = Plan(cfg, Options(sino=sino_mode))
    gm = g.to(torch.bfloat16) if sino_mode == SINO_BF16 else g
    P.mlem_prepare()
    f = P.new_volume(1.0)
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    a.record()
    for _ in range(ITERS - 1):
        P.mlem_iteration(gm, f)
    b.record()
    torch.cuda.synchronize()
    s_per_iter = a.elapsed_time(b) / (ITERS - 1) / 1e3
    f9 = f.cpu().numpy().ravel().copy()
    # iteration 10 in its two halves, timed apart
    e = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
    e[0].record()
    P.mlem_forward(gm, f)
    e[1].record()
    P.mlem_backward_update(f)
    e[2].record()
    torch.cuda.synchronize()
    f10 = f.cpu().numpy().ravel()
    info = {"forward_ms": e[0].elapsed_time(e[1]), "backward_ms": e[1].elapsed_time(e[2]),
            "forward_projector": P.forward_projector, "siddon_bp": P.siddon_bp, "mirror_pairs": P.mirror_pairs}
    if sino_mode == SINO_F32:  # every (ray, voxel) pair of positive length, as each projector takes them
        info["pairs"] = {"walk": P.count_intersections(), "forward": P.count_projector_pairs(PROJECTOR_FORWARD),
                         "back": P.count_projector_pairs(PROJECTOR_BACK)}
    del P
    torch.cuda.empty_cache()
    return s_per_iter, f9, f10, info


def test_large_precision_modes():
    cfg = dict(LARGE)
    nproj = int(cfg["NumProj"])
    dang = np.float32(cfg["DeltaAng"])
    vol = phantom(cfg, device=torch.device("cuda"))
    g = noisy(Plan(cfg).fp_views(vol), cfg["I0"], cfg["seed"])
    del vol
    g_host = g.cpu().numpy()
    geo = O.Geom.from_dict(geom_dict(cfg))
    plane = int(cfg["Xdim"]) * int(cfg["Ydim"])
    out = {"workload": "large_512cube_720x1024x768", "iterations": ITERS, "slab": [Z0, Z1]}
    for name, mode in (("f32_kahan", SINO_F32), ("bf16_sinogram", SINO_BF16)):
        s_it, f9, f10, info = _run(cfg, g, mode)
        t0 = time.time()
        ref = O.x_slab_update(geo, nproj, dang, f9, g_host, Z0, Z1)
        host_s = time.time() - t0
        got = f10[Z0 * plane:Z1 * plane].astype(np.float64)
        err = float(np.linalg.norm(got - ref) / np.linalg.norm(ref))
        out[name] = {"s_per_iteration": s_it, "rel_l2_vs_fp64": err,
                     "max_abs_vs_fp64": float(np.abs(got - ref).max()), "max_abs_ref": float(np.abs(ref).max()),
                     "fp64_host_s": host_s, **info}
    print(json.dumps(out))
    pairs = out["f32_kahan"]["pairs"]
    assert pairs["forward"] == pairs["walk"] and pairs["back"] == pairs["walk"], pairs
    assert out["f32_kahan"]["rel_l2_vs_fp64"] < 1e-5
    assert out["bf16_sinogram"]["rel_l2_vs_fp64"] < 2e-2
