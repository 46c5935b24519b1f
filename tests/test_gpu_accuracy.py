"""Accuracy on the measured workloads, and (ray, voxel) pair counts.

* Pair counts: the forward projector and the gather back projector must give a
  positive length to exactly the pairs the ray walk does
  (recon_count_projector_pairs against recon_count_intersections).  The
  gather finds its candidate detector columns and rows with margins; an equal
  count shows the margins lose no pair.
* The benchmarked workload (256^3 FP32 volume of 0.25 mm voxels, 360 views of a
  512^2 detector of 0.5 mm pixels, 40-ellipsoid phantom, Poisson noise at
  I0 = 1e5, EXACT arithmetic with the back projector the plan picks): 20 MLEM
  iterations from f = 1.  At iterations 1, 10 and 20 the GPU's update of its
  own previous image is compared, on the central 16 slices, with the FP64
  update of the same image (oracle orc_x_slab_update: full-length FP64 line
  integrals of every ray crossing the slab, the slab's FP64 back projection
  and sensitivity).  Bound: 1e-5 relative L2 per iteration.
* The small workload (64^3 x 0.5 mm, 128^2 x 1 mm, 90 views, 10 iterations):
  the full 10 iterations against FP64 MLEM (1e-5 after one iteration, 1e-4
  after ten), and against the reference's own file-driven MLEM
  (siddon_recon::a0_RECON_MLEM, CT_Recon/hf_siddon_recon.hpp:91-108, built
  for sm_100a from its sources) on the same projection files.  The reference
  drops entry segments and skips axes where its FP32 set-up rounds
  (siddon_kernelsMLEM.cuh:153-190, siddon_device_kernelsMLEM.cuh:151-185), so
  that distance is stated, with a loose bound.

Each test prints one JSON line with its measurements.
"""
import json
import os
import time

import numpy as np
import pytest

from conftest import rel_l2, small_cfg

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

from oracle import oracle as O  # noqa: E402
from recon_b200 import (ARITH_COMPAT, FP_COLUMNS, PROJECTOR_BACK, PROJECTOR_FORWARD, SIDDON_BP_GATHER,  # noqa: E402
                        SIDDON_BP_RAY, Options, Plan, mlem_from_cfg)
from recon_b200.configs import CPU_SMALL, PLAIN_GPU, geom_dict, scaled  # noqa: E402
from recon_b200.phantom import noisy, phantom, workload  # noqa: E402

COUNT_GEOMS = {
    "plain": small_cfg(),
    "offset": small_cfg(Dx=0.7, Dz=-0.4, Ry=803.0, M=1.2),
    "anisotropic": small_cfg(XVoxSize=0.8, YVoxSize=1.1, ZVoxSize=0.9, Xdim=30, Ydim=26, Zdim=21, AxPixels=61,
                             TAxPixels=47),
    "rows_apart": small_cfg(TAxPixDim=2.0, TAxPixels=36),
    "z256": small_cfg(Xdim=16, Ydim=16, Zdim=256, ZVoxSize=0.25, TAxPixDim=0.5, TAxPixels=160, NumProj=6),
    "cpu_small": scaled(CPU_SMALL, NumProj=30),
    "thin_ray_walk": small_cfg(ZVoxSize=0.1, TAxPixels=200, TAxPixDim=1.5),
}


@pytest.mark.parametrize("design", ["gather", "ray"])
@pytest.mark.parametrize("name", list(COUNT_GEOMS))
def test_pair_counts_equal(name, design):
    cfg = COUNT_GEOMS[name]
    P = Plan(cfg, Options(siddon_bp=SIDDON_BP_GATHER if design == "gather" else SIDDON_BP_RAY))
    # mirror pairing wherever the z table is symmetric: no Dz, an even slice count
    assert P.mirror_pairs == (cfg["Dz"] == 0.0 and int(cfg["Zdim"]) % 2 == 0)
    walk = P.count_intersections()
    assert walk > 0
    assert P.count_projector_pairs(PROJECTOR_FORWARD) == walk
    assert P.count_projector_pairs(PROJECTOR_BACK) == walk


def _update_errors(P, g, g_host, geo, nproj, dang, iters, checks, z0, z1):
    """Run `iters` MLEM iterations from f = 1; at the iterations in `checks`
    compare the GPU update with the FP64 update of the same image on slices
    [z0, z1)."""
    plane = P.shape_vol[1] * P.shape_vol[2]
    P.mlem_prepare()
    f = P.new_volume(1.0)
    out = {}
    for it in range(1, iters + 1):
        if it in checks:
            f_prev = f.cpu().numpy().ravel().copy()
            P.mlem_iteration(g, f)
            got = f.cpu().numpy().ravel()[z0 * plane:z1 * plane].astype(np.float64)
            t0 = time.time()
            ref = O.x_slab_update(geo, nproj, dang, f_prev, g_host, z0, z1)
            out[it] = {"rel_l2": rel_l2(got, ref), "max_abs": float(np.abs(got - ref).max()),
                       "max_ref": float(np.abs(ref).max()), "fp64_s": round(time.time() - t0, 1)}
        else:
            P.mlem_iteration(g, f)
    return out


def test_plain_gpu_workload_accuracy_and_counts():
    cfg = dict(PLAIN_GPU)
    nproj = int(cfg["NumProj"])
    dang = np.float32(cfg["DeltaAng"])
    vol, g = workload(cfg, "cuda")  # the benchmark's own inputs
    del vol
    P = Plan(cfg)
    # the benchmarked designs: detector-column forward projector, gather back
    # projector, both on mirrored row / voxel pairs
    assert P.forward_projector == FP_COLUMNS and P.siddon_bp == SIDDON_BP_GATHER and P.mirror_pairs
    walk = P.count_intersections()
    pairs = {"walk": walk, "forward": P.count_projector_pairs(PROJECTOR_FORWARD),
             "back": P.count_projector_pairs(PROJECTOR_BACK)}
    geo = O.Geom.from_dict(geom_dict(cfg))
    g_host = g.cpu().numpy()
    errs = _update_errors(P, g, g_host, geo, nproj, dang, 20, (1, 10, 20), 120, 136)
    print(json.dumps({"workload": "plain_gpu_256cube_360x512x512", "slab": [120, 136], "pairs": pairs,
                      "update_vs_fp64": errs}))
    assert pairs["forward"] == walk and pairs["back"] == walk
    for it, e in errs.items():
        assert e["rel_l2"] < 1e-5, (it, e)


def _small_case():
    cfg = dict(CPU_SMALL)
    geo = O.Geom.from_dict(geom_dict(cfg))
    nproj = int(cfg["NumProj"])
    dang = np.float32(cfg["DeltaAng"])
    vol = phantom(cfg)
    p = O.x_fp_all(geo, nproj, dang, vol.astype(np.float64).ravel())
    meas = noisy(p, cfg["I0"], cfg["seed"]).astype(np.float32)
    return cfg, geo, nproj, dang, meas


@pytest.mark.parametrize("design", ["gather", "ray"])
def test_cpu_small_workload_mlem_vs_fp64(design):
    cfg, geo, nproj, dang, meas = _small_case()
    P = Plan(cfg, Options(siddon_bp=SIDDON_BP_GATHER if design == "gather" else SIDDON_BP_RAY))
    g = torch.from_numpy(meas).cuda().reshape(nproj, P.nv, P.nu)
    P.mlem_prepare()
    f = P.new_volume(1.0)
    errs = {}
    done = 0
    for k in (1, 5, 10):
        P.mlem(g, k - done, f, init_ones=False)
        done = k
        f64, _ = O.x_mlem(geo, nproj, dang, meas.ravel(), k)
        errs[k] = rel_l2(f.cpu().numpy(), f64)
    print(json.dumps({"workload": "cpu_small_64cube_90x128x128", "design": design, "mlem_vs_fp64": errs}))
    assert errs[1] < 1e-5, errs
    assert errs[10] < 1e-4, errs


needs_ref = pytest.mark.skipif(O.ref_gpu() is None, reason="reference sm_100a build missing")


@needs_ref
def test_cpu_small_workload_vs_reference_mlem(tmp_path):
    """EXACT and COMPAT file-driven MLEM against the reference's own
    a0_RECON_MLEM on the same projection files, and both against FP64."""
    from tests_helpers import write_cfg

    cfg, geo, nproj, dang, meas = _small_case()
    folder = str(tmp_path)
    meas = meas.reshape(nproj, -1)
    for n in range(nproj):
        meas[n].tofile(os.path.join(folder, f"proj_{n}.bin"))
    outs = {}
    for tag in ("ref", "exact", "compat"):
        d = os.path.join(folder, tag) + "/"
        os.makedirs(d)
        write_cfg(os.path.join(folder, f"{tag}.cfg"), cfg, folder + "/", d)
        outs[tag] = d
    t0 = time.time()
    assert O.ref_gpu().ref_gpu_mlem_cfg((folder + "/").encode(), b"ref.cfg") > 0
    ref_s = time.time() - t0
    mlem_from_cfg(folder, "exact.cfg", Options())
    mlem_from_cfg(folder, "compat.cfg", Options(arith=ARITH_COMPAT))
    nvox = geo.nvox
    table = {}
    for k in (1, 5, 10):
        f64, _ = O.x_mlem(geo, nproj, dang, meas.ravel(), k)
        a = {t: np.fromfile(os.path.join(outs[t], f"recon_{k - 1}.bin"), np.float32) for t in outs}
        assert all(x.size == nvox for x in a.values())
        table[k] = {"exact_vs_ref": rel_l2(a["exact"], a["ref"]), "compat_vs_ref": rel_l2(a["compat"], a["ref"]),
                    "exact_vs_fp64": rel_l2(a["exact"], f64), "ref_vs_fp64": rel_l2(a["ref"], f64),
                    "compat_vs_fp64": rel_l2(a["compat"], f64)}
    print(json.dumps({"workload": "cpu_small_64cube_90x128x128", "reference_mlem_s": round(ref_s, 1),
                      "after_iterations": table}))
    for k, row in table.items():
        assert row["compat_vs_ref"] < 1e-5 * (k + 1), (k, row)
        assert row["exact_vs_fp64"] < 1e-4, (k, row)
        assert row["exact_vs_ref"] < 5e-2, (k, row)  # the reference's own distance from FP64 dominates
