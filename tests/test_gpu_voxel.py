"""Voxel-driven back projection (backward_projection2, CT_Recon/hf_cuda_kernels.cuh:240-284)
against the reference's own sm_100a kernel and the CPU oracle, and MLEM with it."""
import numpy as np
import pytest

from conftest import rel_l2, small_cfg

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

from oracle import oracle as O  # noqa: E402
from recon_b200 import BP_VOXEL, VOXEL_GEOMETRIC, VOXEL_REFERENCE, Options, Plan  # noqa: E402
from recon_b200.configs import CPU_SMALL, geom_dict, scaled  # noqa: E402

REFG = O.ref_gpu()


@pytest.mark.skipif(REFG is None, reason="reference sm_100a build missing")
@pytest.mark.parametrize("pitch", [1.0, 0.5])
def test_reference_mode_vs_reference_kernel(pitch):
    cfg = small_cfg(AxPixDim=pitch, TAxPixDim=pitch)
    P = Plan(cfg)
    g = O.Geom.from_dict(geom_dict(cfg))
    img = np.random.default_rng(20).random(g.npix).astype(np.float32)
    for ang in (0.0, 33.0, 90.0, 200.0):
        ref = np.zeros(g.nvox, np.float32)
        REFG.ref_gpu_voxel_bp2_view(g, ang, img, 12, ref)
        out = P.voxel_bp_view(torch.from_numpy(img).cuda(), ang, 12, VOXEL_REFERENCE).cpu().numpy().ravel()
        assert rel_l2(out, ref) < 1e-6, (ang, rel_l2(out, ref))
        assert rel_l2(out, O.v_bp_view(g, ang, img, 12, 0)) < 1e-5


@pytest.mark.parametrize("mode", [VOXEL_REFERENCE, VOXEL_GEOMETRIC])
def test_modes_vs_oracle(mode):
    cfg = small_cfg(AxPixDim=0.75, TAxPixDim=0.75)
    P = Plan(cfg)
    g = O.Geom.from_dict(geom_dict(cfg))
    img = np.random.default_rng(21).random(g.npix).astype(np.float32)
    for ang in (0.0, 45.0, 123.0):
        out = P.voxel_bp_view(torch.from_numpy(img).cuda(), ang, 12, mode).cpu().numpy().ravel()
        assert rel_l2(out, O.v_bp_view(g, ang, img, 12, int(mode))) < 1e-5


def test_geometric_mode_tracks_siddon_bp():
    # same angle sense and units as the Siddon back projector: the voxel-driven
    # back projection of a smooth sinogram correlates with the Siddon one
    cfg = scaled(CPU_SMALL, Xdim=32, Ydim=32, Zdim=32, XVoxSize=1.0, YVoxSize=1.0, ZVoxSize=1.0, NumProj=30)
    P = Plan(cfg)
    vol = torch.zeros(P.shape_vol, device="cuda")
    vol[10:20, 5:12, 18:27] = 1.0
    sino = P.fp_views(vol)
    a = P.bp_views(sino).ravel()
    Pv = Plan(cfg, Options(bp=BP_VOXEL))
    b = torch.zeros_like(a)
    for n in range(P.nproj):
        b = Pv.voxel_bp_view(sino[n], P.angle(n), P.nproj, VOXEL_GEOMETRIC, accum=b.reshape(P.shape_vol)).ravel()
    c = torch.corrcoef(torch.stack([a, b]))[0, 1].item()
    assert c > 0.95, c


def test_mlem_with_voxel_bp_converges():
    cfg = scaled(CPU_SMALL, Xdim=32, Ydim=32, Zdim=32, XVoxSize=1.0, YVoxSize=1.0, ZVoxSize=1.0, NumProj=45)
    P = Plan(cfg)
    truth = torch.zeros(P.shape_vol, device="cuda")
    truth[8:24, 8:24, 8:24] = 0.02
    truth[12:18, 10:20, 14:20] = 0.05
    g = P.fp_views(truth)
    Pv = Plan(cfg, Options(bp=BP_VOXEL))
    errs = []
    f = Pv.new_volume(1.0)
    Pv.mlem_prepare()
    for it in range(8):
        Pv.mlem_iteration(g, f)
        errs.append(rel_l2(f.cpu().numpy(), truth.cpu().numpy()))
    assert errs[-1] < errs[0] and np.all(np.isfinite(errs))


@pytest.mark.parametrize("zdim", [40, 300])
def test_mlem_iteration_matches_per_view_path(zdim):
    # an EXACT plan's MLEM iteration with the voxel-driven back projector (the
    # ratio in the detector-column layout, read by the column gather kernel) against the
    # same iteration assembled from the forward projector and single-view voxel
    # back projections of row-major images (the texture kernels)
    cfg = small_cfg(Zdim=zdim, ZVoxSize=0.2 if zdim > 100 else 1.0, NumProj=10)
    Pv = Plan(cfg, Options(bp=BP_VOXEL))
    gen = torch.Generator("cuda").manual_seed(61)
    g = torch.rand((Pv.nproj, Pv.nv, Pv.nu), device="cuda", generator=gen) * 2
    f0 = torch.rand(Pv.shape_vol, device="cuda", generator=gen) + 0.5
    f = f0.clone()
    Pv.mlem_prepare()
    Pv.mlem_iteration(g, f)
    hf = Pv.fp_views(f0)
    ratio = torch.where(hf != 0, g / torch.where(hf != 0, hf, torch.ones_like(hf)), torch.zeros_like(hf))
    ht = Pv.new_volume(0.0)
    sens = Pv.new_volume(0.0)
    ones = torch.ones((Pv.nv, Pv.nu), device="cuda")
    for n in range(Pv.nproj):
        Pv.voxel_bp_view(ratio[n].contiguous(), Pv.angle(n), Pv.nproj, VOXEL_GEOMETRIC, accum=ht)
        Pv.voxel_bp_view(ones, Pv.angle(n), Pv.nproj, VOXEL_GEOMETRIC, accum=sens)
    expect = torch.where(sens != 0, f0 * ht / torch.where(sens != 0, sens, torch.ones_like(sens)),
                         torch.zeros_like(sens))
    assert expect.abs().max() > 0
    assert rel_l2(f.cpu().numpy(), expect.cpu().numpy()) < 1e-5
