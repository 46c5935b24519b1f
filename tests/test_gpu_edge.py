"""Edge cases of the EXACT path: empty view ranges, geometries whose rays all
miss the volume, a one-voxel volume, and plans without views (the single-view
calls at arbitrary angles use the plan's scratch slot).

Expected: empty ranges change nothing and copy nothing; a volume no ray
crosses projects to zeros, back projects to zeros, has no (ray, voxel) pairs
in any projector, and MLEM leaves it at zero (0 where the sensitivity is 0,
as divide1 does) without NaN; a one-voxel volume matches the FP64 oracle; a
plan with NumProj = 0 projects single views like any other plan.
"""
import numpy as np
import pytest

from conftest import rel_l2, small_cfg

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

from oracle import oracle as O  # noqa: E402
from recon_b200 import (PROJECTOR_BACK, PROJECTOR_FORWARD, SIDDON_BP_GATHER, SIDDON_BP_RAY, Options,  # noqa: E402
                        Plan)
from recon_b200.configs import geom_dict  # noqa: E402


def test_empty_view_ranges():
    P = Plan(small_cfg())
    vol = torch.rand(P.shape_vol, device="cuda")
    g = P.fp_views(vol)
    P.mlem_prepare()
    f = P.new_volume(1.0)
    out = torch.full_like(g, 7.0)
    P.fp_views(vol, 3, 0, out)
    ht = P.new_volume(5.0)
    P.mlem_backward(ht, 3, 0)  # an empty range back projects to zero
    P.mlem_forward(g, f, 3, 0)
    n = P.upload_sinogram(g.cpu().pin_memory(), out, 3, 0)
    torch.cuda.synchronize()
    assert torch.all(out == 7.0)
    assert torch.all(ht == 0.0)
    assert torch.all(f == 1.0)
    assert n == 0


@pytest.mark.parametrize("design", [SIDDON_BP_GATHER, SIDDON_BP_RAY])
@pytest.mark.parametrize("fp_block", [0, 8])
def test_volume_no_ray_crosses(design, fp_block):
    cfg = small_cfg(Dx=400.0)  # the detector shifted far to the side: every ray misses the volume
    P = Plan(cfg, Options(siddon_bp=design, fp_block=fp_block))
    assert P.count_intersections() == 0
    assert P.count_projector_pairs(PROJECTOR_FORWARD) == 0
    assert P.count_projector_pairs(PROJECTOR_BACK) == 0
    vol = torch.rand(P.shape_vol, device="cuda")
    g = P.fp_views(vol)
    y = torch.rand_like(g)
    b = P.bp_views(y)
    f = P.mlem(y, 2)
    torch.cuda.synchronize()
    assert torch.all(g == 0.0) and torch.all(b == 0.0)
    assert not torch.isnan(f).any() and torch.all(f == 0.0)


def test_one_voxel_volume():
    cfg = small_cfg(Xdim=1, Ydim=1, Zdim=1, XVoxSize=4.0, YVoxSize=4.0, ZVoxSize=4.0)
    P = Plan(cfg)
    g = O.Geom.from_dict(geom_dict(cfg))
    vol = np.array([0.7], np.float32)
    sino = P.fp_views(torch.from_numpy(vol).cuda().reshape(1, 1, 1)).cpu().numpy().ravel()
    ref = O.x_fp_all(g, int(cfg["NumProj"]), np.float32(cfg["DeltaAng"]), vol.astype(np.float64))
    assert np.abs(ref).max() > 0
    assert rel_l2(sino, ref) < 1e-5
    assert P.count_projector_pairs(PROJECTOR_FORWARD) == P.count_intersections() > 0
    assert P.count_projector_pairs(PROJECTOR_BACK) == P.count_intersections()


def test_plan_without_views_projects_single_views():
    cfg = small_cfg(NumProj=0, DeltaAng=0.0)
    P = Plan(cfg)
    g = O.Geom.from_dict(geom_dict(cfg))
    vol = np.random.default_rng(3).random(g.nvox).astype(np.float32)
    dvol = torch.from_numpy(vol).cuda().reshape(P.shape_vol)
    for ang in (0.0, 33.5):
        img = P.fp_view(dvol, ang).cpu().numpy().ravel()
        ref = np.zeros(g.npix)
        O.lib().orc_x_fp_view(g, float(np.float32(ang)), vol.astype(np.float64), ref)
        assert rel_l2(img, ref) < 1e-5, (ang, rel_l2(img, ref))
