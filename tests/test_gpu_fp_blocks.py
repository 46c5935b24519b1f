"""The column forward projector over xy blocks (recon_options_t.fp_block).

Volumes larger than L2 are walked one xy block of voxel columns at a time, the
blocks' shares of each ray sum added in block order.  Against the same plan
walking the whole volume at once (fp_block = -1) and the FP64 oracle:
  * pair counts: the blocked walk's (ray, voxel) pairs equal the ray walk's;
  * projections: rel. L2 <= 1e-6 from the unblocked walk, <= 1e-5 from FP64;
  * views: projecting a view range gives those views of the whole sinogram,
    bit for bit (a pixel's sum does not depend on the other views);
  * the MLEM iteration: rel. L2 <= 1e-6 from the unblocked walk, FP32 and BF16
    ratio sinograms (<= 1e-2 for BF16, whose ratio rounds to 8 bits);
  * a block side giving more than 64 blocks is refused.
"""
import numpy as np
import pytest

from conftest import rel_l2, small_cfg

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

from oracle import oracle as O  # noqa: E402
from recon_b200 import (FP_COLUMN_BLOCKS, FP_COLUMNS, PROJECTOR_FORWARD, SIDDON_BP_GATHER, SIDDON_BP_RAY,  # noqa: E402
                        SINO_BF16, SINO_F32, Options, Plan, ReconError)
from recon_b200.configs import geom_dict  # noqa: E402

GEOMS = {
    # name: (geometry, block side, mirror pairing expected)
    "mirror": (small_cfg(), 8, True),
    "odd_z": (small_cfg(Zdim=25), 8, False),
    "ragged": (small_cfg(Xdim=30, Ydim=27, Zdim=24), 7, True),
    "offset": (small_cfg(Dx=0.7, Dz=-0.4, Ry=803.0), 16, False),
}


def _plans(cfg, side, **kw):
    return Plan(cfg, Options(fp_block=side, **kw)), Plan(cfg, Options(fp_block=-1, **kw))


def _volume(P, seed):
    gen = torch.Generator("cuda").manual_seed(seed)
    return torch.rand(P.shape_vol, device="cuda", generator=gen)


@pytest.mark.parametrize("name", list(GEOMS))
def test_blocked_projection(name):
    cfg, side, mirror = GEOMS[name]
    B, U = _plans(cfg, side)
    assert B.forward_projector == FP_COLUMN_BLOCKS
    assert U.forward_projector == FP_COLUMNS
    assert B.mirror_pairs == mirror
    assert B.count_projector_pairs(PROJECTOR_FORWARD) == B.count_intersections()
    vol = _volume(B, 71)
    sb = B.fp_views(vol)
    su = U.fp_views(vol)
    torch.cuda.synchronize()
    a, b = sb.double().cpu().numpy(), su.double().cpu().numpy()
    assert np.abs(b).max() > 0
    assert rel_l2(a, b) < 1e-6, rel_l2(a, b)
    g = O.Geom.from_dict(geom_dict(cfg))
    n = int(cfg["NumProj"])
    ref = O.x_fp_all(g, n, np.float32(cfg["DeltaAng"]), vol.double().cpu().numpy().ravel()).reshape(a.shape)
    assert rel_l2(a, ref) < 1e-5, rel_l2(a, ref)
    part = B.fp_views(vol, 3, 5)
    torch.cuda.synchronize()
    assert torch.equal(part.view(torch.int32), sb[3:8].view(torch.int32))


# with the gather on the mirror geometry the ratio is kept in mirrored row pairs
# (column_finish_pairs_kernel forms it from the block sums)
@pytest.mark.parametrize("design", [SIDDON_BP_GATHER, SIDDON_BP_RAY])
@pytest.mark.parametrize("sino", [SINO_F32, SINO_BF16])
@pytest.mark.parametrize("name", ["mirror", "offset"])
def test_blocked_mlem_iteration(name, sino, design):
    cfg, side, _ = GEOMS[name]
    B, U = _plans(cfg, side, sino=sino, siddon_bp=design)
    assert B.forward_projector == FP_COLUMN_BLOCKS
    vol = _volume(B, 72) + 0.2
    g = U.fp_views(vol)
    if sino == SINO_BF16:
        g = g.to(torch.bfloat16)
    out = []
    for P in (B, U):
        P.mlem_prepare()
        f = P.new_volume(1.0)
        for _ in range(2):
            P.mlem_forward(g, f)
            P.mlem_backward_update(f)
        out.append(f.double().cpu().numpy())
    err = rel_l2(out[0], out[1])
    assert err < (1e-2 if sino == SINO_BF16 else 1e-6), err


def test_block_count_limit():
    with pytest.raises(ReconError):
        Plan(small_cfg(), Options(fp_block=3))  # 11 x 11 blocks


def test_blocked_osem_voxel_and_batch():
    """The other callers of the forward projector with blocks: OSEM (view
    subsets), the voxel-driven back projector's ratio (g / Hf) and a batch,
    which must give the bits of its plain plans."""
    from recon_b200 import BP_VOXEL, VOXEL_GEOMETRIC, Batch

    cfg, side, _ = GEOMS["mirror"]
    B, U = _plans(cfg, side)
    vol = _volume(B, 73) + 0.2
    g = U.fp_views(vol)
    fb, fu = B.osem(g, 2, 3), U.osem(g, 2, 3)
    err = rel_l2(fb.double().cpu().numpy(), fu.double().cpu().numpy())
    assert err < 1e-6, err
    VB = Plan(cfg, Options(fp_block=side, bp=BP_VOXEL, voxel_mode=VOXEL_GEOMETRIC))
    VU = Plan(cfg, Options(fp_block=-1, bp=BP_VOXEL, voxel_mode=VOXEL_GEOMETRIC))
    assert VB.forward_projector == FP_COLUMN_BLOCKS
    vb, vu = VB.mlem(g, 2), VU.mlem(g, 2)
    err = rel_l2(vb.double().cpu().numpy(), vu.double().cpu().numpy())
    assert err < 1e-6, err
    cfgs = [cfg, small_cfg(Xdim=30, Ydim=27, Zdim=24)]
    opts = Options(fp_block=8)
    plans = [Plan(c, opts) for c in cfgs]
    assert all(P.forward_projector == FP_COLUMN_BLOCKS for P in plans)
    gs = [P.fp_views(_volume(P, 74 + k) + 0.2) for k, P in enumerate(plans)]
    batch = Batch(cfgs, opts).mlem(gs, 3)
    for P, gk, fk in zip(plans, gs, batch):
        ref = P.mlem(gk, 3)
        torch.cuda.synchronize()
        assert torch.equal(fk.view(torch.int32), ref.view(torch.int32))
