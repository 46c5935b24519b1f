"""Views a quarter turn apart (recon_plan_quarter_turns).

A plan whose views come in exact quarter turns about a square volume derives
the ray tables of views N/4 .. N-1 from the first quarter's, so column (x, y)
at view n + N/4 gets exactly the lengths of column (X-1-y, x) at view n.
Checked through the forward projectors: the projection of the volume turned
by a quarter turn, vol_r[z, y, x] = vol[z, X-1-x, y], at view n is the
projection of vol at view n + N/4, bit for bit (the column and ray-walk
forward projectors; to 1e-6 in xy blocks, whose order a turn changes).  The
gather back projector then finds each set of lengths once for the four
columns of an orbit (bp_gather_quarter_kernel); its sums run in another order
than the view-range kernel's, so it is checked against that kernel on two
half ranges (<= 1e-6), against the FP64 oracle (<= 1e-5), by its pair count
(equal to the forward walk's) and through the fused MLEM update.  The forward
projections and MLEM ratios of all views at once equal those of two view
ranges bit for bit (a ray's sum does not depend on the other views).
"""
import numpy as np
import pytest

from conftest import rel_l2, small_cfg

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

from oracle import oracle as O  # noqa: E402
from recon_b200 import (ARITH_COMPAT, FP_RAY_WALK, PROJECTOR_BACK, SIDDON_BP_GATHER, SINO_BF16, Options,  # noqa: E402
                        Plan)
from recon_b200.configs import geom_dict  # noqa: E402

CASES = {
    # name: (geometry, options)
    "mirror": (small_cfg(), {}),
    "odd_z": (small_cfg(Zdim=25), {}),
    "offset_detector": (small_cfg(Dx=0.7), {}),
    "partial_tiles": (small_cfg(Xdim=30, Ydim=30, NumProj=8), {}),
    "two_chunks": (small_cfg(Xdim=16, Ydim=16, Zdim=300, ZVoxSize=0.25, TAxPixDim=0.5, TAxPixels=200, NumProj=8), {}),
    "column_blocks": (small_cfg(), {"fp_block": 8}),
    "ray_walk": (small_cfg(ZVoxSize=0.1, TAxPixels=200, TAxPixDim=1.5), {}),
}


def _turned(vol):
    """vol_r[z, y, x] = vol[z, X-1-x, y] (X = Y)."""
    X = vol.shape[2]
    yy, xx = torch.meshgrid(torch.arange(X, device=vol.device), torch.arange(X, device=vol.device), indexing="ij")
    return vol[:, X - 1 - xx, yy].contiguous()


def test_detection():
    assert Plan(small_cfg()).quarter_turns
    assert Plan(small_cfg(NumProj=8)).quarter_turns
    assert not Plan(small_cfg(Ydim=28)).quarter_turns  # not square
    assert not Plan(small_cfg(Xdim=31, Ydim=31)).quarter_turns  # odd side
    assert not Plan(small_cfg(YVoxSize=0.9)).quarter_turns
    assert not Plan(small_cfg(NumProj=10)).quarter_turns  # not a multiple of 4
    assert not Plan(small_cfg(NumProj=12, DeltaAng=7.5)).quarter_turns  # views 3 apart are 22.5 degrees apart
    assert not Plan(small_cfg(), Options(arith=ARITH_COMPAT)).quarter_turns


@pytest.mark.parametrize("name", list(CASES))
def test_projection_of_turned_volume(name):
    cfg, extra = CASES[name]
    P = Plan(cfg, Options(**extra))
    assert P.quarter_turns
    if name == "ray_walk":
        assert P.forward_projector == FP_RAY_WALK
    gen = torch.Generator("cuda").manual_seed(101)
    vol = torch.rand(P.shape_vol, device="cuda", generator=gen)
    g = P.fp_views(vol)
    gr = P.fp_views(_turned(vol))
    torch.cuda.synchronize()
    n, q = P.nproj, P.nproj // 4
    assert g.abs().sum().item() > 0
    turned = torch.cat([g[q:], g[:q]])
    if extra.get("fp_block", 0) > 0:
        # the blocked walk adds each ray's block shares in block order, which a
        # quarter turn changes: the same lengths, summed in another order
        assert rel_l2(gr.double().cpu().numpy(), turned.double().cpu().numpy()) < 1e-6
        return
    for v in range(n):
        assert torch.equal(gr[v].view(torch.int32), turned[v].view(torch.int32)), v


@pytest.mark.parametrize("name", ["mirror", "offset_detector", "partial_tiles", "two_chunks"])
def test_quarter_forward_equals_view_ranges(name):
    """Projections and MLEM ratios (FP32 and BF16) of all views at once and of
    two view ranges agree bit for bit; the ratios are compared through the
    back projection of all views."""
    cfg, extra = CASES[name]
    P = Plan(cfg, Options(**extra))
    assert P.quarter_turns and P.mirror_pairs
    gen = torch.Generator("cuda").manual_seed(104)
    vol = torch.rand(P.shape_vol, device="cuda", generator=gen)
    n, h = P.nproj, P.nproj // 2
    whole = P.fp_views(vol)
    parts = torch.cat([P.fp_views(vol, 0, h), P.fp_views(vol, h, n - h)])
    torch.cuda.synchronize()
    assert whole.abs().sum().item() > 0
    assert torch.equal(whole.view(torch.int32), parts.view(torch.int32))
    for kw in ({}, {"sino": SINO_BF16}):
        M = Plan(cfg, Options(siddon_bp=SIDDON_BP_GATHER, **extra, **kw))
        g = whole * 1.3 + 0.01
        if kw:
            g = g.to(torch.bfloat16)
        M.mlem_prepare()
        f0 = vol + 0.5
        ht_whole, ht_parts = M.new_volume(), M.new_volume()
        M.mlem_forward(g, f0)  # the ratio of all views at once
        M.mlem_backward(ht_whole)
        M.mlem_forward(g, f0, 0, h)
        M.mlem_forward(g, f0, h, n - h)  # the same ratio in two view ranges
        M.mlem_backward(ht_parts)
        torch.cuda.synchronize()
        assert ht_whole.abs().sum().item() > 0
        assert torch.equal(ht_whole.view(torch.int32), ht_parts.view(torch.int32)), kw


@pytest.mark.parametrize("name", [k for k in CASES if k != "ray_walk"])
def test_quarter_gather(name):
    cfg, extra = CASES[name]
    P = Plan(cfg, Options(siddon_bp=SIDDON_BP_GATHER, **extra))
    assert P.quarter_turns and P.siddon_bp == SIDDON_BP_GATHER
    gen = torch.Generator("cuda").manual_seed(102)
    y = torch.rand((P.nproj, P.nv, P.nu), device="cuda", generator=gen)
    whole = P.bp_views(y)  # all views: the quarter-turn gather where the rows are paired
    h = P.nproj // 2
    halves = P.bp_views(y[:h], 0, h)
    halves += P.bp_views(y[h:], h, P.nproj - h)  # view ranges: the range kernels
    torch.cuda.synchronize()
    assert whole.abs().sum().item() > 0
    assert rel_l2(whole.cpu().numpy(), halves.cpu().numpy()) < 1e-6
    g = O.Geom.from_dict(geom_dict(cfg))
    ref = O.x_bp_all(g, P.nproj, np.float32(cfg["DeltaAng"]), y.cpu().numpy().astype(np.float64).ravel())
    assert rel_l2(whole.cpu().numpy(), ref) < 1e-5
    assert P.count_projector_pairs(PROJECTOR_BACK) == P.count_intersections()


@pytest.mark.parametrize("sino", ["f32", "bf16"])
def test_quarter_mlem(sino):
    cfg = small_cfg()
    kw = {"sino": SINO_BF16} if sino == "bf16" else {}
    P = Plan(cfg, Options(siddon_bp=SIDDON_BP_GATHER, **kw))
    assert P.quarter_turns and P.mirror_pairs
    gen = torch.Generator("cuda").manual_seed(103)
    g = torch.rand((P.nproj, P.nv, P.nu), device="cuda", generator=gen) * 3
    if sino == "bf16":
        g = g.to(torch.bfloat16)
    P.mlem_prepare()
    f0 = torch.rand(P.shape_vol, device="cuda", generator=gen) + 0.5
    P.mlem_forward(g, f0)
    fused = f0.clone()
    P.mlem_backward_update(fused)
    split = f0.clone()
    ht = P.new_volume()
    P.mlem_backward(ht)
    P.mlem_update(split, ht)
    again = f0.clone()
    P.mlem_backward_update(again)
    torch.cuda.synchronize()
    assert fused.abs().sum().item() > 0
    assert torch.equal(fused.view(torch.int32), split.view(torch.int32))
    assert torch.equal(fused.view(torch.int32), again.view(torch.int32))  # deterministic


@pytest.mark.parametrize("sino", ["f32", "bf16"])
def test_quarter_sets(sino):
    """recon_mlem_forward_quarters / recon_mlem_backward_quarters: the views of
    ranks that split the plan by quarter sets (run one after another on this
    GPU) sum to the back projection of all views (<= 1e-6: the sets' sums are
    added at the end); the set of every base view is the all-views call, bit
    for bit; plans without quarter turns refuse."""
    from recon_b200 import ReconError
    from recon_b200.sharding import view_range

    cfg = small_cfg(NumProj=16, DeltaAng=22.5)
    kw = {"sino": SINO_BF16} if sino == "bf16" else {}
    P = Plan(cfg, Options(siddon_bp=SIDDON_BP_GATHER, **kw))
    assert P.quarter_sets
    gen = torch.Generator("cuda").manual_seed(105)
    g = torch.rand((P.nproj, P.nv, P.nu), device="cuda", generator=gen) * 3
    if sino == "bf16":
        g = g.to(torch.bfloat16)
    P.mlem_prepare()
    f = torch.rand(P.shape_vol, device="cuda", generator=gen) + 0.5
    P.mlem_forward(g, f)
    whole = P.new_volume()
    P.mlem_backward(whole)
    q = P.nproj // 4
    all_sets = P.new_volume()
    P.mlem_forward_quarters(g, f, 0, q)
    P.mlem_backward_quarters(all_sets, 0, q)
    torch.cuda.synchronize()
    assert torch.equal(whole.view(torch.int32), all_sets.view(torch.int32))
    for world in (2, 3):
        total = P.new_volume()
        for rank in range(world):
            first, count = view_range(q, rank, world)
            part = P.new_volume(7.0)
            P.mlem_forward_quarters(g, f, first, count)
            P.mlem_backward_quarters(part, first, count)
            total += part
        torch.cuda.synchronize()
        assert rel_l2(total.double().cpu().numpy(), whole.double().cpu().numpy()) < 1e-6, world
    other = Plan(small_cfg(NumProj=10), Options(siddon_bp=SIDDON_BP_GATHER))
    assert not other.quarter_turns and not other.quarter_sets
    other.mlem_prepare()
    with pytest.raises(ReconError):
        other.mlem_backward_quarters(other.new_volume(), 0, 1)
