"""Batched MLEM (recon_batch_*) against per-problem plans and the FP64 oracle.

Every problem of a batch runs the same per-ray and per-column device code as a
single plan, so its image is bit-identical to Plan.mlem on its own geometry,
whatever launch shape the batch's autotuner picks.
"""
import numpy as np
import pytest

from conftest import rel_l2, small_cfg

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

from oracle import oracle as O  # noqa: E402
from recon_b200 import ARITH_COMPAT, SUM_PLAIN, Batch, Options, Plan, ReconError  # noqa: E402
from recon_b200.configs import batched_problems, geom_dict, scaled  # noqa: E402

MIXED = [
    small_cfg(),
    small_cfg(Dx=0.7, Dz=-0.4, Ry=803.0, M=1.2, NumProj=12),
    small_cfg(XVoxSize=0.8, YVoxSize=1.1, ZVoxSize=0.9, Xdim=30, Ydim=26, Zdim=21, AxPixels=61, TAxPixels=47),
    small_cfg(Xdim=20, Ydim=44, Zdim=9, NumProj=5),
    small_cfg(Dz=0.75, NumProj=16),
]


def _sinos(cfgs, seed):
    gen = torch.Generator(device="cuda").manual_seed(seed)
    return [torch.rand((int(c["NumProj"]), int(c["TAxPixels"]), int(c["AxPixels"])), device="cuda",
                       generator=gen) for c in cfgs]


def _bits(t):
    return t.cpu().numpy().view(np.uint32)


@pytest.mark.parametrize("sum_mode", ["kahan", "plain"])
def test_batch_matches_plans_bitwise(sum_mode):
    opt = Options(sum=SUM_PLAIN) if sum_mode == "plain" else Options()
    gs = _sinos(MIXED, 5)
    B = Batch(MIXED, opt)
    fs = B.mlem(gs, 3)
    torch.cuda.synchronize()
    for p, (c, g) in enumerate(zip(MIXED, gs)):
        f = Plan(c, opt).mlem(g, 3)
        assert np.array_equal(_bits(fs[p]), _bits(f)), f"problem {p}: rel {rel_l2(fs[p].cpu(), f.cpu())}"


def test_batch_continues_and_repeats():
    gs = _sinos(MIXED, 6)
    B = Batch(MIXED)
    fs = B.mlem(gs, 2)
    fs = B.mlem(gs, 2, fs=fs, init_ones=False)  # 4 iterations in two calls
    again = Batch(MIXED).mlem(gs, 4)
    for p in range(len(MIXED)):
        f = Plan(MIXED[p]).mlem(gs[p], 4)
        assert np.array_equal(_bits(fs[p]), _bits(f))
        assert np.array_equal(_bits(again[p]), _bits(f))


def test_batch_vs_fp64_oracle():
    cfgs = MIXED[:2]
    rng = np.random.default_rng(7)
    gs_np = [rng.random(int(c["NumProj"]) * int(c["TAxPixels"]) * int(c["AxPixels"])).astype(np.float32)
             for c in cfgs]
    gs = [torch.from_numpy(g).cuda().reshape(int(c["NumProj"]), int(c["TAxPixels"]), int(c["AxPixels"]))
          for g, c in zip(gs_np, cfgs)]
    fs = Batch(cfgs).mlem(gs, 5)
    for c, g, f in zip(cfgs, gs_np, fs):
        geo = O.Geom.from_dict(geom_dict(c))
        f64, _ = O.x_mlem(geo, int(c["NumProj"]), np.float32(c["DeltaAng"]), g, 5)
        assert rel_l2(f.cpu().numpy().ravel(), f64) < 1e-4


def test_batch_of_generated_problems():
    # four problems of the generated batch workload, shrunk so per-problem
    # plans finish quickly; shapes stay mutually different
    cfgs = [scaled(c, Xdim=max(8, int(c["Xdim"]) // 4), Ydim=max(8, int(c["Ydim"]) // 4),
                   Zdim=max(8, int(c["Zdim"]) // 4), AxPixels=int(c["AxPixels"]) // 2,
                   TAxPixels=int(c["TAxPixels"]) // 2, NumProj=int(c["NumProj"]) // 6)
            for c in batched_problems(4, seed=11)]
    gs = _sinos(cfgs, 8)
    fs = Batch(cfgs).mlem(gs, 2)
    for c, g, f in zip(cfgs, gs, fs):
        assert np.array_equal(_bits(f), _bits(Plan(c).mlem(g, 2)))


def test_batch_rejects_unsupported_and_mismatched():
    with pytest.raises(ReconError):
        Batch(MIXED[:1], Options(arith=ARITH_COMPAT))
    pair = [MIXED[0], MIXED[2]]  # different volume and detector shapes
    B = Batch(pair)
    gs = _sinos(pair, 9)
    with pytest.raises(ValueError):
        B.mlem(gs[:1], 1)
    with pytest.raises(ValueError):
        B.mlem([gs[1], gs[0]], 1)


def test_tuned_back_projector_same_choice_and_bits():
    # SIDDON_BP_TUNED measures both back projectors on each geometry at plan
    # creation and keeps the faster, remembered per geometry: the batch's plans
    # and later plain plans of the same geometries choose alike and agree bit for bit
    from recon_b200 import SIDDON_BP_GATHER, SIDDON_BP_RAY, SIDDON_BP_TUNED

    opt = Options(siddon_bp=SIDDON_BP_TUNED)
    gs = _sinos(MIXED, 12)
    fs = Batch(MIXED, opt).mlem(gs, 2)
    torch.cuda.synchronize()
    for p, (c, g) in enumerate(zip(MIXED, gs)):
        P = Plan(c, opt)
        assert P.siddon_bp in (SIDDON_BP_GATHER, SIDDON_BP_RAY)
        assert Plan(c, opt).siddon_bp == P.siddon_bp
        assert np.array_equal(_bits(fs[p]), _bits(P.mlem(g, 2))), p
    # and the tuned plan is the EXACT projector pair: against FP64
    c = MIXED[0]
    geo = O.Geom.from_dict(geom_dict(c))
    y = np.random.default_rng(3).random(int(c["NumProj"]) * geo.npix).astype(np.float32)
    bp = Plan(c, opt).bp_views(torch.from_numpy(y).cuda().reshape(int(c["NumProj"]), -1, int(c["AxPixels"])))
    ref = O.x_bp_all(geo, int(c["NumProj"]), np.float32(c["DeltaAng"]), y.astype(np.float64))
    assert rel_l2(bp.cpu().numpy().ravel(), ref) < 1e-5
