"""EXACT arithmetic on the GPU against the FP64 oracle.

Tolerances (relative L2 against the FP64 exact Siddon of oracle/siddon_oracle.c):
  forward projection, back projection, sensitivity   <= 1e-5
  adjointness <A x, y> = <x, A^T y> (FP32 sums)        <= 1e-5
  MLEM after 10 iterations                             <= 1e-4
Back projection and MLEM are bit-reproducible run to run.  The tests that
involve the back projector run with both of its designs (the column gather,
FP32 sums in a fixed order, and the ray-driven walk into int64 fixed-point
slabs), which assign the same length to every ray-voxel pair.
"""
import numpy as np
import pytest

from conftest import rel_l2, small_cfg

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

from oracle import oracle as O  # noqa: E402
from recon_b200 import (SIDDON_BP_AUTO, SIDDON_BP_GATHER, SIDDON_BP_RAY, SINO_BF16, SUM_PLAIN, Options,  # noqa: E402
                        Plan)
from recon_b200.configs import CPU_SMALL, geom_dict, scaled  # noqa: E402
from recon_b200.phantom import noisy, phantom  # noqa: E402

GEOMS = {
    "plain": small_cfg(),
    "offset": small_cfg(Dx=0.7, Dz=-0.4, Ry=803.0, M=1.2),
    "z_parallel_row": small_cfg(Dz=0.75),
    "anisotropic": small_cfg(XVoxSize=0.8, YVoxSize=1.1, ZVoxSize=0.9, Xdim=30, Ydim=26, Zdim=21, AxPixels=61,
                             TAxPixels=47),
    "cpu_small": scaled(CPU_SMALL, NumProj=18),
    # detector rows 1.2 voxels apart (a short volume, so the automatic choice stays the ray walk)
    "rows_apart": small_cfg(TAxPixDim=2.0, TAxPixels=36),
    # 100 and 256 slices: the gather's 4- and 8-voxel-per-lane variants (the others
    # cover 1, 2 and, in TALL below, 7)
    "z100": small_cfg(Zdim=100, TAxPixels=110, NumProj=8),
    "z256": small_cfg(Xdim=16, Ydim=16, Zdim=256, ZVoxSize=0.25, TAxPixDim=0.5, TAxPixels=160, NumProj=6),
    # a thin slab under steep rows: the ray-walk forward projector with mirrored rows, so the
    # mirror-paired gather reads the detector-column layout (not row pairs)
    "thin_ray_walk": small_cfg(ZVoxSize=0.1, TAxPixels=200, TAxPixDim=1.5),
}
DESIGNS = {"gather": SIDDON_BP_GATHER, "ray": SIDDON_BP_RAY}


def _x_fp(g, cfg, vol64):
    return O.x_fp_all(g, int(cfg["NumProj"]), np.float32(cfg["DeltaAng"]), vol64)


@pytest.mark.parametrize("name", list(GEOMS))
def test_fp_vs_fp64(name):
    cfg = GEOMS[name]
    P = Plan(cfg)
    g = O.Geom.from_dict(geom_dict(cfg))
    vol = np.random.default_rng(10).random(g.nvox).astype(np.float32)
    ref = _x_fp(g, cfg, vol.astype(np.float64))
    out = P.fp_views(torch.from_numpy(vol).cuda().reshape(P.shape_vol)).cpu().numpy().ravel()
    assert rel_l2(out, ref) < 1e-5, rel_l2(out, ref)
    # hits and misses agree ray by ray, except rays grazing the volume's surface
    grazing = (out != 0) != (ref != 0)
    assert grazing.sum() <= max(2, 1e-4 * out.size)
    assert np.all(np.abs(ref[grazing]) < 1e-3)


@pytest.mark.parametrize("design", list(DESIGNS))
@pytest.mark.parametrize("name", list(GEOMS))
def test_bp_and_sensitivity_vs_fp64(name, design):
    cfg = GEOMS[name]
    P = Plan(cfg, Options(siddon_bp=DESIGNS[design]))
    g = O.Geom.from_dict(geom_dict(cfg))
    nproj = int(cfg["NumProj"])
    sino = np.random.default_rng(11).random(nproj * g.npix).astype(np.float32)
    ref = O.x_bp_all(g, nproj, np.float32(cfg["DeltaAng"]), sino.astype(np.float64))
    out = P.bp_views(torch.from_numpy(sino).cuda().reshape(nproj, P.nv, P.nu)).cpu().numpy().ravel()
    assert rel_l2(out, ref) < 1e-5, rel_l2(out, ref)
    sref = O.x_bp_all(g, nproj, np.float32(cfg["DeltaAng"]), np.ones(nproj * g.npix))
    sens = P.sensitivity().cpu().numpy().ravel()
    assert rel_l2(sens, sref) < 1e-5


@pytest.mark.parametrize("design", list(DESIGNS))
@pytest.mark.parametrize("name", ["plain", "offset", "cpu_small", "rows_apart"])
def test_adjoint(name, design):
    cfg = GEOMS[name]
    P = Plan(cfg, Options(siddon_bp=DESIGNS[design]))
    x = torch.rand(P.shape_vol, device="cuda", generator=torch.Generator("cuda").manual_seed(1))
    y = torch.rand((P.nproj, P.nv, P.nu), device="cuda", generator=torch.Generator("cuda").manual_seed(2))
    Ax = P.fp_views(x)
    Aty = P.bp_views(y)
    lhs = torch.dot(Ax.double().ravel(), y.double().ravel()).item()
    rhs = torch.dot(x.double().ravel(), Aty.double().ravel()).item()
    assert abs(lhs - rhs) < 1e-5 * abs(lhs), (lhs, rhs)


@pytest.mark.parametrize("design", list(DESIGNS))
def test_single_view_arbitrary_angle(design):
    cfg = GEOMS["plain"]
    P = Plan(cfg, Options(siddon_bp=DESIGNS[design]))
    g = O.Geom.from_dict(geom_dict(cfg))
    vol = np.random.default_rng(12).random(g.nvox).astype(np.float32)
    dvol = torch.from_numpy(vol).cuda().reshape(P.shape_vol)
    for ang in (12.345, 271.5):
        ref = np.zeros(g.npix)
        O.lib().orc_x_fp_view(g, ang, vol.astype(np.float64), ref)
        out = P.fp_view(dvol, ang).cpu().numpy().ravel()
        assert rel_l2(out, ref) < 1e-5
        img = torch.rand((P.nv, P.nu), device="cuda")
        bp = P.bp_view(img, ang)
        dot1 = torch.dot(P.fp_view(dvol, ang).double().ravel(), img.double().ravel()).item()
        dot2 = torch.dot(dvol.double().ravel(), bp.double().ravel()).item()
        assert abs(dot1 - dot2) < 1e-5 * abs(dot1)


@pytest.mark.parametrize("design", list(DESIGNS))
def test_determinism(design):
    cfg = GEOMS["cpu_small"]
    P = Plan(cfg, Options(siddon_bp=DESIGNS[design]))
    y = torch.rand((P.nproj, P.nv, P.nu), device="cuda")
    a = P.bp_views(y)
    b = P.bp_views(y)
    assert torch.equal(a, b)
    g = torch.rand((P.nproj, P.nv, P.nu), device="cuda") * 2
    f1 = P.mlem(g, 3)
    f2 = P.mlem(g, 3)
    assert torch.equal(f1, f2)


def _mlem_case(cfg, seed):
    g = O.Geom.from_dict(geom_dict(cfg))
    vol = phantom(cfg, seed=seed, n_ellipsoids=8)
    nproj = int(cfg["NumProj"])
    p = O.x_fp_all(g, nproj, np.float32(cfg["DeltaAng"]), vol.astype(np.float64).ravel())
    meas = noisy(p, 1e5, seed)
    return g, vol, meas


@pytest.mark.parametrize("design", list(DESIGNS))
@pytest.mark.parametrize("opts", ["kahan", "plain_sum"])
def test_mlem_vs_fp64(opts, design):
    cfg = scaled(CPU_SMALL, Xdim=48, Ydim=48, Zdim=40, XVoxSize=0.66, YVoxSize=0.66, ZVoxSize=0.66, AxPixels=96,
                 TAxPixels=80, NumProj=45)
    g, vol, meas = _mlem_case(cfg, 3)
    iters = 10
    f64, _ = O.x_mlem(g, 45, np.float32(cfg["DeltaAng"]), meas, iters)
    P = Plan(cfg, Options(sum=SUM_PLAIN if opts == "plain_sum" else 0, siddon_bp=DESIGNS[design]))
    f = P.mlem(torch.from_numpy(meas).cuda().reshape(45, P.nv, P.nu), iters)
    err = rel_l2(f.cpu().numpy(), f64)
    assert err < 1e-4, err


@pytest.mark.parametrize("design", list(DESIGNS))
def test_mlem_bf16_sinogram_error_reported(design):
    cfg = scaled(CPU_SMALL, Xdim=48, Ydim=48, Zdim=40, XVoxSize=0.66, YVoxSize=0.66, ZVoxSize=0.66, AxPixels=96,
                 TAxPixels=80, NumProj=45)
    g, vol, meas = _mlem_case(cfg, 4)
    f64, _ = O.x_mlem(g, 45, np.float32(cfg["DeltaAng"]), meas, 5)
    P = Plan(cfg, Options(sino=SINO_BF16, siddon_bp=DESIGNS[design]))
    gb = torch.from_numpy(meas).cuda().reshape(45, P.nv, P.nu).to(torch.bfloat16)
    f = P.mlem(gb, 5)
    err = rel_l2(f.cpu().numpy(), f64)
    assert err < 2e-2, err  # BF16 storage: ~3 significant digits per ratio value


# A wide, flat volume whose back projection needs two z-slabs (768 x 768 voxels per slice:
# 7 slices fit the 64 MiB accumulator budget), so the slab clipping, the accumulator offsets
# and the per-slab finish are exercised against FP64.
WIDE = small_cfg(Xdim=768, Ydim=768, Zdim=12, XVoxSize=0.05, YVoxSize=0.05, ZVoxSize=0.05, AxPixels=96,
                 TAxPixels=24, AxPixDim=0.64, TAxPixDim=0.1, NumProj=6)


@pytest.mark.parametrize("design", list(DESIGNS))
def test_multi_slab_back_projection_vs_fp64(design):
    cfg = WIDE
    P = Plan(cfg, Options(siddon_bp=DESIGNS[design]))
    g = O.Geom.from_dict(geom_dict(cfg))
    rng = np.random.default_rng(21)
    y = rng.random(6 * g.npix).astype(np.float32)
    bp = P.bp_views(torch.from_numpy(y).cuda().reshape(6, P.nv, P.nu)).cpu().numpy().ravel()
    ref = O.x_bp_all(g, 6, np.float32(cfg["DeltaAng"]), y.astype(np.float64))
    assert rel_l2(bp, ref) < 1e-5, rel_l2(bp, ref)
    sens = P.sensitivity().cpu().numpy().ravel()
    ref_s = O.x_bp_all(g, 6, np.float32(cfg["DeltaAng"]), np.ones(6 * g.npix))
    assert rel_l2(sens, ref_s) < 1e-5, rel_l2(sens, ref_s)
    x = rng.random(g.nvox).astype(np.float32)
    fp = P.fp_views(torch.from_numpy(x).cuda().reshape(P.shape_vol)).cpu().numpy().ravel()
    assert abs(np.dot(fp.astype(np.float64), y) - np.dot(x.astype(np.float64), bp)) < 1e-5 * abs(np.dot(fp, y))


@pytest.mark.parametrize("design", list(DESIGNS))
def test_multi_slab_mlem_vs_fp64(design):
    cfg = WIDE
    g = O.Geom.from_dict(geom_dict(cfg))
    meas = (np.random.default_rng(22).random(6 * g.npix) * 0.05).astype(np.float32)
    f64, _ = O.x_mlem(g, 6, np.float32(cfg["DeltaAng"]), meas, 3)
    P = Plan(cfg, Options(siddon_bp=DESIGNS[design]))
    f = P.mlem(torch.from_numpy(meas).cuda().reshape(6, P.nv, P.nu), 3).cpu().numpy().ravel()
    assert rel_l2(f, f64) < 1e-4, rel_l2(f, f64)


@pytest.mark.parametrize("design", list(DESIGNS))
def test_truncated_detector_vs_fp64(design):
    # a detector narrower and shorter than the volume's shadow: rays cover part of it
    cfg = small_cfg(AxPixels=16, TAxPixels=12, NumProj=8)
    P = Plan(cfg, Options(siddon_bp=DESIGNS[design]))
    g = O.Geom.from_dict(geom_dict(cfg))
    vol = np.random.default_rng(23).random(g.nvox).astype(np.float32)
    fp = P.fp_views(torch.from_numpy(vol).cuda().reshape(P.shape_vol)).cpu().numpy().ravel()
    assert rel_l2(fp, _x_fp(g, cfg, vol.astype(np.float64))) < 1e-5
    y = np.random.default_rng(24).random(8 * g.npix).astype(np.float32)
    bp = P.bp_views(torch.from_numpy(y).cuda().reshape(8, P.nv, P.nu)).cpu().numpy().ravel()
    assert rel_l2(bp, O.x_bp_all(g, 8, np.float32(cfg["DeltaAng"]), y.astype(np.float64))) < 1e-5


@pytest.mark.parametrize("design", list(DESIGNS))
def test_non_finite_input(design):
    # a non-finite value on a ray through the volume makes the voxels it crosses
    # non-finite (the ray design's shared fixed-point scale makes every voxel NaN)
    cfg = small_cfg(NumProj=4)
    P = Plan(cfg, Options(siddon_bp=DESIGNS[design]))
    y = torch.rand((4, P.nv, P.nu), device="cuda")
    c = (1, P.nv // 2, P.nu // 2)
    for bad in (float("nan"), float("inf")):
        y[c] = bad
        out = P.bp_views(y)
        assert not torch.isfinite(out).all()
        if design == "ray":
            assert torch.isnan(out).all()
        else:
            assert torch.isfinite(out).any()
    y[c] = 0.5  # finite again: the plan is not left in a bad state
    assert torch.isfinite(P.bp_views(y)).all()


def test_automatic_design_choice():
    # rows 1 to 1.4 voxels apart on a tall volume pick the gather; rows closer than a
    # voxel, or a short volume, the ray walk
    y_seed, x_seed = 31, 32
    for name, expect in (("z256", SIDDON_BP_GATHER), ("plain", SIDDON_BP_RAY), ("rows_apart", SIDDON_BP_RAY)):
        cfg = GEOMS[name]
        auto, forced = Plan(cfg, Options(siddon_bp=SIDDON_BP_AUTO)), Plan(cfg, Options(siddon_bp=expect))
        assert auto.siddon_bp == expect and forced.siddon_bp == expect
        y = torch.rand((auto.nproj, auto.nv, auto.nu), device="cuda",
                       generator=torch.Generator("cuda").manual_seed(y_seed))
        assert torch.equal(auto.bp_views(y), forced.bp_views(y))
        g = torch.rand((auto.nproj, auto.nv, auto.nu), device="cuda",
                       generator=torch.Generator("cuda").manual_seed(x_seed)) * 2
        assert torch.equal(auto.mlem(g, 2), forced.mlem(g, 2))


@pytest.mark.parametrize("name", ["plain", "rows_apart", "anisotropic"])
def test_designs_agree(name):
    # both designs sum the same lengths; they differ only in FP32 summation order
    cfg = GEOMS[name]
    Pg, Pr = Plan(cfg, Options(siddon_bp=SIDDON_BP_GATHER)), Plan(cfg, Options(siddon_bp=SIDDON_BP_RAY))
    y = torch.rand((Pg.nproj, Pg.nv, Pg.nu), device="cuda", generator=torch.Generator("cuda").manual_seed(33))
    a, b = Pg.bp_views(y).double(), Pr.bp_views(y).double()
    assert ((a - b).norm() / b.norm()).item() < 2e-6
    a, b = Pg.sensitivity().double(), Pr.sensitivity().double()
    assert ((a - b).norm() / b.norm()).item() < 2e-6


@pytest.mark.parametrize("name", ["plain", "offset", "anisotropic", "rows_apart", "z100"])
def test_mlem_iteration_designs_agree(name):
    # one MLEM iteration: the gather reads the ratio transposed into detector columns
    # (tiles outside each view's ray rectangle skipped), the ray design reads it as
    # the forward projector writes it; the images differ only by summation order
    cfg = GEOMS[name]
    gen = torch.Generator("cuda").manual_seed(34)
    fs = []
    for design in (SIDDON_BP_GATHER, SIDDON_BP_RAY):
        P = Plan(cfg, Options(siddon_bp=design))
        if not fs:
            g = torch.rand((P.nproj, P.nv, P.nu), device="cuda", generator=gen) * 2
            f0 = torch.rand(P.shape_vol, device="cuda", generator=gen) + 0.5
        f = f0.clone()
        P.mlem_prepare()
        P.mlem_iteration(g, f)
        fs.append(f.double())
    assert fs[1].norm() > 0
    assert ((fs[0] - fs[1]).norm() / fs[1].norm()).item() < 1e-5


def test_odd_height_gather_vs_fp64():
    # 255 slices in one chunk of 8 voxels per lane: the middle voxel straddles the
    # source plane, so the gather takes both ends of each piece for its row bounds
    cfg = small_cfg(Xdim=16, Ydim=16, Zdim=255, ZVoxSize=0.25, TAxPixDim=0.5, TAxPixels=160, NumProj=6)
    P = Plan(cfg, Options(siddon_bp=SIDDON_BP_GATHER))
    g = O.Geom.from_dict(geom_dict(cfg))
    nproj = int(cfg["NumProj"])
    sino = np.random.default_rng(13).random(nproj * g.npix).astype(np.float32)
    ref = O.x_bp_all(g, nproj, np.float32(cfg["DeltaAng"]), sino.astype(np.float64))
    out = P.bp_views(torch.from_numpy(sino).cuda().reshape(nproj, P.nv, P.nu)).cpu().numpy().ravel()
    assert rel_l2(out, ref) < 1e-5, rel_l2(out, ref)
    # the slices around the one straddling z = 0 on their own: an error in the
    # middle voxel's row bounds would be diluted in the whole volume's norm.  A
    # slice no ray crosses (rows 0.31 mm apart at the isocentre, voxels 0.25 mm
    # tall) must stay exactly zero
    plane = 16 * 16
    for k in (125, 126, 127, 128, 129):
        a, b = out[k * plane:(k + 1) * plane], ref[k * plane:(k + 1) * plane]
        if not np.any(b):
            assert not np.any(a), k
            continue
        assert np.abs(a - b).max() < 1e-5 * np.abs(b).max(), (k, np.abs(a - b).max(), np.abs(b).max())
        assert rel_l2(a, b) < 1e-5, (k, rel_l2(a, b))


# A tall, thin volume: the gather works through the column in five z-chunks of 224 slices.
TALL = small_cfg(Xdim=4, Ydim=4, Zdim=1100, XVoxSize=0.05, YVoxSize=0.05, ZVoxSize=0.05, AxPixels=8,
                 TAxPixels=900, AxPixDim=0.1, TAxPixDim=0.1, NumProj=4)


@pytest.mark.parametrize("design", list(DESIGNS))
def test_tall_volume_vs_fp64(design):
    cfg = TALL
    P = Plan(cfg, Options(siddon_bp=DESIGNS[design]))
    g = O.Geom.from_dict(geom_dict(cfg))
    y = np.random.default_rng(25).random(4 * g.npix).astype(np.float32)
    bp = P.bp_views(torch.from_numpy(y).cuda().reshape(4, P.nv, P.nu)).cpu().numpy().ravel()
    ref = O.x_bp_all(g, 4, np.float32(cfg["DeltaAng"]), y.astype(np.float64))
    assert rel_l2(bp, ref) < 1e-5, rel_l2(bp, ref)
    meas = (np.random.default_rng(26).random(4 * g.npix) * 0.05).astype(np.float32)
    f64, _ = O.x_mlem(g, 4, np.float32(cfg["DeltaAng"]), meas, 2)
    f = P.mlem(torch.from_numpy(meas).cuda().reshape(4, P.nv, P.nu), 2).cpu().numpy().ravel()
    assert rel_l2(f, f64) < 1e-4, rel_l2(f, f64)


def test_gather_with_many_detector_rows():
    # 4000 rows: the rows' z-plane table (64 KB) needs the large shared-memory opt-in;
    # the gather must agree with the ray walk.  Past 12288 rows a forced gather is refused.
    cfg = small_cfg(Xdim=8, Ydim=8, Zdim=200, ZVoxSize=0.2, AxPixels=16, TAxPixels=4000, TAxPixDim=0.05,
                    NumProj=3)
    Pg, Pr = Plan(cfg, Options(siddon_bp=SIDDON_BP_GATHER)), Plan(cfg, Options(siddon_bp=SIDDON_BP_RAY))
    y = torch.rand((3, Pg.nv, Pg.nu), device="cuda", generator=torch.Generator("cuda").manual_seed(35))
    a, b = Pg.bp_views(y).double(), Pr.bp_views(y).double()
    assert b.norm() > 0 and ((a - b).norm() / b.norm()).item() < 2e-6
    with pytest.raises(Exception):
        Plan(small_cfg(AxPixels=2, TAxPixels=12289), Options(siddon_bp=SIDDON_BP_GATHER))
    assert Plan(small_cfg(AxPixels=2, TAxPixels=12289)).siddon_bp == SIDDON_BP_RAY
