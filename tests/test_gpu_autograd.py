"""Differentiable projector (128^3 volume, 180 views, 256^2 detector):
autograd gradient of 0.5||Ax - b||^2 against FP64 central differences, the
dot-product adjoint test, and the gradient through unrolled MLEM with
per-iteration checkpointing with respect to the relaxation weight."""
import numpy as np
import pytest

from conftest import rel_l2

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

from oracle import oracle as O  # noqa: E402
from recon_b200 import Plan  # noqa: E402
from recon_b200.autograd import backproject, mlem_unrolled, project  # noqa: E402
from recon_b200.configs import CPU_SMALL, DIFFERENTIABLE, geom_dict, scaled  # noqa: E402
from recon_b200.phantom import phantom  # noqa: E402


@pytest.fixture(scope="module")
def diff_case():
    cfg = dict(DIFFERENTIABLE)
    P = Plan(cfg)
    g = O.Geom.from_dict(geom_dict(cfg))
    x = phantom(cfg, seed=3)
    rng = np.random.default_rng(40)
    b = (O.x_fp_all(g, 180, np.float32(cfg["DeltaAng"]), x.astype(np.float64).ravel()) *
         (1.0 + 0.05 * rng.standard_normal(180 * g.npix))).astype(np.float32)
    return cfg, P, g, x, b


def test_dot_product_adjoint(diff_case):
    cfg, P, g, _, _ = diff_case
    gen = torch.Generator("cuda").manual_seed(7)
    x = torch.rand(P.shape_vol, device="cuda", generator=gen)
    y = torch.rand((180, P.nv, P.nu), device="cuda", generator=gen)
    lhs = torch.dot(project(x, P).double().ravel(), y.double().ravel()).item()
    rhs = torch.dot(x.double().ravel(), backproject(y, P).double().ravel()).item()
    assert abs(lhs - rhs) < 1e-5 * abs(lhs)


def test_gradient_vs_fp64_central_differences(diff_case):
    cfg, P, g, x, b = diff_case
    xt = torch.from_numpy(x).cuda().requires_grad_(True)
    bt = torch.from_numpy(b).cuda().reshape(180, P.nv, P.nu)
    loss = 0.5 * ((project(xt, P) - bt) ** 2).sum()
    loss.backward()
    grad = xt.grad.double().cpu().numpy().ravel()
    # FP64: r = A x - b; for L = 0.5 ||A x - b||^2 the central difference
    # (L(x + e a_i) - L(x - e a_i)) / (2 e) with e = 1e-3 is exact up to rounding
    r = O.x_fp_all(g, 180, np.float32(cfg["DeltaAng"]), x.astype(np.float64).ravel()) - b.astype(np.float64)
    rng = np.random.default_rng(41)
    cand = np.flatnonzero(x.ravel() > 0)
    voxels = rng.choice(cand, 64, replace=False)
    eps = 1e-3
    fd, ad = [], []
    for vx in voxels:
        view, pix, ln = O.x_voxel_column(g, 180, np.float32(cfg["DeltaAng"]), int(vx))
        rows = view.astype(np.int64) * g.npix + pix
        rp = r[rows] + eps * ln
        rm = r[rows] - eps * ln
        fd.append((0.5 * np.dot(rp, rp) - 0.5 * np.dot(rm, rm)) / (2 * eps))
        ad.append(grad[vx])
    fd, ad = np.array(fd), np.array(ad)
    assert rel_l2(ad, fd) < 1e-4, rel_l2(ad, fd)


def _fp64_relaxed_mlem(g, cfg, meas, iters, w):
    nproj, dang = int(cfg["NumProj"]), np.float32(cfg["DeltaAng"])
    s = O.x_bp_all(g, nproj, dang, np.ones(nproj * g.npix))
    f = np.ones(g.nvox)
    for _ in range(iters):
        hf = O.x_fp_all(g, nproj, dang, f)
        ratio = np.where(hf != 0, meas / np.where(hf != 0, hf, 1.0), 0.0)
        ht = O.x_bp_all(g, nproj, dang, ratio)
        upd = np.where(s != 0, ht / np.where(s != 0, s, 1.0), 0.0)
        f = f * (1.0 - w + w * upd)
    return f


def test_unrolled_mlem_gradient_wrt_relaxation():
    cfg = scaled(CPU_SMALL, NumProj=60, AxPixels=96, TAxPixels=96, AxPixDim=1.25, TAxPixDim=1.25, N_iteration=10)
    P = Plan(cfg)
    g = O.Geom.from_dict(geom_dict(cfg))
    truth = phantom(cfg, seed=5)
    meas = O.x_fp_all(g, 60, np.float32(cfg["DeltaAng"]), truth.astype(np.float64).ravel()).astype(np.float32)
    gt = torch.from_numpy(meas).cuda().reshape(60, P.nv, P.nu)
    tt = torch.from_numpy(truth).cuda()
    w = torch.tensor(0.8, device="cuda", requires_grad=True)
    f = mlem_unrolled(P, gt, 10, w, use_checkpoint=True)
    loss = 0.5 * ((f - tt) ** 2).sum()
    loss.backward()
    dw = w.grad.item()
    # the same without checkpointing
    w2 = torch.tensor(0.8, device="cuda", requires_grad=True)
    loss2 = 0.5 * ((mlem_unrolled(P, gt, 10, w2, use_checkpoint=False) - tt) ** 2).sum()
    loss2.backward()
    assert abs(w2.grad.item() - dw) <= 1e-5 * abs(dw)
    # FP64 central difference through 10 unrolled iterations
    eps = 1e-3
    lp = 0.5 * np.sum((_fp64_relaxed_mlem(g, cfg, meas.astype(np.float64), 10, 0.8 + eps) - truth.ravel()) ** 2)
    lm = 0.5 * np.sum((_fp64_relaxed_mlem(g, cfg, meas.astype(np.float64), 10, 0.8 - eps) - truth.ravel()) ** 2)
    fd = (lp - lm) / (2 * eps)
    assert abs(dw - fd) < 2e-3 * abs(fd), (dw, fd)


def test_unrolled_mlem_gradient_at_differentiable_size(diff_case):
    """The relaxation-weight gradient through 10 unrolled, checkpointed MLEM
    iterations on the differentiable workload itself (128^3, 180 views, 256^2):
    checkpointed against plain autograd, and against the FP64 central
    difference of the same 10 relaxed iterations (a few minutes of host FP64)."""
    cfg, P, g, x, b = diff_case
    bt = torch.from_numpy(b).cuda().reshape(180, P.nv, P.nu)
    tt = torch.from_numpy(x).cuda()
    w = torch.tensor(0.8, device="cuda", requires_grad=True)
    loss = 0.5 * ((mlem_unrolled(P, bt, 10, w, use_checkpoint=True) - tt) ** 2).sum()
    loss.backward()
    dw = w.grad.item()
    w2 = torch.tensor(0.8, device="cuda", requires_grad=True)
    loss2 = 0.5 * ((mlem_unrolled(P, bt, 10, w2, use_checkpoint=False) - tt) ** 2).sum()
    loss2.backward()
    assert abs(w2.grad.item() - dw) <= 1e-5 * abs(dw)
    eps = 1e-3
    meas = b.astype(np.float64)
    lp = 0.5 * np.sum((_fp64_relaxed_mlem(g, cfg, meas, 10, 0.8 + eps) - x.ravel()) ** 2)
    lm = 0.5 * np.sum((_fp64_relaxed_mlem(g, cfg, meas, 10, 0.8 - eps) - x.ravel()) ** 2)
    fd = (lp - lm) / (2 * eps)
    assert abs(dw - fd) < 2e-3 * abs(fd), (dw, fd)
