"""recon_compat_bp_view_noalloc: COMPAT back projection with no device allocation.

Collected last (file name), so it runs both alone and after every other test
has loaded and used the library.  Each case makes two calls in a row through
the allocation-free entry point and compares both, bit for bit, with
recon_bp_view on a COMPAT plan of the same geometry; the second call also
shows that the shared scratch starts clean.
"""
import ctypes as C

import numpy as np
import pytest

from conftest import small_cfg

from recon_b200 import ARITH_COMPAT, Options, Plan, ReconError
from recon_b200 import _lib as L
from recon_b200.api import compat_bp_view_noalloc, geometry


def test_oversize_volume_rejected_before_device_work():
    # 129^3 voxels > RECON_NOALLOC_MAX_VOXELS; rejected on the host (no GPU needed)
    g = geometry(small_cfg(Xdim=129, Ydim=129, Zdim=129))
    dummy = C.c_void_p(256)
    st = L.lib().recon_compat_bp_view_noalloc(C.byref(g), dummy, 0.0, dummy, None)
    assert st == 2  # RECON_ERR_UNSUPPORTED
    assert b"RECON_NOALLOC_MAX_VOXELS" in L.lib().recon_last_error()
    st = L.lib().recon_compat_bp_view_noalloc(None, dummy, 0.0, dummy, None)
    assert st == 1  # RECON_ERR_INVALID_ARGUMENT


CASES = {
    "plain": small_cfg(),
    "offset_tilt": small_cfg(Dx=0.7, Dz=-0.4, Ry=803.0, M=1.2, xangle=0.01, zangle=-0.02),
    "max_voxels": small_cfg(Xdim=128, Ydim=128, Zdim=128, XVoxSize=0.25, YVoxSize=0.25, ZVoxSize=0.25),
}


@pytest.mark.gpu
@pytest.mark.parametrize("name", list(CASES))
def test_two_calls_match_plan_bitwise(name):
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    cfg = CASES[name]
    P = Plan(cfg, Options(arith=ARITH_COMPAT))
    rng = np.random.default_rng(40)
    imgs = [torch.from_numpy(rng.random((P.nv, P.nu), dtype=np.float32)).cuda() for _ in range(2)]
    angles = [P.angle(1), 123.25]  # a plan view and an arbitrary angle
    outs = [torch.full(P.shape_vol, -7.0, device="cuda") for _ in range(2)]
    for img, ang, out in zip(imgs, angles, outs):
        compat_bp_view_noalloc(cfg, img, ang, out)
    for img, ang, out in zip(imgs, angles, outs):
        ref = P.bp_view(img, ang)
        torch.cuda.synchronize()
        a = out.cpu().numpy().view(np.uint32)
        b = ref.cpu().numpy().view(np.uint32)
        assert np.array_equal(a, b), f"{name} angle {ang}: {np.count_nonzero(a != b)} voxels differ"
        assert float(ref.abs().sum()) > 0.0


@pytest.mark.gpu
def test_steady_state_allocates_no_device_memory():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    cfg = CASES["plain"]
    img = torch.rand((int(cfg["TAxPixels"]), int(cfg["AxPixels"])), device="cuda")
    out = torch.empty((int(cfg["Zdim"]), int(cfg["Ydim"]), int(cfg["Xdim"])), device="cuda")
    compat_bp_view_noalloc(cfg, img, 10.0, out)  # set-up call
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for ang in (20.0, 30.0):
        compat_bp_view_noalloc(cfg, img, ang, out)
    torch.cuda.synchronize()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0


@pytest.mark.gpu
def test_invalid_geometry_reports_error():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    cfg = small_cfg(R=-1.0)
    img = torch.zeros((int(cfg["TAxPixels"]), int(cfg["AxPixels"])), device="cuda")
    out = torch.zeros((int(cfg["Zdim"]), int(cfg["Ydim"]), int(cfg["Xdim"])), device="cuda")
    with pytest.raises(ReconError):
        compat_bp_view_noalloc(cfg, img, 0.0, out)
