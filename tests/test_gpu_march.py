"""Ray-marching forward projection (recon_march_fp_view).

REFERENCE mode against the reference's own kernel: forward_projection
(CT_Recon/hf_cuda_kernels.cuh:126-180), built for sm_100a from its sources
(oracle/_ref/libref_gpu.so) with its 3D texture replaced by a point-sampled,
border-addressed stand-in over normalised coordinates (oracle/ref_shim/common/
ref_prelude_gpu.h), launched once per depth plane: bit-identical images.
Both modes against the FP64 restatement (orc_m_fp_view):
GEOMETRIC: trilinear plane samples; FP32 against FP64, rel. L2 <= 1e-5.
REFERENCE: point samples of normalised coordinates; a sample whose coordinate
lies within FP32 rounding of a texel boundary may take the neighbouring texel,
so the bound is rel. L2 <= 1e-3 with at least 99 % of pixels within 1e-4 of
the oracle.
"""
import numpy as np
import pytest

from conftest import rel_l2, small_cfg

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

from oracle import oracle as O  # noqa: E402
from recon_b200 import ARITH_COMPAT, VOXEL_GEOMETRIC, VOXEL_REFERENCE, Options, Plan  # noqa: E402
from recon_b200.configs import geom_dict  # noqa: E402

GEOMS = {
    "plain": (small_cfg(Zdim=32), Options()),
    "offset": (small_cfg(Dx=0.7, Dz=-0.4, Ry=803.0, M=1.2, Zdim=32), Options()),
    # tilted detector: a COMPAT plan (EXACT plans refuse tilt); the projector takes any plan
    "tilted": (small_cfg(xangle=0.4, yangle=-0.3, zangle=0.2, Zdim=32), Options(arith=ARITH_COMPAT)),
}


@pytest.mark.parametrize("name", list(GEOMS))
@pytest.mark.parametrize("mode", [VOXEL_GEOMETRIC, VOXEL_REFERENCE])
def test_march_vs_oracle(name, mode):
    cfg, opts = GEOMS[name]
    P = Plan(cfg, opts)
    g = O.Geom.from_dict(geom_dict(cfg))
    vol = np.random.default_rng(41).random(g.nvox).astype(np.float32)
    dvol = torch.from_numpy(vol).cuda().reshape(P.shape_vol)
    for ang in (0.0, 37.5, 90.0, 211.25):
        out = P.march_fp_view(dvol, ang, mode).cpu().numpy().ravel().astype(np.float64)
        ref = O.m_fp_view(g, ang, mode, vol)
        err = rel_l2(out, ref)
        if mode == VOXEL_GEOMETRIC:
            assert err < 1e-5, (ang, err)
        else:
            assert err < 1e-3, (ang, err)
            close = np.abs(out - ref) <= 1e-4 * np.abs(ref).max()
            assert close.mean() >= 0.99, (ang, close.mean())


def test_march_rejects_bad_arguments():
    P = Plan(small_cfg())
    vol = P.new_volume(1.0)
    with pytest.raises(Exception):
        P.march_fp_view(vol, 0.0, 7)
    with pytest.raises(Exception):
        P.march_fp_view(vol, float("nan"), VOXEL_GEOMETRIC)


REFG = O.ref_gpu()


@pytest.mark.skipif(REFG is None or not hasattr(REFG, "ref_gpu_march_fp_view"),
                    reason="reference sm_100a build missing")
@pytest.mark.parametrize("name", list(GEOMS))
def test_reference_mode_vs_reference_kernel(name):
    cfg, opts = GEOMS[name]
    P = Plan(cfg, opts)
    g = O.Geom.from_dict(geom_dict(cfg))
    vol = np.random.default_rng(43).random(g.nvox).astype(np.float32)
    dvol = torch.from_numpy(vol).cuda().reshape(P.shape_vol)
    for ang in (0.0, 37.5, 90.0, 211.25, 359.0):
        out = P.march_fp_view(dvol, ang, VOXEL_REFERENCE).cpu().numpy().ravel()
        ref = np.zeros(g.npix, np.float32)
        REFG.ref_gpu_march_fp_view(g, ang, vol, ref)
        assert np.any(ref != 0), ang
        assert np.array_equal(out.view(np.uint32), ref.view(np.uint32)), (ang, rel_l2(out, ref))
