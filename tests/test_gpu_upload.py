"""recon_upload_sinogram: only the detector rows the plan's rays can read.

The measured sinogram is uploaded into a device buffer filled with NaN, so
every row the upload skips holds NaN.  MLEM from that buffer must give the
image of MLEM from a full copy bit for bit: for every forward design (detector
columns, in xy blocks, the ray walk), both Siddon back projectors, the
voxel-driven back projector, BF16 sinograms and COMPAT arithmetic (which
copies whole views).  The bytes reported are the rows v_min..v_max of every
view for EXACT plans, whole views for COMPAT.
"""
import pytest

from conftest import small_cfg

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

from recon_b200 import (ARITH_COMPAT, BP_VOXEL, FP_RAY_WALK, SIDDON_BP_RAY, SINO_BF16, VOXEL_GEOMETRIC,  # noqa: E402
                        Options, Plan)

TALL_DET = small_cfg(TAxPixels=96)
THIN = small_cfg(ZVoxSize=0.1, TAxPixels=200, TAxPixDim=1.5)  # a 2.4 mm slab: the ray walk
CASES = {
    "columns": (TALL_DET, Options()),
    "column_blocks": (TALL_DET, Options(fp_block=8)),
    "ray_bp": (TALL_DET, Options(siddon_bp=SIDDON_BP_RAY)),
    "voxel_bp": (TALL_DET, Options(bp=BP_VOXEL, voxel_mode=VOXEL_GEOMETRIC)),
    "ray_walk": (THIN, Options()),
    "bf16": (TALL_DET, Options(sino=SINO_BF16)),
    "compat": (TALL_DET, Options(arith=ARITH_COMPAT)),
}


@pytest.mark.parametrize("name", list(CASES))
def test_upload_reads_only_what_the_plan_reads(name):
    cfg, opts = CASES[name]
    P = Plan(cfg, opts)
    if name == "ray_walk":
        assert P.forward_projector == FP_RAY_WALK
    gen = torch.Generator("cuda").manual_seed(81)
    vol = torch.rand(P.shape_vol, device="cuda", generator=gen) + 0.1
    g = Plan(cfg).fp_views(vol)
    if opts.sino == SINO_BF16:
        g = g.to(torch.bfloat16)
    g_host = g.cpu().pin_memory()
    full = g.clone()
    part = torch.full_like(g, float("nan"))
    n = P.upload_sinogram(g_host, part)
    torch.cuda.synchronize()
    view_bytes = g[0].numel() * g.element_size()
    rows_read = ~torch.isnan(part.float()).all(dim=2).all(dim=0)  # rows the upload wrote
    assert n == int(rows_read.sum()) * P.nu * g.element_size() * P.nproj
    if opts.arith == ARITH_COMPAT:
        assert n == view_bytes * P.nproj
    else:
        assert n < view_bytes * P.nproj  # this detector is taller than the volume's shadow
    f_full = P.mlem(full, 2)
    f_part = P.mlem(part, 2)
    torch.cuda.synchronize()
    assert f_full.abs().sum().item() > 0
    assert torch.equal(f_full.view(torch.int32), f_part.view(torch.int32))


def test_upload_view_range_and_arguments():
    P = Plan(TALL_DET)
    g = torch.rand((P.nproj, P.nv, P.nu), device="cuda")
    g_host = g.cpu().pin_memory()
    part = torch.zeros_like(g)
    n = P.upload_sinogram(g_host, part, 3, 4)
    torch.cuda.synchronize()
    assert n > 0
    assert torch.all(part[:3] == 0) and torch.all(part[7:] == 0)
    rows = (part[3:7] != 0).any(dim=2).any(dim=0)
    assert torch.equal(part[3:7][:, rows], g[3:7][:, rows])
    with pytest.raises(ValueError):
        P.upload_sinogram(g, part)  # the source must be host memory
    with pytest.raises(Exception):
        P.upload_sinogram(g_host, part, P.nproj - 1, 2)  # past the last view
