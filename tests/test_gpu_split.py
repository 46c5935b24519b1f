"""The split MLEM iteration (forward and back projection over view ranges, then
the update), as view sharding across GPUs calls it, against the whole iteration.

Two view ranges are projected and back projected separately and their partial
images summed; the update then gives the same image as recon_mlem_iteration up
to FP32 summation order (rel. L2 <= 1e-6), for both back projectors and both
sinogram precisions.
"""
import pytest

from conftest import small_cfg

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

from recon_b200 import SIDDON_BP_GATHER, SIDDON_BP_RAY, SINO_BF16, SINO_F32, Options, Plan  # noqa: E402

# a tall volume whose rows are 1.2 voxels apart (the gather's geometry), 9 views split 4 + 5
CFG = small_cfg(Xdim=16, Ydim=16, Zdim=160, ZVoxSize=0.25, TAxPixDim=0.5, TAxPixels=110, NumProj=9)


@pytest.mark.parametrize("sino", [SINO_F32, SINO_BF16])
@pytest.mark.parametrize("design", [SIDDON_BP_GATHER, SIDDON_BP_RAY])
def test_split_iteration_matches_whole(design, sino):
    P = Plan(CFG, Options(siddon_bp=design, sino=sino))
    gen = torch.Generator("cuda").manual_seed(51)
    g = torch.rand((P.nproj, P.nv, P.nu), device="cuda", generator=gen) * 3
    if sino == SINO_BF16:
        g = g.to(torch.bfloat16)
    P.mlem_prepare()
    f_whole = P.new_volume(1.0)
    P.mlem_iteration(g, f_whole)
    f_split = P.new_volume(1.0)
    ht = P.new_volume(0.0)
    ht_part = P.new_volume(0.0)
    for first, count in ((0, 4), (4, 5)):
        P.mlem_forward(g, f_split, first, count)
    for first, count in ((0, 4), (4, 5)):
        P.mlem_backward(ht_part, first, count)
        ht += ht_part
    P.mlem_update(f_split, ht)
    a, b = f_split.double(), f_whole.double()
    assert b.norm() > 0
    assert ((a - b).norm() / b.norm()).item() < 1e-6
