"""The gather back projector's fused MLEM update against its two halves.

recon_mlem_backward_update runs the gather with the update in its epilogue:
each CTA stages its tile's sums in shared memory and writes the tile along x,
one float4 per (plane, row) when the width is a multiple of 4 and the image and
sensitivity are 16-byte aligned, one voxel per thread otherwise.
recon_mlem_backward over all views (the same sums, written as Ht) followed by
recon_mlem_update (update_kernel) must give the same image bit for bit.
Geometries: mirrored voxel pairs (ratio in mirrored row pairs, or in detector
columns behind the ray-walk forward projector) and plain, one and several z
chunks, widths that are and are not multiples of 4, a partial tile row (odd
height in y), and an image 4 bytes off a 16-byte boundary.
"""
import pytest

from conftest import small_cfg

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

from recon_b200 import SIDDON_BP_GATHER, Options, Plan  # noqa: E402

CASES = {
    # name: (geometry, expected mirror pairing)
    "mirror_vec4": (small_cfg(), True),
    "plain_odd_z": (small_cfg(Zdim=25), False),
    "mirror_partial_tiles": (small_cfg(Xdim=30, Ydim=27), True),
    "plain_partial_tiles": (small_cfg(Xdim=30, Ydim=27, Zdim=23), False),
    "mirror_two_chunks": (small_cfg(Xdim=16, Ydim=16, Zdim=300, ZVoxSize=0.25, TAxPixDim=0.5, TAxPixels=200,
                                    NumProj=6), True),
    "plain_two_chunks": (small_cfg(Xdim=16, Ydim=18, Zdim=301, ZVoxSize=0.25, TAxPixDim=0.5, TAxPixels=200,
                                   NumProj=6), False),
    # the ray-walk forward projector: the mirror-paired gather on the detector-column layout
    "mirror_columns_layout": (small_cfg(ZVoxSize=0.1, TAxPixels=200, TAxPixDim=1.5), True),
}


def _volume(P, offset: int):
    """A volume tensor whose data starts `offset` floats into its allocation."""
    buf = torch.empty(P.shape_vol[0] * P.shape_vol[1] * P.shape_vol[2] + 4, device="cuda")
    return buf[offset:offset + buf.numel() - 4].view(P.shape_vol)


@pytest.mark.parametrize("offset", [0, 1])
@pytest.mark.parametrize("name", list(CASES))
def test_fused_update_equals_backward_then_update(name, offset):
    cfg, mirror = CASES[name]
    P = Plan(cfg, Options(siddon_bp=SIDDON_BP_GATHER))
    assert P.siddon_bp == SIDDON_BP_GATHER
    assert P.mirror_pairs == mirror
    gen = torch.Generator("cuda").manual_seed(61)
    g = torch.rand((P.nproj, P.nv, P.nu), device="cuda", generator=gen) * 3
    P.mlem_prepare()
    f0 = torch.rand(P.shape_vol, device="cuda", generator=gen) + 0.5
    P.mlem_forward(g, f0)  # the ratio both halves read
    fused = _volume(P, offset)
    fused.copy_(f0)
    P.mlem_backward_update(fused)
    split = _volume(P, offset)
    split.copy_(f0)
    ht = _volume(P, offset)
    P.mlem_backward(ht)
    P.mlem_update(split, ht)
    torch.cuda.synchronize()
    assert fused.abs().sum().item() > 0
    assert torch.equal(fused.view(torch.int32), split.view(torch.int32))
