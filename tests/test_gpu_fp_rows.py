"""Detector rows per CTA of the column forward projector (recon_options_t.fp_rows).

Each lane walks one detector row whatever the CTA's size, so projections and
MLEM images are bit-identical with 32, 64 and 128 rows per CTA: with mirrored
row pairs and without, in xy blocks, and for a detector whose columns hold
more rows than one CTA.  AUTO takes the fewest of 32, 64, 128 that cover a
column's rows; RECON_SIDDON_BP_TUNED measures the three and keeps the choice
for the geometry (a second plan makes the same choice).
"""
import pytest

from conftest import small_cfg

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

from recon_b200 import FP_RAY_WALK, SIDDON_BP_GATHER, SIDDON_BP_TUNED, Options, Plan  # noqa: E402

CASES = {
    "mirror": (small_cfg(), {}),
    "odd_z": (small_cfg(Zdim=25), {}),
    "tall_detector": (small_cfg(TAxPixels=300, TAxPixDim=0.25, Zdim=40), {}),
    "blocks": (small_cfg(), {"fp_block": 8}),
}


@pytest.mark.parametrize("name", list(CASES))
def test_results_do_not_depend_on_rows_per_cta(name):
    cfg, extra = CASES[name]
    gen = torch.Generator("cuda").manual_seed(91)
    images, sinos = [], []
    for rows in (32, 64, 128):
        P = Plan(cfg, Options(fp_rows=rows, siddon_bp=SIDDON_BP_GATHER, **extra))
        assert P.forward_projector != FP_RAY_WALK
        assert P.column_rows == rows
        if not images:
            vol = torch.rand(P.shape_vol, device="cuda", generator=gen) + 0.1
        sinos.append(P.fp_views(vol))
        images.append(P.mlem(sinos[0], 2))
    torch.cuda.synchronize()
    for s, f in zip(sinos[1:], images[1:]):
        assert torch.equal(s.view(torch.int32), sinos[0].view(torch.int32))
        assert torch.equal(f.view(torch.int32), images[0].view(torch.int32))


def test_auto_and_tuned_rows():
    assert Plan(small_cfg()).column_rows == 32  # 24 lower rows of 48: one warp covers a column
    assert Plan(small_cfg(TAxPixels=300, TAxPixDim=0.25, Zdim=40)).column_rows == 128
    cfg = small_cfg(TAxPixels=160, TAxPixDim=0.5, Zdim=64)
    a = Plan(cfg, Options(siddon_bp=SIDDON_BP_TUNED))
    b = Plan(cfg, Options(siddon_bp=SIDDON_BP_TUNED))
    assert a.column_rows in (32, 64, 128)
    assert b.column_rows == a.column_rows
