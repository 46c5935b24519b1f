"""OSEM (recon_osem) against the FP64 oracle and against MLEM.

The reference defines OSEM only through its parameter structs and their
check (hf_cpp_functions.hpp:298-375): the subsets split NumProj evenly and a
subset is a contiguous arc of views.  Tolerance: relative L2 <= 1e-4 against
FP64 OSEM after 3 passes.
"""
import numpy as np
import pytest

from conftest import rel_l2, small_cfg

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

from oracle import oracle as O  # noqa: E402
from recon_b200 import ARITH_COMPAT, Options, Plan, ReconError  # noqa: E402
from recon_b200.configs import geom_dict  # noqa: E402


def _problem(cfg, seed):
    g = O.Geom.from_dict(geom_dict(cfg))
    sino = np.random.default_rng(seed).random(int(cfg["NumProj"]) * g.npix).astype(np.float32)
    return g, sino, torch.from_numpy(sino).cuda().reshape(int(cfg["NumProj"]), int(cfg["TAxPixels"]),
                                                          int(cfg["AxPixels"]))


def test_one_subset_is_mlem_bitwise():
    cfg = small_cfg()
    _, _, g = _problem(cfg, 1)
    P = Plan(cfg)
    a = P.osem(g, 3, 1).cpu().numpy().view(np.uint32)
    b = Plan(cfg).mlem(g, 3).cpu().numpy().view(np.uint32)
    assert np.array_equal(a, b)


@pytest.mark.parametrize("subsets", [2, 3, 4])
def test_osem_vs_fp64(subsets):
    cfg = small_cfg(NumProj=12)
    geo, sino, g = _problem(cfg, 2)
    f = Plan(cfg).osem(g, 3, subsets).cpu().numpy().ravel()
    ref = O.x_osem(geo, 12, np.float32(cfg["DeltaAng"]), sino, 3, subsets)
    assert rel_l2(f, ref) < 1e-4, rel_l2(f, ref)


def test_repeat_and_subset_count_change():
    cfg = small_cfg(NumProj=12)
    _, _, g = _problem(cfg, 3)
    P = Plan(cfg)
    a = P.osem(g, 2, 4).cpu().numpy()
    P.osem(g, 1, 3)  # another subset count re-derives the subset sensitivities
    b = P.osem(g, 2, 4).cpu().numpy()
    assert np.array_equal(a.view(np.uint32), b.view(np.uint32))


def test_rejects_bad_subsets_and_compat():
    cfg = small_cfg(NumProj=12)
    _, _, g = _problem(cfg, 4)
    P = Plan(cfg)
    with pytest.raises(ReconError):
        P.osem(g, 1, 5)
    with pytest.raises(ReconError):
        P.osem(g, 1, 0)
    with pytest.raises(ReconError):
        Plan(cfg, Options(arith=ARITH_COMPAT)).osem(g, 1, 2)
