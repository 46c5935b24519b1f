"""Plans used from several host threads at once (each thread its own plan and
stream) give the same results as one thread: plans share no mutable state,
including the voxel-driven back projector's texture cache, and batches their
autotuning cache under a lock."""
import threading

import numpy as np
import pytest

from conftest import small_cfg

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

from recon_b200 import BP_VOXEL, Batch, Options, Plan  # noqa: E402

CFGS = [small_cfg(), small_cfg(Xdim=30, Ydim=26, Zdim=21, AxPixels=61, TAxPixels=47),
        small_cfg(Dx=0.7, Dz=-0.4, NumProj=16), small_cfg(NumProj=8)]


def _work(cfg, opts, g):
    P = Plan(cfg, opts)
    f = P.mlem(g, 3)
    return f.cpu().numpy()


def _inputs(seed):
    gen = torch.Generator(device="cuda").manual_seed(seed)
    return [torch.rand((int(c["NumProj"]), int(c["TAxPixels"]), int(c["AxPixels"])), device="cuda", generator=gen)
            for c in CFGS]


@pytest.mark.parametrize("bp", ["siddon", "voxel"])
def test_concurrent_plans_match_sequential(bp):
    opts = Options(bp=BP_VOXEL) if bp == "voxel" else Options()
    gs = _inputs(11)
    torch.cuda.synchronize()
    expect = [_work(c, opts, g) for c, g in zip(CFGS, gs)]
    got = [None] * len(CFGS)
    errors = []

    def run(i):
        try:
            with torch.cuda.stream(torch.cuda.Stream()):
                got[i] = _work(CFGS[i], opts, gs[i])
        except Exception as e:  # pragma: no cover - reported below
            errors.append(e)

    threads = [threading.Thread(target=run, args=(i,)) for i in range(len(CFGS))]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    assert not errors, errors
    for a, b in zip(got, expect):
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32))


def test_concurrent_batches():
    gs = _inputs(12)
    torch.cuda.synchronize()
    expect = [f.cpu().numpy() for f in Batch(CFGS).mlem(gs, 2)]
    results, errors = [None, None], []

    def run(i):
        try:
            with torch.cuda.stream(torch.cuda.Stream()):
                fs = Batch(CFGS).mlem(gs, 2)
                torch.cuda.current_stream().synchronize()
                results[i] = [f.cpu().numpy() for f in fs]
        except Exception as e:  # pragma: no cover
            errors.append(e)

    threads = [threading.Thread(target=run, args=(i,)) for i in range(2)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    assert not errors, errors
    for r in results:
        for a, b in zip(r, expect):
            assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
