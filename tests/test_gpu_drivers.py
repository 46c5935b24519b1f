"""The file-driven forward and back projection drivers against the reference's own.

recon_forward_projection_from_cfg / recon_backward_projection_from_cfg (COMPAT
arithmetic) and the reference's siddon_recon::a1_FORWARD_PROJECTION /
a1_BACKWARD_PROJECTION (CT_Recon/hf_siddon_recon.hpp:146-182, 515-592), built
for sm_100a from its sources (oracle/_ref/libref_gpu.so), run on the same
configuration and files:
  * per-view projection files <ProjFileFolder><ProjFileNameRoot>_<n><suffix>:
    bit-identical;
  * per-view back projections <ProjFileFolder><BpFileNameRoot>_<n><suffix>:
    relative L2 <= 1e-6 (the reference sums with float atomics, in an order
    that changes run to run);
  * the total back projection <ProjFileFolder><BpFileNameRoot><suffix>:
    against the sum of the reference's per-view files (the reference adds its
    views into an image it allocates without clearing, hf_siddon_recon.hpp:425,
    568, so its own total depends on what that memory held);
  * the .info parameter echoes (hf_siddon_class.hpp:483-643): the same keys with
    the same values.
The EXACT drivers' per-view files are checked against the FP64 oracle.
"""
import os

import numpy as np
import pytest

from conftest import rel_l2, small_cfg

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

from oracle import oracle as O  # noqa: E402
from recon_b200 import ARITH_COMPAT, Options, backward_projection_from_cfg, forward_projection_from_cfg  # noqa: E402
from recon_b200.configs import geom_dict  # noqa: E402
from recon_b200.phantom import phantom  # noqa: E402
from tests_helpers import write_cfg  # noqa: E402

REF = O.ref_gpu()
needs_ref = pytest.mark.skipif(REF is None or not hasattr(REF, "ref_gpu_backward_projection_cfg"),
                               reason="reference sm_100a build missing")


def _info(path: str) -> dict:
    """key -> value of a `key = value  # comment` parameter echo."""
    out = {}
    for line in open(path):
        line = line.split("#", 1)[0]
        if "=" in line:
            k, v = line.split("=", 1)
            out[k.strip()] = v.strip()
    return out


def _case(tmp_path, cfg):
    root = str(tmp_path)
    vol = phantom(cfg, seed=5, n_ellipsoids=6).astype(np.float32)
    vol.tofile(os.path.join(root, "object.bin"))
    dirs = {}
    for tag in ("ref", "new"):
        d = os.path.join(root, tag) + "/"
        os.makedirs(d)  # the reference asks on stdin before creating a missing folder
        write_cfg(os.path.join(root, f"{tag}.cfg"), cfg, d, root + "/recon/", obj_folder=root + "/")
        dirs[tag] = d
    return root, vol, dirs


@needs_ref
def test_forward_and_backward_drivers_vs_reference(tmp_path):
    cfg = small_cfg(NumProj=12)
    root, vol, dirs = _case(tmp_path, cfg)
    n = int(cfg["NumProj"])
    REF.ref_gpu_forward_projection_cfg((root + "/").encode(), b"ref.cfg")
    forward_projection_from_cfg(root, "new.cfg", Options(arith=ARITH_COMPAT))
    for k in range(n):
        a = np.fromfile(os.path.join(dirs["new"], f"proj_{k}.bin"), np.float32)
        b = np.fromfile(os.path.join(dirs["ref"], f"proj_{k}.bin"), np.float32)
        assert a.size == b.size == cfg["AxPixels"] * cfg["TAxPixels"]
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), k
    ia, ib = _info(os.path.join(dirs["new"], "proj.info")), _info(os.path.join(dirs["ref"], "proj.info"))
    assert set(ia) == set(ib)
    for k in ia:
        if k != "ProjFileFolder":
            assert ia[k] == ib[k], (k, ia[k], ib[k])
    # back projection of the same (bit-identical) projection files
    REF.ref_gpu_backward_projection_cfg((root + "/").encode(), b"ref.cfg", 1)
    backward_projection_from_cfg(root, "new.cfg", True, Options(arith=ARITH_COMPAT))
    nvox = cfg["Xdim"] * cfg["Ydim"] * cfg["Zdim"]
    total_ref = np.zeros(nvox, np.float64)
    for k in range(n):
        a = np.fromfile(os.path.join(dirs["new"], f"bp_{k}.bin"), np.float32)
        b = np.fromfile(os.path.join(dirs["ref"], f"bp_{k}.bin"), np.float32)
        assert a.size == b.size == nvox
        assert rel_l2(a, b) < 1e-6, (k, rel_l2(a, b))
        total_ref += b
    total = np.fromfile(os.path.join(dirs["new"], "bp.bin"), np.float32)
    assert rel_l2(total, total_ref) < 1e-6, rel_l2(total, total_ref)
    ia, ib = _info(os.path.join(dirs["new"], "bp.info")), _info(os.path.join(dirs["ref"], "bp.info"))
    assert set(ia) == set(ib)
    for k in ia:
        if k != "ProjFileFolder":
            assert ia[k] == ib[k], (k, ia[k], ib[k])


def test_exact_drivers_vs_fp64(tmp_path):
    cfg = small_cfg(NumProj=8)
    root, vol, dirs = _case(tmp_path, cfg)
    g = O.Geom.from_dict(geom_dict(cfg))
    n = int(cfg["NumProj"])
    forward_projection_from_cfg(root, "new.cfg", Options())
    dang = np.float32(cfg["DeltaAng"])
    ref = O.x_fp_all(g, n, dang, vol.astype(np.float64).ravel()).reshape(n, -1)
    sino = np.stack([np.fromfile(os.path.join(dirs["new"], f"proj_{k}.bin"), np.float32) for k in range(n)])
    assert rel_l2(sino, ref) < 1e-5, rel_l2(sino, ref)
    backward_projection_from_cfg(root, "new.cfg", False, Options())
    bp = np.fromfile(os.path.join(dirs["new"], "bp.bin"), np.float32)
    bref = O.x_bp_all(g, n, dang, sino.astype(np.float64).ravel())
    assert rel_l2(bp, bref) < 1e-5, rel_l2(bp, bref)
