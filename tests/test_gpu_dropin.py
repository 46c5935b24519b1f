"""The drop-in C++ headers: a caller written against the reference's class
interface (tests/cpp/drop_in_main.cpp) is compiled against include/ and
linked with librecon_b200.so; its outputs equal the Python binding's results
for the same library calls, bit for bit."""
import os
import shutil
import subprocess

import numpy as np
import pytest

from conftest import ROOT, small_cfg

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")
if not torch.cuda.is_available():
    pytest.skip("no CUDA device", allow_module_level=True)

from recon_b200 import ARITH_COMPAT, VOXEL_REFERENCE, Options, Plan  # noqa: E402
from tests_helpers import write_case, write_cfg  # noqa: E402


def test_reference_style_caller(tmp_path):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    exe = os.path.join(str(tmp_path), "drop_in")
    libdir = os.path.join(ROOT, "recon_b200")
    subprocess.run([nvcc, "-std=c++17", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "cpp", "drop_in_main.cpp"), "-o", exe, "-L", libdir,
                    "-lrecon_b200", "-Xlinker", f"-rpath={libdir}"], check=True)
    cfg = small_cfg(NumProj=8, N_iteration=3)
    folder = write_case(tmp_path, cfg, seed=30)
    out = os.path.join(folder, "out")
    os.makedirs(out)
    write_cfg(os.path.join(folder, "c.cfg"), cfg, folder, out + "/", obj_folder=folder)
    res = subprocess.run([exe, folder, "c.cfg", out], capture_output=True, text=True, timeout=600)
    assert res.returncode == 0, res.stdout + res.stderr
    assert "Do reconstruction" in res.stdout and "drop-in ok" in res.stdout

    P = Plan(cfg, Options(arith=ARITH_COMPAT))
    npix, nvox = P.nu * P.nv, int(np.prod(P.shape_vol))
    g = np.stack([np.fromfile(os.path.join(folder, f"proj_{n}.bin"), np.float32) for n in range(8)])
    f = P.mlem(torch.from_numpy(g).cuda().reshape(8, P.nv, P.nu), 3).cpu().numpy().ravel()
    assert np.array_equal(f, np.fromfile(os.path.join(out, "recon_2.bin"), np.float32))
    vol = torch.from_numpy(np.fromfile(os.path.join(folder, "object.bin"), np.float32)).cuda().reshape(P.shape_vol)
    for n in range(8):
        fp = P.fp_view(vol, P.angle(n))
        assert np.array_equal(fp.cpu().numpy().ravel(), np.fromfile(os.path.join(out, f"fp_{n}.bin"), np.float32))
        bp = P.bp_view(fp, P.angle(n))
        assert np.array_equal(bp.cpu().numpy().ravel(), np.fromfile(os.path.join(out, f"bp_{n}.bin"), np.float32))
    vb = P.voxel_bp_view(fp, P.angle(7), 8, VOXEL_REFERENCE)
    assert np.array_equal(vb.cpu().numpy().ravel(), np.fromfile(os.path.join(out, "voxel_bp.bin"), np.float32))
    assert nvox == vb.numel() and npix == fp.numel()


def test_mlem_from_cfg_resumes_from_saved_iterate(tmp_path):
    """InitialVolume + StartIteration continue a file-driven run from a written
    iterate: iterations 2 and 3 resumed from recon_1 are bit-identical to an
    uninterrupted run."""
    from recon_b200 import mlem_from_cfg

    cfg = small_cfg(NumProj=8, N_iteration=4)
    folder = write_case(tmp_path, cfg, seed=31)
    full, resumed = os.path.join(folder, "full"), os.path.join(folder, "resumed")
    os.makedirs(full)
    os.makedirs(resumed)
    write_cfg(os.path.join(folder, "full.cfg"), cfg, folder + "/", full + "/")
    mlem_from_cfg(folder + "/", "full.cfg")
    write_cfg(os.path.join(folder, "resume.cfg"), cfg, folder + "/", resumed + "/")
    with open(os.path.join(folder, "resume.cfg"), "a") as fh:
        fh.write(f"InitialVolume = {os.path.join(full, 'recon_1.bin')}\nStartIteration = 2\n")
    mlem_from_cfg(folder + "/", "resume.cfg")
    assert not os.path.exists(os.path.join(resumed, "recon_1.bin"))
    for it in (2, 3):
        a = np.fromfile(os.path.join(full, f"recon_{it}.bin"), np.float32)
        b = np.fromfile(os.path.join(resumed, f"recon_{it}.bin"), np.float32)
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
