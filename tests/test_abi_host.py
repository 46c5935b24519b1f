"""C ABI and host logic, no GPU needed: the library loads and exports every
function include/recon_b200.h declares; options, configuration parsing and the
drivers' host-side failure paths behave as specified (status codes, never an
exit or a prompt)."""
import ctypes as C
import os
import re

import numpy as np
import pytest

from conftest import ROOT, have_gpu, small_cfg
from recon_b200 import _lib as L
from recon_b200.api import geometry, geometry_from_cfg
from tests_helpers import write_cfg


def header_functions():
    names = set()
    for h in os.listdir(os.path.join(ROOT, "include")):
        if not h.endswith(".h"):
            continue
        txt = open(os.path.join(ROOT, "include", h)).read()
        txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
        names |= set(re.findall(r"^\s*(?:recon_status_t|void|int|size_t|const char\*)\s+(recon_[a-z0-9_]+)\s*\(",
                                txt, flags=re.M))
    return sorted(names)


def test_exports_every_declared_function():
    lib = L.lib()
    declared = header_functions()
    assert len(declared) >= 20
    for name in declared:
        assert hasattr(lib, name), name
    assert sorted(L.exported_symbols()) == declared
    assert lib.recon_abi_version() == L.ABI_VERSION
    header = open(os.path.join(ROOT, "include", "recon_b200.h")).read()
    assert f"#define RECON_B200_ABI_VERSION {L.ABI_VERSION}\n" in header


def test_default_options():
    o = L.Options()
    assert L.lib().recon_default_options(C.byref(o)) == 0
    assert (o.arith, o.sum, o.sino, o.bp, o.voxel_mode, o.device, o.siddon_bp, o.fp_block, o.fp_rows) == (
        L.ARITH_EXACT, L.SUM_KAHAN, L.SINO_F32, L.BP_SIDDON, L.VOXEL_GEOMETRIC, 0, L.SIDDON_BP_AUTO, 0, 0)


def _cfg_text(extra=""):
    return """
################################
#### Calibration Parameters ####
################################
R   = 1105.7000   # millimeters, source to detector
Rf  = 907.45      # source to rotation axis
Ry  = 1105.7
Dx  = 0.25
Dz  = -0.5
xangle = 0.0
yangle = 0.0
zangle = 0.0
M   = 13.1024

TAxPixels = 512   # rows
AxPixels  = 1024  # columns
TAxPixDim = 0.0065
AxPixDim  = 0.0065

Xdim = 64
Ydim = 64
Zdim = 32
XVoxSize = 0.2
YVoxSize = 0.2
ZVoxSize = 0.25

N_iteration = 2
NumProj  = 180
DeltaAng = 2.0000

ProjFileFolder   = H:\\data\\sim
ProjFileNameRoot = fp_phantom
ProjFileSuffix   = .bin
ReconFileFolder  = out/
ReconFileNameRoot = recon_fp
ReconFileSuffix  = .bin
ObjFileFolder = objs
ObjFileName = phantom.bin
BpFileNameRoot = bp
BpFileSuffix = .bin
""" + extra


def test_cfg_parser_values(tmp_path):
    p = tmp_path / "a.cfg"
    p.write_text(_cfg_text())
    g, paths = geometry_from_cfg(str(p))
    assert g["R"] == np.float32(1105.7) and g["Rf"] == np.float32(907.45) and g["Dz"] == np.float32(-0.5)
    assert (g["AxPixels"], g["TAxPixels"], g["Xdim"], g["Zdim"]) == (1024, 512, 64, 32)
    assert g["NumProj"] == 180 and g["DeltaAng"] == 2.0 and g["N_iteration"] == 2
    assert paths["ProjFileFolder"] == "H:\\data\\sim"  # raw value; folders are corrected by the drivers
    assert paths["ReconFileNameRoot"] == "recon_fp"


def test_cfg_parser_overwrite_comment_continuation_sentry(tmp_path):
    p = tmp_path / "b.cfg"
    p.write_text(_cfg_text("Xdim = 96   # later key wins\nObjFileName = part1\n  part2   # continues\n\n"
                           "EndConfigFile\nYdim = 7\n"))
    g, paths = geometry_from_cfg(str(p))
    assert g["Xdim"] == 96
    assert g["Ydim"] == 64  # after the sentry nothing is read
    assert paths["ObjFileName"] == "part1\n  part2"


def test_cfg_missing_key_and_file(tmp_path):
    p = tmp_path / "c.cfg"
    p.write_text(_cfg_text().replace("NumProj  = 180", ""))
    with pytest.raises(L.ReconError) as e:
        geometry_from_cfg(str(p))
    assert e.value.status == 6 and "NumProj" in str(e.value)
    with pytest.raises(L.ReconError) as e:
        geometry_from_cfg(str(tmp_path / "nope.cfg"))
    assert e.value.status == 5
    p.write_text(_cfg_text().replace("Xdim = 64", "Xdim = sixty"))
    with pytest.raises(L.ReconError) as e:
        geometry_from_cfg(str(p))
    assert e.value.status == 1


def test_plan_rejects_bad_geometry():
    lib = L.lib()
    h = C.c_void_p()
    for bad in (dict(Xdim=0), dict(AxPixDim=-1.0), dict(R=float("nan")), dict(AxPixels=1)):
        g = geometry(small_cfg(**bad))
        st = lib.recon_plan_create(C.byref(g), None, C.byref(h))
        assert st == 1, bad
        assert lib.recon_last_error()
    # exact arithmetic needs an untilted detector and source / detector outside the volume
    o = L.Options(0, 0, 0, 0, 1, 0)
    assert lib.recon_plan_create(C.byref(geometry(small_cfg(yangle=0.01))), C.byref(o), C.byref(h)) == 2
    assert lib.recon_plan_create(C.byref(geometry(small_cfg(Rf=10.0))), C.byref(o), C.byref(h)) == 2
    o.arith = 7
    assert lib.recon_plan_create(C.byref(geometry(small_cfg())), C.byref(o), C.byref(h)) == 1
    o.arith, o.siddon_bp = 0, 4  # 0..3 are AUTO, GATHER, RAY, TUNED
    assert lib.recon_plan_create(C.byref(geometry(small_cfg())), C.byref(o), C.byref(h)) == 1
    o.siddon_bp = 0
    for bad_block in (-2, 3):  # -1 = never, 0 = AUTO; 3 gives 11 x 11 > 64 blocks of the 32 x 32 columns
        o.fp_block = bad_block
        assert lib.recon_plan_create(C.byref(geometry(small_cfg())), C.byref(o), C.byref(h)) == 1, bad_block
        assert "fp_block" in lib.recon_last_error().decode()
    o.fp_block = 0
    for bad_rows in (-32, 16, 96, 256):
        o.fp_rows = bad_rows
        assert lib.recon_plan_create(C.byref(geometry(small_cfg())), C.byref(o), C.byref(h)) == 1, bad_rows
        assert "fp_rows" in lib.recon_last_error().decode()


@pytest.mark.skipif(have_gpu(), reason="checks the no-device path")
def test_plan_without_device_reports_no_device():
    h = C.c_void_p()
    st = L.lib().recon_plan_create(C.byref(geometry(small_cfg())), None, C.byref(h))
    assert st == 9 and not h.value


def test_drivers_fail_on_host_before_any_gpu_work(tmp_path):
    cfg = small_cfg(NumProj=4, N_iteration=1)
    folder = str(tmp_path)
    write_cfg(os.path.join(folder, "r.cfg"), cfg, folder, folder + "/out/")
    lib = L.lib()
    # missing projection files: check_projection_files
    st = lib.recon_mlem_from_cfg(folder.encode(), b"r.cfg", None)
    assert st == 5 and b"proj_0.bin" in lib.recon_last_error()
    npix = cfg["AxPixels"] * cfg["TAxPixels"]
    for n in range(4):
        np.zeros(npix, np.float32).tofile(os.path.join(folder, f"proj_{n}.bin"))
    np.zeros(npix - 1, np.float32).tofile(os.path.join(folder, "proj_2.bin"))  # short file
    st = lib.recon_mlem_from_cfg(folder.encode(), b"r.cfg", None)
    assert st == 7 and b"proj_2.bin" in lib.recon_last_error()
    st = lib.recon_backward_projection_from_cfg(folder.encode(), b"r.cfg", 0, None)
    assert st == 7
    # forward projection: missing / wrong-size object file
    st = lib.recon_forward_projection_from_cfg(folder.encode(), b"r.cfg", None)
    assert st == 5
    np.zeros(10, np.float32).tofile(os.path.join(folder, "object.bin"))
    write_cfg(os.path.join(folder, "r.cfg"), cfg, folder, folder + "/out/", obj_folder=folder)
    st = lib.recon_forward_projection_from_cfg(folder.encode(), b"r.cfg", None)
    assert st == 7
    # missing configuration
    assert lib.recon_mlem_from_cfg(folder.encode(), b"missing.cfg", None) == 5


def test_elementwise_argument_checks():
    lib = L.lib()
    assert lib.recon_set_ones(None, 0, None) == 0
    assert lib.recon_set_ones(None, 5, None) == 1
    assert lib.recon_divide1(None, None, 3, None) == 1


def test_plan_queries_reject_null():
    """The plan queries refuse a NULL plan or output before touching either."""
    lib = L.lib()
    out = C.c_int(-7)
    for name in ("recon_plan_siddon_bp", "recon_plan_forward_projector", "recon_plan_mirror_pairs",
                 "recon_plan_quarter_turns", "recon_plan_column_rows"):
        fn = getattr(lib, name)
        assert fn(None, C.byref(out)) == 1, name
        assert out.value == -7, name
