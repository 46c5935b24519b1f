"""ctypes binding of ``librecon_b200.so`` (the C ABI in ``include/recon_b200.h``).

The library is loaded from the package directory; if it is missing the import
fails with an error that says how to build it -- there is no fallback path.
"""
from __future__ import annotations

import ctypes as C
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "librecon_b200.so")

RECON_OK = 0
STATUS_NAMES = {
    0: "RECON_OK", 1: "RECON_ERR_INVALID_ARGUMENT", 2: "RECON_ERR_UNSUPPORTED", 3: "RECON_ERR_CUDA",
    4: "RECON_ERR_OUT_OF_MEMORY", 5: "RECON_ERR_FILE_NOT_FOUND", 6: "RECON_ERR_KEY_NOT_FOUND",
    7: "RECON_ERR_SIZE_MISMATCH", 8: "RECON_ERR_IO", 9: "RECON_ERR_NO_DEVICE",
}

ARITH_EXACT, ARITH_COMPAT = 0, 1
SUM_KAHAN, SUM_PLAIN = 0, 1
SINO_F32, SINO_BF16 = 0, 1
BP_SIDDON, BP_VOXEL = 0, 1
VOXEL_REFERENCE, VOXEL_GEOMETRIC = 0, 1
SIDDON_BP_AUTO, SIDDON_BP_GATHER, SIDDON_BP_RAY, SIDDON_BP_TUNED = 0, 1, 2, 3
NOALLOC_MAX_VOXELS = 2097152  # RECON_NOALLOC_MAX_VOXELS
PROJECTOR_FORWARD = 0  # RECON_PROJECTOR_FORWARD
PROJECTOR_BACK = 1  # RECON_PROJECTOR_BACK
FP_RAY_WALK = 0  # RECON_FP_RAY_WALK
FP_COLUMNS = 1  # RECON_FP_COLUMNS
FP_COLUMN_BLOCKS = 2  # RECON_FP_COLUMN_BLOCKS
ABI_VERSION = 4  # RECON_B200_ABI_VERSION: the layout of the structures above


class ReconError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


class Calibration(C.Structure):
    _fields_ = [(n, C.c_float) for n in ("R", "Rf", "Ry", "Dx", "Dz", "xangle", "yangle", "zangle", "M")]


class Detector(C.Structure):
    _fields_ = [("NumTAxPixels", C.c_uint), ("NumAxPixels", C.c_uint), ("TAxPixDimMm", C.c_float),
                ("AxPixDimMm", C.c_float)]


class Volume(C.Structure):
    _fields_ = [("Xdim", C.c_uint), ("Ydim", C.c_uint), ("Zdim", C.c_uint), ("XVoxSize", C.c_float),
                ("YVoxSize", C.c_float), ("ZVoxSize", C.c_float)]


class Scan(C.Structure):
    _fields_ = [("N_iteration", C.c_uint), ("NumProj", C.c_uint), ("DeltaAng", C.c_float)]


class Geometry(C.Structure):
    _fields_ = [("cal", Calibration), ("det", Detector), ("vox", Volume), ("scan", Scan)]


PATH_MAX = 1024
_PATH_KEYS = ["ProjFileFolder", "ProjFileNameRoot", "ProjFileSuffix", "ReconFileFolder", "ReconFileNameRoot",
              "ReconFileSuffix", "ObjFileFolder", "ObjFileName", "BpFileNameRoot", "BpFileSuffix"]


class FilePaths(C.Structure):
    _fields_ = [(k, C.c_char * PATH_MAX) for k in _PATH_KEYS]


class Options(C.Structure):
    _fields_ = [("arith", C.c_int), ("sum", C.c_int), ("sino", C.c_int), ("bp", C.c_int),
                ("voxel_mode", C.c_int), ("device", C.c_int), ("siddon_bp", C.c_int), ("fp_block", C.c_int),
                ("fp_rows", C.c_int)]


_lib = None


def lib() -> C.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise ImportError(f"{LIB_PATH} is missing: build it with `python -m recon_b200.build` "
                          "(or __graft_entry__.build())")
    L = C.CDLL(LIB_PATH)
    P = C.c_void_p
    f = C.c_float
    u = C.c_uint
    st = C.c_int
    fp = C.POINTER(C.c_float)
    up = C.POINTER(C.c_uint)
    ip = C.POINTER(C.c_int)
    sigs = {
        "recon_abi_version": (C.c_int, []),
        "recon_last_error": (C.c_char_p, []),
        "recon_default_options": (st, [C.POINTER(Options)]),
        "recon_geometry_from_cfg": (st, [C.c_char_p, C.POINTER(Geometry), C.POINTER(FilePaths)]),
        "recon_plan_create": (st, [C.POINTER(Geometry), C.POINTER(Options), C.POINTER(P)]),
        "recon_plan_destroy": (None, [P]),
        "recon_plan_device_bytes": (C.c_size_t, [P]),
        "recon_plan_siddon_bp": (st, [P, ip]),
        "recon_plan_forward_projector": (st, [P, C.POINTER(C.c_int)]),
        "recon_plan_mirror_pairs": (st, [P, C.POINTER(C.c_int)]),
        "recon_plan_quarter_turns": (st, [P, C.POINTER(C.c_int)]),
        "recon_plan_column_rows": (st, [P, C.POINTER(C.c_int)]),
        "recon_march_fp_view": (st, [P, P, f, C.c_int, P, P]),
        "recon_fp_view": (st, [P, P, f, P, P]),
        "recon_fp_views": (st, [P, P, u, u, P, P]),
        "recon_bp_view": (st, [P, P, f, P, P]),
        "recon_bp_views": (st, [P, P, u, u, P, P]),
        "recon_sensitivity": (st, [P, P, P]),
        "recon_voxel_bp_view": (st, [P, P, f, u, C.c_int, P, P]),
        "recon_mlem": (st, [P, P, u, P, C.c_int, P]),
        "recon_mlem_prepare": (st, [P, P]),
        "recon_osem": (st, [P, P, u, u, P, C.c_int, P]),
        "recon_mlem_iteration": (st, [P, P, P, P]),
        "recon_upload_sinogram": (st, [P, P, P, u, u, C.POINTER(C.c_size_t), P]),
        "recon_mlem_forward": (st, [P, P, P, u, u, P]),
        "recon_mlem_backward": (st, [P, u, u, P, P]),
        "recon_mlem_update": (st, [P, P, P, P]),
        "recon_mlem_forward_quarters": (st, [P, P, P, u, u, P]),
        "recon_mlem_backward_quarters": (st, [P, u, u, P, P]),
        "recon_mlem_backward_update": (st, [P, P, P]),
        "recon_count_intersections": (st, [P, C.POINTER(C.c_ulonglong)]),
        "recon_count_projector_pairs": (st, [P, C.c_int, C.POINTER(C.c_ulonglong)]),
        "recon_view_step_count": (st, [P, f, up]),
        "recon_set_ones": (st, [P, C.c_size_t, P]),
        "recon_divide1": (st, [P, P, C.c_size_t, P]),
        "recon_multiply1": (st, [P, P, C.c_size_t, P]),
        "recon_add": (st, [P, P, C.c_size_t, P]),
        "recon_compat_setup_view": (st, [P, f, fp, fp, fp, up, fp, fp, fp, fp, fp, up, up]),
        "recon_compat_trace": (st, [P, f, C.c_int, ip, C.c_int, ip, fp, up]),
        "recon_mlem_from_cfg": (st, [C.c_char_p, C.c_char_p, C.POINTER(Options)]),
        "recon_forward_projection_from_cfg": (st, [C.c_char_p, C.c_char_p, C.POINTER(Options)]),
        "recon_backward_projection_from_cfg": (st, [C.c_char_p, C.c_char_p, C.c_int, C.POINTER(Options)]),
        "recon_batch_create": (st, [C.POINTER(Geometry), C.c_int, C.POINTER(Options), C.POINTER(P)]),
        "recon_batch_destroy": (None, [P]),
        "recon_batch_mlem": (st, [P, C.POINTER(P), C.POINTER(P), u, C.c_int, P]),
        "recon_compat_bp_view_noalloc": (st, [C.POINTER(Geometry), P, f, P, P]),
    }
    for name, (res, args) in sigs.items():
        fn = getattr(L, name, None)
        if fn is None:
            continue
        fn.restype = res
        fn.argtypes = args
    _lib = L
    return L


def exported_symbols() -> list[str]:
    """Names of the C ABI functions this binding expects (all of include/recon_b200.h)."""
    return [
        "recon_abi_version", "recon_last_error", "recon_default_options", "recon_geometry_from_cfg",
        "recon_plan_create", "recon_plan_destroy", "recon_plan_device_bytes", "recon_plan_siddon_bp", "recon_plan_forward_projector", "recon_plan_mirror_pairs", "recon_plan_quarter_turns", "recon_plan_column_rows", "recon_fp_view", "recon_fp_views",
        "recon_bp_view", "recon_bp_views", "recon_sensitivity", "recon_voxel_bp_view", "recon_march_fp_view", "recon_mlem",
        "recon_mlem_prepare", "recon_mlem_iteration", "recon_mlem_forward", "recon_mlem_backward",
        "recon_mlem_update", "recon_mlem_forward_quarters", "recon_mlem_backward_quarters", "recon_mlem_backward_update", "recon_count_intersections", "recon_count_projector_pairs", "recon_set_ones", "recon_divide1", "recon_multiply1",
        "recon_add", "recon_compat_setup_view", "recon_compat_trace", "recon_view_step_count", "recon_mlem_from_cfg",
        "recon_forward_projection_from_cfg", "recon_backward_projection_from_cfg", "recon_batch_create",
        "recon_batch_destroy", "recon_batch_mlem", "recon_compat_bp_view_noalloc", "recon_osem",
        "recon_upload_sinogram",
    ]


def check(status: int) -> None:
    if status != RECON_OK:
        msg = lib().recon_last_error()
        raise ReconError(status, msg.decode() if msg else "")
