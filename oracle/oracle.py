"""ctypes wrapper for the checker libraries (test infrastructure only).

Only tests/, ``__graft_entry__.smoke()``, the cpu_baseline / reference legs
of bench.py and oracle/time_ref_gpu.py (a timing of the reference's own GPU
build) import this module.  It loads:

* ``oracle/liboracle.so``        -- the CPU restatement (siddon_oracle.c);
* ``oracle/_ref/libref_cpu.so``  -- the reference's kernels built for the host;
* ``oracle/_ref/libref_gpu.so``  -- the reference's CUDA sources built for sm_100a.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))

_f32p = np.ctypeslib.ndpointer(np.float32, flags="C_CONTIGUOUS")
_f64p = np.ctypeslib.ndpointer(np.float64, flags="C_CONTIGUOUS")
_u32p = np.ctypeslib.ndpointer(np.uint32, flags="C_CONTIGUOUS")
_i32p = np.ctypeslib.ndpointer(np.int32, flags="C_CONTIGUOUS")
_i64p = np.ctypeslib.ndpointer(np.int64, flags="C_CONTIGUOUS")


class Geom(C.Structure):
    """CalibrationParam + Detector + VoxVolParam (CT_Recon/CTSystemElements_HF.h:13-99)."""

    _fields_ = [
        ("R", C.c_float), ("Rf", C.c_float), ("Ry", C.c_float), ("Dx", C.c_float),
        ("Dz", C.c_float), ("xangle", C.c_float), ("yangle", C.c_float),
        ("zangle", C.c_float), ("M", C.c_float),
        ("NumTAxPixels", C.c_uint), ("NumAxPixels", C.c_uint),
        ("TAxPixDimMm", C.c_float), ("AxPixDimMm", C.c_float),
        ("Xdim", C.c_uint), ("Ydim", C.c_uint), ("Zdim", C.c_uint),
        ("XVoxSize", C.c_float), ("YVoxSize", C.c_float), ("ZVoxSize", C.c_float),
    ]

    @classmethod
    def from_dict(cls, d: dict) -> "Geom":
        g = cls()
        for name, _ in cls._fields_:
            setattr(g, name, d[name])
        return g

    @property
    def npix(self) -> int:
        return int(self.NumAxPixels) * int(self.NumTAxPixels)

    @property
    def nvox(self) -> int:
        return int(self.Xdim) * int(self.Ydim) * int(self.Zdim)


class XRay(C.Structure):
    _fields_ = [("p1", C.c_double * 3), ("p2", C.c_double * 3), ("d12", C.c_double)]


_GP = C.POINTER(Geom)
_lib = None
_ref_cpu = None
_ref_gpu = None


def lib():
    global _lib
    if _lib is None:
        path = os.path.join(HERE, "liboracle.so")
        if not os.path.exists(path):
            from oracle.build_oracle import build_oracle  # noqa: WPS433

            build_oracle()
        L = C.CDLL(path)
        L.orc_rotation_matrix.argtypes = [C.c_float, C.c_float, C.c_float, _f32p]
        L.orc_c_set_device_model.argtypes = [C.c_int]
        L.orc_c_pixel_iterate2.argtypes = [C.c_float, C.c_float, C.c_float, C.c_int]
        L.orc_c_pixel_iterate2.restype = C.c_float
        L.orc_c_setup_view.argtypes = [_GP, _f32p, C.c_float] + [_f32p] * 3 + [_u32p] + [_f32p] * 5 + [_u32p]
        L.orc_c_setup_view.restype = C.c_uint32
        L.orc_c_loopN.argtypes = [_GP, _f32p, C.c_float]
        L.orc_c_loopN.restype = C.c_uint32
        L.orc_c_trace.argtypes = [_GP, _f32p, C.c_float, C.c_int, C.c_int, C.c_uint32, _i32p, _f32p, C.c_int]
        L.orc_c_trace.restype = C.c_int
        L.orc_c_fp_view.argtypes = [_GP, _f32p, C.c_float, _f32p, _f32p]
        L.orc_c_bp_view.argtypes = [_GP, _f32p, C.c_float, _f32p, _f32p]
        L.orc_c_mlem.argtypes = [_GP, C.c_uint, C.c_float, _f32p, C.c_uint, _f32p, _f32p, C.c_void_p]
        L.orc_x_ray_geom.argtypes = [_GP, C.c_float, C.c_int, C.c_int, C.POINTER(XRay)]
        L.orc_x_trace.argtypes = [_GP, C.c_float, C.c_int, C.c_int, _i64p, _f64p, C.c_int]
        L.orc_x_trace.restype = C.c_int
        L.orc_x_fp_view.argtypes = [_GP, C.c_float, _f64p, _f64p]
        L.orc_x_fp_all.argtypes = [_GP, C.c_uint, C.c_float, _f64p, _f64p, C.c_int]
        L.orc_x_bp_all.argtypes = [_GP, C.c_uint, C.c_float, _f64p, _f64p, C.c_int]
        L.orc_x_mlem.argtypes = [_GP, C.c_uint, C.c_float, _f32p, C.c_uint, _f64p, C.c_void_p, C.c_int]
        L.orc_x_osem.argtypes = [_GP, C.c_uint, C.c_float, _f32p, C.c_uint, C.c_uint, _f64p, C.c_int]
        L.orc_x_osem.restype = C.c_int
        L.orc_x_slab_update.argtypes = [_GP, C.c_uint, C.c_float, _f32p, _f32p, C.c_uint, C.c_uint, _f64p, C.c_int]
        L.orc_x_slab_update.restype = C.c_int
        L.orc_x_count_isects.argtypes = [_GP, C.c_uint, C.c_float, C.c_int]
        L.orc_x_count_isects.restype = C.c_int64
        L.orc_x_voxel_column.argtypes = [_GP, C.c_uint, C.c_float, C.c_int64, _i32p, _i32p, _f64p, C.c_int]
        L.orc_x_voxel_column.restype = C.c_int
        L.orc_v_bp_view.argtypes = [_GP, _f32p, C.c_float, _f32p, C.c_uint, C.c_int, _f32p]
        L.orc_m_fp_view.argtypes = [_GP, _f32p, C.c_float, C.c_int, _f32p, _f64p]
        _lib = L
    return _lib


def ref_cpu():
    """The reference's kernels compiled for the host, or None if not built."""
    global _ref_cpu
    if _ref_cpu is None:
        path = os.path.join(HERE, "_ref", "libref_cpu.so")
        if not os.path.exists(path):
            return None
        L = C.CDLL(path)
        L.ref_cpu_set_threads.argtypes = [C.c_int]
        L.ref_cpu_setup.argtypes = [_GP, C.c_float] + [_f32p] * 3 + [_u32p] + [_f32p] * 5 + [_u32p]
        L.ref_cpu_setup.restype = C.c_uint
        L.ref_cpu_fp_view.argtypes = [_GP, C.c_float, C.c_uint, _f32p, _f32p]
        L.ref_cpu_bp_view.argtypes = [_GP, C.c_float, C.c_uint, _f32p, _f32p]
        L.ref_cpu_trace.argtypes = [_GP, C.c_float, C.c_uint, C.c_int, _i32p, _i32p, _f32p]
        L.ref_cpu_mlem.argtypes = [_GP, C.c_uint, C.c_float, _u32p, _f32p, C.c_uint, _f32p, _f32p, C.c_void_p]
        L.ref_cpu_mlem_view.argtypes = [_GP, C.c_float, C.c_uint, _f32p, _f32p, _f32p]
        L.ref_cpu_mlem_view_steps.argtypes = [_GP, C.c_float, C.c_uint, _f32p, _f32p, _f32p]
        _ref_cpu = L
    return _ref_cpu


def ref_gpu():
    """The reference's CUDA sources built for sm_100a, or None if not built."""
    global _ref_gpu
    if _ref_gpu is None:
        path = os.path.join(HERE, "_ref", "libref_gpu.so")
        if not os.path.exists(path):
            return None
        L = C.CDLL(path)
        L.ref_gpu_setup.argtypes = [_GP, C.c_float] + [_f32p] * 3 + [_u32p] + [_f32p] * 5 + [_u32p]
        L.ref_gpu_setup.restype = C.c_uint
        L.ref_gpu_fp_view.argtypes = [_GP, C.c_float, _f32p, _f32p]
        L.ref_gpu_fp_view.restype = C.c_uint
        L.ref_gpu_bp_view.argtypes = [_GP, C.c_float, _f32p, _f32p]
        L.ref_gpu_bp_view.restype = C.c_uint
        L.ref_gpu_trace.argtypes = [_GP, C.c_float, C.c_int, _i32p, C.c_int, _i32p, _f32p]
        L.ref_gpu_trace.restype = C.c_uint
        L.ref_gpu_mlem_cfg.argtypes = [C.c_char_p, C.c_char_p]
        L.ref_gpu_mlem_cfg.restype = C.c_float
        L.ref_gpu_forward_projection_cfg.argtypes = [C.c_char_p, C.c_char_p]
        if hasattr(L, "ref_gpu_backward_projection_cfg"):
            L.ref_gpu_backward_projection_cfg.argtypes = [C.c_char_p, C.c_char_p, C.c_int]
        L.ref_gpu_voxel_bp2_view.argtypes = [_GP, C.c_float, _f32p, C.c_uint, _f32p]
        if hasattr(L, "ref_gpu_march_fp_view"):
            L.ref_gpu_march_fp_view.argtypes = [_GP, C.c_float, _f32p, _f32p]
        _ref_gpu = L
    return _ref_gpu


# ---------------------------------------------------------------------------
# convenience wrappers
# ---------------------------------------------------------------------------

def rotation_matrix(g: Geom) -> np.ndarray:
    RM = np.zeros(9, np.float32)
    lib().orc_rotation_matrix(g.xangle, g.yangle, g.zangle, RM)
    return RM


def _setup_arrays(n: int) -> dict:
    return {
        "alpha_min": np.zeros(n, np.float32), "alpha_max": np.zeros(n, np.float32),
        "d12": np.zeros(n, np.float32), "mask": np.zeros(n, np.uint32),
        "alpha_i": np.zeros(3 * n, np.float32), "alpha_f": np.zeros(3 * n, np.float32),
        "delta_alpha": np.zeros(3 * n, np.float32), "p1": np.zeros(3 * n, np.float32),
        "p2": np.zeros(3 * n, np.float32), "delta_index": np.zeros(n, np.uint32),
    }


_SETUP_ORDER = ["alpha_min", "alpha_max", "d12", "mask", "alpha_i", "alpha_f", "delta_alpha",
                "p1", "p2", "delta_index"]


def c_setup_view(g: Geom, angle: float) -> tuple[int, dict]:
    a = _setup_arrays(g.npix)
    loopN = lib().orc_c_setup_view(C.byref(g), rotation_matrix(g), angle, *[a[k] for k in _SETUP_ORDER])
    return int(loopN), a


def ref_cpu_setup_view(g: Geom, angle: float) -> tuple[int, dict]:
    a = _setup_arrays(g.npix)
    loopN = ref_cpu().ref_cpu_setup(C.byref(g), angle, *[a[k] for k in _SETUP_ORDER])
    return int(loopN), a


def ref_gpu_setup_view(g: Geom, angle: float) -> tuple[int, dict]:
    a = _setup_arrays(g.npix)
    loopN = ref_gpu().ref_gpu_setup(C.byref(g), angle, *[a[k] for k in _SETUP_ORDER])
    return int(loopN), a


def c_loopN(g: Geom, angle: float) -> int:
    return int(lib().orc_c_loopN(C.byref(g), rotation_matrix(g), angle))


def c_fp_view(g: Geom, angle: float, vol: np.ndarray) -> np.ndarray:
    img = np.zeros(g.npix, np.float32)
    lib().orc_c_fp_view(C.byref(g), rotation_matrix(g), angle, np.ascontiguousarray(vol, np.float32).ravel(), img)
    return img


def c_bp_view(g: Geom, angle: float, img: np.ndarray) -> np.ndarray:
    vol = np.zeros(g.nvox, np.float32)
    lib().orc_c_bp_view(C.byref(g), rotation_matrix(g), angle, np.ascontiguousarray(img, np.float32).ravel(), vol)
    return vol


def c_trace(g: Geom, angle: float, u: int, v: int, loopN: int | None = None):
    if loopN is None:
        loopN = c_loopN(g, angle)
    cap = loopN + 2
    idx = np.zeros(cap, np.int32)
    ln = np.zeros(cap, np.float32)
    n = lib().orc_c_trace(C.byref(g), rotation_matrix(g), angle, u, v, loopN, idx, ln, cap)
    assert n >= 0
    return idx[:n], ln[:n]


def c_mlem(g: Geom, nproj: int, dang: float, sino: np.ndarray, iters: int, history: bool = False):
    f = np.zeros(g.nvox, np.float32)
    sens = np.zeros(g.nvox, np.float32)
    hist = np.zeros(iters * g.nvox, np.float32) if history else None
    lib().orc_c_mlem(C.byref(g), nproj, dang, np.ascontiguousarray(sino, np.float32).ravel(), iters, f, sens,
                     hist.ctypes.data_as(C.c_void_p) if hist is not None else None)
    return f, sens, (hist.reshape(iters, -1) if hist is not None else None)


def x_ray(g: Geom, angle: float, u: int, v: int) -> XRay:
    r = XRay()
    lib().orc_x_ray_geom(C.byref(g), angle, u, v, C.byref(r))
    return r


def x_trace(g: Geom, angle: float, u: int, v: int, cap: int = 4096):
    idx = np.zeros(cap, np.int64)
    ln = np.zeros(cap, np.float64)
    n = lib().orc_x_trace(C.byref(g), angle, u, v, idx, ln, cap)
    assert n >= 0
    return idx[:n], ln[:n]


def x_fp_all(g: Geom, nproj: int, dang: float, vol: np.ndarray, threads: int = 0) -> np.ndarray:
    sino = np.zeros(nproj * g.npix, np.float64)
    lib().orc_x_fp_all(C.byref(g), nproj, dang, np.ascontiguousarray(vol, np.float64).ravel(), sino, threads)
    return sino


def x_bp_all(g: Geom, nproj: int, dang: float, sino: np.ndarray, threads: int = 0) -> np.ndarray:
    vol = np.zeros(g.nvox, np.float64)
    lib().orc_x_bp_all(C.byref(g), nproj, dang, np.ascontiguousarray(sino, np.float64).ravel(), vol, threads)
    return vol


def x_mlem(g: Geom, nproj: int, dang: float, sino: np.ndarray, iters: int, threads: int = 0):
    f = np.zeros(g.nvox, np.float64)
    sens = np.zeros(g.nvox, np.float64)
    lib().orc_x_mlem(C.byref(g), nproj, dang, np.ascontiguousarray(sino, np.float32).ravel(), iters, f,
                     sens.ctypes.data_as(C.c_void_p), threads)
    return f, sens


def x_osem(g: Geom, nproj: int, dang: float, sino: np.ndarray, iters: int, subsets: int, threads: int = 0):
    """FP64 OSEM, contiguous subsets (orc_x_osem)."""
    f = np.zeros(g.nvox, np.float64)
    rc = lib().orc_x_osem(C.byref(g), nproj, dang, np.ascontiguousarray(sino, np.float32).ravel(), iters, subsets,
                          f, threads)
    if rc != 0:
        raise ValueError(f"{subsets} subsets do not divide {nproj} views")
    return f


def x_slab_update(g: Geom, nproj: int, dang: float, f: np.ndarray, sino: np.ndarray, z0: int, z1: int,
                  threads: int = 0) -> np.ndarray:
    """FP64 MLEM update of the slab z in [z0, z1) from an FP32 image (orc_x_slab_update)."""
    out = np.zeros((z1 - z0) * g.Xdim * g.Ydim, np.float64)
    rc = lib().orc_x_slab_update(C.byref(g), nproj, dang, np.ascontiguousarray(f, np.float32).ravel(),
                                 np.ascontiguousarray(sino, np.float32).ravel(), z0, z1, out, threads)
    if rc != 0:
        raise ValueError("bad slab or out of memory")
    return out


def x_count_isects(g: Geom, nproj: int, dang: float, threads: int = 0) -> int:
    return int(lib().orc_x_count_isects(C.byref(g), nproj, dang, threads))


def x_voxel_column(g: Geom, nproj: int, dang: float, voxel: int, cap: int = 1 << 16):
    view = np.zeros(cap, np.int32)
    pix = np.zeros(cap, np.int32)
    ln = np.zeros(cap, np.float64)
    n = lib().orc_x_voxel_column(C.byref(g), nproj, dang, voxel, view, pix, ln, cap)
    assert n >= 0
    return view[:n], pix[:n], ln[:n]


def v_bp_view(g: Geom, angle: float, img: np.ndarray, nproj: int, mode: int, vol=None) -> np.ndarray:
    out = np.zeros(g.nvox, np.float32) if vol is None else np.ascontiguousarray(vol, np.float32).copy()
    lib().orc_v_bp_view(C.byref(g), rotation_matrix(g), angle, np.ascontiguousarray(img, np.float32).ravel(),
                        nproj, mode, out)
    return out


def m_fp_view(g: Geom, angle: float, mode: int, vol: np.ndarray) -> np.ndarray:
    """Ray-marching forward projection of one view (plane samples), FP64."""
    out = np.zeros(g.npix, np.float64)
    lib().orc_m_fp_view(C.byref(g), rotation_matrix(g), angle, mode, np.ascontiguousarray(vol, np.float32).ravel(),
                        out)
    return out
