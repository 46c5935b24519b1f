"""Python face of the C ABI, over torch CUDA tensors.

The calls mirror the reference's projector / recon surface
(CT_Recon/hf_siddon_class.hpp, hf_siddon_recon.hpp): a :class:`Plan` plays
``siddon_commons`` + ``forward`` + ``backward``; :func:`mlem_from_cfg` is
``siddon_recon::a0_RECON_MLEM``.  Every tensor argument must be a contiguous
float32 (or bfloat16 for BF16 sinograms) CUDA tensor on the plan's device;
work is queued on torch's current stream.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass

import numpy as np

from . import _lib as L
from ._lib import check, lib


@dataclass
class Options:
    arith: int = L.ARITH_EXACT
    sum: int = L.SUM_KAHAN
    sino: int = L.SINO_F32
    bp: int = L.BP_SIDDON
    voxel_mode: int = L.VOXEL_GEOMETRIC
    device: int = 0
    siddon_bp: int = L.SIDDON_BP_AUTO
    fp_block: int = 0
    fp_rows: int = 0

    def c(self) -> L.Options:
        return L.Options(self.arith, self.sum, self.sino, self.bp, self.voxel_mode, self.device, self.siddon_bp,
                         self.fp_block, self.fp_rows)


def geometry(cfg: dict) -> L.Geometry:
    """C geometry from a dict with the reference configuration keys
    (R, Rf, Ry, Dx, Dz, xangle, yangle, zangle, M, TAxPixels, AxPixels,
    TAxPixDim, AxPixDim, Xdim..ZVoxSize, N_iteration, NumProj, DeltaAng)."""
    g = L.Geometry()
    for k in ("R", "Rf", "Ry", "Dx", "Dz", "xangle", "yangle", "zangle", "M"):
        setattr(g.cal, k, float(cfg[k]))
    g.det.NumTAxPixels = int(cfg["TAxPixels"])
    g.det.NumAxPixels = int(cfg["AxPixels"])
    g.det.TAxPixDimMm = float(cfg["TAxPixDim"])
    g.det.AxPixDimMm = float(cfg["AxPixDim"])
    for k in ("Xdim", "Ydim", "Zdim"):
        setattr(g.vox, k, int(cfg[k]))
    for k in ("XVoxSize", "YVoxSize", "ZVoxSize"):
        setattr(g.vox, k, float(cfg[k]))
    g.scan.N_iteration = int(cfg.get("N_iteration", 0))
    g.scan.NumProj = int(cfg.get("NumProj", 0))
    g.scan.DeltaAng = float(cfg.get("DeltaAng", 0.0))
    return g


def geometry_from_cfg(path: str) -> tuple[dict, dict]:
    """Parse a reference-format configuration file with the library's parser.

    Returns (geometry dict, file paths dict)."""
    g = L.Geometry()
    p = L.FilePaths()
    check(lib().recon_geometry_from_cfg(path.encode(), C.byref(g), C.byref(p)))
    d = dict(R=g.cal.R, Rf=g.cal.Rf, Ry=g.cal.Ry, Dx=g.cal.Dx, Dz=g.cal.Dz, xangle=g.cal.xangle,
             yangle=g.cal.yangle, zangle=g.cal.zangle, M=g.cal.M, TAxPixels=g.det.NumTAxPixels,
             AxPixels=g.det.NumAxPixels, TAxPixDim=g.det.TAxPixDimMm, AxPixDim=g.det.AxPixDimMm,
             Xdim=g.vox.Xdim, Ydim=g.vox.Ydim, Zdim=g.vox.Zdim, XVoxSize=g.vox.XVoxSize,
             YVoxSize=g.vox.YVoxSize, ZVoxSize=g.vox.ZVoxSize, N_iteration=g.scan.N_iteration,
             NumProj=g.scan.NumProj, DeltaAng=g.scan.DeltaAng)
    paths = {k: getattr(p, k).decode() for k, _ in L.FilePaths._fields_}
    return d, paths


def _ptr(t) -> int:
    import torch

    if not isinstance(t, torch.Tensor):
        raise TypeError("expected a torch tensor")
    if not t.is_cuda:
        raise ValueError("tensor must live on a CUDA device")
    if not t.is_contiguous():
        raise ValueError("tensor must be contiguous")
    return t.data_ptr()


def _stream() -> int:
    import torch

    return torch.cuda.current_stream().cuda_stream


class Plan:
    """siddon_commons + forward + backward (hf_siddon_class.hpp:18-368) for one geometry."""

    def __init__(self, cfg: dict, options: Options | None = None):
        self.cfg = dict(cfg)
        self.options = options or Options()
        self._geom = geometry(cfg)
        h = C.c_void_p()
        check(lib().recon_plan_create(C.byref(self._geom), C.byref(self.options.c()), C.byref(h)))
        self._h = h
        self.nu = int(cfg["AxPixels"])
        self.nv = int(cfg["TAxPixels"])
        self.shape_vol = (int(cfg["Zdim"]), int(cfg["Ydim"]), int(cfg["Xdim"]))
        self.nproj = int(cfg.get("NumProj", 0))
        self.dang = np.float32(cfg.get("DeltaAng", 0.0))

    def close(self) -> None:
        if getattr(self, "_h", None):
            lib().recon_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self) -> C.c_void_p:
        return self._h

    def angle(self, n: int) -> float:
        return float(np.float32(n) * self.dang)

    @property
    def device_bytes(self) -> int:
        return int(lib().recon_plan_device_bytes(self._h))

    @property
    def siddon_bp(self) -> int:
        """The Siddon back projector of an EXACT plan: SIDDON_BP_GATHER or SIDDON_BP_RAY."""
        d = C.c_int(-1)
        check(lib().recon_plan_siddon_bp(self._h, C.byref(d)))
        return int(d.value)

    @property
    def column_rows(self) -> int:
        """recon_plan_column_rows: detector rows per CTA of the column forward projector (0: another)."""
        d = C.c_int()
        check(lib().recon_plan_column_rows(self._h, C.byref(d)))
        return int(d.value)

    @property
    def mirror_pairs(self) -> bool:
        """True when the EXACT projectors pair rows / voxels mirrored about z = 0."""
        d = C.c_int(0)
        check(lib().recon_plan_mirror_pairs(self._h, C.byref(d)))
        return bool(d.value)

    @property
    def quarter_turns(self) -> bool:
        """True when an EXACT plan's views come in exact quarter turns about a square volume."""
        return self._quarter_level() >= 1

    @property
    def quarter_sets(self) -> bool:
        """True when the MLEM back projection also takes quarter sets of views
        (recon_mlem_backward_quarters): recon_plan_quarter_turns reports 2."""
        return self._quarter_level() == 2

    def _quarter_level(self) -> int:
        d = C.c_int(0)
        check(lib().recon_plan_quarter_turns(self._h, C.byref(d)))
        return int(d.value)

    @property
    def forward_projector(self) -> int:
        """The forward projector of an EXACT plan: FP_COLUMNS or FP_RAY_WALK."""
        d = C.c_int(-1)
        check(lib().recon_plan_forward_projector(self._h, C.byref(d)))
        return int(d.value)

    # --- tensors ---
    def new_volume(self, fill: float = 0.0):
        import torch

        return torch.full(self.shape_vol, fill, dtype=torch.float32, device=f"cuda:{self.options.device}")

    def new_sinogram(self, views: int | None = None, dtype=None):
        import torch

        v = self.nproj if views is None else views
        return torch.zeros((v, self.nv, self.nu), dtype=dtype or torch.float32, device=f"cuda:{self.options.device}")

    # --- projectors ---
    def fp_view(self, vol, angle: float, out=None):
        out = self.new_sinogram(1)[0] if out is None else out
        check(lib().recon_fp_view(self._h, _ptr(vol), float(angle), _ptr(out), _stream()))
        return out

    def fp_views(self, vol, first: int = 0, count: int | None = None, out=None):
        count = self.nproj - first if count is None else count
        out = self.new_sinogram(count) if out is None else out
        check(lib().recon_fp_views(self._h, _ptr(vol), first, count, _ptr(out), _stream()))
        return out

    def bp_view(self, img, angle: float, out=None):
        out = self.new_volume() if out is None else out
        check(lib().recon_bp_view(self._h, _ptr(img), float(angle), _ptr(out), _stream()))
        return out

    def bp_views(self, sino, first: int = 0, count: int | None = None, out=None):
        count = self.nproj - first if count is None else count
        out = self.new_volume() if out is None else out
        check(lib().recon_bp_views(self._h, _ptr(sino), first, count, _ptr(out), _stream()))
        return out

    def sensitivity(self, out=None):
        out = self.new_volume() if out is None else out
        check(lib().recon_sensitivity(self._h, _ptr(out), _stream()))
        return out

    def voxel_bp_view(self, img, angle: float, nproj: int, mode: int, accum=None):
        accum = self.new_volume() if accum is None else accum
        check(lib().recon_voxel_bp_view(self._h, _ptr(img), float(angle), int(nproj), int(mode), _ptr(accum),
                                        _stream()))
        return accum

    def march_fp_view(self, vol, angle: float, mode: int, out=None):
        """Ray-marching forward projection of one view (plane samples; see recon_march_fp_view)."""
        out = self.new_sinogram(1)[0] if out is None else out
        check(lib().recon_march_fp_view(self._h, _ptr(vol), float(angle), int(mode), _ptr(out), _stream()))
        return out

    # --- MLEM ---
    def mlem(self, g, iters: int, f=None, init_ones: bool = True):
        f = self.new_volume() if f is None else f
        check(lib().recon_mlem(self._h, _ptr(g), int(iters), _ptr(f), 1 if init_ones else 0, _stream()))
        return f

    def osem(self, g, iters: int, subsets: int, f=None, init_ones: bool = True):
        """recon_osem: `iters` passes over `subsets` contiguous view subsets."""
        f = self.new_volume() if f is None else f
        check(lib().recon_osem(self._h, _ptr(g), int(iters), int(subsets), _ptr(f), 1 if init_ones else 0,
                               _stream()))
        return f

    def mlem_prepare(self) -> None:
        check(lib().recon_mlem_prepare(self._h, _stream()))

    def mlem_iteration(self, g, f) -> None:
        check(lib().recon_mlem_iteration(self._h, _ptr(g), _ptr(f), _stream()))

    def upload_sinogram(self, g_host, g_dev, first: int = 0, count: int | None = None) -> int:
        """recon_upload_sinogram: views [first, first + count) of the host sinogram
        g_host into g_dev (both [NumProj][TAxPixels][AxPixels] in the plan's
        sinogram type), only the rows the plan's rays can read; returns the
        bytes copied.  Asynchronous on the current stream."""
        count = self.nproj - first if count is None else count
        if g_host.is_cuda or not g_dev.is_cuda:
            raise ValueError("g_host must be in host memory and g_dev on the device")
        if tuple(g_host.shape) != (self.nproj, self.nv, self.nu) or g_dev.shape != g_host.shape:
            raise ValueError("g_host and g_dev must both be [NumProj][TAxPixels][AxPixels]")
        es = 2 if self.options.sino == L.SINO_BF16 else 4
        if g_host.dtype != g_dev.dtype or g_host.element_size() != es:
            raise ValueError("g_host and g_dev must both have the plan's sinogram type")
        if not g_host.is_contiguous():
            raise ValueError("g_host must be contiguous")
        n = C.c_size_t()
        check(lib().recon_upload_sinogram(self._h, g_host.data_ptr(), _ptr(g_dev), first, count, C.byref(n),
                                          _stream()))
        return int(n.value)

    def mlem_forward(self, g, f, first: int = 0, count: int | None = None) -> None:
        count = self.nproj - first if count is None else count
        check(lib().recon_mlem_forward(self._h, _ptr(g), _ptr(f), first, count, _stream()))

    def mlem_backward(self, ht, first: int = 0, count: int | None = None) -> None:
        count = self.nproj - first if count is None else count
        check(lib().recon_mlem_backward(self._h, first, count, _ptr(ht), _stream()))

    def mlem_forward_quarters(self, g, f, first: int, count: int) -> None:
        """recon_mlem_forward_quarters: the ratio of base views first .. first+count-1 of each quarter."""
        check(lib().recon_mlem_forward_quarters(self._h, _ptr(g), _ptr(f), first, count, _stream()))

    def mlem_backward_quarters(self, ht, first: int, count: int) -> None:
        """recon_mlem_backward_quarters: ht = the back projection of that quarter set's ratio."""
        check(lib().recon_mlem_backward_quarters(self._h, first, count, _ptr(ht), _stream()))

    def mlem_update(self, f, ht) -> None:
        check(lib().recon_mlem_update(self._h, _ptr(f), _ptr(ht), _stream()))

    def mlem_backward_update(self, f) -> None:
        check(lib().recon_mlem_backward_update(self._h, _ptr(f), _stream()))

    def count_intersections(self) -> int:
        n = C.c_ulonglong()
        check(lib().recon_count_intersections(self._h, C.byref(n)))
        return int(n.value)

    def count_projector_pairs(self, projector: int) -> int:
        """(ray, voxel) pairs of positive length as PROJECTOR_FORWARD or
        PROJECTOR_BACK assigns them (recon_count_projector_pairs)."""
        n = C.c_ulonglong()
        check(lib().recon_count_projector_pairs(self._h, int(projector), C.byref(n)))
        return int(n.value)

    # --- parity (COMPAT) ---
    def compat_setup_view(self, angle: float) -> tuple[int, dict]:
        n = self.nu * self.nv
        a = {k: np.zeros(n, np.float32) for k in ("alpha_min", "alpha_max", "d12")}
        a["mask"] = np.zeros(n, np.uint32)
        for k in ("alpha_i", "alpha_f", "delta_alpha", "p1", "p2"):
            a[k] = np.zeros(3 * n, np.float32)
        a["delta_index"] = np.zeros(n, np.uint32)
        loopN = C.c_uint()
        fptr = lambda x: x.ctypes.data_as(C.POINTER(C.c_float))  # noqa: E731
        uptr = lambda x: x.ctypes.data_as(C.POINTER(C.c_uint))  # noqa: E731
        check(lib().recon_compat_setup_view(
            self._h, float(angle), fptr(a["alpha_min"]), fptr(a["alpha_max"]), fptr(a["d12"]), uptr(a["mask"]),
            fptr(a["alpha_i"]), fptr(a["alpha_f"]), fptr(a["delta_alpha"]), fptr(a["p1"]), fptr(a["p2"]),
            uptr(a["delta_index"]), C.byref(loopN)))
        return int(loopN.value), a

    def compat_trace(self, angle: float, rays, cap_steps: int):
        rays = np.ascontiguousarray(rays, np.int32)
        idx = np.zeros(len(rays) * cap_steps, np.int32)
        ln = np.zeros(len(rays) * cap_steps, np.float32)
        loopN = C.c_uint()
        check(lib().recon_compat_trace(self._h, float(angle), len(rays), rays.ctypes.data_as(C.POINTER(C.c_int)),
                                       int(cap_steps), idx.ctypes.data_as(C.POINTER(C.c_int)),
                                       ln.ctypes.data_as(C.POINTER(C.c_float)), C.byref(loopN)))
        return int(loopN.value), idx.reshape(len(rays), cap_steps), ln.reshape(len(rays), cap_steps)


class Batch:
    """Many independent MLEM reconstructions run together (recon_batch_*).

    Each problem has its own geometry; every iteration of every problem is two
    persistent kernels over one work queue.  The reference has no batch call:
    this replaces a loop of siddon_recon::a0_RECON_MLEM over many scans.
    """

    def __init__(self, cfgs: list[dict], options: Options | None = None):
        self.cfgs = [dict(c) for c in cfgs]
        self.options = options or Options()
        geoms = (L.Geometry * len(cfgs))(*[geometry(c) for c in cfgs])
        h = C.c_void_p()
        check(lib().recon_batch_create(geoms, len(cfgs), C.byref(self.options.c()), C.byref(h)))
        self._h = h
        self.shapes_vol = [(int(c["Zdim"]), int(c["Ydim"]), int(c["Xdim"])) for c in cfgs]
        self.shapes_sino = [(int(c["NumProj"]), int(c["TAxPixels"]), int(c["AxPixels"])) for c in cfgs]

    def close(self) -> None:
        if getattr(self, "_h", None):
            lib().recon_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __len__(self) -> int:
        return len(self.cfgs)

    def new_volumes(self, fill: float = 0.0):
        import torch

        dev = torch.device("cuda", self.options.device)
        return [torch.full(s, fill, dtype=torch.float32, device=dev) for s in self.shapes_vol]

    def mlem(self, gs, iters: int, fs=None, init_ones: bool = True):
        """Run `iters` iterations of every problem; gs[p] is problem p's sinogram."""
        if len(gs) != len(self.cfgs):
            raise ValueError(f"expected {len(self.cfgs)} sinograms, got {len(gs)}")
        fs = self.new_volumes() if fs is None else fs
        for p, (g, f) in enumerate(zip(gs, fs)):
            if tuple(g.shape) != self.shapes_sino[p] or tuple(f.shape) != self.shapes_vol[p]:
                raise ValueError(f"problem {p}: sinogram {tuple(g.shape)} / image {tuple(f.shape)} do not match "
                                 f"{self.shapes_sino[p]} / {self.shapes_vol[p]}")
        n = len(self.cfgs)
        gp = (C.c_void_p * n)(*[_ptr(g) for g in gs])
        fp = (C.c_void_p * n)(*[_ptr(f) for f in fs])
        check(lib().recon_batch_mlem(self._h, gp, fp, int(iters), 1 if init_ones else 0, _stream()))
        return fs


def compat_bp_view_noalloc(cfg: dict, img, angle: float, out):
    """recon_compat_bp_view_noalloc: COMPAT back projection of one view into
    `out` on the current CUDA device, with no device allocation by the library
    (at most L.NOALLOC_MAX_VOXELS voxels; overlapping calls on one device
    share its scratch and must not run concurrently)."""
    import torch

    g = geometry(cfg)
    nv, nu = int(cfg["TAxPixels"]), int(cfg["AxPixels"])
    shape_vol = (int(cfg["Zdim"]), int(cfg["Ydim"]), int(cfg["Xdim"]))
    dev = torch.cuda.current_device()
    for name, t, shape in (("img", img, (nv, nu)), ("out", out, shape_vol)):
        if not isinstance(t, torch.Tensor) or t.dtype != torch.float32 or not t.is_cuda:
            raise ValueError(f"{name} must be a float32 CUDA tensor")
        if t.device.index != dev:
            raise ValueError(f"{name} is on cuda:{t.device.index}, the current device is cuda:{dev}")
        if tuple(t.shape) != shape or not t.is_contiguous():
            raise ValueError(f"{name} must be a contiguous {shape} tensor, got {tuple(t.shape)}")
    check(lib().recon_compat_bp_view_noalloc(C.byref(g), _ptr(img), float(angle), _ptr(out), _stream()))
    return out


def mlem_from_cfg(folder: str, cfg: str, options: Options | None = None) -> None:
    """siddon_recon::a0_RECON_MLEM(folder, cfg) (hf_siddon_recon.hpp:91-108)."""
    o = (options or Options()).c()
    check(lib().recon_mlem_from_cfg(folder.encode() if folder else None, cfg.encode(), C.byref(o)))


def forward_projection_from_cfg(folder: str, cfg: str, options: Options | None = None) -> None:
    """siddon_recon::a1_FORWARD_PROJECTION (hf_siddon_recon.hpp:146-163)."""
    o = (options or Options()).c()
    check(lib().recon_forward_projection_from_cfg(folder.encode() if folder else None, cfg.encode(), C.byref(o)))


def backward_projection_from_cfg(folder: str, cfg: str, write_per_angle: bool = False,
                                 options: Options | None = None) -> None:
    """siddon_recon::a1_BACKWARD_PROJECTION (hf_siddon_recon.hpp:165-182)."""
    o = (options or Options()).c()
    check(lib().recon_backward_projection_from_cfg(folder.encode() if folder else None, cfg.encode(),
                                                   1 if write_per_angle else 0, C.byref(o)))
