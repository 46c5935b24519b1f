"""The CPU oracle against the reference's own kernels (host build) and against
analytic known answers.  No GPU needed.

The reference ships no tests, fixtures or golden vectors, so the FP32
restatement (oracle/siddon_oracle.c) is pinned by running the reference's
kernel sources themselves, compiled for the host (oracle/_ref/libref_cpu.so,
built from the reference's sources by oracle/build_oracle.py): set-up arrays,
per-step traces, projections, back projections and MLEM must agree bit for bit.
The FP64 oracle is pinned by analytic intersection lengths.
"""
import numpy as np
import pytest

from conftest import small_cfg
from oracle import oracle as O
from recon_b200.configs import geom_dict

REF = O.ref_cpu()
needs_ref = pytest.mark.skipif(REF is None, reason="reference host build missing (oracle/_ref/libref_cpu.so)")

ANGLES = [0.0, 4.0, 37.0, 90.0, 133.0, 180.0, 215.0, 359.0]


def bits(a):
    return np.ascontiguousarray(a).view(np.uint32)


def geoms():
    yield "plain", small_cfg()
    # misaligned detector: offsets and tilts (siddon_device_kernelsMLEM.cuh:315-316 overwrite order)
    yield "misaligned", small_cfg(Dx=0.7, Dz=-0.4, xangle=0.01, yangle=-0.02, zangle=0.015, Ry=803.0)
    # a detector offset that puts row 23 at z = 0: that row's rays are parallel
    # to the z planes (p2.z == p1.z).  (Odd detector sizes would do the same,
    # but the reference's 4-wide launch grids cannot cover them.)
    yield "z_parallel_row", small_cfg(Dz=0.75)
    # magnification and non-cubic voxels
    yield "anisotropic", small_cfg(M=1.3, XVoxSize=0.8, YVoxSize=1.1, ZVoxSize=0.9, Zdim=20)


@needs_ref
@pytest.mark.parametrize("name,cfg", list(geoms()))
def test_setup_bitexact(name, cfg):
    REF.ref_cpu_set_threads(1)
    g = O.Geom.from_dict(geom_dict(cfg))
    for ang in ANGLES:
        l1, a = O.c_setup_view(g, ang)
        l2, b = O.ref_cpu_setup_view(g, ang)
        for k in a:
            assert np.array_equal(bits(a[k]), bits(b[k])), (name, ang, k)


@needs_ref
@pytest.mark.parametrize("name,cfg", list(geoms()))
def test_fp_bp_bitexact(name, cfg):
    REF.ref_cpu_set_threads(1)
    g = O.Geom.from_dict(geom_dict(cfg))
    rng = np.random.default_rng(1)
    vol = rng.random(g.nvox).astype(np.float32)
    img = rng.random(g.npix).astype(np.float32)
    for ang in ANGLES[:5]:
        loopN = O.c_loopN(g, ang)
        f1 = O.c_fp_view(g, ang, vol)
        f2 = np.zeros(g.npix, np.float32)
        REF.ref_cpu_fp_view(g, ang, loopN, vol, f2)
        assert np.array_equal(bits(f1), bits(f2)), (name, ang)
        b1 = O.c_bp_view(g, ang, img)
        b2 = np.zeros(g.nvox, np.float32)
        REF.ref_cpu_bp_view(g, ang, loopN, img, b2)
        assert np.array_equal(bits(b1), bits(b2)), (name, ang)
        assert f1.max() > 0 and b1.max() > 0


@needs_ref
def test_trace_bitexact_every_ray():
    REF.ref_cpu_set_threads(1)
    cfg = small_cfg(AxPixels=32, TAxPixels=24)
    g = O.Geom.from_dict(geom_dict(cfg))
    for ang in (0.0, 37.0, 90.0):
        loopN = O.c_loopN(g, ang)
        rays = np.arange(g.npix, dtype=np.int32)
        idx = np.zeros(len(rays) * (loopN + 1), np.int32)
        val = np.zeros(len(rays) * (loopN + 1), np.float32)
        REF.ref_cpu_trace(g, ang, loopN, len(rays), rays, idx, val)
        idx = idx.reshape(len(rays), -1)
        val = val.reshape(len(rays), -1)
        for n in rays:
            ti, tl = O.c_trace(g, ang, int(n % g.NumAxPixels), int(n // g.NumAxPixels), loopN)
            k = len(ti) - 1  # steps taken before the fixed point; last record = end segment
            assert np.array_equal(ti[:-1], idx[n, :k])
            assert np.array_equal(bits(tl[:-1]), bits(val[n, :k]))
            assert np.all(idx[n, k:loopN] == -1) and np.all(val[n, k:loopN] == 0)
            assert ti[-1] == idx[n, loopN] and bits(tl[-1:])[0] == bits(val[n, loopN:])[0]


@needs_ref
def test_mlem_bitexact():
    REF.ref_cpu_set_threads(1)
    cfg = small_cfg(AxPixels=32, TAxPixels=24, Xdim=16, Ydim=16, Zdim=12, XVoxSize=2.0, YVoxSize=2.0,
                    ZVoxSize=2.0, AxPixDim=2.0, TAxPixDim=2.0, NumProj=12)
    g = O.Geom.from_dict(geom_dict(cfg))
    nproj, dang = 12, np.float32(30.0)
    sino = (np.random.default_rng(2).random(nproj * g.npix) * 5).astype(np.float32)
    f1, s1, h1 = O.c_mlem(g, nproj, dang, sino, 3, history=True)
    loopN = np.array([O.c_loopN(g, np.float32(n) * dang) for n in range(nproj)], np.uint32)
    f2 = np.zeros(g.nvox, np.float32)
    s2 = np.zeros(g.nvox, np.float32)
    REF.ref_cpu_mlem(g, nproj, dang, loopN, sino, 3, f2, s2, None)
    assert np.array_equal(bits(s1), bits(s2))
    assert np.array_equal(bits(f1), bits(f2))
    assert np.all(np.isfinite(h1))


def test_pixel_centres_rounded():
    # pixel_iterate2 rounds centres to 1e-5 mm (hf_cuda_kernels.cuh:92-97)
    L = O.lib()
    for N, d in ((512, 0.5), (128, 1.0), (1024, 0.0065)):
        for i in (0, 1, N // 2, N - 1):
            c = L.orc_c_pixel_iterate2(float(N), d, 1.0, i)
            ideal = -(N - 1) / 2.0 * d + i * d
            assert abs(c - ideal) < 2e-5 + abs(ideal) * 1e-6


# ---- FP64 exact Siddon: analytic answers ---------------------------------------------------

def _chord(r, half):
    p1, p2 = np.array(r.p1), np.array(r.p2)
    d = p2 - p1
    lo, hi = 0.0, 1.0
    for k in range(3):
        if d[k] == 0:
            if not (-half[k] <= p1[k] < half[k]):
                return 0.0
            continue
        a0, a1 = (-half[k] - p1[k]) / d[k], (half[k] - p1[k]) / d[k]
        lo, hi = max(lo, min(a0, a1)), min(hi, max(a0, a1))
    return max(0.0, hi - lo) * r.d12


@pytest.mark.parametrize("ang", [0.0, 30.0, 45.0, 90.0, 123.0, 270.0])
def test_fp64_lengths_sum_to_chord(ang):
    cfg = small_cfg(Xdim=8, Ydim=8, Zdim=8, AxPixels=8, TAxPixels=6, AxPixDim=4.0, TAxPixDim=4.0)
    g = O.Geom.from_dict(geom_dict(cfg))
    half = [4.0, 4.0, 4.0]
    for u in range(8):
        for v in range(6):
            idx, ln = O.x_trace(g, ang, u, v)
            r = O.x_ray(g, ang, u, v)
            assert abs(ln.sum() - _chord(r, half)) < 1e-9
            assert np.all(ln > 0) and len(set(idx.tolist())) == len(idx)


def test_fp64_axis_aligned_ray():
    # a ray along y through voxel centres: every voxel of the row gets exactly one voxel length
    cfg = small_cfg(Xdim=8, Ydim=8, Zdim=8, AxPixels=9, TAxPixels=9, AxPixDim=1.0, TAxPixDim=1.0)
    g = O.Geom.from_dict(geom_dict(cfg))
    idx, ln = O.x_trace(g, 0.0, 4, 4)  # central pixel of an odd detector: x = z = 0, on voxel planes
    assert len(idx) == 8
    assert np.allclose(ln, 1.0, atol=1e-12)


def test_fp64_fp_bp_adjoint():
    cfg = small_cfg(Xdim=16, Ydim=16, Zdim=12, AxPixels=24, TAxPixels=20, AxPixDim=2.0, TAxPixDim=2.0, NumProj=6)
    g = O.Geom.from_dict(geom_dict(cfg))
    rng = np.random.default_rng(3)
    x = rng.random(g.nvox)
    y = rng.random(6 * g.npix)
    Ax = O.x_fp_all(g, 6, np.float32(60.0), x)
    Aty = O.x_bp_all(g, 6, np.float32(60.0), y)
    assert abs(np.dot(Ax, y) - np.dot(x, Aty)) < 1e-11 * abs(np.dot(Ax, y))


def test_fp64_voxel_column_matches_traversal():
    cfg = small_cfg(Xdim=12, Ydim=12, Zdim=8, AxPixels=20, TAxPixels=16, AxPixDim=2.0, TAxPixDim=2.0, NumProj=5)
    g = O.Geom.from_dict(geom_dict(cfg))
    voxel = 5 + 7 * 12 + 3 * 144
    e = np.zeros(g.nvox)
    e[voxel] = 1.0
    col = O.x_fp_all(g, 5, np.float32(72.0), e)
    view, pix, ln = O.x_voxel_column(g, 5, np.float32(72.0), voxel)
    dense = np.zeros_like(col)
    dense[view * g.npix + pix] = ln
    assert np.allclose(dense, col, rtol=1e-12, atol=1e-12)


def test_compat_vs_fp64_close():
    # the reference arithmetic differs from the exact Siddon only by its documented quirks
    cfg = small_cfg()
    g = O.Geom.from_dict(geom_dict(cfg))
    vol = np.random.default_rng(4).random(g.nvox).astype(np.float32)
    for ang in (0.0, 37.0):
        c = O.c_fp_view(g, ang, vol).astype(np.float64)
        x = np.zeros(g.npix)
        O.lib().orc_x_fp_view(g, ang, vol.astype(np.float64), x)
        err = np.linalg.norm(c - x) / np.linalg.norm(x)
        assert err < 5e-2, err


def test_fp64_osem_one_subset_is_mlem_and_checks_subsets():
    # OSEM of the oracle (contiguous subsets, osem_input_values / check_recon_inputs,
    # hf_cpp_functions.hpp:298-375): one subset is MLEM exactly; a subset count
    # that does not divide the views is refused
    cfg = small_cfg(Xdim=12, Ydim=12, Zdim=8, AxPixels=20, TAxPixels=16, AxPixDim=2.0, TAxPixDim=2.0, NumProj=6)
    g = O.Geom.from_dict(geom_dict(cfg))
    sino = np.random.default_rng(5).random(6 * g.npix).astype(np.float32)
    f_mlem, _ = O.x_mlem(g, 6, np.float32(60.0), sino, 2)
    assert np.array_equal(O.x_osem(g, 6, np.float32(60.0), sino, 2, 1), f_mlem)
    f3 = O.x_osem(g, 6, np.float32(60.0), sino, 2, 3)
    assert np.all(np.isfinite(f3)) and not np.array_equal(f3, f_mlem)
    with pytest.raises(ValueError):
        O.x_osem(g, 6, np.float32(60.0), sino, 1, 4)
