// voxel.cu -- voxel-driven back projection (the reference's
// backward_projection / backward_projection2, CT_Recon/hf_cuda_kernels.cuh:
// 183-284) as a deterministic gather: a loop over views inside the thread,
// the running sums in registers (added in view order, as the reference's
// per-view launches add into the volume), and the MLEM update
// f <- f * Ht / sens fused into the epilogue when requested.  One thread per
// voxel in general; one thread per (x, y) column and z-chunk in GEOMETRIC mode
// without detector tilt, where a column projects to one detector column.
//
// REFERENCE mode keeps backward_projection2's arithmetic and its flat-array
// bilinear taps (a tap beyond the image end reads 0).  GEOMETRIC mode uses the
// Siddon projector's angle sense and pixel units and samples the view image
// through a texture object (point fetches, FP32 bilinear weights -- hardware
// linear filtering has 8-bit weights); the reference samples through a legacy
// texture reference with the Ruijters cubic B-spline library, which is not
// part of the reference, so that variant cannot be reproduced.
#include <climits>

#include "internal.h"

namespace rb {
namespace voxel {

struct VGeom {
    int X, Y, Z, Nu, Nv;
    float vox[3];
    float R, Rf, Ry, Dx, Dz, M, du_mm, dv_mm;  // pitches in mm (not times M)
    float RM[9];
};

// pixel_iterate (hf_cuda_kernels.cuh:83-87)
__device__ __forceinline__ float center(float NumPixels, float PixelsDimMm, float Mag, int iterator)
{
    return -(NumPixels - 1.0f) / 2.0f * PixelsDimMm * Mag + (float)iterator * PixelsDimMm * Mag;
}

template <bool TEX>
__device__ __forceinline__ float tap(const float* img, cudaTextureObject_t tex, int u, int v, int Nu)
{
    if (TEX) return tex2D<float>(tex, (float)u + 0.5f, (float)v + 0.5f);
    return __ldg(img + (size_t)v * Nu + u);
}

// MODE 0: vol += sum over views; MODE 1: sensitivity (ones images);
// MODE 2: MLEM update f = (s != 0) ? f * Ht / s : 0.
template <int VMODE, int MODE, bool TEX>
__global__ void __launch_bounds__(128) bp_kernel(VGeom G, const float* __restrict__ angles, unsigned view0,
                                                  unsigned nview, unsigned Nproj, const float* __restrict__ sino,
                                                  const cudaTextureObject_t* __restrict__ texs,
                                                  float* __restrict__ vol, const float* __restrict__ sens)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int z = blockIdx.z;
    if (x >= G.X || y >= G.Y) return;
    const size_t n = (size_t)x + (size_t)y * G.X + (size_t)z * G.X * G.Y;
    const size_t npix = (size_t)G.Nu * G.Nv;
    const float xo = center((float)G.X, G.vox[0], 1.0f, x);
    const float yo = center((float)G.Y, G.vox[1], 1.0f, y);
    const float zo = center((float)G.Z, G.vox[2], 1.0f, z);
    const float* RM = G.RM;
    const float R = G.R, Rf = G.Rf, Ry = G.Ry;
    float acc = (MODE == 0) ? vol[n] : 0.0f;
    for (unsigned vi = 0; vi < nview; ++vi) {
        const float alpha = angles[view0 + vi];
        const float* img = sino + vi * npix;
        cudaTextureObject_t tex = TEX ? texs[vi] : 0;
        if (VMODE == RECON_VOXEL_REFERENCE) {
            // backward_projection2 (hf_cuda_kernels.cuh:240-284), as written
            const float sin_alpha = sinf(alpha * (float)3.1415927 / 180.0f);
            const float cos_alpha = cosf(alpha * (float)3.1415927 / 180.0f);
            const float x_alpha = xo * cos_alpha + yo * sin_alpha;
            const float y_alpha = -xo * sin_alpha + yo * cos_alpha;
            const float u_id = __fdividef(R * x_alpha, y_alpha + Rf);
            const float v_id = __fdividef(R * zo, y_alpha + Rf);
            const float detQ = (RM[0] - RM[3] * u_id / R) * (RM[8] - RM[5] * v_id / R) -
                               (RM[2] - RM[5] * u_id / R) * (RM[6] - RM[3] * v_id / R);
            const float u = __fdividef(1, detQ) * ((RM[8] - RM[5] * v_id / R) * (Ry / R * u_id - G.Dx) -
                                                   (RM[2] - RM[5] * u_id / R) * (Ry / R * v_id - G.Dz));
            const float v = __fdividef(1, detQ) * (-(RM[6] - RM[3] * v_id / R) * (Ry / R * u_id - G.Dx) +
                                                   (RM[0] - RM[3] * u_id / R) * (Ry / R * v_id - G.Dz));
            const float u_pix = u + (float)(G.Nu - 1) / 2.0f * G.du_mm * G.M;
            const float v_pix = v + (float)(G.Nv - 1) / 2.0f * G.dv_mm * G.M;
            const unsigned u_int = __float2uint_rd(u_pix);
            const unsigned v_int = __float2uint_rd(v_pix);
            const float u_weight = (u_pix - (float)u_int);
            const float v_weight = (v_pix - (float)v_int);
            if (u_pix >= 0.0 && u_pix <= (float)(G.Nu - 1) * G.du_mm * G.M && v_pix >= 0.0f &&
                v_pix <= (float)(G.Nv - 1) * G.dv_mm * G.M) {
                float t[4];
                const size_t q00 = u_int + (size_t)v_int * G.Nu, q10 = u_int + 1 + (size_t)v_int * G.Nu;
                const size_t q01 = u_int + (size_t)(v_int + 1) * G.Nu, q11 = u_int + 1 + (size_t)(v_int + 1) * G.Nu;
                if (MODE == 1) {
                    t[0] = q00 < npix ? 1.0f : 0.0f; t[1] = q10 < npix ? 1.0f : 0.0f;
                    t[2] = q01 < npix ? 1.0f : 0.0f; t[3] = q11 < npix ? 1.0f : 0.0f;
                } else {
                    t[0] = q00 < npix ? __ldg(img + q00) : 0.0f; t[1] = q10 < npix ? __ldg(img + q10) : 0.0f;
                    t[2] = q01 < npix ? __ldg(img + q01) : 0.0f; t[3] = q11 < npix ? __ldg(img + q11) : 0.0f;
                }
                acc = acc + __fdividef((t[0] * (1 - u_weight) + t[1] * u_weight) * (1 - v_weight) +
                                           (t[2] * (1 - u_weight) + t[3] * u_weight) * v_weight,
                                       (float)Nproj);
            }
        } else {
            // geometric: Siddon angle sense, pixel units, taps inside the image
            const float c = cospif(alpha / 180.0f), s = sinpif(alpha / 180.0f);
            const float xa = xo * c - yo * s;
            const float ya = xo * s + yo * c;
            const float u_id = __fdividef(R * xa, ya + Rf);
            const float v_id = __fdividef(R * zo, ya + Rf);
            const float detQ = (RM[0] - RM[3] * u_id / R) * (RM[8] - RM[5] * v_id / R) -
                               (RM[2] - RM[5] * u_id / R) * (RM[6] - RM[3] * v_id / R);
            const float uu = __fdividef(1, detQ) * ((RM[8] - RM[5] * v_id / R) * (Ry / R * u_id - G.Dx) -
                                                    (RM[2] - RM[5] * u_id / R) * (Ry / R * v_id - G.Dz));
            const float vv = __fdividef(1, detQ) * (-(RM[6] - RM[3] * v_id / R) * (Ry / R * u_id - G.Dx) +
                                                    (RM[0] - RM[3] * u_id / R) * (Ry / R * v_id - G.Dz));
            const float u_pix = uu / (G.du_mm * G.M) + (float)(G.Nu - 1) * 0.5f;
            const float v_pix = vv / (G.dv_mm * G.M) + (float)(G.Nv - 1) * 0.5f;
            if (u_pix >= 0.0f && u_pix <= (float)(G.Nu - 1) && v_pix >= 0.0f && v_pix <= (float)(G.Nv - 1)) {
                const int ui = min(max((int)floorf(u_pix), 0), G.Nu - 2);
                const int vj = min(max((int)floorf(v_pix), 0), G.Nv - 2);
                const float uw = u_pix - (float)ui, vw = v_pix - (float)vj;
                float t00 = 1.0f, t10 = 1.0f, t01 = 1.0f, t11 = 1.0f;
                if (MODE != 1) {
                    t00 = tap<TEX>(img, tex, ui, vj, G.Nu);
                    t10 = tap<TEX>(img, tex, ui + 1, vj, G.Nu);
                    t01 = tap<TEX>(img, tex, ui, vj + 1, G.Nu);
                    t11 = tap<TEX>(img, tex, ui + 1, vj + 1, G.Nu);
                }
                const float val = (t00 * (1.0f - uw) + t10 * uw) * (1.0f - vw) + (t01 * (1.0f - uw) + t11 * uw) * vw;
                acc = acc + val / (float)Nproj;
            }
        }
    }
    if (MODE == 2) {
        const float sv = sens[n];
        const float f = vol[n];
        vol[n] = (sv != 0.0f) ? __fdiv_rn(__fmul_rn(f, acc), sv) : 0.0f;
    } else {
        vol[n] = acc;
    }
}

// GEOMETRIC mode without detector tilt (RM = I): the detector coordinates
// of voxel (x, y, z) at a view are
//   u = (Ry * xa / (ya + Rf) - Dx) / (du * M) + (Nu - 1) / 2,
//   v = (Ry * z / (ya + Rf) - Dz) / (dv * M) + (Nv - 1) / 2,
// with (xa, ya) the voxel's x-y centre rotated to the view, so u is the same
// for a whole (x, y) column and v is linear in z.  One thread per column and
// z-chunk of ZC voxels: per view it projects the column once, then steps v
// along the chunk, with the ZC sums in registers.  Taps, bounds and update as
// in bp_kernel.
template <int ZC, int MODE, bool TEX>
__global__ void __launch_bounds__(128) bp_column_kernel(VGeom G, const float* __restrict__ angles, unsigned view0,
                                                         unsigned nview, unsigned Nproj,
                                                         const float* __restrict__ sino,
                                                         const cudaTextureObject_t* __restrict__ texs,
                                                         float* __restrict__ vol, const float* __restrict__ sens)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int k0 = blockIdx.z * ZC;
    if (x >= G.X || y >= G.Y) return;
    const size_t npix = (size_t)G.Nu * G.Nv, plane = (size_t)G.X * G.Y;
    const size_t n0 = (size_t)x + (size_t)y * G.X + (size_t)k0 * plane;
    const int nz = min(ZC, G.Z - k0);
    const float xo = center((float)G.X, G.vox[0], 1.0f, x);
    const float yo = center((float)G.Y, G.vox[1], 1.0f, y);
    const float z0 = center((float)G.Z, G.vox[2], 1.0f, k0);
    const float inv_du = 1.0f / (G.du_mm * G.M), inv_dv = 1.0f / (G.dv_mm * G.M);
    const float cu = (float)(G.Nu - 1) * 0.5f, cv = (float)(G.Nv - 1) * 0.5f;
    const float umax = (float)(G.Nu - 1), vmax = (float)(G.Nv - 1);
    const float inv_n = 1.0f / (float)Nproj;
    float acc[ZC];
#pragma unroll
    for (int k = 0; k < ZC; ++k) acc[k] = (MODE == 0 && k < nz) ? vol[n0 + (size_t)k * plane] : 0.0f;
    for (unsigned vi = 0; vi < nview; ++vi) {
        const float alpha = angles[view0 + vi];
        const float c = cospif(alpha / 180.0f), s = sinpif(alpha / 180.0f);
        const float xa = xo * c - yo * s;
        const float ya = xo * s + yo * c;
        const float inv = 1.0f / (ya + G.Rf);
        const float u_pix = (G.Ry * xa * inv - G.Dx) * inv_du + cu;
        if (!(u_pix >= 0.0f && u_pix <= umax)) continue;
        const int ui = min(max((int)floorf(u_pix), 0), G.Nu - 2);
        const float uw = u_pix - (float)ui;
        const float vB = G.Ry * inv * G.vox[2] * inv_dv;
        const float vA = (G.Ry * inv * z0 - G.Dz) * inv_dv + cv;
        const float* img = sino + vi * npix;
        cudaTextureObject_t tex = TEX ? texs[vi] : 0;
        // taps of rows `row` (t00, t10) and row + 1 (t01, t11), reused by the
        // next voxel when it samples the same rows or one row further
        int row = INT_MIN;
        float t00 = 1.0f, t10 = 1.0f, t01 = 1.0f, t11 = 1.0f;
#pragma unroll
        for (int k = 0; k < ZC; ++k) {
            const float v_pix = fmaf((float)k, vB, vA);
            if (k < nz && v_pix >= 0.0f && v_pix <= vmax) {
                const int vj = min(max((int)floorf(v_pix), 0), G.Nv - 2);
                const float vw = v_pix - (float)vj;
                if (MODE != 1 && vj != row) {
                    if (vj == row + 1) {
                        t00 = t01;
                        t10 = t11;
                    } else {
                        t00 = tap<TEX>(img, tex, ui, vj, G.Nu);
                        t10 = tap<TEX>(img, tex, ui + 1, vj, G.Nu);
                    }
                    t01 = tap<TEX>(img, tex, ui, vj + 1, G.Nu);
                    t11 = tap<TEX>(img, tex, ui + 1, vj + 1, G.Nu);
                    row = vj;
                }
                const float val = (t00 * (1.0f - uw) + t10 * uw) * (1.0f - vw) + (t01 * (1.0f - uw) + t11 * uw) * vw;
                acc[k] = fmaf(val, inv_n, acc[k]);
            }
        }
    }
#pragma unroll
    for (int k = 0; k < ZC; ++k) {
        if (k >= nz) break;
        const size_t n = n0 + (size_t)k * plane;
        if (MODE == 2) {
            const float sv = sens[n];
            vol[n] = (sv != 0.0f) ? __fdiv_rn(__fmul_rn(vol[n], acc[k]), sv) : 0.0f;
        } else {
            vol[n] = acc[k];
        }
    }
}

// GEOMETRIC mode without tilt, gathered per column by a warp (the layout of
// the Siddon gather back projector, exact.cu): lane l owns the voxels
// k0 + l + 32 s (s < SLOTS) of a column chunk and keeps their sums in
// registers.  Per view the column's detector column u_pix and the row of its
// bottom voxel centre vA (with the row step per voxel vB) are set up 32 views
// at a time, one per lane, in shared memory; then every lane samples its
// voxels' rows v = vA + k vB with the same bilinear arithmetic as
// bp_column_kernel.  The view images are read in the detector-column layout
// [view][u][v] (view_stride elements per view), so one tap of all 32 lanes
// (about 26 consecutive rows of one detector column) lies in one or two
// 128-byte lines.  The taps of four voxels are loaded before any is used.  MODE
// as in bp_kernel; MODE 1 reads nothing.
constexpr int kVoxelWarps = 8;  // a 4 x 2 tile of columns per CTA

template <int MODE, int SLOTS>
__global__ void __launch_bounds__(kVoxelWarps * 32, 3) bp_gather_kernel(VGeom G, const float* __restrict__ angles,
                                                                       unsigned view0, unsigned nview, unsigned Nproj,
                                                                       const float* __restrict__ rg, size_t view_stride,
                                                                       float* __restrict__ vol,
                                                                       const float* __restrict__ sens)
{
    __shared__ float4 sview[kVoxelWarps][32];  // per view: {u_pix, vA, vB, -}
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int x = blockIdx.x * 4 + (warp & 3), y = blockIdx.y * 2 + (warp >> 2);
    if (x >= G.X || y >= G.Y) return;  // whole warps; no block barrier
    float4* sv = sview[warp];
    const size_t plane = (size_t)G.X * G.Y;
    const float xo = center((float)G.X, G.vox[0], 1.0f, x);
    const float yo = center((float)G.Y, G.vox[1], 1.0f, y);
    const float inv_du = 1.0f / (G.du_mm * G.M), inv_dv = 1.0f / (G.dv_mm * G.M);
    const float cu = (float)(G.Nu - 1) * 0.5f, cv = (float)(G.Nv - 1) * 0.5f;
    const float umax = (float)(G.Nu - 1), vmax = (float)(G.Nv - 1);
    const float inv_n = 1.0f / (float)Nproj;
    for (int k0 = 0; k0 < G.Z; k0 += 32 * SLOTS) {
        const float z0 = center((float)G.Z, G.vox[2], 1.0f, k0);
        float acc[SLOTS];
#pragma unroll
        for (int s = 0; s < SLOTS; ++s) {
            const int k = k0 + lane + 32 * s;
            acc[s] = (MODE == 0 && k < G.Z) ? vol[(size_t)x + (size_t)y * G.X + (size_t)k * plane] : 0.0f;
        }
        for (unsigned vb = 0; vb < nview; vb += 32) {
            const unsigned nb = min(32u, nview - vb);
            if ((unsigned)lane < nb) {
                const float alpha = angles[view0 + vb + lane];
                const float c = cospif(alpha / 180.0f), sn = sinpif(alpha / 180.0f);
                const float xa = xo * c - yo * sn;
                const float ya = xo * sn + yo * c;
                const float inv = 1.0f / (ya + G.Rf);
                sv[lane] = make_float4((G.Ry * xa * inv - G.Dx) * inv_du + cu, (G.Ry * inv * z0 - G.Dz) * inv_dv + cv,
                                       G.Ry * inv * G.vox[2] * inv_dv, 0.0f);
            }
            __syncwarp();
            for (unsigned q = 0; q < nb; ++q) {
                const float4 V = sv[q];
                const float u_pix = V.x;
                if (!(u_pix >= 0.0f && u_pix <= umax)) continue;
                const int ui = min(max((int)floorf(u_pix), 0), G.Nu - 2);
                const float uw = u_pix - (float)ui;
                const float* __restrict__ col = rg + (size_t)(vb + q) * view_stride + (size_t)ui * G.Nv;
                const float vbase = fmaf((float)lane, V.z, V.y);
                // taps of PH voxels at a time, loaded before any is used: rows are
                // clamped to the image, so every address is valid, and voxels whose
                // row lies outside the image are dropped when adding
                constexpr int PH = SLOTS < 4 ? SLOTS : 4;
#pragma unroll
                for (int p0 = 0; p0 < SLOTS; p0 += PH) {
                    float t00[PH], t10[PH], t01[PH], t11[PH], vw[PH];
                    bool ok[PH];
#pragma unroll
                    for (int jj = 0; jj < PH; ++jj) {
                        const int s = p0 + jj;
                        if (s >= SLOTS) break;
                        const float v_pix = fmaf((float)(32 * s), V.z, vbase);
                        ok[jj] = v_pix >= 0.0f && v_pix <= vmax;
                        // floor, saturated at 0 by the conversion to unsigned (NaN gives 0)
                        const int vj = (int)min(__float2uint_rd(v_pix), (unsigned)G.Nv - 2u);
                        vw[jj] = v_pix - (float)vj;
                        if (MODE != 1) {
                            const float* r0 = col + vj;
                            t00[jj] = __ldg(r0);
                            t10[jj] = __ldg(r0 + G.Nv);
                            t01[jj] = __ldg(r0 + 1);
                            t11[jj] = __ldg(r0 + 1 + G.Nv);
                        }
                    }
#pragma unroll
                    for (int jj = 0; jj < PH; ++jj) {
                        const int s = p0 + jj;
                        if (s >= SLOTS) break;
                        if (!ok[jj]) continue;
                        float val = 1.0f;
                        if (MODE != 1)
                            val = (t00[jj] * (1.0f - uw) + t10[jj] * uw) * (1.0f - vw[jj]) +
                                  (t01[jj] * (1.0f - uw) + t11[jj] * uw) * vw[jj];
                        acc[s] = fmaf(val, inv_n, acc[s]);
                    }
                }
            }
            __syncwarp();  // the next batch rewrites sv
        }
#pragma unroll
        for (int s = 0; s < SLOTS; ++s) {
            const int k = k0 + lane + 32 * s;
            if (k >= G.Z) continue;
            const size_t n = (size_t)x + (size_t)y * G.X + (size_t)k * plane;
            if (MODE == 2) {
                const float svv = sens[n];
                vol[n] = (svv != 0.0f) ? __fdiv_rn(__fmul_rn(vol[n], acc[s]), svv) : 0.0f;
            } else {
                vol[n] = acc[s];
            }
        }
    }
}

}  // namespace voxel

// ---- host side ----------------------------------------------------------------------

static voxel::VGeom vgeom(const Plan& P)
{
    voxel::VGeom G;
    const recon_geometry_t& g = P.geom;
    G.X = (int)g.vox.Xdim;
    G.Y = (int)g.vox.Ydim;
    G.Z = (int)g.vox.Zdim;
    G.Nu = (int)g.det.NumAxPixels;
    G.Nv = (int)g.det.NumTAxPixels;
    G.vox[0] = g.vox.XVoxSize;
    G.vox[1] = g.vox.YVoxSize;
    G.vox[2] = g.vox.ZVoxSize;
    G.R = g.cal.R;
    G.Rf = g.cal.Rf;
    G.Ry = g.cal.Ry;
    G.Dx = g.cal.Dx;
    G.Dz = g.cal.Dz;
    G.M = g.cal.M;
    G.du_mm = g.det.AxPixDimMm;
    G.dv_mm = g.det.TAxPixDimMm;
    for (int k = 0; k < 9; ++k) G.RM[k] = P.RM[k];
    return G;
}

// Texture objects over the views of a device sinogram (pitched linear 2D
// resources, point filtering, clamp addressing, unnormalised coordinates).
// Returns false (no textures) when the base address or row pitch does not
// meet the device's texture alignment; the caller then reads through the
// read-only data path instead.
static bool make_view_textures(const Plan& P, const float* sino, unsigned count, std::vector<cudaTextureObject_t>& out)
{
    int talign = 512, palign = 32;
    cudaDeviceGetAttribute(&talign, cudaDevAttrTextureAlignment, P.device);
    cudaDeviceGetAttribute(&palign, cudaDevAttrTexturePitchAlignment, P.device);
    const size_t row = (size_t)P.geom.det.NumAxPixels * sizeof(float);
    const size_t view_bytes = P.npix * sizeof(float);
    if (row % (size_t)palign != 0) return false;
    if (reinterpret_cast<uintptr_t>(sino) % (uintptr_t)talign != 0) return false;
    if (count > 1 && view_bytes % (size_t)talign != 0) return false;
    out.resize(count);
    for (unsigned n = 0; n < count; ++n) {
        cudaResourceDesc rd{};
        rd.resType = cudaResourceTypePitch2D;
        rd.res.pitch2D.devPtr = const_cast<float*>(sino) + (size_t)n * P.npix;
        rd.res.pitch2D.desc = cudaCreateChannelDesc<float>();
        rd.res.pitch2D.width = P.geom.det.NumAxPixels;
        rd.res.pitch2D.height = P.geom.det.NumTAxPixels;
        rd.res.pitch2D.pitchInBytes = row;
        cudaTextureDesc td{};
        td.addressMode[0] = cudaAddressModeClamp;
        td.addressMode[1] = cudaAddressModeClamp;
        td.filterMode = cudaFilterModePoint;
        td.readMode = cudaReadModeElementType;
        td.normalizedCoords = 0;
        if (cudaCreateTextureObject(&out[n], &rd, &td, nullptr) != cudaSuccess) {
            cudaGetLastError();
            for (unsigned q = 0; q < n; ++q) cudaDestroyTextureObject(out[q]);
            out.clear();
            return false;
        }
    }
    return true;
}

static void release_textures(TexCache& c)
{
    for (auto h : c.handles) cudaDestroyTextureObject(h);
    if (c.d_handles) cudaFree(c.d_handles);
    c = TexCache{};
}

void release_plan_textures(Plan* P) { release_textures(P->tex); }

// columns: sino is in the detector-column layout [view][u][v] (the MLEM ratio
// of an EXACT plan with this back projector), else [view][v][u].
template <int VMODE, int MODE>
static recon_status_t launch_voxel(Plan& P, const float* sino, const float* angles, unsigned first, unsigned count,
                                   unsigned Nproj, float* vol, const float* sens, bool cache_textures,
                                   bool columns, cudaStream_t s)
{
    voxel::VGeom G = vgeom(P);
    dim3 blk(32, 4, 1), grid((G.X + 31) / 32, (G.Y + 3) / 4, G.Z);
    bool tex = false;
    cudaTextureObject_t* d_handles = nullptr;
    std::vector<cudaTextureObject_t> local;
    cudaTextureObject_t* d_local = nullptr;
    if (VMODE == RECON_VOXEL_GEOMETRIC && MODE != 1 && sino && !columns) {
        if (cache_textures) {
            TexCache& c = P.tex;
            if (c.base != sino || c.count != count) {
                release_textures(c);
                if (make_view_textures(P, sino, count, c.handles)) {
                    RB_CUDA(cudaMalloc(&c.d_handles, count * sizeof(cudaTextureObject_t)));
                    RB_CUDA(cudaMemcpy(c.d_handles, c.handles.data(), count * sizeof(cudaTextureObject_t),
                                       cudaMemcpyHostToDevice));
                    c.base = sino;
                    c.count = count;
                }
            }
            if (c.d_handles) {
                tex = true;
                d_handles = c.d_handles;
            }
        } else if (make_view_textures(P, sino, count, local)) {
            RB_CUDA(cudaMalloc(&d_local, count * sizeof(cudaTextureObject_t)));
            RB_CUDA(cudaMemcpyAsync(d_local, local.data(), count * sizeof(cudaTextureObject_t), cudaMemcpyHostToDevice,
                                    s));
            tex = true;
            d_handles = d_local;
        }
    }
    const bool untilted = P.geom.cal.xangle == 0.0f && P.geom.cal.yangle == 0.0f && P.geom.cal.zangle == 0.0f;
    if (VMODE == RECON_VOXEL_GEOMETRIC && untilted && (MODE == 1 || columns)) {
        const dim3 ggrid((G.X + 3) / 4, (G.Y + 1) / 2);
        const size_t stride = P.npix;
        switch (gather_slots(G.Z)) {
#define RB_VOXEL_SLOTS(n)                                                                                          \
    case n:                                                                                                        \
        voxel::bp_gather_kernel<MODE, n><<<ggrid, voxel::kVoxelWarps * 32, 0, s>>>(G, angles, first, count, Nproj, \
                                                                                  sino, stride, vol, sens);        \
        break
            RB_VOXEL_SLOTS(1);
            RB_VOXEL_SLOTS(2);
            RB_VOXEL_SLOTS(3);
            RB_VOXEL_SLOTS(4);
            RB_VOXEL_SLOTS(5);
            RB_VOXEL_SLOTS(6);
            RB_VOXEL_SLOTS(7);
            default: RB_VOXEL_SLOTS(8);
#undef RB_VOXEL_SLOTS
        }
        RB_CUDA(cudaGetLastError());
        return RECON_OK;
    }
    if (VMODE == RECON_VOXEL_GEOMETRIC && untilted) {
        constexpr int ZC = 16;
        const dim3 cgrid((G.X + 31) / 32, (G.Y + 3) / 4, (G.Z + ZC - 1) / ZC);
        if (tex)
            voxel::bp_column_kernel<ZC, MODE, true><<<cgrid, blk, 0, s>>>(G, angles, first, count, Nproj, sino,
                                                                          d_handles, vol, sens);
        else
            voxel::bp_column_kernel<ZC, MODE, false><<<cgrid, blk, 0, s>>>(G, angles, first, count, Nproj, sino,
                                                                           nullptr, vol, sens);
    } else if (tex) {
        voxel::bp_kernel<VMODE, MODE, true><<<grid, blk, 0, s>>>(G, angles, first, count, Nproj, sino, d_handles, vol,
                                                                  sens);
    } else {
        voxel::bp_kernel<VMODE, MODE, false><<<grid, blk, 0, s>>>(G, angles, first, count, Nproj, sino, nullptr, vol,
                                                                   sens);
    }
    cudaError_t e = cudaGetLastError();
    if (d_local) {
        // the per-call textures must outlive the kernel
        cudaStreamSynchronize(s);
        for (auto h : local) cudaDestroyTextureObject(h);
        cudaFree(d_local);
    }
    if (e != cudaSuccess) return cuda_fail(e, "voxel back projection launch");
    return RECON_OK;
}

__global__ void voxel_set_angle_kernel(float* p, float v) { *p = v; }

recon_status_t voxel_bp(Plan& P, const float* sino, unsigned first, unsigned count, bool scratch_slot,
                        float angle_scratch, unsigned Nproj, int mode, bool ones, float* vol_accum,
                        const float* sens, float* f_update, cudaStream_t s, bool columns)
{
    if (scratch_slot) {
        voxel_set_angle_kernel<<<1, 1, 0, s>>>(P.d_angles + P.nviews, angle_scratch);
        first = P.nviews;
        count = 1;
    }
    const bool ref = (mode == RECON_VOXEL_REFERENCE);
    const bool cache = !scratch_slot;
    if (ones) {
        return ref ? launch_voxel<RECON_VOXEL_REFERENCE, 1>(P, nullptr, P.d_angles, first, count, Nproj, vol_accum,
                                                             nullptr, false, false, s)
                   : launch_voxel<RECON_VOXEL_GEOMETRIC, 1>(P, nullptr, P.d_angles, first, count, Nproj, vol_accum,
                                                             nullptr, false, false, s);
    }
    if (f_update) {
        return ref ? launch_voxel<RECON_VOXEL_REFERENCE, 2>(P, sino, P.d_angles, first, count, Nproj, f_update, sens,
                                                             cache, columns, s)
                   : launch_voxel<RECON_VOXEL_GEOMETRIC, 2>(P, sino, P.d_angles, first, count, Nproj, f_update, sens,
                                                             cache, columns, s);
    }
    return ref ? launch_voxel<RECON_VOXEL_REFERENCE, 0>(P, sino, P.d_angles, first, count, Nproj, vol_accum, nullptr,
                                                         cache, columns, s)
               : launch_voxel<RECON_VOXEL_GEOMETRIC, 0>(P, sino, P.d_angles, first, count, Nproj, vol_accum, nullptr,
                                                         cache, columns, s);
}

}  // namespace rb
