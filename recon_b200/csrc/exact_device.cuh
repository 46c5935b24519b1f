// exact_device.cuh -- device functions of the EXACT projector pair, shared by
// the single-problem kernels (exact.cu) and the batched persistent kernels
// (batch.cu).  See exact.cu for the ray parameterisation.
#pragma once

#include <cuda_bf16.h>

#include <climits>

#include "internal.h"

namespace rb {
namespace exact {

// ---- shared device helpers -------------------------------------------------------------

__device__ __forceinline__ float plane_t(int k, float S, float O, int kc) { return fmaf((float)(k - kc), S, O); }

// Voxel i in [lo, hi) along an axis: the voxel whose t-interval [t_i, t_i+1)
// contains t (entry: t_i <= t < t_i+1) or (t_i, t_i+1] (exit), ends ordered,
// found from an FP64 estimate and corrected against the FP32 plane values.
template <bool ENTRY>
__device__ __forceinline__ int locate_in(float t, float S, float O, int kc, int lo, int hi, double invS)
{
    double kf = (double)kc + ((double)t - (double)O) * invS;
    int i = (int)floor(fmin(fmax(kf, (double)lo - 1.0), (double)hi));
    i = min(max(i, lo), hi - 1);
    const int up = (S > 0.0f) ? 1 : -1;  // index step toward larger t
#pragma unroll 1
    for (int it = 0; it < 6; ++it) {
        float t0 = plane_t(i, S, O, kc), t1 = plane_t(i + 1, S, O, kc);
        float a = fminf(t0, t1), b = fmaxf(t0, t1);
        bool before = ENTRY ? (t < a) : (t <= a);
        bool after = ENTRY ? (t >= b) : (t > b);
        int ni = before ? i - up : (after ? i + up : i);
        if (ni == i || ni < lo || ni >= hi) break;
        i = ni;
    }
    return i;
}

// The same over the whole axis of N voxels.
template <bool ENTRY>
__device__ __forceinline__ int locate(float t, float S, float O, int kc, int N, double invS)
{
    return locate_in<ENTRY>(t, S, O, kc, 0, N, invS);
}

template <class T>
__device__ __forceinline__ float load_val(const T* p);
template <>
__device__ __forceinline__ float load_val<float>(const float* p) { return __ldg(p); }
template <>
__device__ __forceinline__ float load_val<__nv_bfloat16>(const __nv_bfloat16* p)
{
    // BF16 is the upper half of an FP32: widening is a shift (plain code, so a
    // predicated load stays a predicated load)
    return __uint_as_float((unsigned)__ldg(reinterpret_cast<const unsigned short*>(p)) << 16);
}
// A value as stored (load_raw) and widened to FP32 later (widen), so that a
// batch of loads can be issued before any of them is used.
__device__ __forceinline__ float load_raw(const float* p) { return __ldg(p); }
__device__ __forceinline__ unsigned short load_raw(const __nv_bfloat16* p)
{
    return __ldg(reinterpret_cast<const unsigned short*>(p));
}
__device__ __forceinline__ float widen(float x) { return x; }
__device__ __forceinline__ float widen(unsigned short h) { return __uint_as_float((unsigned)h << 16); }
template <class T>
__device__ __forceinline__ void store_val(T* p, float v);
template <>
__device__ __forceinline__ void store_val<float>(float* p, float v) { *p = v; }
template <>
__device__ __forceinline__ void store_val<__nv_bfloat16>(__nv_bfloat16* p, float v) { *p = __float2bfloat16_rn(v); }

// Two values kept together (mirrored row pairs): one 8-byte access for float,
// one 4-byte access for bf16; p is aligned to the pair.  load_pair_raw keeps
// the stored form, widen_lo / widen_hi give the first and second value.
template <class T>
__device__ __forceinline__ void store_pair(T* p, float a, float b);
template <>
__device__ __forceinline__ void store_pair<float>(float* p, float a, float b)
{
    *reinterpret_cast<float2*>(p) = make_float2(a, b);
}
template <>
__device__ __forceinline__ void store_pair<__nv_bfloat16>(__nv_bfloat16* p, float a, float b)
{
    *reinterpret_cast<__nv_bfloat162*>(p) = __floats2bfloat162_rn(a, b);
}
__device__ __forceinline__ float2 load_pair_raw(const float* p) { return __ldg(reinterpret_cast<const float2*>(p)); }
__device__ __forceinline__ unsigned load_pair_raw(const __nv_bfloat16* p)
{
    return __ldg(reinterpret_cast<const unsigned*>(p));
}
__device__ __forceinline__ float widen_lo(float2 x) { return x.x; }
__device__ __forceinline__ float widen_hi(float2 x) { return x.y; }
__device__ __forceinline__ float widen_lo(unsigned x) { return __uint_as_float(x << 16); }
__device__ __forceinline__ float widen_hi(unsigned x) { return __uint_as_float(x & 0xffff0000u); }

// ---- ray blocks ---------------------------------------------------------------------------

// Rays are launched in blocks of 32 (u) x 4 (v).  A CTA's block comes from a
// tile list ({view, tu | tv << 16}, the blocks whose rays can cross the
// volume; blockIdx.x indexes it) or, when tiles is null, from the full grid
// (blockIdx.x, blockIdx.y, view view0 + blockIdx.z).
struct RayPos {
    int u, v;
    unsigned view;
};

__device__ __forceinline__ RayPos ray_pos(const uint2* __restrict__ tiles, unsigned view0)
{
    if (tiles) {
        const uint2 t = tiles[blockIdx.x];
        return RayPos{(int)(t.y & 0xffffu) * 32 + (int)threadIdx.x, (int)(t.y >> 16) * 4 + (int)threadIdx.y, t.x};
    }
    return RayPos{(int)(blockIdx.x * 32 + threadIdx.x), (int)(blockIdx.y * 4 + threadIdx.y), view0 + blockIdx.z};
}

// ---- forward projection --------------------------------------------------------------------

// The volume as the forward walk reads it: voxel (x, y, z) at
// base[x*ux + y*uy + z*X*Y].  ux = 1, uy = X is the image layout; ux = Y,
// uy = 1 is its xy-transposed copy, read for views whose detector rows run
// mostly along y (|sin| > |cos|), so that the 32 rays of a warp (adjacent
// detector columns) read adjacent addresses in either case.
struct VolView {
    const float* __restrict__ base;
    int ux, uy;
};

__device__ __forceinline__ VolView vol_view_for(const float2 cs, const float* vol, const float* vol_t, int X, int Y)
{
    if (vol_t && fabsf(cs.y) > fabsf(cs.x)) return VolView{vol_t, Y, 1};
    return VolView{vol, 1, X};
}

// Sum over the voxels the ray crosses of (t_exit - t_entry) * f[voxel] (the
// projection divided by w): entry and exit voxels located per ray, the step
// count known before the walk, one axis advanced per step.
template <bool KAHAN>
__device__ __forceinline__ float fp_ray_sum(const ExactGeom& G, const float4 T, const int2 K, const ZParam Z,
                                            const VolView V)
{
    const float* __restrict__ vol = V.base;
    // entry / exit planes of the volume
    float x0 = plane_t(0, T.x, T.y, K.x), x1 = plane_t(G.X, T.x, T.y, K.x);
    float y0 = plane_t(0, T.z, T.w, K.y), y1 = plane_t(G.Y, T.z, T.w, K.y);
    float z0 = plane_t(0, Z.S, Z.O, Z.kc), z1 = plane_t(G.Z, Z.S, Z.O, Z.kc);
    const float t_in = fmaxf(fmaxf(fminf(x0, x1), fminf(y0, y1)), fminf(z0, z1));
    const float t_out = fminf(fminf(fmaxf(x0, x1), fmaxf(y0, y1)), fmaxf(z0, z1));
    float acc = 0.0f;
    if (t_in < t_out) {
        const double ivx = 1.0 / (double)T.x, ivy = 1.0 / (double)T.z, ivz = 1.0 / (double)Z.S;
        int ix = locate<true>(t_in, T.x, T.y, K.x, G.X, ivx), ex = locate<false>(t_out, T.x, T.y, K.x, G.X, ivx);
        int iy = locate<true>(t_in, T.z, T.w, K.y, G.Y, ivy), ey = locate<false>(t_out, T.z, T.w, K.y, G.Y, ivy);
        int iz = locate<true>(t_in, Z.S, Z.O, Z.kc, G.Z, ivz), ez = locate<false>(t_out, Z.S, Z.O, Z.kc, G.Z, ivz);
        const int nsteps = abs(ex - ix) + abs(ey - iy) + abs(ez - iz) + 1;
        const int dx = T.x > 0.0f ? 1 : -1, dy = T.z > 0.0f ? 1 : -1, dz = Z.S > 0.0f ? 1 : -1;
        // float offsets (plane - kc) of each axis's next plane
        float kx = (float)((dx > 0 ? ix + 1 : ix) - K.x);
        float ky = (float)((dy > 0 ? iy + 1 : iy) - K.y);
        float kz = (float)((dz > 0 ? iz + 1 : iz) - Z.kc);
        float tx = fmaf(kx, T.x, T.y), ty = fmaf(ky, T.z, T.w), tz = fmaf(kz, Z.S, Z.O);
        const float fdx = (float)dx, fdy = (float)dy, fdz = (float)dz;
        const int sx = dx * V.ux, sy = dy * V.uy, sz = dz * G.X * G.Y;
        const unsigned vmax = (unsigned)(G.X * G.Y * G.Z - 1);
        int idx = ix * V.ux + iy * V.uy + iz * G.X * G.Y;
        float cur = t_in, comp = 0.0f;
#pragma unroll 4  // 2 and 8 measured 2 % slower, 3 slower still
        for (int s = 0; s < nsteps; ++s) {
            const float m = fminf(tx, fminf(ty, tz));
            const float fv = __ldg(vol + min((unsigned)idx, vmax));
            const float L = m - cur;
            if (KAHAN) {
                const float y = fmaf(L, fv, -comp);
                const float t = acc + y;
                comp = (t - acc) - y;
                acc = t;
            } else {
                acc = fmaf(L, fv, acc);
            }
            cur = m;
            // advance the axis whose plane was crossed (x before y before z
            // on ties), without divergent branches
            const bool bx = (tx == m);
            const bool by = !bx && (ty == m);
            const bool bz = !bx && !by;
            kx = bx ? kx + fdx : kx;
            ky = by ? ky + fdy : ky;
            kz = bz ? kz + fdz : kz;
            tx = bx ? fmaf(kx, T.x, T.y) : tx;
            ty = by ? fmaf(ky, T.z, T.w) : ty;
            tz = bz ? fmaf(kz, Z.S, Z.O) : tz;
            idx += bx ? sx : (by ? sy : sz);
        }
    }
    return acc;
}

// ---- back projection (ray-driven, exact fixed-point sums) -----------------------------------
//
// Each ray walks the voxels it crosses exactly as the forward projector does,
// restricted to a z-slab [k0, k1) of the volume, and adds L * value to each
// voxel's 64-bit fixed-point accumulator with an integer atomic.  Integer sums
// do not depend on the order of the additions, so the result is
// deterministic, and every (ray, voxel) length is the forward projector's, so
// the pair is an exact transpose.  The scale 2^F is chosen per call so that
// no voxel sum can overflow: |L * value| < 2^e (max |value| times the longest
// segment) and at most 2^count_bits contributions per voxel give
// |sum| < 2^(e + F + count_bits) = 2^62.  A slab's accumulators are sized to
// stay resident in L2.  Views whose detector rows run mostly along y add into
// a second, xy-transposed accumulator, so that the 32 rays of a warp (adjacent
// detector columns) update adjacent addresses in either case.

// F for the fixed-point scale, or INT_MIN when the input is all zero or not
// finite (nothing is accumulated then).
__device__ __forceinline__ int fix_exponent(unsigned maxabs_bits, float max_len, int count_bits)
{
    const float m = __uint_as_float(maxabs_bits);
    if (!(m > 0.0f) || !isfinite(m)) return INT_MIN;
    int e;
    frexp((double)m * (double)max_len, &e);
    return min(62 - count_bits - e, 120);
}

// One ray's contributions to the slab [k0, k1): cval = value * 2^F.  acc is
// the slab in image layout [z-k0][y][x]; acc_t the transposed one
// [z-k0][x][y], used when `transposed`.
__device__ __forceinline__ void bp_ray_slab(const ExactGeom& G, const float4 T, const int2 K, const ZParam Z,
                                            int k0, int k1, float cval, bool transposed, unsigned long long* acc,
                                            unsigned long long* acc_t)
{
    const float x0 = plane_t(0, T.x, T.y, K.x), x1 = plane_t(G.X, T.x, T.y, K.x);
    const float y0 = plane_t(0, T.z, T.w, K.y), y1 = plane_t(G.Y, T.z, T.w, K.y);
    const float z0 = plane_t(k0, Z.S, Z.O, Z.kc), z1 = plane_t(k1, Z.S, Z.O, Z.kc);
    const float t_in = fmaxf(fmaxf(fminf(x0, x1), fminf(y0, y1)), fminf(z0, z1));
    const float t_out = fminf(fminf(fmaxf(x0, x1), fmaxf(y0, y1)), fmaxf(z0, z1));
    if (!(t_in < t_out)) return;
    const double ivx = 1.0 / (double)T.x, ivy = 1.0 / (double)T.z, ivz = 1.0 / (double)Z.S;
    const int ix = locate<true>(t_in, T.x, T.y, K.x, G.X, ivx), ex = locate<false>(t_out, T.x, T.y, K.x, G.X, ivx);
    const int iy = locate<true>(t_in, T.z, T.w, K.y, G.Y, ivy), ey = locate<false>(t_out, T.z, T.w, K.y, G.Y, ivy);
    const int iz = min(max(locate<true>(t_in, Z.S, Z.O, Z.kc, G.Z, ivz), k0), k1 - 1);
    const int ez = min(max(locate<false>(t_out, Z.S, Z.O, Z.kc, G.Z, ivz), k0), k1 - 1);
    const int nsteps = abs(ex - ix) + abs(ey - iy) + abs(ez - iz) + 1;
    const int dx = T.x > 0.0f ? 1 : -1, dy = T.z > 0.0f ? 1 : -1, dz = Z.S > 0.0f ? 1 : -1;
    float kx = (float)((dx > 0 ? ix + 1 : ix) - K.x);
    float ky = (float)((dy > 0 ? iy + 1 : iy) - K.y);
    float kz = (float)((dz > 0 ? iz + 1 : iz) - Z.kc);
    float tx = fmaf(kx, T.x, T.y), ty = fmaf(ky, T.z, T.w), tz = fmaf(kz, Z.S, Z.O);
    const float fdx = (float)dx, fdy = (float)dy, fdz = (float)dz;
    const int ux = transposed ? G.Y : 1, uy = transposed ? 1 : G.X;
    unsigned long long* __restrict__ A = transposed ? acc_t : acc;
    const int sx = dx * ux, sy = dy * uy, sz = dz * G.X * G.Y;
    const unsigned lmax = (unsigned)(G.X * G.Y * (k1 - k0) - 1);
    int l = ix * ux + iy * uy + (iz - k0) * G.X * G.Y;
    float cur = t_in;
#pragma unroll 2
    for (int s = 0; s < nsteps; ++s) {
        const float m = fminf(tx, fminf(ty, tz));
        const long long q = __float2ll_rn((m - cur) * cval);
        if (q != 0) atomicAdd(A + min((unsigned)l, lmax), (unsigned long long)q);
        cur = m;
        // advance the axis whose plane was crossed (x before y before z on
        // ties), as the forward walk does
        const bool bx = (tx == m);
        const bool by = !bx && (ty == m);
        const bool bz = !bx && !by;
        kx = bx ? kx + fdx : kx;
        ky = by ? ky + fdy : ky;
        kz = bz ? kz + fdz : kz;
        tx = bx ? fmaf(kx, T.x, T.y) : tx;
        ty = by ? fmaf(ky, T.z, T.w) : ty;
        tz = bz ? fmaf(kz, Z.S, Z.O) : tz;
        l += bx ? sx : (by ? sy : sz);
    }
}

}  // namespace exact
}  // namespace rb
