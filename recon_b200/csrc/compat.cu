// compat.cu -- COMPAT arithmetic: the reference's FP32 Siddon traversal,
// reproduced operation for operation, with one thread per ray and the whole
// traversal in registers.
//
// The reference runs every traversal step as separate launches over all rays
// (siddon_sort_alpha, siddon_fp_calc_ray_path / siddon_bp_calc_ray_path,
// siddon_add, the atomic scatter kernel and a full-volume siddon_add_bp per
// step; CT_Recon/hf_siddon_class.hpp:195-225, 313-347), with a blocking
// device-to-host copy per view to find the step count.  Here each thread
// carries one ray from set-up to its end segment: no per-step launches, no
// memsets, no host synchronisation.  The per-ray arithmetic is the
// reference's own: every expression below keeps the operand order of the
// reference line it restates, so that the compiler forms the same FMAs and
// the intrinsics (__fdividef, __fdiv_rz, cospif, sinpif, __float2int_rz) see
// the same operands.  Float-to-unsigned conversions of run-time values
// (float plane indices passed as unsigned) are made explicit with the
// saturating device conversion (NaN -> 0), which is what the hardware does.
// The reference also stores the constant CUDART_NAN_F into its unsigned
// ray mask (calc_mask, the parallel-axis branch of siddon_calc_indices,
// bound_index).  Converting NaN to an integer is undefined behaviour in C++,
// and nvcc's optimizer drops those stores: the reference's sm_100a build
// keeps mask = 1 for every ray (measured on all test geometries, misses and
// axis-parallel rays included).  COMPAT reproduces the GPU build, so the mask
// is never cleared here either.
//
// Back projection keeps the reference's ray-driven scatter, but accumulates
// each view's contributions len*img in 64-bit fixed point (integer atomics,
// exact and order independent) and rounds once to float, so the result is
// deterministic; the reference sums with float atomics in arbitrary order.
#include "internal.h"

#include <cfloat>
#include <cmath>

namespace rb {
namespace compat {

#define RB_CUDART_NAN_F __int_as_float(0x7FFFFFFF)

struct Ray {
    float p1[3], p2[3];
    float d12, amin, amax;
    unsigned mask;
    float ai[3], af[3], da[3];
    unsigned dindex;
};

// pixel_iterate2 (hf_cuda_kernels.cuh:92-97)
__device__ __forceinline__ float pixel_center(float NumPixels, float PixelsDimMm, float Mag, int iterator)
{
    float result = __fdividef(-(NumPixels - 1.0f), 2.0f) * PixelsDimMm * Mag +
                   __fdividef((float)iterator, NumPixels) * NumPixels * PixelsDimMm * Mag;
    return __fdiv_rz(rintf(result * 100000.0f), 100000.0f);
}

// find_index (siddon_device_kernelsMLEM.cuh:151-185)
__device__ __forceinline__ float plane_index(float index, float amin, float amax, float p1, float p2,
                                             float plane1, float dplane)
{
    if (index > 0.0f) {
        float low = floorf(index), high = ceilf(index);
        float plane_low = (plane1 + dplane * (low - 1.0f));
        float plane_high = (plane1 + dplane * (high - 1.0f));
        float alow = __fdividef(plane_low - p1, p2 - p1);
        float ahigh = __fdividef(plane_high - p1, p2 - p1);
        if (alow >= amin && alow <= amax) return low;
        else if (ahigh >= amin && ahigh <= amax) return high;
        else return RB_CUDART_NAN_F;
    }
    return RB_CUDART_NAN_F;
}

// alpha_float (siddon_device_kernelsMLEM.cuh:218-237); mn, mx arrive unsigned
__device__ __forceinline__ float plane_alpha(unsigned mn, unsigned mx, float p1, float p2, float plane1,
                                            float dplane)
{
    float plane;
    if ((p2 - p1) > 0 && (mx - mn) > 0) {
        plane = plane1 + dplane * ((float)mn - 1.0f);
        return __fdividef(plane - p1, p2 - p1);
    } else if ((p2 - p1) < 0 && (mx - mn) > 0) {
        plane = plane1 + dplane * ((float)mx - 1.0f);
        return __fdividef(plane - p1, p2 - p1);
    }
    return RB_CUDART_NAN_F;
}

// siddon_calc_indices (siddon_device_kernelsMLEM.cuh:240-270) with bound_index (:50-58)
__device__ __forceinline__ unsigned axis_indices(float& ai, float& af, unsigned& mask, float p1, float p2,
                                                 float plane1, float plane2, float Nplanes, float amin,
                                                 float amax, float dplane)
{
    float ix, iy;
    if ((p2 - p1) > 0) {
        ix = Nplanes - __fdividef((plane2 - amin * (p2 - p1) - p1), dplane);
        iy = 1.0f + __fdividef((p1 + amax * (p2 - p1) - plane1), dplane);
    } else if ((p2 - p1) < 0) {
        ix = Nplanes - __fdividef((plane2 - amax * (p2 - p1) - p1), dplane);
        iy = 1.0f + __fdividef((p1 + amin * (p2 - p1) - plane1), dplane);
    } else {
        ix = 0;
        iy = 0;  // (the reference's mask store here is dropped by nvcc)
    }
    ix = (float)mask * plane_index(ix, amin, amax, p1, p2, plane1, dplane);
    iy = (float)mask * plane_index(iy, amin, amax, p1, p2, plane1, dplane);
    if ((iy - ix) < 0 && ix <= 1 && iy <= 1) {
        ix = 0;
        iy = 0;  // bound_index; its mask store is dropped likewise
    }
    ai = (float)mask * plane_alpha(__float2uint_rz(ix), __float2uint_rz(iy), p1, p2, plane1, dplane);
    af = (float)mask * plane_alpha(__float2uint_rz(iy), __float2uint_rz(ix), p1, p2, plane1, dplane);
    return __float2uint_rz(iy - ix);
}

// calc_points12 (siddon_device_kernelsMLEM.cuh:305-331) + siddon_alpha_limits
// (siddon_kernelsMLEM.cuh:103-149)
__device__ __forceinline__ void setup(const CompatGeom& G, float angle, int u, int v, Ray& r)
{
    float det_x = pixel_center(G.NumAxPixels_f, G.AxPixDimMm, G.M, u);
    float det_y = G.R - G.Rf;
    float det_z = pixel_center(G.NumTAxPixels_f, G.TAxPixDimMm, G.M, v);
    det_x = __fdividef(G.R, (G.Ry + G.RM[3] * det_x + G.RM[5] * det_z)) * (G.RM[0] * det_x + G.RM[2] * det_z + G.Dx);
    det_z = __fdividef(G.R, (G.Ry + G.RM[3] * det_x + G.RM[5] * det_z)) * (G.RM[6] * det_x + G.RM[8] * det_z + G.Dz);
    float cos_a = cospif(__fdividef(angle, 180.0f));
    float sin_a = sinpif(__fdividef(angle, 180.0f));
    r.p1[0] = G.Xs[0] * cos_a + G.Xs[1] * sin_a;
    r.p1[1] = -G.Xs[0] * sin_a + G.Xs[1] * cos_a;
    r.p1[2] = G.Xs[2];
    r.p2[0] = det_x * cos_a + det_y * sin_a;
    r.p2[1] = -det_x * sin_a + det_y * cos_a;
    r.p2[2] = det_z;
    r.d12 = sqrtf((r.p2[0] - r.p1[0]) * (r.p2[0] - r.p1[0]) + (r.p2[1] - r.p1[1]) * (r.p2[1] - r.p1[1]) +
                  (r.p2[2] - r.p1[2]) * (r.p2[2] - r.p1[2]));
    float a1[3], aN[3];
    for (int k = 0; k < 3; ++k) {  // calc_alpha_1N (siddon_device_kernelsMLEM.cuh:71-85)
        if ((r.p2[k] - r.p1[k]) != 0) {
            a1[k] = __fdividef(G.Pi[k] - r.p1[k], r.p2[k] - r.p1[k]);
            aN[k] = __fdividef(G.Pf[k] - r.p1[k], r.p2[k] - r.p1[k]);
        } else {
            a1[k] = RB_CUDART_NAN_F;
            aN[k] = RB_CUDART_NAN_F;
        }
    }
    float amin = fmaxf(fmaxf(fmaxf(0, fminf(a1[0], aN[0])), fminf(a1[1], aN[1])), fminf(a1[2], aN[2]));
    float amax = fminf(fminf(fminf(1, fmaxf(a1[0], aN[0])), fmaxf(a1[1], aN[1])), fmaxf(a1[2], aN[2]));
    unsigned mask = 1u;  // calc_mask (:88-98) as the GPU build evaluates it
    amin = (float)mask * amin;
    amax = (float)mask * amax;
    unsigned idx[3];
#pragma unroll
    for (int k = 0; k < 3; ++k)
        idx[k] = axis_indices(r.ai[k], r.af[k], mask, r.p1[k], r.p2[k], G.Pi[k], G.Pf[k], (float)G.dims[k] + 1.0f,
                              amin, amax, G.Pd[k]);
    r.dindex = idx[0] + 1 + idx[1] + 1 + idx[2] + 1 + 1;
#pragma unroll
    for (int k = 0; k < 3; ++k) r.da[k] = fabsf(__fdividef(G.Pd[k], r.p2[k] - r.p1[k]));  // delta_alpha (:100-113)
    r.mask = mask;
    r.amin = amin;
    r.amax = amax;
}

// alpha_bound (siddon_device_kernelsMLEM.cuh:134-148)
__device__ __forceinline__ float clamp_alpha(float a, float ai, float af, float amax)
{
    if (a >= ai && a <= af) return a;
    else if (a > af) return amax;
    return RB_CUDART_NAN_F;
}

__device__ __forceinline__ bool same_bits(float a, float b) { return __float_as_uint(a) == __float_as_uint(b); }

struct State {
    float a[3];
    float cur, next;
};

// siddon_begin (siddon_kernelsMLEM.cuh:283-303)
__device__ __forceinline__ void begin(const Ray& r, State& s)
{
    s.a[0] = r.mask * r.ai[0];
    s.a[1] = r.mask * r.ai[1];
    s.a[2] = r.mask * r.ai[2];
    s.next = fminf(fminf(r.ai[0], r.ai[1]), r.ai[2]);
    s.cur = RB_CUDART_NAN_F;
}

// siddon_sort_alpha (siddon_kernelsMLEM.cuh:153-190).  Returns true when the
// step left the state unchanged with next == current: every later step
// repeats it and yields a zero-length segment, so the caller may stop.
__device__ __forceinline__ bool step(const Ray& r, State& s)
{
    const float a0 = s.a[0], a1 = s.a[1], a2 = s.a[2], n0 = s.next;
    s.cur = s.next;
    if (s.cur == s.a[0]) {
        s.a[0] = s.a[0] + r.da[0];
        s.a[0] = clamp_alpha(s.a[0], r.ai[0], r.af[0], r.amax);
    } else if (s.cur == s.a[1]) {
        s.a[1] = s.a[1] + r.da[1];
        s.a[1] = clamp_alpha(s.a[1], r.ai[1], r.af[1], r.amax);
    } else if (s.cur == s.a[2]) {
        s.a[2] = s.a[2] + r.da[2];
        s.a[2] = clamp_alpha(s.a[2], r.ai[2], r.af[2], r.amax);
    }
    s.next = fminf(fminf(s.a[0], s.a[1]), s.a[2]);
    return same_bits(a0, s.a[0]) && same_bits(a1, s.a[1]) && same_bits(a2, s.a[2]) && same_bits(n0, s.next) &&
           same_bits(s.next, s.cur);
}

// Segment of siddon_fp_calc_ray_path / siddon_bp_calc_ray_path /
// siddon_fp_end / siddon_bp_end (siddon_kernelsMLEM.cuh:193-279, 307-411):
// midpoint voxel and length; -1 when there is no in-range segment.
__device__ __forceinline__ int segment(const CompatGeom& G, const Ray& r, float a_hi, float a_lo, float& len)
{
    int ix = -1, iy = -1, iz = -1;
    float ray_length = 0.0f;
    if (a_hi > a_lo) {
        float alpha_mid = __fdividef((a_hi + a_lo), 2.0f);
        ray_length = r.d12 * (a_hi - a_lo);
        ix = __float2int_rz((__fdividef((r.p1[0] + alpha_mid * (r.p2[0] - r.p1[0]) - G.Pi[0]), G.Pd[0])));
        iy = __float2int_rz((__fdividef((r.p1[1] + alpha_mid * (r.p2[1] - r.p1[1]) - G.Pi[1]), G.Pd[1])));
        iz = __float2int_rz((__fdividef((r.p1[2] + alpha_mid * (r.p2[2] - r.p1[2]) - G.Pi[2]), G.Pd[2])));
    }
    len = ray_length;
    if (ix >= 0 && ix < G.dims[0] && iy >= 0 && iy < G.dims[1] && iz >= 0 && iz < G.dims[2])
        return (int)((unsigned)iz * (unsigned)(G.dims[1] * G.dims[0]) + (unsigned)iy * (unsigned)G.dims[0] + (unsigned)ix);
    return -1;
}

// ---- kernels -------------------------------------------------------------------

__device__ __forceinline__ float view_angle(const float* angles, unsigned view) { return angles[view]; }

// Per-view loopN = max delta_index (siddon_commons::a_calc_initial_limits,
// hf_siddon_class.hpp:93-106), computed on the device.
__global__ void loopn_kernel(CompatGeom G, const float* __restrict__ angles, unsigned view0,
                             unsigned* __restrict__ loopN)
{
    const int u = blockIdx.x * blockDim.x + threadIdx.x;
    const int v = blockIdx.y * blockDim.y + threadIdx.y;
    const unsigned view = view0 + blockIdx.z;
    unsigned d = 0;
    if (u < G.Nu && v < G.Nv) {
        Ray r;
        setup(G, view_angle(angles, view), u, v, r);
        d = r.dindex;
    }
    for (int o = 16; o > 0; o >>= 1) d = max(d, __shfl_xor_sync(0xffffffffu, d, o));
    if ((threadIdx.x & 31) == 0 && d) atomicMax(&loopN[view], d);
}

__global__ void setup_dump_kernel(CompatGeom G, float angle, float* amin, float* amax, float* d12, unsigned* mask,
                                  float* ai, float* af, float* da, float* p1, float* p2, unsigned* dindex)
{
    const int u = blockIdx.x * blockDim.x + threadIdx.x;
    const int v = blockIdx.y * blockDim.y + threadIdx.y;
    if (u >= G.Nu || v >= G.Nv) return;
    const size_t n = (size_t)u + (size_t)v * G.Nu;
    Ray r;
    setup(G, angle, u, v, r);
    amin[n] = r.amin;
    amax[n] = r.amax;
    d12[n] = r.d12;
    mask[n] = r.mask;
    dindex[n] = r.dindex;
    for (int k = 0; k < 3; ++k) {
        ai[3 * n + k] = r.ai[k];
        af[3 * n + k] = r.af[k];
        da[3 * n + k] = r.da[k];
        p1[3 * n + k] = r.p1[k];
        p2[3 * n + k] = r.p2[k];
    }
}

__global__ void trace_kernel(CompatGeom G, float angle, unsigned loopN, int nrays, const int* __restrict__ rays,
                             int cap, int* __restrict__ idx_out, float* __restrict__ len_out)
{
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= nrays) return;
    const int n = rays[q];
    Ray r;
    setup(G, angle, n % G.Nu, n / G.Nu, r);
    State s;
    begin(r, s);
    int* io = idx_out + (size_t)q * cap;
    float* lo = len_out + (size_t)q * cap;
    for (int k = 0; k < cap; ++k) {
        io[k] = -1;
        lo[k] = 0.0f;
    }
    unsigned k = 0;
    bool fixed = false;
    for (; k < loopN && !fixed; ++k) {
        fixed = step(r, s);
        float len;
        int id = segment(G, r, s.next, s.cur, len);
        if ((int)k < cap) {
            io[k] = id;
            lo[k] = id >= 0 ? len : 0.0f;
        }
    }
    float len;
    int id = segment(G, r, r.amax, s.cur, len);
    if ((int)loopN < cap) {
        io[loopN] = id;
        lo[loopN] = id >= 0 ? len : 0.0f;
    }
}

// Forward projection: image = sum over steps, in step order, of len*f[idx],
// each product and each sum rounded once (siddon_fp_calc_ray_path writes the
// product, siddon_add adds it).  mode 0: store Hf; mode 1: store
// divide1(g, Hf) (hf_cuda_kernels.cuh:370-387) and track max |ratio| per view.
template <int MODE>
__global__ void fp_kernel(CompatGeom G, const float* __restrict__ angles, const unsigned* __restrict__ loopN,
                          unsigned view0, const float* __restrict__ vol, const float* __restrict__ g,
                          float* __restrict__ out, unsigned* __restrict__ maxabs)
{
    const int u = blockIdx.x * blockDim.x + threadIdx.x;
    const int v = blockIdx.y * blockDim.y + threadIdx.y;
    const unsigned view = view0 + blockIdx.z;
    if (u >= G.Nu || v >= G.Nv) return;
    const size_t n = (size_t)blockIdx.z * G.Nu * G.Nv + (size_t)u + (size_t)v * G.Nu;
    Ray r;
    setup(G, view_angle(angles, view), u, v, r);
    // Rays with mask 0 are not skipped: when a later axis clears the mask the
    // traversal can still produce segments, exactly as in the reference.
    float acc = 0.0f;
    {
        State s;
        begin(r, s);
        const unsigned L = loopN[view];
        bool fixed = false;
        for (unsigned k = 0; k < L && !fixed; ++k) {
            fixed = step(r, s);
            float len;
            int id = segment(G, r, s.next, s.cur, len);
            float t = id >= 0 ? __fmul_rn(len, __ldg(vol + id)) : 0.0f;
            acc = __fadd_rn(acc, t);
        }
        float len;
        int id = segment(G, r, r.amax, s.cur, len);
        float t = id >= 0 ? __fmul_rn(len, __ldg(vol + id)) : 0.0f;
        acc = __fadd_rn(acc, t);
    }
    if (MODE == 0) {
        out[n] = acc;
    } else {
        float gv = g[n];
        float ratio = (acc != 0) ? __fdividef(gv, acc) : 0.0f;
        out[n] = ratio;
        // one atomic per warp: every ray of the block belongs to this view, and a
        // max does not depend on the order it is taken in
        const unsigned active = __activemask();
        const unsigned bits = __reduce_max_sync(active, __float_as_uint(fabsf(ratio)));
        const unsigned lane = (threadIdx.x + threadIdx.y * blockDim.x) & 31u;
        if (bits && (active & ((1u << lane) - 1u)) == 0u) atomicMax(&maxabs[view], bits);
    }
}

__global__ void maxabs_kernel(const float* __restrict__ img, size_t n, unsigned* __restrict__ out)
{
    unsigned m = 0;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
        m = max(m, __float_as_uint(fabsf(img[i])));
    for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0 && m) atomicMax(out, m);
}

// Fixed-point scale for a view.  Every segment lies on its ray, so
// |len*img| <= maxabs * max_len with max_len >= every source-detector
// distance; a voxel receives at most 2^count_bits contributions (one per ray
// of the view), so with scale = 2^F, F = 62 - count_bits - e and
// maxabs*max_len < 2^e, the per-voxel sum stays below 2^62.
__device__ __forceinline__ double fix_scale(unsigned maxabs_bits, float max_len, int count_bits)
{
    float m = __uint_as_float(maxabs_bits);
    if (!(m > 0.0f) || !isfinite(m)) return 0.0;
    int e;
    frexp((double)m * (double)max_len, &e);
    int F = 62 - count_bits - e;
    if (F > 200) F = 200;
    return ldexp(1.0, F);
}

// Back projection scatter: per in-range segment, len*img[n] added in 64-bit
// fixed point (siddon_bp_calc_ray_path + the atomic kernel,
// siddon_kernelsMLEM.cuh:307-365).
// Views view0 + blockIdx.z, view z reading img + z * img_stride, all scaled by
// maxabs[slot] (one view's bound, or the bound over all the views launched).
__global__ void bp_scatter_kernel(CompatGeom G, const float* __restrict__ angles, const unsigned* __restrict__ loopN,
                                  unsigned view0, const float* __restrict__ img, size_t img_stride,
                                  const unsigned* __restrict__ maxabs, unsigned slot, float chord, int count_bits,
                                  unsigned long long* __restrict__ acc)
{
    const int u = blockIdx.x * blockDim.x + threadIdx.x;
    const int v = blockIdx.y * blockDim.y + threadIdx.y;
    if (u >= G.Nu || v >= G.Nv) return;
    const unsigned view = view0 + blockIdx.z;
    const size_t n = (size_t)blockIdx.z * img_stride + (size_t)u + (size_t)v * G.Nu;
    const double scale = fix_scale(maxabs[slot], chord, count_bits);
    if (scale == 0.0) return;
    Ray r;
    setup(G, view_angle(angles, view), u, v, r);
    const float gi = img[n];
    State s;
    begin(r, s);
    const unsigned L = loopN[view];
    bool fixed = false;
    for (unsigned k = 0; k < L && !fixed; ++k) {
        fixed = step(r, s);
        float len;
        int id = segment(G, r, s.next, s.cur, len);
        if (id >= 0) {
            float c = __fmul_rn(len, gi);
            long long q = __double2ll_rn((double)c * scale);
            if (q) atomicAdd(acc + id, (unsigned long long)q);
        }
    }
    float len;
    int id = segment(G, r, r.amax, s.cur, len);
    if (id >= 0) {
        float c = __fmul_rn(len, gi);
        long long q = __double2ll_rn((double)c * scale);
        if (q) atomicAdd(acc + id, (unsigned long long)q);
    }
}

// Fixed point -> float (one rounding), then out = v (overwrite) or
// out = out + v (siddon_add_bp into the running sum); the accumulator is
// cleared for the next view.
__global__ void bp_finish_kernel(unsigned long long* __restrict__ acc, size_t n, const unsigned* __restrict__ maxabs,
                                 unsigned view, float chord, int count_bits, float* __restrict__ out, int accumulate)
{
    const double scale = fix_scale(maxabs[view], chord, count_bits);
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        float v = 0.0f;
        if (scale != 0.0) {
            long long q = (long long)acc[i];
            v = (float)((double)q / scale);
            acc[i] = 0ull;
        }
        out[i] = accumulate ? __fadd_rn(out[i], v) : v;
    }
}

// out = max over views of maxabs[0 .. n) (non-negative floats as unsigned bits)
__global__ void max_views_kernel(const unsigned* __restrict__ maxabs, unsigned n, unsigned* __restrict__ out)
{
    unsigned m = 0;
    for (unsigned i = threadIdx.x; i < n; i += blockDim.x) m = max(m, maxabs[i]);
    m = __reduce_max_sync(0xffffffffu, m);
    __shared__ unsigned w[32];
    if ((threadIdx.x & 31) == 0) w[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned r = 0;
        for (unsigned k = 0; k < (blockDim.x + 31) / 32; ++k) r = max(r, w[k]);
        *out = r;
    }
}

}  // namespace compat

// ---- host side ---------------------------------------------------------------------

static dim3 ray_block() { return dim3(32, 4, 1); }
static dim3 ray_grid(const Plan& P, unsigned views)
{
    return dim3((P.cg.Nu + 31) / 32, (P.cg.Nv + 3) / 4, views);
}
static unsigned elem_blocks(size_t n) { return (unsigned)std::min<size_t>((n + 255) / 256, 148 * 16); }

// Upper bound of any source-to-pixel distance (every segment is part of one).
static float max_ray_length(const Plan& P)
{
    const recon_geometry_t& g = P.geom;
    double hu = 0.5 * g.det.NumAxPixels * (double)g.det.AxPixDimMm * std::fabs((double)g.cal.M) + std::fabs(g.cal.Dx);
    double hv = 0.5 * g.det.NumTAxPixels * (double)g.det.TAxPixDimMm * std::fabs((double)g.cal.M) + std::fabs(g.cal.Dz);
    double sc = std::fabs((double)g.cal.R) / std::max(1e-6, std::fabs((double)g.cal.Ry) - hu - hv);
    double R = std::fabs((double)g.cal.R) + std::fabs((double)g.cal.Rf);
    return (float)(2.0 * (R + sc * (hu + hv)) + 1.0);
}
static int count_bits(const Plan& P)
{
    int b = 0;
    while ((size_t(1) << b) < P.npix) ++b;
    return b + 1;
}

// Scale bounds for the sum over all plan views (compat_bp_all).  A segment
// lies on its ray between the volume's entry and exit, so it is no longer
// than the volume's diagonal.  A contribution to a voxel comes from a ray
// whose segment midpoint falls in it, i.e. a ray through the voxel's box (up
// to the index rounding): with an untilted detector those are the pixels in
// the box's shadow, at most W x H on the detector from the nearest depth the
// volume reaches, widened by three pixels each way, with at most four segments
// each.  A tilted detector falls back to one contribution per ray of the view.
static float volume_diagonal(const Plan& P)
{
    const recon_geometry_t& g = P.geom;
    const double x = g.vox.Xdim * (double)g.vox.XVoxSize, y = g.vox.Ydim * (double)g.vox.YVoxSize,
                 z = g.vox.Zdim * (double)g.vox.ZVoxSize;
    return (float)(std::sqrt(x * x + y * y + z * z) * 1.001 + 1e-3);
}

static int count_bits_all(const Plan& P)
{
    const recon_geometry_t& g = P.geom;
    double per_view = std::ldexp(1.0, count_bits(P));
    if (g.cal.xangle == 0.0f && g.cal.yangle == 0.0f && g.cal.zangle == 0.0f) {
        const double vx = std::fabs((double)g.vox.XVoxSize), vy = std::fabs((double)g.vox.YVoxSize),
                     vz = std::fabs((double)g.vox.ZVoxSize);
        const double rmax = 0.5 * std::hypot(g.vox.Xdim * vx, g.vox.Ydim * vy);
        const double dmin = std::fabs((double)g.cal.Rf) - rmax;
        const double pu = std::fabs((double)g.det.AxPixDimMm * g.cal.M), pv = std::fabs((double)g.det.TAxPixDimMm * g.cal.M);
        if (dmin > 0.0 && pu > 0.0 && pv > 0.0) {
            const double mag = std::max(std::fabs((double)g.cal.R), std::fabs((double)g.cal.Ry)) / dmin;
            const double diag = std::hypot(vx, vy), zmax = 0.5 * g.vox.Zdim * vz;
            const double W = diag * mag, H = (vz + diag * zmax / dmin) * mag;
            per_view = std::min(per_view, 4.0 * (std::ceil(W / pu) + 6.0) * (std::ceil(H / pv) + 6.0));
        }
    }
    const double total = per_view * std::max(1u, P.nviews);
    int b = 0;
    while (std::ldexp(1.0, b) < total) ++b;
    return b + 1;
}

__global__ void set_value_kernel(float* p, float v) { *p = v; }

static float* angles_dev(Plan& P) { return P.d_angles; }

recon_status_t build_compat_tables(Plan& P, cudaStream_t s)
{
    if (P.nviews == 0) return RECON_OK;
    RB_CUDA(cudaMemsetAsync(P.d_loopN, 0, (P.nviews + 1) * sizeof(unsigned), s));
    compat::loopn_kernel<<<ray_grid(P, P.nviews), ray_block(), 0, s>>>(P.cg, angles_dev(P), 0u, P.d_loopN);
    RB_CUDA(cudaGetLastError());
    return RECON_OK;
}

recon_status_t compat_view_loopN(Plan& P, float angle, unsigned slot, cudaStream_t s)
{
    float* ang = angles_dev(P);
    set_value_kernel<<<1, 1, 0, s>>>(ang + slot, angle);
    RB_CUDA(cudaMemsetAsync(P.d_loopN + slot, 0, sizeof(unsigned), s));
    compat::loopn_kernel<<<ray_grid(P, 1), ray_block(), 0, s>>>(P.cg, ang, slot, P.d_loopN);
    RB_CUDA(cudaGetLastError());
    return RECON_OK;
}

recon_status_t compat_fp(Plan& P, const float* vol, unsigned first, unsigned count, bool scratch_slot,
                         float angle_scratch, float* out, cudaStream_t s)
{
    if (scratch_slot) {
        RB_CHECK(compat_view_loopN(P, angle_scratch, P.nviews, s));
        first = P.nviews;
        count = 1;
    }
    compat::fp_kernel<0><<<ray_grid(P, count), ray_block(), 0, s>>>(P.cg, angles_dev(P), P.d_loopN, first, vol,
                                                                     nullptr, out, nullptr);
    RB_CUDA(cudaGetLastError());
    return RECON_OK;
}

static recon_status_t compat_bp_into(Plan& P, const float* img, unsigned view, float* out, bool accumulate,
                                     bool have_maxabs, cudaStream_t s)
{
    const float chord = max_ray_length(P);
    const int cbits = count_bits(P);
    if (!have_maxabs) {
        RB_CUDA(cudaMemsetAsync(P.d_maxabs + view, 0, sizeof(unsigned), s));
        compat::maxabs_kernel<<<elem_blocks(P.npix), 256, 0, s>>>(img, P.npix, P.d_maxabs + view);
        RB_CUDA(cudaGetLastError());
    }
    compat::bp_scatter_kernel<<<ray_grid(P, 1), ray_block(), 0, s>>>(P.cg, angles_dev(P), P.d_loopN, view, img, 0,
                                                                      P.d_maxabs, view, chord, cbits, P.d_fix);
    RB_CUDA(cudaGetLastError());
    compat::bp_finish_kernel<<<elem_blocks(P.nvox), 256, 0, s>>>(P.d_fix, P.nvox, P.d_maxabs, view, chord, cbits,
                                                                  out, accumulate ? 1 : 0);
    RB_CUDA(cudaGetLastError());
    return RECON_OK;
}

recon_status_t compat_bp_view(Plan& P, const float* img, unsigned view, bool scratch_slot, float angle_scratch,
                              float* out, bool accumulate, cudaStream_t s)
{
    if (scratch_slot) {
        RB_CHECK(compat_view_loopN(P, angle_scratch, P.nviews, s));
        view = P.nviews;
    }
    return compat_bp_into(P, img, view, out, accumulate, false, s);
}

// Back projection of every plan view's image (img + n * img_stride) summed in
// one 64-bit fixed-point accumulator, scaled by the bound over all views
// (maxabs[nviews + 1], which the caller sets), and rounded to float once into
// out.  The reference adds each view's back projection into a float image
// (hf_siddon_recon.hpp:437-476); one rounding of the exact sum differs from
// that by float rounding only.
static recon_status_t compat_bp_all(Plan& P, const float* img, size_t img_stride, float* out, cudaStream_t s)
{
    const float chord = volume_diagonal(P);
    const int cbits = count_bits_all(P);
    const unsigned all = P.nviews + 1;
    compat::bp_scatter_kernel<<<ray_grid(P, P.nviews), ray_block(), 0, s>>>(P.cg, angles_dev(P), P.d_loopN, 0u, img,
                                                                             img_stride, P.d_maxabs, all, chord, cbits,
                                                                             P.d_fix);
    RB_CUDA(cudaGetLastError());
    compat::bp_finish_kernel<<<elem_blocks(P.nvox), 256, 0, s>>>(P.d_fix, P.nvox, P.d_maxabs, all, chord, cbits, out,
                                                                  0);
    RB_CUDA(cudaGetLastError());
    return RECON_OK;
}

recon_status_t compat_sensitivity(Plan& P, float* sens, cudaStream_t s)
{
    if (P.nviews == 0) {
        RB_CUDA(cudaMemsetAsync(sens, 0, P.nvox * sizeof(float), s));
        return RECON_OK;
    }
    RB_CHECK(launch_fill(P.d_view_img, 1.0f, P.npix, s));
    set_value_kernel<<<1, 1, 0, s>>>(reinterpret_cast<float*>(P.d_maxabs + P.nviews + 1), 1.0f);
    RB_CUDA(cudaGetLastError());
    return compat_bp_all(P, P.d_view_img, 0, sens, s);
}

// m_mlem_single_iteration (hf_siddon_recon.hpp:437-476): FP and ratio of every
// view (the image is fixed within the iteration, so the views' order does not
// matter), the back projections of all ratios summed exactly, then
// f = f*Ht; f = divide1(f, sens).
recon_status_t compat_mlem_iteration(Plan& P, const float* g, float* f, cudaStream_t s)
{
    if (P.nviews == 0) return RECON_OK;
    RB_CUDA(cudaMemsetAsync(P.d_maxabs, 0, (P.nviews + 2) * sizeof(unsigned), s));
    float* ratio = static_cast<float*>(P.d_ratio);
    compat::fp_kernel<1><<<ray_grid(P, P.nviews), ray_block(), 0, s>>>(P.cg, angles_dev(P), P.d_loopN, 0u, f, g, ratio,
                                                                        P.d_maxabs);
    RB_CUDA(cudaGetLastError());
    compat::max_views_kernel<<<1, 256, 0, s>>>(P.d_maxabs, P.nviews, P.d_maxabs + P.nviews + 1);
    RB_CUDA(cudaGetLastError());
    RB_CHECK(compat_bp_all(P, ratio, P.npix, P.d_ht, s));
    return launch_update(f, P.d_ht, P.d_sens, P.nvox, true, s);
}

// divide1(g, FP(f)) for every view, into a full ratio sinogram (input of the
// voxel-driven back projector).
recon_status_t compat_fp_ratio_all(Plan& P, const float* vol, const float* g, float* ratio, cudaStream_t s)
{
    RB_CUDA(cudaMemsetAsync(P.d_maxabs, 0, (P.nviews + 1) * sizeof(unsigned), s));
    compat::fp_kernel<1><<<ray_grid(P, P.nviews), ray_block(), 0, s>>>(P.cg, angles_dev(P), P.d_loopN, 0u, vol, g,
                                                                        ratio, P.d_maxabs);
    RB_CUDA(cudaGetLastError());
    return RECON_OK;
}

// ---- parity entry points --------------------------------------------------------------

recon_status_t compat_setup_dump(Plan& P, float angle, float* h[10], unsigned* loopN)
{
    cudaStream_t s = 0;
    const size_t n = P.npix;
    float *amin, *amax, *d12, *ai, *af, *da, *p1, *p2;
    unsigned *mask, *dindex;
    size_t bytes = n * (3 * 4 + 4 + 4 + 5 * 12) + 16;
    char* base = nullptr;
    RB_CUDA(cudaMalloc(&base, bytes));
    char* q = base;
    auto take = [&](size_t b) { char* r = q; q += b; return r; };
    amin = (float*)take(n * 4); amax = (float*)take(n * 4); d12 = (float*)take(n * 4);
    mask = (unsigned*)take(n * 4); ai = (float*)take(n * 12); af = (float*)take(n * 12);
    da = (float*)take(n * 12); p1 = (float*)take(n * 12); p2 = (float*)take(n * 12);
    dindex = (unsigned*)take(n * 4);
    compat::setup_dump_kernel<<<ray_grid(P, 1), ray_block(), 0, s>>>(P.cg, angle, amin, amax, d12, mask, ai, af, da,
                                                                      p1, p2, dindex);
    cudaError_t e = cudaGetLastError();
    if (e == cudaSuccess) e = cudaStreamSynchronize(cudaStreamLegacy);
    void* dev[10] = {amin, amax, d12, mask, ai, af, da, p1, p2, dindex};
    size_t sz[10] = {n * 4, n * 4, n * 4, n * 4, n * 12, n * 12, n * 12, n * 12, n * 12, n * 4};
    for (int k = 0; k < 10 && e == cudaSuccess; ++k) e = cudaMemcpy(h[k], dev[k], sz[k], cudaMemcpyDeviceToHost);
    cudaFree(base);
    if (e != cudaSuccess) return cuda_fail(e, "compat setup dump");
    unsigned mx = 0;
    const unsigned* di = reinterpret_cast<const unsigned*>(h[9]);
    for (size_t i = 0; i < n; ++i) mx = std::max(mx, di[i]);
    *loopN = mx;
    return RECON_OK;
}

recon_status_t compat_trace(Plan& P, float angle, int nrays, const int* rays, int cap, int* idx, float* len,
                            unsigned* loopN_out)
{
    RB_CHECK(compat_view_loopN(P, angle, P.nviews, 0));
    unsigned loopN = 0;
    RB_CUDA(cudaMemcpy(&loopN, P.d_loopN + P.nviews, sizeof(unsigned), cudaMemcpyDeviceToHost));
    int *d_rays = nullptr, *d_idx = nullptr;
    float* d_len = nullptr;
    cudaError_t e = cudaMalloc(&d_rays, sizeof(int) * std::max(1, nrays));
    if (e == cudaSuccess) e = cudaMalloc(&d_idx, sizeof(int) * (size_t)std::max(1, nrays) * cap);
    if (e == cudaSuccess) e = cudaMalloc(&d_len, sizeof(float) * (size_t)std::max(1, nrays) * cap);
    if (e == cudaSuccess) e = cudaMemcpy(d_rays, rays, sizeof(int) * nrays, cudaMemcpyHostToDevice);
    if (e == cudaSuccess && nrays > 0) {
        compat::trace_kernel<<<(nrays + 127) / 128, 128>>>(P.cg, angle, loopN, nrays, d_rays, cap, d_idx, d_len);
        e = cudaGetLastError();
        if (e == cudaSuccess) e = cudaStreamSynchronize(cudaStreamLegacy);
        if (e == cudaSuccess) e = cudaMemcpy(idx, d_idx, sizeof(int) * (size_t)nrays * cap, cudaMemcpyDeviceToHost);
        if (e == cudaSuccess) e = cudaMemcpy(len, d_len, sizeof(float) * (size_t)nrays * cap, cudaMemcpyDeviceToHost);
    }
    cudaFree(d_rays);
    cudaFree(d_idx);
    cudaFree(d_len);
    if (e != cudaSuccess) return cuda_fail(e, "compat trace");
    *loopN_out = loopN;
    return RECON_OK;
}

}  // namespace rb
