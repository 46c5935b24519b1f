// exact.cu -- EXACT arithmetic: a true Siddon projector pair.
//
// Ray parameterisation.  A ray runs from the source p1 to the pixel centre p2;
// the reference parameterises it by alpha in [0,1]
// (siddon_device_kernelsMLEM.cuh:71-85).  Here the parameter is
// t = R*alpha - Rf, the ray's depth along the view's central axis in mm,
// which is 0 at the isocentre plane, so the plane crossings inside the volume
// all have |t| of a few tens of mm and FP32 resolves them to ~4e-6 mm.  Plane
// k of an axis crosses the ray at t(k) = fmaf(float(k - kc), S, O); S, O and
// kc are computed once per ray in FP64 (kc = the plane nearest t = 0), and
// every later use -- forward traversal, back-projection gather, entry and
// exit -- evaluates planes with that same expression.  Both projectors
// therefore assign every (ray, voxel) pair the same FP32 length
//     L = w * (min(hi_x, hi_y, hi_z) - max(lo_x, lo_y, lo_z)),
// w = |p2 - p1| / R, and are exact transposes of each other.
//
// Separability.  With no detector tilt the x/y crossings of ray (u, v) depend
// only on (view, u) and the z crossings only on v (the source lies in z = 0),
// so the tables are [view][u] for x and y, [v] for z and [v][u] for w.
//
// Forward projection: one thread per ray, the voxel walk fully in registers,
// the step count known before the loop (no exit test on planes); views whose
// detector rows run along y read an xy-transposed copy of the volume so that
// a warp's gathers stay coalesced.  Back projection: the same walk per ray,
// z-slab by z-slab, adding L * value to 64-bit fixed-point accumulators with
// integer atomics (exact, order-independent sums, so results are
// bit-reproducible); a finishing pass per slab converts to float and applies
// the MLEM update f <- f * Ht / sens.
#include "exact_device.cuh"
#include "internal.h"

#include <algorithm>
#include <climits>
#include <cmath>
#include <cstdio>
#include <map>
#include <mutex>
#include <string>
#include <type_traits>

namespace rb {
namespace exact {

// ---- FP64 table set-up --------------------------------------------------------------

struct GeomD {
    double R, Rf, Ry, Dx, Dz;
    double du, dv;  // pixel pitch * M
    int Nu, Nv;
    int dims[3];
    double vox[3], P0[3];
};

// Pixel centre of pixel_iterate2 (hf_cuda_kernels.cuh:92-97) in FP64: the
// nominal centre rounded to the 1e-5 mm grid.
__device__ __forceinline__ double pixel_center_d(int N, double d, int i)
{
    double c = -((double)N - 1.0) / 2.0 * d + (double)i * d;
    return rint(c * 1e5) / 1e5;
}

// Plane parameters of one axis: p1 + alpha*dp crosses plane P0 + k*vox at
// t = R*alpha - Rf.
__device__ __forceinline__ void axis_params(const GeomD& G, double p1, double dp, double P0, double vox, float& S,
                                            float& O, int& kc)
{
    const double tiny = 1e-9 * G.R;
    if (fabs(dp) < tiny) dp = (dp < 0.0) ? -tiny : tiny;  // axis-parallel ray: push its planes far away
    double kstar = (p1 + (G.Rf / G.R) * dp - P0) / vox;     // plane index at t = 0
    if (kstar > 1048576.0) kstar = 1048576.0;
    if (kstar < -1048576.0) kstar = -1048576.0;
    double k = rint(kstar);
    S = (float)(G.R * vox / dp);
    O = (float)(G.R * (P0 + k * vox - p1) / dp - G.Rf);
    kc = (int)k;
}

__global__ void xy_table_kernel(GeomD G, const float* __restrict__ angles, unsigned view0, unsigned nview,
                                float4* __restrict__ txy, int2* __restrict__ kxy, float2* __restrict__ cs)
{
    const int u = blockIdx.x * blockDim.x + threadIdx.x;
    const unsigned view = view0 + blockIdx.y;
    if (u >= G.Nu || blockIdx.y >= nview) return;
    const double th = (double)angles[view] / 180.0;
    const double c = cospi(th), s = sinpi(th);
    // detector x of column u after the misalignment shift/scale (no tilt):
    // calc_points12, siddon_device_kernelsMLEM.cuh:310-316
    const double det_x = G.R / G.Ry * (pixel_center_d(G.Nu, G.du, u) + G.Dx);
    const double det_y = G.R - G.Rf;
    const double p1x = -G.Rf * s, p1y = -G.Rf * c;
    const double p2x = det_x * c + det_y * s, p2y = -det_x * s + det_y * c;
    float4 T;
    int2 K;
    axis_params(G, p1x, p2x - p1x, G.P0[0], G.vox[0], T.x, T.y, K.x);
    axis_params(G, p1y, p2y - p1y, G.P0[1], G.vox[1], T.z, T.w, K.y);
    txy[(size_t)view * G.Nu + u] = T;
    kxy[(size_t)view * G.Nu + u] = K;
    if (u == 0) cs[view] = make_float2((float)c, (float)s);
}

// Views a quarter turn apart.  With a square volume (X = Y, equal x and y voxel
// sizes, P0 = -X vox / 2 on both axes) and view n + q at angle(n) + 90 degrees,
// ray (view n + q, u) is ray (view n, u) turned about the z axis, (x, y) ->
// (y, -x) by xy_table_kernel's formulas: its x planes are view n's y planes
// and its y plane k is view n's x plane X - k.  So its entries are
//     {Sx, Ox, Sy, Oy}' = {Sy, Oy, -Sx, Ox},  {kcx, kcy}' = {kcy, X - kcx},
// as fmaf(k - (X - kc), -S, O) = fmaf((X - k) - kc, S, O) bit for bit.  Views
// q .. 4q-1 are derived this way from views 0 .. q-1 (one thread per (view n <
// q, u)), which makes every length either projector gives to (column (i, j),
// view n + q) the one it gives to (column (X-1-j, i), view n), bit for bit.
__global__ void quarter_turn_table_kernel(int X, int Nu, unsigned q, float4* __restrict__ txy, int2* __restrict__ kxy,
                                          float2* __restrict__ cs)
{
    const int u = blockIdx.x * blockDim.x + threadIdx.x;
    const unsigned n = blockIdx.y;
    if (u >= Nu) return;
    float4 T = txy[(size_t)n * Nu + u];
    int2 K = kxy[(size_t)n * Nu + u];
    float2 c = cs[n];
    for (unsigned r = 1; r < 4; ++r) {
        T = make_float4(T.z, T.w, -T.x, T.y);
        K = make_int2(K.y, X - K.x);
        c = make_float2(-c.y, c.x);  // {cos, sin} of the angle plus 90 degrees
        txy[(size_t)(n + r * q) * Nu + u] = T;
        kxy[(size_t)(n + r * q) * Nu + u] = K;
        if (u == 0) cs[n + r * q] = c;
    }
}

__global__ void z_table_kernel(GeomD G, ZParam* __restrict__ zp)
{
    const int v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= G.Nv) return;
    const double det_z = G.R / G.Ry * (pixel_center_d(G.Nv, G.dv, v) + G.Dz);
    ZParam z;
    axis_params(G, 0.0, det_z, G.P0[2], G.vox[2], z.S, z.O, z.kc);
    z.inv_S = (float)(1.0 / (double)z.S);
    zp[v] = z;
}

// w = |p2 - p1| / R per ray, stored [v][u] (w) and in the detector-column layout
// [u][v] (wq)
__global__ void w_table_kernel(GeomD G, float* __restrict__ w, float* __restrict__ wq)
{
    const int u = blockIdx.x * blockDim.x + threadIdx.x;
    const int v = blockIdx.y;
    if (u >= G.Nu) return;
    const double det_x = G.R / G.Ry * (pixel_center_d(G.Nu, G.du, u) + G.Dx);
    const double det_z = G.R / G.Ry * (pixel_center_d(G.Nv, G.dv, v) + G.Dz);
    const float wv = (float)(sqrt(det_x * det_x + G.R * G.R + det_z * det_z) / G.R);
    w[(size_t)v * G.Nu + u] = wv;
    wq[(size_t)u * G.Nv + v] = wv;
}

// MODE 0: out = projection (w * sum L_t * f).  MODE 1 (MLEM): out = w * ratio
// with ratio = g / Hf (0 where Hf == 0), the Siddon back projector's input.
// MODE 2: out = ratio (input of the voxel-driven back projector).  All stored
// [view][v][u], so that a warp's 32 rays (adjacent detector columns) store 128
// contiguous bytes; the gather back projectors read a transposed copy
// (to_columns_kernel).
template <bool KAHAN, int MODE, class GT, class OT>
__global__ void __launch_bounds__(128, 10) fp_kernel(ExactGeom G, const float4* __restrict__ txy,
                                                  const int2* __restrict__ kxy, const ZParam* __restrict__ zp,
                                                  const float* __restrict__ wtab, const float2* __restrict__ cs,
                                                  const uint2* __restrict__ tiles, unsigned view0,
                                                  const float* __restrict__ vol, const float* __restrict__ vol_t,
                                                  const GT* __restrict__ g, OT* __restrict__ out)
{
    const RayPos R = ray_pos(tiles, view0);
    const int u = R.u, v = R.v;
    const unsigned view = R.view;
    if (u >= G.Nu || v >= G.Nv) return;
    const VolView V = vol_view_for(__ldg(cs + view), vol, vol_t, G.X, G.Y);
    const size_t pix = (size_t)u + (size_t)v * G.Nu;
    const size_t n = (size_t)(view - view0) * G.Nu * G.Nv + pix;
    const float4 T = __ldg(txy + (size_t)view * G.Nu + u);
    const int2 K = __ldg(kxy + (size_t)view * G.Nu + u);
    const ZParam Z = zp[v];
    const float w = __ldg(wtab + pix);

    const float acc = fp_ray_sum<KAHAN>(G, T, K, Z, V);
    const float hf = w * acc;
    if (MODE == 0) {
        store_val<OT>(out + n, hf);
    } else {
        const float gv = load_val<GT>(g + n);
        const float ratio = (hf != 0.0f) ? __fdiv_rn(gv, hf) : 0.0f;
        store_val<OT>(out + n, MODE == 1 ? ratio * w : ratio);
    }
}

// ---- back projection (gather, one warp per (x, y) column) -----------------------------------
//
// A warp owns the column of voxels (i, j, *) and gathers, view by view, every
// ray that crosses it; lane l owns the voxels k = k0 + l + 32 s (s < SLOTS) of
// a chunk of 32 * SLOTS slices and keeps their sums in registers.  Per view the
// column's four corners, projected from the source, give the detector columns
// u whose rays can cross it; for each, [A, B] is the column's piece of those
// rays in t (from the x and y planes, evaluated as the forward walk does).  A
// ray of row v crosses heights z = dz_v * (t + Rf) / R there, so it can meet
// voxel [z_k, z_k+1] only if dz_v lies between min(z_k R / (A+Rf), z_k R /
// (B+Rf)) and max(z_k+1 R / (A+Rf), z_k+1 R / (B+Rf)): a few FMAs per voxel
// give its candidate rows (one, sometimes none or two, where rows are further
// apart than voxels), widened by 0.002 row.  Each candidate's length
//     L = min(B, hi_z) - max(A, lo_z)
// takes the row's z planes exactly as the forward walk does, so the pair
// stays an exact transpose, and is added as acc = fmaf(L, value, acc) in the
// order views, u: each voxel's first candidate rows into a register, any
// further ones into a shared-memory sum, and Ht = register + shared sum, so
// the result is deterministic.
//
// Values are read in the detector-column layout [view][u][v] (view_stride
// elements per view; 0 for the weights w of the sensitivity): a warp's loads of
// nearby rows of one detector column fall in one or two 128-byte lines, and a
// row's element is one add from its column.  EPI 1 (MLEM update):
// f = (sens != 0) ? f * Ht / sens : 0; EPI 0: vol = Ht; EPI 2: no image, the
// number of (ray, voxel) pairs given a positive length is added to *npairs
// (a check that the candidate margins drop no pair of the forward walk).
constexpr int kGatherWarps = 8;  // a kGatherTileX x (8 / kGatherTileX) tile of columns per CTA
constexpr int kGatherTileX = 4;
// SLOTS: voxels per lane and chunk (chunks of 32 * SLOTS slices; 8 unless the
// volume is shorter)

struct GatherConst {
    float eu, ou;  // detector column of a point (a, b) of the view frame: a / (b + Rf) * eu + ou
    float ez, oz;  // detector row of height z at depth d (t = d - Rf):      z / d * ez + oz
    int vec4;      // X % 4 == 0 and the volume, sensitivity 16-byte aligned: float4 epilogue
};

// MLEM update of one voxel, as update_kernel computes it
__device__ __forceinline__ float gather_update(float f, float ht, float sens)
{
    return (sens != 0.0f) ? __fdiv_rn(__fmul_rn(f, ht), sens) : 0.0f;
}

// The CTA's epilogue for one chunk of planes, coalesced along x.  Warp
// w = xl + kGatherTileX * yl (column i0 + xl, j0 + yl) has left its sum for
// entry e in stage[w * NE + e]; entry e belongs to plane zplane(e), or to none
// when that is negative.  EPI 0 writes the sums, EPI 1 the updated image.  With
// C.vec4 a thread moves the tile's four x-neighbours of one (plane, row) as one
// float4, otherwise one voxel, the CTA's threads walking (x, y, entry) x fastest.
template <int EPI, int NE, class ZPlane>
__device__ __forceinline__ void gather_tile_epilogue(const ExactGeom& G, bool vec4, const float* stage, int i0,
                                                     int j0, ZPlane zplane, float* __restrict__ vol,
                                                     const float* __restrict__ sens)
{
    constexpr int tx = kGatherTileX, ty = kGatherWarps / kGatherTileX;
    static_assert(tx == 4, "the float4 epilogue moves four x-neighbours");
    const size_t plane = (size_t)G.X * G.Y;
    if (vec4) {
        for (int q = threadIdx.x; q < NE * ty; q += blockDim.x) {
            const int yl = q % ty, e = q / ty;
            const int k = zplane(e), j = j0 + yl;
            if (k < 0 || j >= G.Y) continue;
            const size_t v = (size_t)k * plane + (size_t)j * G.X + (size_t)i0;
            const float* h = stage + yl * tx * NE + e;
            float4 o = make_float4(h[0], h[NE], h[2 * NE], h[3 * NE]);
            if (EPI == 1) {
                const float4 f = *reinterpret_cast<const float4*>(vol + v);
                const float4 sv = *reinterpret_cast<const float4*>(sens + v);
                o = make_float4(gather_update(f.x, o.x, sv.x), gather_update(f.y, o.y, sv.y),
                                gather_update(f.z, o.z, sv.z), gather_update(f.w, o.w, sv.w));
            }
            *reinterpret_cast<float4*>(vol + v) = o;
        }
    } else {
        for (int q = threadIdx.x; q < NE * ty * tx; q += blockDim.x) {
            const int xl = q % tx, yl = (q / tx) % ty, e = q / (tx * ty);
            const int k = zplane(e), i = i0 + xl, j = j0 + yl;
            if (k < 0 || i >= G.X || j >= G.Y) continue;
            const size_t v = (size_t)k * plane + (size_t)j * G.X + (size_t)i;
            const float h = stage[(yl * tx + xl) * NE + e];
            vol[v] = (EPI == 1) ? gather_update(vol[v], h, sens[v]) : h;
        }
    }
}

// A warp's column seen from one view: detector columns u_lo..u_hi and, for the
// first two (sl = 0, 1), the column's piece [A, B] of their rays, the row
// coefficients ca = ez / (A + Rf), cb = ez / (B + Rf) and the per-slot steps
// pa = 32 vz ca, pb = 32 vz cb of the row bounds.  flags: bit sl = the rays of
// u_lo + sl cross the column (A < B); bit 2 + sl = no voxel of the column has
// a second candidate row there; bit 4 + sl = the piece lies behind the source
// (every row is a candidate).
struct GatherView {
    float4 ab[2];  // {A, B, pa, pb}
    float2 c[2];   // {ca, cb}
    int u_lo, u_hi;
    unsigned flags;
    unsigned view;  // the view's index (fills the struct's 16-byte alignment)
};

// Column (i, j) of the volume, [Xa, Xb] x [Ya, Yb], seen from one view (see
// GatherView); margin = the candidate rows' total widening (0.004 row).
__device__ __forceinline__ GatherView gather_view(const ExactGeom& G, const GatherConst& C,
                                                  const float4* __restrict__ txy, const int2* __restrict__ kxy,
                                                  const float2* __restrict__ cs, unsigned view, int i, int j, float Xa,
                                                  float Xb, float Ya, float Yb, float margin, float dz32)
{
    const float2 CS = __ldg(cs + view);
    float umin = 3.0e38f, umax = -3.0e38f;
    bool behind = false;
#pragma unroll
    for (int c4 = 0; c4 < 4; ++c4) {
        const float X = (c4 & 1) ? Xb : Xa, Y = (c4 & 2) ? Yb : Ya;
        const float a = X * CS.x - Y * CS.y, b = X * CS.y + Y * CS.x;
        const float d = b + G.Rf;
        behind |= !(d > 1e-3f * G.Rf);
        const float uf = a / d * C.eu + C.ou;
        umin = fminf(umin, uf);
        umax = fmaxf(umax, uf);
    }
    GatherView V;
    V.flags = 0u;
    V.view = view;
    if (behind) {  // not for a volume in front of the source; stays exact anyway
        V.u_lo = 0;
        V.u_hi = G.Nu - 1;
    } else {
        V.u_lo = min(max(0, __float2int_ru(umin - 0.01f)), G.Nu);
        V.u_hi = min(G.Nu - 1, __float2int_rd(umax + 0.01f));
    }
#pragma unroll
    for (int sl = 0; sl < 2; ++sl) {
        const int u = min(V.u_lo + sl, G.Nu - 1);
        const float4 T = __ldg(txy + (size_t)view * G.Nu + u);
        const int2 K = __ldg(kxy + (size_t)view * G.Nu + u);
        const float xa = plane_t(i, T.x, T.y, K.x), xb = plane_t(i + 1, T.x, T.y, K.x);
        const float ya = plane_t(j, T.z, T.w, K.y), yb = plane_t(j + 1, T.z, T.w, K.y);
        const float A = fmaxf(fminf(xa, xb), fminf(ya, yb));
        const float B = fminf(fmaxf(xa, xb), fmaxf(ya, yb));
        const float ca = C.ez / (A + G.Rf), cb = C.ez / (B + G.Rf);
        V.ab[sl] = make_float4(A, B, dz32 * ca, dz32 * cb);
        V.c[sl] = make_float2(ca, cb);
        if (A < B) V.flags |= 1u << sl;
        // a voxel's candidate interval [f0, f1] (row units) has a length
        // convex in its height, largest at the column's bottom or top voxel
        const float zb = G.P0[2], zt = G.P0[2] + (float)G.Z * G.vox[2];
        const float len_b = fmaxf((zb + G.vox[2]) * ca, (zb + G.vox[2]) * cb) - fminf(zb * ca, zb * cb);
        const float len_t = fmaxf(zt * ca, zt * cb) - fminf((zt - G.vox[2]) * ca, (zt - G.vox[2]) * cb);
        if (fmaxf(len_b, len_t) + margin < 0.99f) V.flags |= 1u << (2 + sl);
        if (!(A + G.Rf > 1e-3f * G.Rf)) V.flags |= 1u << (4 + sl);
    }
    return V;
}

template <int EPI, class ST, int SLOTS>
__global__ void __launch_bounds__(kGatherWarps * 32, 3) bp_gather_kernel(
    ExactGeom G, GatherConst C, const float4* __restrict__ txy, const int2* __restrict__ kxy,
    const float2* __restrict__ cs, const ZParam* __restrict__ zp, unsigned view0, unsigned nview,
    const ST* __restrict__ vals, size_t view_stride, float* __restrict__ vol, const float* __restrict__ sens,
    unsigned long long* __restrict__ npairs)
{
    // row v's z planes: voxel k spans t in [fmaf(k - z, S, O), fmaf(k - w, S, O)]
    // with {S, O, z, w} = szq[v] (z = kc, w = kc - 1 when S > 0; swapped when S < 0)
    extern __shared__ float4 szq[];
    __shared__ GatherView sview[kGatherWarps][32];
    __shared__ float sacc2[kGatherWarps][SLOTS * 32];  // sums of the further candidates
    for (int q = threadIdx.x; q < G.Nv; q += blockDim.x) {
        const ZParam z = zp[q];
        const float kc = (float)z.kc;
        szq[q] = (z.S > 0.0f) ? make_float4(z.S, z.O, kc, kc - 1.0f) : make_float4(z.S, z.O, kc - 1.0f, kc);
    }
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int i0 = blockIdx.x * kGatherTileX, j0 = blockIdx.y * (kGatherWarps / kGatherTileX);
    const int i = i0 + warp % kGatherTileX, j = j0 + warp / kGatherTileX;
    // a warp past the volume's edge takes no view but joins the epilogue's barriers
    const unsigned nview_w = (i < G.X && j < G.Y) ? nview : 0u;
    GatherView* sv = sview[warp];
    float* acc2 = sacc2[warp];
    const float Xa = G.P0[0] + i * G.vox[0], Xb = Xa + G.vox[0];
    const float Ya = G.P0[1] + j * G.vox[1], Yb = Ya + G.vox[1];
    // candidate rows are widened by 0.002 row on either side: about ten times the
    // FP32 error of the row bounds (values of a few hundred rows, a few roundings),
    // small enough that a voxel rarely shows a second candidate that is not one
    const float oz_lo = C.oz - 0.002f, oz_hi = C.oz + 0.002f;
    const float dz32 = 32.0f * G.vox[2];
    for (int k0 = 0; k0 < G.Z; k0 += 32 * SLOTS) {
        // Slots below the source plane z = 0 (voxels k < Z/2, the volume being centred)
        // when that is the same count for every lane, else -1.  The bound f0 of voxel k
        // is min over the piece of z_k * c and f1 the max of z_k+1 * c: c = ez / (depth)
        // is larger at the piece's near end, so the near end gives f0 below z = 0 and
        // f1 above, the far end the others.  Z must be even: for odd Z the middle voxel
        // straddles z = 0 (its bottom below, its top above).  Rounding can make the
        // other end's value pass by an ulp, which moves a bound only where it lies a
        // row's 0.002 margin away from the voxel: the row it adds or drops has no
        // length there.
        const int rel = G.Z / 2 - k0;
        const int split = (G.Z & 1) ? -1
                          : rel <= 0 ? 0 : (rel >= 32 * SLOTS ? SLOTS : (rel % 32 == 0 ? rel / 32 : -1));
        const float fk0 = (float)(k0 + lane);
        const float zl0 = fmaf(fk0, G.vox[2], G.P0[2]), zh0 = zl0 + G.vox[2];
        const int nslot = min(SLOTS, max(0, (G.Z - k0 - lane + 31) / 32));
        float acc[SLOTS];
#pragma unroll
        for (int s = 0; s < SLOTS; ++s) {
            acc[s] = 0.0f;
            acc2[s * 32 + lane] = 0.0f;
        }
        // the views' contributions to this chunk; SPLIT as `split`, a constant of
        // the chunk's code
        auto chunk = [&](auto split_tag) {
            constexpr int SPLIT = decltype(split_tag)::value;
            // detector column u of one view: its piece [A, B], row coefficients and
            // steps; col = the view's values from row 0 of column u
            auto piece = [&](float A, float B, float ca, float cb, float pa, float pb, bool single, bool behind,
                             const ST* __restrict__ col) {
                auto add = [&](int s, int v, float x) {
                    const float4 zr = szq[v];
                    const float t = fk0 + (float)(32 * s);
                    const float lo = fmaf(t - zr.z, zr.x, zr.y), hi = fmaf(t - zr.w, zr.x, zr.y);
                    const float L = fminf(B, hi) - fmaxf(A, lo);
                    if (L > 0.0f) acc[s] = (EPI == 2) ? acc[s] + 1.0f : fmaf(L, x, acc[s]);
                };
                if (behind) {  // a piece behind the source: every row is a candidate
#pragma unroll
                    for (int s = 0; s < SLOTS; ++s)
                        if (s < nslot)
                            for (int v = 0; v < G.Nv; ++v) add(s, v, load_val<ST>(col + v));
                    return;
                }
                // row bounds of slot s: f0 = min over the piece of the voxel's bottom
                // row, f1 = max of its top row, both affine in s
                const float P0a = fmaf(zl0, ca, oz_lo), P0b = fmaf(zl0, cb, oz_lo);
                const float P1a = single ? 0.0f : fmaf(zh0, ca, oz_hi), P1b = single ? 0.0f : fmaf(zh0, cb, oz_hi);
                // first candidate row of every voxel (loads issued together); a row that
                // misses the voxel gives L <= 0 and adds nothing
                auto first_rows = [&](auto single_tag) -> unsigned {
                    constexpr bool SINGLE = decltype(single_tag)::value;
                    unsigned more = 0u;
                    int vl[SLOTS];
                    decltype(load_raw(col)) x[SLOTS];
#pragma unroll
                    for (int s = 0; s < SLOTS; ++s) {
                        // the lower of the two bounds: the piece's near end (a) for
                        // voxels below the source plane, its far end (b) above it,
                        // where the slot is on one side for every lane (SPLIT >= 0)
                        const float f0 = SPLIT < 0 ? fminf(fmaf((float)s, pa, P0a), fmaf((float)s, pb, P0b))
                                                   : (s < SPLIT ? fmaf((float)s, pa, P0a) : fmaf((float)s, pb, P0b));
                        // clamped to a detector row, so every load is in bounds: a row
                        // that is no candidate gives L <= 0, and the sums of slots past
                        // the volume's top are never written out.  The conversion to
                        // unsigned saturates (negative rows and NaN give 0), which leaves
                        // one min for the clamp
                        const int a = (int)min(__float2uint_ru(f0), (unsigned)G.Nv - 1u);
                        vl[s] = a;
                        x[s] = load_raw(col + a);
                        if (!SINGLE) {  // the higher top bound: far end below z = 0, near end above
                            const float f1 = SPLIT < 0
                                                 ? fmaxf(fmaf((float)s, pa, P1a), fmaf((float)s, pb, P1b))
                                                 : (s < SPLIT ? fmaf((float)s, pb, P1b) : fmaf((float)s, pa, P1a));
                            if ((float)(a + 1) <= f1) more |= 1u << s;
                        }
                    }
#pragma unroll
                    for (int s = 0; s < SLOTS; ++s) add(s, vl[s], widen(x[s]));
                    return more;
                };
                if (single) {
                    first_rows(std::true_type{});
                    return;
                }
                const unsigned more = first_rows(std::false_type{});
                // further candidates (rare): summed apart, in shared memory
                if (__any_sync(0xffffffffu, more != 0u)) {
                    for (unsigned m = more; m != 0u; m &= m - 1u) {
                        const int s = __ffs(m) - 1;
                        const float f0 = fminf(fmaf((float)s, pa, P0a), fmaf((float)s, pb, P0b));
                        const float f1 = fmaxf(fmaf((float)s, pa, P1a), fmaf((float)s, pb, P1b));
                        const int a = max(0, __float2int_ru(f0));
                        const int b = min(G.Nv - 1, __float2int_rd(f1));
                        const float t = fk0 + (float)(32 * s);
                        float sum = acc2[s * 32 + lane];
                        for (int v = a + 1; v <= b; ++v) {
                            const float4 zr = szq[v];
                            const float lo = fmaf(t - zr.z, zr.x, zr.y), hi = fmaf(t - zr.w, zr.x, zr.y);
                            const float L = fminf(B, hi) - fmaxf(A, lo);
                            if (L > 0.0f) sum = (EPI == 2) ? sum + 1.0f : fmaf(L, load_val<ST>(col + v), sum);
                        }
                        acc2[s * 32 + lane] = sum;
                    }
                }
            };
            for (unsigned vb = 0; vb < nview_w; vb += 32) {
                const unsigned nb = min(32u, nview_w - vb);
                if ((unsigned)lane < nb)  // lane q sets up view vb + q
                    sv[lane] = gather_view(G, C, txy, kxy, cs, view0 + vb + lane, i, j, Xa, Xb, Ya, Yb, oz_hi - oz_lo,
                                           dz32);
                __syncwarp();
                for (unsigned q = 0; q < nb; ++q) {
                    const unsigned vi = vb + q;
                    const int ulo = sv[q].u_lo, uhi = sv[q].u_hi;
                    const unsigned fl = sv[q].flags;
                    // the first two detector columns, set up with the view
#pragma unroll 1
                    for (int sl = 0; sl < 2; ++sl) {
                        if (ulo + sl > uhi) break;
                        if (!((fl >> sl) & 1u)) continue;  // the rays miss the column
                        const float4 ab = sv[q].ab[sl];
                        const float2 cc = sv[q].c[sl];
                        piece(ab.x, ab.y, cc.x, cc.y, ab.z, ab.w, (fl >> (2 + sl)) & 1u, (fl >> (4 + sl)) & 1u,
                              vals + (size_t)vi * view_stride + (size_t)(ulo + sl) * G.Nv);
                    }
                    // a column wider than two detector pitches: set up here
                    for (int u = ulo + 2; u <= uhi; ++u) {
                        const unsigned view = view0 + vi;
                        const float4 T = __ldg(txy + (size_t)view * G.Nu + u);
                        const int2 K = __ldg(kxy + (size_t)view * G.Nu + u);
                        const float xa = plane_t(i, T.x, T.y, K.x), xb = plane_t(i + 1, T.x, T.y, K.x);
                        const float ya = plane_t(j, T.z, T.w, K.y), yb = plane_t(j + 1, T.z, T.w, K.y);
                        const float A = fmaxf(fminf(xa, xb), fminf(ya, yb));
                        const float B = fminf(fmaxf(xa, xb), fmaxf(ya, yb));
                        if (!(A < B)) continue;
                        const float ca = C.ez / (A + G.Rf), cb = C.ez / (B + G.Rf);
                        piece(A, B, ca, cb, dz32 * ca, dz32 * cb, false, !(A + G.Rf > 1e-3f * G.Rf),
                              vals + (size_t)vi * view_stride + (size_t)u * G.Nv);
                    }
                }
                __syncwarp();  // the next batch rewrites sv
            }
        };
        if (SLOTS == 8 && split == 0)
            chunk(std::integral_constant<int, 0>{});
        else if (SLOTS == 8 && split == SLOTS / 2)
            chunk(std::integral_constant<int, SLOTS / 2>{});
        else if (SLOTS == 8 && split == SLOTS)
            chunk(std::integral_constant<int, SLOTS>{});
        else
            chunk(std::integral_constant<int, -1>{});
        if (EPI == 2) {  // pair counts (exact: a voxel's count stays far below 2^24)
            unsigned long long c = 0;
#pragma unroll
            for (int s = 0; s < SLOTS; ++s)
                if (s < nslot) c += (unsigned long long)(acc[s] + acc2[s * 32 + lane]);
            for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
            if (lane == 0 && c) atomicAdd(npairs, c);
        } else {
            // the sums into the staging entries (each lane its own), then the
            // CTA's coalesced epilogue
#pragma unroll
            for (int s = 0; s < SLOTS; ++s) acc2[s * 32 + lane] += acc[s];
            __syncthreads();
            gather_tile_epilogue<EPI, SLOTS * 32>(
                G, C.vec4 != 0, &sacc2[0][0], i0, j0, [&](int e) { return k0 + e < G.Z ? k0 + e : -1; }, vol, sens);
            __syncthreads();  // the next chunk clears the entries
        }
    }
}

// The gather for geometries mirror-symmetric about the source plane z = 0: no
// vertical detector offset, so row Nv-1-v's z planes are row v's mirrored,
// bit for bit (S -> -S, O unchanged, kc -> Z - kc, checked on the plan's
// table before this kernel is chosen).  Then row Nv-1-a gives voxel Z-1-k
// exactly the length that row a gives voxel k: fmaf(-q, -S, O) = fmaf(q, S, O).
// A lane owns the pairs (k, Z-1-k) for k = k0 + lane + 32 s < Z/2 (s < PS);
// each pair's candidate rows and lengths are found once, for the lower voxel,
// and each length is applied to both values, row a for voxel k and row
// Nv-1-a for its mirror.  All the lower voxels lie below the source plane, so
// a slot's row bounds come from one end of the piece each.  Sums, the sums'
// order (views, detector columns, rows) and the epilogue are those of
// bp_gather_kernel, so the results are deterministic too.
template <int EPI, class ST, int PS>
__global__ void __launch_bounds__(kGatherWarps * 32, 3) bp_gather_mirror_kernel(
    ExactGeom G, GatherConst C, const float4* __restrict__ txy, const int2* __restrict__ kxy,
    const float2* __restrict__ cs, const ZParam* __restrict__ zp, unsigned view0, unsigned nview,
    const ST* __restrict__ vals, size_t view_stride, float* __restrict__ vol, const float* __restrict__ sens,
    unsigned long long* __restrict__ npairs)
{
    extern __shared__ float4 szq[];  // as in bp_gather_kernel
    __shared__ GatherView sview[kGatherWarps][32];
    __shared__ float sacc2[kGatherWarps][2][PS * 32];  // further candidates: lower voxels, mirrors
    for (int q = threadIdx.x; q < G.Nv; q += blockDim.x) {
        const ZParam z = zp[q];
        const float kc = (float)z.kc;
        szq[q] = (z.S > 0.0f) ? make_float4(z.S, z.O, kc, kc - 1.0f) : make_float4(z.S, z.O, kc - 1.0f, kc);
    }
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int i0 = blockIdx.x * kGatherTileX, j0 = blockIdx.y * (kGatherWarps / kGatherTileX);
    const int i = i0 + warp % kGatherTileX, j = j0 + warp / kGatherTileX;
    const unsigned nview_w = (i < G.X && j < G.Y) ? nview : 0u;  // as in bp_gather_kernel
    GatherView* sv = sview[warp];
    float* acc2 = sacc2[warp][0];
    float* acc2m = sacc2[warp][1];
    const float Xa = G.P0[0] + i * G.vox[0], Xb = Xa + G.vox[0];
    const float Ya = G.P0[1] + j * G.vox[1], Yb = Ya + G.vox[1];
    const float oz_lo = C.oz - 0.002f, oz_hi = C.oz + 0.002f;  // margins as in bp_gather_kernel
    const float dz32 = 32.0f * G.vox[2];
    const int Zh = G.Z / 2;
    const unsigned top = (unsigned)G.Nv - 1u;
    for (int k0 = 0; k0 < Zh; k0 += 32 * PS) {
        const float fk0 = (float)(k0 + lane);
        const float zl0 = fmaf(fk0, G.vox[2], G.P0[2]), zh0 = zl0 + G.vox[2];
        const int nslot = min(PS, max(0, (Zh - k0 - lane + 31) / 32));
        float acc[PS], accm[PS];
#pragma unroll
        for (int s = 0; s < PS; ++s) {
            acc[s] = 0.0f;
            accm[s] = 0.0f;
            acc2[s * 32 + lane] = 0.0f;
            acc2m[s * 32 + lane] = 0.0f;
        }
        // detector column u of one view: its piece [A, B], row coefficients and
        // steps; col = the view's values from row 0 of column u
        auto piece = [&](float A, float B, float ca, float cb, float pa, float pb, bool single, bool behind,
                         const ST* __restrict__ col) {
            // row v's length through lower voxel s of this lane
            auto length = [&](int s, int v) {
                const float4 zr = szq[v];
                const float t = fk0 + (float)(32 * s);
                const float lo = fmaf(t - zr.z, zr.x, zr.y), hi = fmaf(t - zr.w, zr.x, zr.y);
                return fminf(B, hi) - fmaxf(A, lo);
            };
            if (behind) {  // a piece behind the source: every row is a candidate
#pragma unroll
                for (int s = 0; s < PS; ++s)
                    if (s < nslot)
                        for (int v = 0; v < G.Nv; ++v) {
                            const float L = length(s, v);
                            if (L > 0.0f) {
                                acc[s] = (EPI == 2) ? acc[s] + 1.0f : fmaf(L, load_val<ST>(col + v), acc[s]);
                                accm[s] = (EPI == 2) ? accm[s] + 1.0f : fmaf(L, load_val<ST>(col + (top - v)), accm[s]);
                            }
                        }
                return;
            }
            // row bounds of a lower voxel: f0 = its bottom row at the piece's near
            // end, f1 = its top row at the far end (the voxel lies below z = 0)
            const float P0a = fmaf(zl0, ca, oz_lo);
            const float P1b = single ? 0.0f : fmaf(zh0, cb, oz_hi);
            auto first_rows = [&](auto single_tag) -> unsigned {
                constexpr bool SINGLE = decltype(single_tag)::value;
                unsigned more = 0u;
                int vl[PS];
                decltype(load_raw(col)) x[PS], xm[PS];
#pragma unroll
                for (int s = 0; s < PS; ++s) {
                    const float f0 = fmaf((float)s, pa, P0a);
                    // clamped to a detector row: every load is in bounds, a row that
                    // is no candidate has no positive length (see bp_gather_kernel)
                    const unsigned a = min(__float2uint_ru(f0), top);
                    vl[s] = (int)a;
                    x[s] = load_raw(col + a);
                    xm[s] = load_raw(col + (top - a));
                    if (!SINGLE) {
                        const float f1 = fmaf((float)s, pb, P1b);
                        if ((float)(a + 1u) <= f1) more |= 1u << s;
                    }
                }
#pragma unroll
                for (int s = 0; s < PS; ++s) {
                    const float L = length(s, vl[s]);
                    if (L > 0.0f) {
                        acc[s] = (EPI == 2) ? acc[s] + 1.0f : fmaf(L, widen(x[s]), acc[s]);
                        accm[s] = (EPI == 2) ? accm[s] + 1.0f : fmaf(L, widen(xm[s]), accm[s]);
                    }
                }
                return more;
            };
            if (single) {
                first_rows(std::true_type{});
                return;
            }
            const unsigned more = first_rows(std::false_type{});
            // further candidates (rare): summed apart, in shared memory, over the
            // bounds of both piece ends as bp_gather_kernel takes them
            if (__any_sync(0xffffffffu, more != 0u)) {
                const float P0b = fmaf(zl0, cb, oz_lo), P1a = fmaf(zh0, ca, oz_hi);
                for (unsigned m = more; m != 0u; m &= m - 1u) {
                    const int s = __ffs(m) - 1;
                    const float f0 = fminf(fmaf((float)s, pa, P0a), fmaf((float)s, pb, P0b));
                    const float f1 = fmaxf(fmaf((float)s, pa, P1a), fmaf((float)s, pb, P1b));
                    const int a = max(0, __float2int_ru(f0));
                    const int b = min(G.Nv - 1, __float2int_rd(f1));
                    float sum = acc2[s * 32 + lane], summ = acc2m[s * 32 + lane];
                    for (int v = a + 1; v <= b; ++v) {
                        const float L = length(s, v);
                        if (L > 0.0f) {
                            sum = (EPI == 2) ? sum + 1.0f : fmaf(L, load_val<ST>(col + v), sum);
                            summ = (EPI == 2) ? summ + 1.0f : fmaf(L, load_val<ST>(col + (top - v)), summ);
                        }
                    }
                    acc2[s * 32 + lane] = sum;
                    acc2m[s * 32 + lane] = summ;
                }
            }
        };
        for (unsigned vb = 0; vb < nview_w; vb += 32) {
            const unsigned nb = min(32u, nview_w - vb);
            if ((unsigned)lane < nb)  // lane q sets up view vb + q
                sv[lane] = gather_view(G, C, txy, kxy, cs, view0 + vb + lane, i, j, Xa, Xb, Ya, Yb, oz_hi - oz_lo,
                                       dz32);
            __syncwarp();
            for (unsigned q = 0; q < nb; ++q) {
                const unsigned vi = vb + q;
                const int ulo = sv[q].u_lo, uhi = sv[q].u_hi;
                const unsigned fl = sv[q].flags;
#pragma unroll 1
                for (int sl = 0; sl < 2; ++sl) {
                    if (ulo + sl > uhi) break;
                    if (!((fl >> sl) & 1u)) continue;  // the rays miss the column
                    const float4 ab = sv[q].ab[sl];
                    const float2 cc = sv[q].c[sl];
                    piece(ab.x, ab.y, cc.x, cc.y, ab.z, ab.w, (fl >> (2 + sl)) & 1u, (fl >> (4 + sl)) & 1u,
                          vals + (size_t)vi * view_stride + (size_t)(ulo + sl) * G.Nv);
                }
                // a column wider than two detector pitches: set up here
                for (int u = ulo + 2; u <= uhi; ++u) {
                    const unsigned view = view0 + vi;
                    const float4 T = __ldg(txy + (size_t)view * G.Nu + u);
                    const int2 K = __ldg(kxy + (size_t)view * G.Nu + u);
                    const float xa = plane_t(i, T.x, T.y, K.x), xb = plane_t(i + 1, T.x, T.y, K.x);
                    const float ya = plane_t(j, T.z, T.w, K.y), yb = plane_t(j + 1, T.z, T.w, K.y);
                    const float A = fmaxf(fminf(xa, xb), fminf(ya, yb));
                    const float B = fminf(fmaxf(xa, xb), fmaxf(ya, yb));
                    if (!(A < B)) continue;
                    const float ca = C.ez / (A + G.Rf), cb = C.ez / (B + G.Rf);
                    piece(A, B, ca, cb, dz32 * ca, dz32 * cb, false, !(A + G.Rf > 1e-3f * G.Rf),
                          vals + (size_t)vi * view_stride + (size_t)u * G.Nv);
                }
            }
            __syncwarp();  // the next batch rewrites sv
        }
        if (EPI == 2) {  // pair counts
            unsigned long long c = 0;
#pragma unroll
            for (int s = 0; s < PS; ++s)
                if (s < nslot)
                    c += (unsigned long long)(acc[s] + acc2[s * 32 + lane]) +
                         (unsigned long long)(accm[s] + acc2m[s * 32 + lane]);
            for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
            if (lane == 0 && c) atomicAdd(npairs, c);
        } else {
            // entries [0, 32 PS) the lower voxels k0 + e, [32 PS, 64 PS) their mirrors
#pragma unroll
            for (int s = 0; s < PS; ++s) {
                acc2[s * 32 + lane] += acc[s];
                acc2m[s * 32 + lane] += accm[s];
            }
            __syncthreads();
            gather_tile_epilogue<EPI, 64 * PS>(
                G, C.vec4 != 0, &sacc2[0][0][0], i0, j0,
                [&](int e) {
                    const int k = k0 + (e < 32 * PS ? e : e - 32 * PS);
                    return k >= Zh ? -1 : (e < 32 * PS ? k : G.Z - 1 - k);
                },
                vol, sens);
            __syncthreads();  // the next chunk clears the entries
        }
    }
}

// bp_gather_mirror_kernel reading its values in mirrored row pairs
// (kLayoutPairs: per detector column, pair p = {row p, row Nv-1-p} for p = 0 ..
// Nv/2, even Nv): a lower voxel's candidate row a and the mirror row Nv-1-a
// come in one load.  Lengths, sums and their order are bp_gather_mirror_kernel's,
// so both give the same bits.
template <int EPI, class ST, int PS>
__global__ void __launch_bounds__(kGatherWarps * 32, 3) bp_gather_pairs_kernel(
    ExactGeom G, GatherConst C, const float4* __restrict__ txy, const int2* __restrict__ kxy,
    const float2* __restrict__ cs, const ZParam* __restrict__ zp, unsigned view0, unsigned nview,
    const ST* __restrict__ vals, size_t view_stride, float* __restrict__ vol, const float* __restrict__ sens,
    unsigned long long* __restrict__ npairs)
{
    extern __shared__ float4 szq[];  // as in bp_gather_kernel
    __shared__ GatherView sview[kGatherWarps][32];
    __shared__ float sacc2[kGatherWarps][2][PS * 32];  // further candidates: lower voxels, mirrors
    for (int q = threadIdx.x; q < G.Nv; q += blockDim.x) {
        const ZParam z = zp[q];
        const float kc = (float)z.kc;
        szq[q] = (z.S > 0.0f) ? make_float4(z.S, z.O, kc, kc - 1.0f) : make_float4(z.S, z.O, kc - 1.0f, kc);
    }
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int i0 = blockIdx.x * kGatherTileX, j0 = blockIdx.y * (kGatherWarps / kGatherTileX);
    const int i = i0 + warp % kGatherTileX, j = j0 + warp / kGatherTileX;
    const unsigned nview_w = (i < G.X && j < G.Y) ? nview : 0u;  // as in bp_gather_kernel
    GatherView* sv = sview[warp];
    float* acc2 = sacc2[warp][0];
    float* acc2m = sacc2[warp][1];
    const float Xa = G.P0[0] + i * G.vox[0], Xb = Xa + G.vox[0];
    const float Ya = G.P0[1] + j * G.vox[1], Yb = Ya + G.vox[1];
    const float oz_lo = C.oz - 0.002f, oz_hi = C.oz + 0.002f;  // margins as in bp_gather_kernel
    const float dz32 = 32.0f * G.vox[2];
    const int Zh = G.Z / 2;
    const unsigned top = (unsigned)G.Nv - 1u;
    const unsigned Nh = (unsigned)G.Nv / 2u, Np = Nh + 1u;  // pairs per detector column
    for (int k0 = 0; k0 < Zh; k0 += 32 * PS) {
        const float fk0 = (float)(k0 + lane);
        const float zl0 = fmaf(fk0, G.vox[2], G.P0[2]), zh0 = zl0 + G.vox[2];
        const int nslot = min(PS, max(0, (Zh - k0 - lane + 31) / 32));
        float acc[PS], accm[PS];
#pragma unroll
        for (int s = 0; s < PS; ++s) {
            acc[s] = 0.0f;
            accm[s] = 0.0f;
            acc2[s * 32 + lane] = 0.0f;
            acc2m[s * 32 + lane] = 0.0f;
        }
        // detector column u of one view: its piece [A, B], row coefficients and
        // steps; col = the view's values from row 0 of column u
        auto piece = [&](float A, float B, float ca, float cb, float pa, float pb, bool single, bool behind,
                         const ST* __restrict__ col) {
            // row v's length through lower voxel s of this lane
            auto length = [&](int s, int v) {
                const float4 zr = szq[v];
                const float t = fk0 + (float)(32 * s);
                const float lo = fmaf(t - zr.z, zr.x, zr.y), hi = fmaf(t - zr.w, zr.x, zr.y);
                return fminf(B, hi) - fmaxf(A, lo);
            };
            if (behind) {  // a piece behind the source: every row is a candidate
#pragma unroll
                for (int s = 0; s < PS; ++s)
                    if (s < nslot)
                        for (int v = 0; v < G.Nv; ++v) {
                            const float L = length(s, v);
                            if (L > 0.0f) {
                                // row v and its mirror from pair min(v, Nv-1-v), in order
                                const bool lower = (unsigned)v < Nh;
                                const auto p = load_pair_raw(col + 2u * (lower ? (unsigned)v : top - v));
                                const float xv = lower ? widen_lo(p) : widen_hi(p), xm = lower ? widen_hi(p) : widen_lo(p);
                                acc[s] = (EPI == 2) ? acc[s] + 1.0f : fmaf(L, xv, acc[s]);
                                accm[s] = (EPI == 2) ? accm[s] + 1.0f : fmaf(L, xm, accm[s]);
                            }
                        }
                return;
            }
            // row bounds of a lower voxel: f0 = its bottom row at the piece's near
            // end, f1 = its top row at the far end (the voxel lies below z = 0)
            const float P0a = fmaf(zl0, ca, oz_lo);
            const float P1b = single ? 0.0f : fmaf(zh0, cb, oz_hi);
            auto first_rows = [&](auto single_tag) -> unsigned {
                constexpr bool SINGLE = decltype(single_tag)::value;
                unsigned more = 0u;
                int vl[PS];
                decltype(load_pair_raw(col)) x[PS];
#pragma unroll
                for (int s = 0; s < PS; ++s) {
                    const float f0 = fmaf((float)s, pa, P0a);
                    // a lower voxel's rows lie at or below row Nv/2 (its z is at or below
                    // the source plane; the pair table's last entry is row Nv/2): clamped
                    // there, every load is in bounds, and a row that is no candidate has
                    // no positive length (see bp_gather_kernel)
                    const unsigned a = min(__float2uint_ru(f0), Nh);
                    vl[s] = (int)a;
                    x[s] = load_pair_raw(col + 2u * a);
                    if (!SINGLE) {
                        const float f1 = fmaf((float)s, pb, P1b);
                        if ((float)(a + 1u) <= f1) more |= 1u << s;
                    }
                }
#pragma unroll
                for (int s = 0; s < PS; ++s) {
                    const float L = length(s, vl[s]);
                    if (L > 0.0f) {
                        acc[s] = (EPI == 2) ? acc[s] + 1.0f : fmaf(L, widen_lo(x[s]), acc[s]);
                        accm[s] = (EPI == 2) ? accm[s] + 1.0f : fmaf(L, widen_hi(x[s]), accm[s]);
                    }
                }
                return more;
            };
            if (single) {
                first_rows(std::true_type{});
                return;
            }
            const unsigned more = first_rows(std::false_type{});
            // further candidates (rare): summed apart, in shared memory, over the
            // bounds of both piece ends as bp_gather_kernel takes them
            if (__any_sync(0xffffffffu, more != 0u)) {
                const float P0b = fmaf(zl0, cb, oz_lo), P1a = fmaf(zh0, ca, oz_hi);
                for (unsigned m = more; m != 0u; m &= m - 1u) {
                    const int s = __ffs(m) - 1;
                    const float f0 = fminf(fmaf((float)s, pa, P0a), fmaf((float)s, pb, P0b));
                    const float f1 = fmaxf(fmaf((float)s, pa, P1a), fmaf((float)s, pb, P1b));
                    const int a = max(0, __float2int_ru(f0));
                    const int b = min((int)Nh, __float2int_rd(f1));
                    float sum = acc2[s * 32 + lane], summ = acc2m[s * 32 + lane];
                    for (int v = a + 1; v <= b; ++v) {
                        const float L = length(s, v);
                        if (L > 0.0f) {
                            const auto p = load_pair_raw(col + 2 * v);
                            sum = (EPI == 2) ? sum + 1.0f : fmaf(L, widen_lo(p), sum);
                            summ = (EPI == 2) ? summ + 1.0f : fmaf(L, widen_hi(p), summ);
                        }
                    }
                    acc2[s * 32 + lane] = sum;
                    acc2m[s * 32 + lane] = summ;
                }
            }
        };
        for (unsigned vb = 0; vb < nview_w; vb += 32) {
            const unsigned nb = min(32u, nview_w - vb);
            if ((unsigned)lane < nb)  // lane q sets up view vb + q
                sv[lane] = gather_view(G, C, txy, kxy, cs, view0 + vb + lane, i, j, Xa, Xb, Ya, Yb, oz_hi - oz_lo,
                                       dz32);
            __syncwarp();
            for (unsigned q = 0; q < nb; ++q) {
                const unsigned vi = vb + q;
                const int ulo = sv[q].u_lo, uhi = sv[q].u_hi;
                const unsigned fl = sv[q].flags;
#pragma unroll 1
                for (int sl = 0; sl < 2; ++sl) {
                    if (ulo + sl > uhi) break;
                    if (!((fl >> sl) & 1u)) continue;  // the rays miss the column
                    const float4 ab = sv[q].ab[sl];
                    const float2 cc = sv[q].c[sl];
                    piece(ab.x, ab.y, cc.x, cc.y, ab.z, ab.w, (fl >> (2 + sl)) & 1u, (fl >> (4 + sl)) & 1u,
                          vals + (size_t)vi * view_stride + (size_t)(ulo + sl) * Np * 2);
                }
                // a column wider than two detector pitches: set up here
                for (int u = ulo + 2; u <= uhi; ++u) {
                    const unsigned view = view0 + vi;
                    const float4 T = __ldg(txy + (size_t)view * G.Nu + u);
                    const int2 K = __ldg(kxy + (size_t)view * G.Nu + u);
                    const float xa = plane_t(i, T.x, T.y, K.x), xb = plane_t(i + 1, T.x, T.y, K.x);
                    const float ya = plane_t(j, T.z, T.w, K.y), yb = plane_t(j + 1, T.z, T.w, K.y);
                    const float A = fmaxf(fminf(xa, xb), fminf(ya, yb));
                    const float B = fminf(fmaxf(xa, xb), fmaxf(ya, yb));
                    if (!(A < B)) continue;
                    const float ca = C.ez / (A + G.Rf), cb = C.ez / (B + G.Rf);
                    piece(A, B, ca, cb, dz32 * ca, dz32 * cb, false, !(A + G.Rf > 1e-3f * G.Rf),
                          vals + (size_t)vi * view_stride + (size_t)u * Np * 2);
                }
            }
            __syncwarp();  // the next batch rewrites sv
        }
        if (EPI == 2) {  // pair counts
            unsigned long long c = 0;
#pragma unroll
            for (int s = 0; s < PS; ++s)
                if (s < nslot)
                    c += (unsigned long long)(acc[s] + acc2[s * 32 + lane]) +
                         (unsigned long long)(accm[s] + acc2m[s * 32 + lane]);
            for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
            if (lane == 0 && c) atomicAdd(npairs, c);
        } else {
            // entries [0, 32 PS) the lower voxels k0 + e, [32 PS, 64 PS) their mirrors
#pragma unroll
            for (int s = 0; s < PS; ++s) {
                acc2[s * 32 + lane] += acc[s];
                acc2m[s * 32 + lane] += accm[s];
            }
            __syncthreads();
            gather_tile_epilogue<EPI, 64 * PS>(
                G, C.vec4 != 0, &sacc2[0][0][0], i0, j0,
                [&](int e) {
                    const int k = k0 + (e < 32 * PS ? e : e - 32 * PS);
                    return k >= Zh ? -1 : (e < 32 * PS ? k : G.Z - 1 - k);
                },
                vol, sens);
            __syncthreads();  // the next chunk clears the entries
        }
    }
}


// The pair gather over a quarter set of a plan's views (base views m0 .. m0 +
// mc - 1 and their turns by one, two and three quarters; all views for m0 = 0,
// mc = N/4) where views a quarter turn apart are exact rotations of each other (Plan::quarter, tables from
// quarter_turn_table_kernel: N = 4Q views, column c at view n + Q is column
// rho(c) = (X-1-j, i) at view n, bit for bit).  The candidate rows and lengths
// found for base column c0 = (i, j) at view m therefore serve the four columns
// of its orbit
//     d_0 = (i, j),  d_1 = (j, X-1-i),  d_2 = (X-1-i, X-1-j),  d_3 = (X-1-j, i)
// (d_r = rho^-r(c0)) at views m, m + Q, m + 2Q, m + 3Q (mod N): a lane finds a
// voxel pair's rows and lengths once and loads four value pairs for them, one
// per view.  Base columns tile the quadrant i, j < X/2 (one orbit each); a
// CTA's 4 x 2 base columns are 8 warps as in bp_gather_pairs_kernel.  Over all
// views column d_r sums its views in the order rQ .. N-1, 0 .. rQ-1, each
// piece's further candidate rows after its first ones, into the same
// registers: deterministic, the same lengths as bp_gather_pairs_kernel, the
// sums in another order.
// Dynamic shared memory: the rows' z planes (Nv float4), then the epilogue's
// staging area [warp][d_r][lower voxels, mirrors][PS * 32].
template <int EPI, class ST, int PS, bool SET = false>
__global__ void __launch_bounds__(kGatherWarps * 32, PS <= 2 ? 3 : 2) bp_gather_quarter_kernel(
    ExactGeom G, GatherConst C, const float4* __restrict__ txy, const int2* __restrict__ kxy,
    const float2* __restrict__ cs, const ZParam* __restrict__ zp, unsigned nview, unsigned m0, unsigned mc,
    const ST* __restrict__ vals, size_t view_stride, float* __restrict__ vol, const float* __restrict__ sens,
    unsigned long long* __restrict__ npairs)
{
    extern __shared__ float4 szq[];
    __shared__ GatherView sview[kGatherWarps][32];
    constexpr int NE = 8 * PS * 32;  // staged entries per warp
    float* const stage = reinterpret_cast<float*>(szq + G.Nv);
    for (int q = threadIdx.x; q < G.Nv; q += blockDim.x) {
        const ZParam z = zp[q];
        const float kc = (float)z.kc;
        szq[q] = (z.S > 0.0f) ? make_float4(z.S, z.O, kc, kc - 1.0f) : make_float4(z.S, z.O, kc - 1.0f, kc);
    }
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int H = G.X / 2;
    const int i0 = blockIdx.x * kGatherTileX, j0 = blockIdx.y * (kGatherWarps / kGatherTileX);
    const int i = i0 + warp % kGatherTileX, j = j0 + warp / kGatherTileX;
    const bool active = i < H && j < H;
    const unsigned Q = nview / 4u;
    // the views summed: all views (item i is view i), or with SET base views m0 ..
    // m0 + mc - 1 of each quarter, item i being view m0 + i % mc + (i / mc) Q (the
    // set is closed under quarter turns, so every turned column gets the same views)
    const unsigned nview_w = active ? (SET ? 4u * mc : nview) : 0u;
    auto view_of = [&](unsigned it) { return SET ? m0 + it % mc + (it / mc) * Q : it; };
    GatherView* sv = sview[warp];
    const float Xa = G.P0[0] + i * G.vox[0], Xb = Xa + G.vox[0];
    const float Ya = G.P0[1] + j * G.vox[1], Yb = Ya + G.vox[1];
    const float oz_lo = C.oz - 0.002f, oz_hi = C.oz + 0.002f;  // margins as in bp_gather_kernel
    const float dz32 = 32.0f * G.vox[2];
    const int Zh = G.Z / 2;
    const unsigned top = (unsigned)G.Nv - 1u;
    const unsigned Nh = (unsigned)G.Nv / 2u, Np = Nh + 1u;  // pairs per detector column
    for (int k0 = 0; k0 < Zh; k0 += 32 * PS) {
        const float fk0 = (float)(k0 + lane);
        const float zl0 = fmaf(fk0, G.vox[2], G.P0[2]), zh0 = zl0 + G.vox[2];
        const int nslot = min(PS, max(0, (Zh - k0 - lane + 31) / 32));
        float acc[4][PS], accm[4][PS];
#pragma unroll
        for (int r = 0; r < 4; ++r)
#pragma unroll
            for (int s = 0; s < PS; ++s) {
                acc[r][s] = 0.0f;
                accm[r][s] = 0.0f;
            }
        // one pair of rows {a, Nv-1-a} (a <= Nv/2) of the four views, length L
        auto add4 = [&](int s, float L, const ST* const* cols, unsigned a) {
#pragma unroll
            for (int r = 0; r < 4; ++r) {
                const auto p = load_pair_raw(cols[r] + 2u * a);
                acc[r][s] = (EPI == 2) ? acc[r][s] + 1.0f : fmaf(L, widen_lo(p), acc[r][s]);
                accm[r][s] = (EPI == 2) ? accm[r][s] + 1.0f : fmaf(L, widen_hi(p), accm[r][s]);
            }
        };
        // detector column u of view m: its piece [A, B], row coefficients and
        // steps; cols[r] = view m + rQ's values from pair 0 of column u
        auto piece = [&](float A, float B, float ca, float cb, float pa, float pb, bool single, bool behind,
                         const ST* const* cols) {
            auto length = [&](int s, int v) {  // row v's length through lower voxel s of this lane
                const float4 zr = szq[v];
                const float t = fk0 + (float)(32 * s);
                const float lo = fmaf(t - zr.z, zr.x, zr.y), hi = fmaf(t - zr.w, zr.x, zr.y);
                return fminf(B, hi) - fmaxf(A, lo);
            };
            if (behind) {  // a piece behind the source: every row is a candidate
#pragma unroll
                for (int s = 0; s < PS; ++s)
                    if (s < nslot)
                        for (int v = 0; v < G.Nv; ++v) {
                            const float L = length(s, v);
                            if (!(L > 0.0f)) continue;
                            // row v and its mirror from pair min(v, Nv-1-v), in order
                            const bool lower = (unsigned)v < Nh;
                            const unsigned a = lower ? (unsigned)v : top - v;
#pragma unroll
                            for (int r = 0; r < 4; ++r) {
                                const auto p = load_pair_raw(cols[r] + 2u * a);
                                const float xv = lower ? widen_lo(p) : widen_hi(p);
                                const float xm = lower ? widen_hi(p) : widen_lo(p);
                                acc[r][s] = (EPI == 2) ? acc[r][s] + 1.0f : fmaf(L, xv, acc[r][s]);
                                accm[r][s] = (EPI == 2) ? accm[r][s] + 1.0f : fmaf(L, xm, accm[r][s]);
                            }
                        }
                return;
            }
            // first candidate row of every lower voxel, clamped to row Nv/2 as in
            // bp_gather_pairs_kernel: lengths found once, then four loads each
            const float P0a = fmaf(zl0, ca, oz_lo);
            const float P1b = single ? 0.0f : fmaf(zh0, cb, oz_hi);
            unsigned av[PS], more = 0u;
            float L[PS];
#pragma unroll
            for (int s = 0; s < PS; ++s) {
                const float f0 = fmaf((float)s, pa, P0a);
                av[s] = min(__float2uint_ru(f0), Nh);
                L[s] = length(s, (int)av[s]);
                if (!single) {
                    const float f1 = fmaf((float)s, pb, P1b);
                    if ((float)(av[s] + 1u) <= f1) more |= 1u << s;
                }
            }
#pragma unroll
            for (int r = 0; r < 4; ++r) {
                decltype(load_pair_raw(cols[0])) x[PS];
#pragma unroll
                for (int s = 0; s < PS; ++s) x[s] = load_pair_raw(cols[r] + 2u * av[s]);
#pragma unroll
                for (int s = 0; s < PS; ++s)
                    if (L[s] > 0.0f) {
                        acc[r][s] = (EPI == 2) ? acc[r][s] + 1.0f : fmaf(L[s], widen_lo(x[s]), acc[r][s]);
                        accm[r][s] = (EPI == 2) ? accm[r][s] + 1.0f : fmaf(L[s], widen_hi(x[s]), accm[r][s]);
                    }
            }
            // further candidates (rare), over the bounds of both piece ends
            if (__any_sync(0xffffffffu, more != 0u)) {
                const float P0b = fmaf(zl0, cb, oz_lo), P1a = fmaf(zh0, ca, oz_hi);
#pragma unroll
                for (int s = 0; s < PS; ++s) {
                    if (!((more >> s) & 1u)) continue;
                    const float f0 = fminf(fmaf((float)s, pa, P0a), fmaf((float)s, pb, P0b));
                    const float f1 = fmaxf(fmaf((float)s, pa, P1a), fmaf((float)s, pb, P1b));
                    const int a = max(0, __float2int_ru(f0));
                    const int b = min((int)Nh, __float2int_rd(f1));
                    for (int v = a + 1; v <= b; ++v) {
                        const float Lv = length(s, v);
                        if (Lv > 0.0f) add4(s, Lv, cols, (unsigned)v);
                    }
                }
            }
        };
        for (unsigned vb = 0; vb < nview_w; vb += 32) {
            const unsigned nb = min(32u, nview_w - vb);
            if ((unsigned)lane < nb)  // lane q sets up view vb + q
                sv[lane] = gather_view(G, C, txy, kxy, cs, view_of(vb + lane), i, j, Xa, Xb, Ya, Yb, oz_hi - oz_lo,
                                       dz32);
            __syncwarp();
            for (unsigned q = 0; q < nb; ++q) {
                const unsigned m = SET ? sv[q].view : vb + q;
                const ST* vm[4];  // views m + rQ (mod N) from detector column 0
#pragma unroll
                for (int r = 0; r < 4; ++r) {
                    unsigned w = m + (unsigned)r * Q;
                    if (w >= nview) w -= nview;
                    vm[r] = vals + (size_t)w * view_stride;
                }
                auto column = [&](int u, const ST** cols) {
#pragma unroll
                    for (int r = 0; r < 4; ++r) cols[r] = vm[r] + (size_t)u * Np * 2;
                };
                const int ulo = sv[q].u_lo, uhi = sv[q].u_hi;
                const unsigned fl = sv[q].flags;
#pragma unroll 1
                for (int sl = 0; sl < 2; ++sl) {
                    if (ulo + sl > uhi) break;
                    if (!((fl >> sl) & 1u)) continue;  // the rays miss the column
                    const float4 ab = sv[q].ab[sl];
                    const float2 cc = sv[q].c[sl];
                    const ST* cols[4];
                    column(ulo + sl, cols);
                    piece(ab.x, ab.y, cc.x, cc.y, ab.z, ab.w, (fl >> (2 + sl)) & 1u, (fl >> (4 + sl)) & 1u, cols);
                }
                // a column wider than two detector pitches: set up here
                for (int u = ulo + 2; u <= uhi; ++u) {
                    const float4 T = __ldg(txy + (size_t)m * G.Nu + u);
                    const int2 K = __ldg(kxy + (size_t)m * G.Nu + u);
                    const float xa = plane_t(i, T.x, T.y, K.x), xb = plane_t(i + 1, T.x, T.y, K.x);
                    const float ya = plane_t(j, T.z, T.w, K.y), yb = plane_t(j + 1, T.z, T.w, K.y);
                    const float A = fmaxf(fminf(xa, xb), fminf(ya, yb));
                    const float B = fminf(fmaxf(xa, xb), fmaxf(ya, yb));
                    if (!(A < B)) continue;
                    const float ca = C.ez / (A + G.Rf), cb = C.ez / (B + G.Rf);
                    const ST* cols[4];
                    column(u, cols);
                    piece(A, B, ca, cb, dz32 * ca, dz32 * cb, false, !(A + G.Rf > 1e-3f * G.Rf), cols);
                }
            }
            __syncwarp();  // the next batch rewrites sv
        }
        if (EPI == 2) {  // pair counts of the four columns
            unsigned long long c = 0;
#pragma unroll
            for (int r = 0; r < 4; ++r)
#pragma unroll
                for (int s = 0; s < PS; ++s)
                    if (s < nslot) c += (unsigned long long)acc[r][s] + (unsigned long long)accm[r][s];
            for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
            if (lane == 0 && c) atomicAdd(npairs, c);
            continue;
        }
        // entry ((r * 2 + h) * PS + s) * 32 + lane: column d_r, lower voxel (h = 0)
        // k0 + lane + 32 s or its mirror (h = 1)
        float* const st = stage + warp * NE;
#pragma unroll
        for (int r = 0; r < 4; ++r)
#pragma unroll
            for (int s = 0; s < PS; ++s) {
                st[((r * 2) * PS + s) * 32 + lane] = acc[r][s];
                st[((r * 2 + 1) * PS + s) * 32 + lane] = accm[r][s];
            }
        __syncthreads();
        // the CTA's epilogue, one voxel per thread, warps fastest (a column
        // tile's x neighbours adjacent)
        const size_t plane = (size_t)G.X * G.Y;
        for (int q = threadIdx.x; q < kGatherWarps * NE; q += blockDim.x) {
            const int w = q % kGatherWarps, e = q / kGatherWarps;
            const int bi = i0 + w % kGatherTileX, bj = j0 + w / kGatherTileX;
            if (bi >= H || bj >= H) continue;
            const int r = e / (2 * PS * 32), h = (e / (PS * 32)) & 1, k = k0 + e % (PS * 32);
            if (k >= Zh) continue;
            const int x = (r == 0) ? bi : (r == 1) ? bj : (r == 2) ? G.X - 1 - bi : G.X - 1 - bj;
            const int y = (r == 0) ? bj : (r == 1) ? G.X - 1 - bi : (r == 2) ? G.X - 1 - bj : bi;
            const int z = h ? G.Z - 1 - k : k;
            const size_t v = (size_t)z * plane + (size_t)y * G.X + (size_t)x;
            const float hv = stage[w * NE + e];
            vol[v] = (EPI == 1) ? gather_update(vol[v], hv, sens[v]) : hv;
        }
        __syncthreads();  // the next chunk rewrites the staging area
    }
}

// A sinogram [view][v][u] times w into mirrored row pairs (kLayoutPairs), 32 (u)
// x 32 (pair) tiles: both rows of each pair read along u through shared memory,
// w (detector columns, wq) and the pairs along the pair index.
template <class T>
__global__ void __launch_bounds__(256) to_pairs_kernel(const T* __restrict__ in, const float* __restrict__ wq, int Nu,
                                                        int Nv, T* __restrict__ out)
{
    __shared__ float lo[32][33], hi[32][33];
    const int Np = Nv / 2 + 1;
    const int u0 = blockIdx.x * 32, p0 = blockIdx.y * 32;
    const size_t base = (size_t)blockIdx.z * Nu * Nv;
    for (int r = threadIdx.y; r < 32; r += 8) {
        const int u = u0 + threadIdx.x, p = p0 + r;
        if (u < Nu && p < Np) {
            lo[r][threadIdx.x] = load_val<T>(in + base + (size_t)p * Nu + u);
            hi[r][threadIdx.x] = load_val<T>(in + base + (size_t)(Nv - 1 - p) * Nu + u);
        }
    }
    __syncthreads();
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const int u = u0 + threadIdx.y + 8 * q, p = p0 + threadIdx.x;
        if (u >= Nu || p >= Np) continue;
        const float wa = wq ? __ldg(wq + (size_t)u * Nv + p) : 1.0f;
        const float wb = wq ? __ldg(wq + (size_t)u * Nv + (Nv - 1 - p)) : 1.0f;
        store_pair<T>(out + (((size_t)blockIdx.z * Nu + u) * Np + p) * 2, lo[threadIdx.x][threadIdx.y + 8 * q] * wa,
                      hi[threadIdx.x][threadIdx.y + 8 * q] * wb);
    }
}

// wq (detector columns [u][v]) into mirrored row pairs.
__global__ void wq_pairs_kernel(const float* __restrict__ wq, int Nu, int Nv, float* __restrict__ out)
{
    const int Np = Nv / 2 + 1;
    const size_t n = (size_t)Nu * Np;
    for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x) {
        const size_t u = q / Np;
        const int p = (int)(q % Np);
        out[2 * q] = wq[u * Nv + p];
        out[2 * q + 1] = wq[u * Nv + (Nv - 1 - p)];
    }
}

// A sinogram [view][v][u] (times w when w is given) into the detector-column
// layout [view][u][v] that the gather back projectors read: 32x32 (u, v) tiles
// through shared memory, read and written along rows of 128 bytes.  With rect
// (per view {u_min, u_max, v_min, v_max}), tiles wholly outside a view's
// rectangle are skipped: the MLEM ratio is zero there in both layouts.
template <class T>
__global__ void __launch_bounds__(256) to_columns_kernel(const T* __restrict__ in, const float* __restrict__ w, int Nu,
                                                         int Nv, const int4* __restrict__ rect, T* __restrict__ out)
{
    __shared__ T tile[32][33];
    const size_t view = blockIdx.z;
    const int u0 = blockIdx.x * 32, v0 = blockIdx.y * 32;
    if (rect) {  // the same for the whole block: no barrier is skipped by part of it
        const int4 r = rect[view];
        if (u0 > r.y || u0 + 31 < r.x || v0 > r.w || v0 + 31 < r.z) return;
    }
    const T* __restrict__ src = in + view * Nu * Nv;
    T* __restrict__ dst = out + view * Nu * Nv;
    for (int r = threadIdx.y; r < 32; r += 8) {
        const int u = u0 + threadIdx.x, v = v0 + r;
        if (u < Nu && v < Nv) {
            T x = src[(size_t)v * Nu + u];
            if (w) x = T(float(x) * __ldg(w + (size_t)v * Nu + u));
            tile[r][threadIdx.x] = x;
        }
    }
    __syncthreads();
    for (int r = threadIdx.y; r < 32; r += 8) {
        const int v = v0 + threadIdx.x, u = u0 + r;
        if (u < Nu && v < Nv) dst[(size_t)u * Nv + v] = tile[threadIdx.x][r];
    }
}

// ---- back projection (ray-driven, into a z-slab) ---------------------------------------------

// MODE 0: sinogram values (times w when WEIGHTED; the MLEM ratio already
// carries w); MODE 1: the value is w (the sensitivity).  One thread per ray
// (ray_pos), rays with a zero value skipped; sino holds views from view0 on.
template <int MODE, bool WEIGHTED, class ST>
__global__ void __launch_bounds__(128) bp_ray_kernel(ExactGeom G, const float4* __restrict__ txy,
                                                      const int2* __restrict__ kxy, const float2* __restrict__ cs,
                                                      const ZParam* __restrict__ zp, const float* __restrict__ wtab,
                                                      const uint2* __restrict__ tiles, unsigned view0,
                                                      const ST* __restrict__ sino,
                                                      const unsigned* __restrict__ maxabs, float max_len,
                                                      int count_bits, int k0, int k1, unsigned long long* acc,
                                                      unsigned long long* acc_t)
{
    const RayPos R = ray_pos(tiles, view0);
    const int u = R.u, v = R.v;
    const unsigned view = R.view;
    if (u >= G.Nu || v >= G.Nv) return;
    const size_t pix = (size_t)u + (size_t)v * G.Nu;
    // every load the ray needs is issued before any is used
    const unsigned mbits = __ldg(maxabs);
    float val = (MODE == 1) ? __ldg(wtab + pix) : load_val<ST>(sino + (size_t)(view - view0) * G.Nu * G.Nv + pix);
    const float wv = (WEIGHTED && MODE != 1) ? __ldg(wtab + pix) : 1.0f;
    const float2 C = __ldg(cs + view);
    const float4 T = __ldg(txy + (size_t)view * G.Nu + u);
    const int2 K = __ldg(kxy + (size_t)view * G.Nu + u);
    const ZParam Z = zp[v];
    const int F = fix_exponent(mbits, max_len, count_bits);
    if (F == INT_MIN) return;
    if (WEIGHTED && MODE != 1) val *= wv;
    if (val == 0.0f) return;
    bp_ray_slab(G, T, K, Z, k0, k1, val * ldexpf(1.0f, F), fabsf(C.y) > fabsf(C.x), acc, acc_t);
}

// Slab [k0, k1) of the result from the accumulators, 32x32 (x, y) tiles of
// one z slice per CTA of 32x8 threads (the transposed accumulator is read and
// cleared through shared memory so that both are accessed coalesced):
// MODE 0: vol = Ht; MODE 2: f = (sens != 0) ? f * Ht / sens : 0 (MLEM update).
template <int MODE>
__global__ void __launch_bounds__(256) bp_finish_kernel(ExactGeom G, const unsigned* __restrict__ maxabs,
                                                         float max_len, int count_bits, int k0,
                                                         unsigned long long* __restrict__ acc,
                                                         unsigned long long* __restrict__ acc_t,
                                                         float* __restrict__ vol, const float* __restrict__ sens)
{
    __shared__ unsigned long long tile[32][33];
    const int x0 = blockIdx.x * 32, y0 = blockIdx.y * 32, zs = blockIdx.z;
    const size_t plane = (size_t)G.X * G.Y, slab_off = (size_t)zs * plane;
    // all loads first: the transposed accumulator (y along the warp), then
    // this thread's accumulator, sensitivity and image values (x along the warp)
    unsigned long long qt[4], qa[4];
    float sv[4], fv[4];
#pragma unroll
    for (int r = 0; r < 4; ++r) {
        const int x = x0 + threadIdx.y + 8 * r, y = y0 + threadIdx.x;
        qt[r] = (x < G.X && y < G.Y) ? acc_t[slab_off + (size_t)x * G.Y + y] : 0ull;
    }
#pragma unroll
    for (int r = 0; r < 4; ++r) {
        const int x = x0 + threadIdx.x, y = y0 + threadIdx.y + 8 * r;
        const bool in = x < G.X && y < G.Y;
        const size_t i = slab_off + (size_t)y * G.X + x;
        qa[r] = in ? acc[i] : 0ull;
        sv[r] = (MODE == 2 && in) ? sens[i + (size_t)k0 * plane] : 0.0f;
        fv[r] = (MODE == 2 && in) ? vol[i + (size_t)k0 * plane] : 0.0f;
    }
    const unsigned mbits = __ldg(maxabs);
    const int F = fix_exponent(mbits, max_len, count_bits);
    // a non-finite input value makes every voxel NaN (as a float sum would)
    const bool nonfinite = !isfinite(__uint_as_float(mbits));
#pragma unroll
    for (int r = 0; r < 4; ++r) {
        const int x = x0 + threadIdx.y + 8 * r, y = y0 + threadIdx.x;
        tile[threadIdx.x][threadIdx.y + 8 * r] = qt[r];  // [y - y0][x - x0]
        if (x < G.X && y < G.Y) acc_t[slab_off + (size_t)x * G.Y + y] = 0ull;
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < 4; ++r) {
        const int x = x0 + threadIdx.x, y = y0 + threadIdx.y + 8 * r;
        if (x >= G.X || y >= G.Y) continue;
        const size_t i = slab_off + (size_t)y * G.X + x;
        const long long q = (long long)(qa[r] + tile[threadIdx.y + 8 * r][threadIdx.x]);
        acc[i] = 0ull;
        const float ht = nonfinite ? __int_as_float(0x7fffffff) : (F != INT_MIN) ? (float)ldexp((double)q, -F) : 0.0f;
        const size_t vox = i + (size_t)k0 * plane;
        if (MODE == 2) vol[vox] = (sv[r] != 0.0f) ? __fdiv_rn(__fmul_rn(fv[r], ht), sv[r]) : 0.0f;
        else vol[vox] = ht;
    }
}

// max |value| (times w when w != nullptr) over n values, as float bits, into
// *out (atomicMax of non-negative floats ordered as unsigned integers)
template <class ST>
__global__ void maxabs_kernel(const ST* __restrict__ a, size_t n, const float* __restrict__ w, size_t npix,
                              unsigned* __restrict__ out)
{
    unsigned m = 0;
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
        float v = fabsf(load_val<ST>(a + i));
        if (w) v *= __ldg(w + i % npix);
        m = max(m, __float_as_uint(v));
    }
    for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0 && m) atomicMax(out, m);
}

}  // namespace exact

// ---- host side -------------------------------------------------------------------------------

static exact::GeomD geom_d(const Plan& P)
{
    const recon_geometry_t& g = P.geom;
    exact::GeomD G;
    G.R = g.cal.R;
    G.Rf = g.cal.Rf;
    G.Ry = g.cal.Ry;
    G.Dx = g.cal.Dx;
    G.Dz = g.cal.Dz;
    G.du = (double)g.det.AxPixDimMm * (double)g.cal.M;
    G.dv = (double)g.det.TAxPixDimMm * (double)g.cal.M;
    G.Nu = (int)g.det.NumAxPixels;
    G.Nv = (int)g.det.NumTAxPixels;
    G.dims[0] = (int)g.vox.Xdim;
    G.dims[1] = (int)g.vox.Ydim;
    G.dims[2] = (int)g.vox.Zdim;
    G.vox[0] = g.vox.XVoxSize;
    G.vox[1] = g.vox.YVoxSize;
    G.vox[2] = g.vox.ZVoxSize;
    for (int k = 0; k < 3; ++k) G.P0[k] = -(double)G.dims[k] / 2.0 * G.vox[k];
    return G;
}

// The plan's views come in quarter turns of a square volume (see
// quarter_turn_table_kernel): N = 4q views, view n + q at exactly angle(n) + 90
// degrees.
static bool quarter_turn_suits(const Plan& P)
{
    const recon_geometry_t& g = P.geom;
    if (P.nviews < 4 || P.nviews % 4 != 0) return false;
    if (g.vox.Xdim != g.vox.Ydim || g.vox.Xdim % 2 != 0 || g.vox.XVoxSize != g.vox.YVoxSize) return false;
    const unsigned q = P.nviews / 4;
    for (unsigned n = 0; n < 3 * q; ++n)
        if ((double)P.view_angles[n + q] != (double)P.view_angles[n] + 90.0) return false;
    return true;
}

recon_status_t build_exact_tables(Plan& P, cudaStream_t s)
{
    exact::GeomD G = geom_d(P);
    P.quarter = quarter_turn_suits(P);
    if (P.nviews) {
        const unsigned direct = P.quarter ? P.nviews / 4 : P.nviews;  // views computed from their angles
        exact::xy_table_kernel<<<dim3((G.Nu + 127) / 128, direct), 128, 0, s>>>(G, P.d_angles, 0u, direct, P.d_txy,
                                                                              P.d_kxy, P.d_cs);
        RB_CUDA(cudaGetLastError());
        if (P.quarter) {
            exact::quarter_turn_table_kernel<<<dim3((G.Nu + 127) / 128, direct), 128, 0, s>>>(
                G.dims[0], G.Nu, direct, P.d_txy, P.d_kxy, P.d_cs);
            RB_CUDA(cudaGetLastError());
        }
    }
    exact::z_table_kernel<<<(G.Nv + 127) / 128, 128, 0, s>>>(G, P.d_zp);
    RB_CUDA(cudaGetLastError());
    exact::w_table_kernel<<<dim3((G.Nu + 127) / 128, G.Nv), 128, 0, s>>>(G, P.d_w, P.d_wq);
    RB_CUDA(cudaGetLastError());
    return RECON_OK;
}

__global__ void exact_set_angle_kernel(float* p, float v) { *p = v; }

recon_status_t exact_view_table(Plan& P, float angle, cudaStream_t s)
{
    exact::GeomD G = geom_d(P);
    exact_set_angle_kernel<<<1, 1, 0, s>>>(P.d_angles + P.nviews, angle);
    exact::xy_table_kernel<<<dim3((G.Nu + 127) / 128, 1), 128, 0, s>>>(G, P.d_angles, P.nviews, 1u, P.d_txy,
                                                                       P.d_kxy, P.d_cs);
    RB_CUDA(cudaGetLastError());
    return RECON_OK;
}

static dim3 fp_block() { return dim3(32, 4, 1); }
static dim3 fp_grid(const Plan& P, unsigned views) { return dim3((P.eg.Nu + 31) / 32, (P.eg.Nv + 3) / 4, views); }

namespace exact {
// f[z][y][x] -> ft[z][x][y], 32x32 tiles through shared memory
__global__ void __launch_bounds__(256) transpose_xy_kernel(const float* __restrict__ in, float* __restrict__ out,
                                                           int X, int Y)
{
    __shared__ float tile[32][33];
    const size_t slab = (size_t)X * Y * blockIdx.z;
    const int x0 = blockIdx.x * 32, y0 = blockIdx.y * 32;
    for (int r = threadIdx.y; r < 32; r += 8) {
        const int x = x0 + threadIdx.x, y = y0 + r;
        if (x < X && y < Y) tile[r][threadIdx.x] = in[slab + (size_t)y * X + x];
    }
    __syncthreads();
    for (int r = threadIdx.y; r < 32; r += 8) {
        const int y = y0 + threadIdx.x, x = x0 + r;
        if (x < X && y < Y) out[slab + (size_t)x * Y + y] = tile[threadIdx.x][r];
    }
}
}  // namespace exact

recon_status_t exact_transpose(const float* vol, float* vol_t, int X, int Y, int Z, cudaStream_t s)
{
    exact::transpose_xy_kernel<<<dim3((X + 31) / 32, (Y + 31) / 32, Z), dim3(32, 8), 0, s>>>(vol, vol_t, X, Y);
    RB_CUDA(cudaGetLastError());
    return RECON_OK;
}

// ---- ray culling ---------------------------------------------------------------------------

namespace exact {
// Bounding rectangle {u_min, u_max, v_min, v_max} per view of the rays that
// cross the box x in [0, X), y in [0, Y), z in [k0, k1): the clip test of the
// walks themselves, so no ray with a non-empty walk falls outside.
__global__ void __launch_bounds__(128) hit_rect_kernel(ExactGeom G, const float4* __restrict__ txy,
                                                        const int2* __restrict__ kxy, const ZParam* __restrict__ zp,
                                                        int k0, int k1, int4* __restrict__ rect)
{
    const int u = blockIdx.x * blockDim.x + threadIdx.x;
    const int v = blockIdx.y * blockDim.y + threadIdx.y;
    const unsigned view = blockIdx.z;
    if (u >= G.Nu || v >= G.Nv) return;
    const float4 T = txy[(size_t)view * G.Nu + u];
    const int2 K = kxy[(size_t)view * G.Nu + u];
    const ZParam Z = zp[v];
    const float x0 = plane_t(0, T.x, T.y, K.x), x1 = plane_t(G.X, T.x, T.y, K.x);
    const float y0 = plane_t(0, T.z, T.w, K.y), y1 = plane_t(G.Y, T.z, T.w, K.y);
    const float z0 = plane_t(k0, Z.S, Z.O, Z.kc), z1 = plane_t(k1, Z.S, Z.O, Z.kc);
    const float t_in = fmaxf(fmaxf(fminf(x0, x1), fminf(y0, y1)), fminf(z0, z1));
    const float t_out = fminf(fminf(fmaxf(x0, x1), fmaxf(y0, y1)), fmaxf(z0, z1));
    if (!(t_in < t_out)) return;
    atomicMin(&rect[view].x, u);
    atomicMax(&rect[view].y, u);
    atomicMin(&rect[view].z, v);
    atomicMax(&rect[view].w, v);
}
}  // namespace exact

// Tile list of the 32x4 ray blocks inside each plan view's rectangle of rays
// crossing the box z in [k0, k1).  Synchronous (plan creation).
static recon_status_t build_ray_tiles(Plan& P, int k0, int k1, RayTiles& T, int4** keep_rect = nullptr,
                                      std::vector<int4>* host_rect = nullptr)
{
    const unsigned nv = P.nviews;
    T.prefix.assign(nv + 1, 0);
    if (nv == 0) return RECON_OK;
    std::vector<int4> rect(nv, make_int4(INT_MAX, -1, INT_MAX, -1));
    int4* d_rect = nullptr;
    RB_CUDA(cudaMalloc(&d_rect, nv * sizeof(int4)));
    cudaError_t e = cudaMemcpy(d_rect, rect.data(), nv * sizeof(int4), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        exact::hit_rect_kernel<<<fp_grid(P, nv), fp_block()>>>(P.eg, P.d_txy, P.d_kxy, P.d_zp, k0, k1, d_rect);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(rect.data(), d_rect, nv * sizeof(int4), cudaMemcpyDeviceToHost);
    cudaFree(d_rect);
    if (e != cudaSuccess) return cuda_fail(e, "ray culling");
    if (host_rect) *host_rect = rect;
    if (keep_rect) {  // the rectangles on the device too
        RB_CHECK(P.alloc(keep_rect, nv, "ray rectangles"));
        RB_CUDA(cudaMemcpy(*keep_rect, rect.data(), nv * sizeof(int4), cudaMemcpyHostToDevice));
    }
    std::vector<uint2> tiles;
    for (unsigned n = 0; n < nv; ++n) {
        T.prefix[n] = (unsigned)tiles.size();
        const int4 r = rect[n];
        if (r.y < r.x) continue;  // no ray of this view crosses the box
        for (int tv = r.z / 4; tv <= r.w / 4; ++tv)
            for (int tu = r.x / 32; tu <= r.y / 32; ++tu) tiles.push_back(make_uint2(n, (unsigned)tu | ((unsigned)tv << 16)));
    }
    T.prefix[nv] = (unsigned)tiles.size();
    if (tiles.empty()) return RECON_OK;
    RB_CHECK(P.alloc(&T.d, tiles.size(), "ray tiles"));
    RB_CUDA(cudaMemcpy(T.d, tiles.data(), tiles.size() * sizeof(uint2), cudaMemcpyHostToDevice));
    return RECON_OK;
}

recon_status_t build_exact_culling(Plan& P)
{
    std::vector<int4> rect;
    RB_CHECK(build_ray_tiles(P, 0, P.eg.Z, P.fp_tiles, &P.d_view_rect, &rect));
    P.sino_v0 = INT_MAX;
    P.sino_v1 = -1;
    for (const int4& r : rect)
        if (r.y >= r.x) {
            P.sino_v0 = std::min(P.sino_v0, r.z);
            P.sino_v1 = std::max(P.sino_v1, r.w);
        }
    P.sino_rows_known = true;
    P.view_rect_host = rect;
    if (P.fp_column && P.nviews) {
        P.col_rows = P.opt.fp_rows ? P.opt.fp_rows : exact_column_rows_default(P, rect);
        RB_CHECK(build_column_tiles(P, rect));
    }
    P.bp_tiles.clear();
    if (P.bp_gather) return RECON_OK;  // the gather back projector needs no ray blocks
    const int depth = bp_slab_depth(P);
    for (int k0 = 0; k0 < P.eg.Z; k0 += depth) {
        P.bp_tiles.emplace_back();
        RB_CHECK(build_ray_tiles(P, k0, std::min(k0 + depth, P.eg.Z), P.bp_tiles.back()));
    }
    return RECON_OK;
}

// Launch shape for views [first, first+count): the tiles of `T` when those
// are plan views (culled), else the full grid.  *tiles is null for the full
// grid; *n_launch = 0 when no ray can contribute.
static void ray_launch(const Plan& P, const RayTiles& T, unsigned first, unsigned count, dim3* grid,
                       const uint2** tiles, unsigned* n_launch)
{
    if (first + count <= P.nviews && T.prefix.size() == P.nviews + 1) {
        const unsigned t0 = T.prefix[first], nt = T.prefix[first + count] - t0;
        *grid = dim3(std::max(nt, 1u), 1, 1);
        *tiles = T.d + t0;
        *n_launch = nt;
    } else {
        *grid = fp_grid(P, count);
        *tiles = nullptr;
        *n_launch = count;
    }
}

// Forward projection of views [first, first+count) (table slots), reading the
// volume in the layout that suits each view (the transposed copy is made
// here, once per call).  Only ray blocks that can cross the volume are
// launched; the other pixels of `out` are zeroed first, except for the MLEM
// ratio (MODE 1 and 3), whose buffer is zero outside the blocks from allocation on.
template <int MODE, class GT, class OT>
static recon_status_t launch_fp(Plan& P, const float* vol, unsigned first, unsigned count, const GT* g, OT* out,
                                cudaStream_t s)
{
    if (count == 0) return RECON_OK;
    dim3 grid;
    const uint2* tiles;
    unsigned n_launch;
    ray_launch(P, P.fp_tiles, first, count, &grid, &tiles, &n_launch);
    if (tiles && MODE != 1 && MODE != 3 && MODE != 4) RB_CUDA(cudaMemsetAsync(out, 0, (size_t)count * P.npix * sizeof(OT), s));
    if (n_launch == 0) return RECON_OK;
    RB_CHECK(exact_transpose(vol, P.d_vol_t, P.eg.X, P.eg.Y, P.eg.Z, s));
    const dim3 blk = fp_block();
    if (P.opt.sum == RECON_SUM_KAHAN)
        exact::fp_kernel<true, MODE, GT, OT><<<grid, blk, 0, s>>>(P.eg, P.d_txy, P.d_kxy, P.d_zp, P.d_w, P.d_cs,
                                                                  tiles, first, vol, P.d_vol_t, g, out);
    else
        exact::fp_kernel<false, MODE, GT, OT><<<grid, blk, 0, s>>>(P.eg, P.d_txy, P.d_kxy, P.d_zp, P.d_w, P.d_cs,
                                                                   tiles, first, vol, P.d_vol_t, g, out);
    RB_CUDA(cudaGetLastError());
    return RECON_OK;
}

recon_status_t exact_fp(Plan& P, const float* vol, unsigned first, unsigned count, bool scratch_slot, float* out,
                        cudaStream_t s)
{
    if (scratch_slot) {
        first = P.nviews;
        count = 1;
    }
    if (P.fp_column) return exact_fp_column(P, vol, first, count, out, s);
    return launch_fp<0, float, float>(P, vol, first, count, nullptr, out, s);
}

// Views [0, count) of a sinogram [view][v][u] (times w when given) into the
// detector-column layout.
// rect: per view from the first, the rectangles of rays crossing the volume
// (tiles outside them are left as they are), or null for every tile.
template <class T>
static recon_status_t to_columns(const Plan& P, const T* in, const float* w, unsigned count, const int4* rect, T* out,
                                 cudaStream_t s)
{
    for (unsigned v0 = 0; v0 < count; v0 += 65535) {
        const unsigned nv = std::min(count - v0, 65535u);
        exact::to_columns_kernel<T><<<dim3((P.eg.Nu + 31) / 32, (P.eg.Nv + 31) / 32, nv), dim3(32, 8), 0, s>>>(
            in + (size_t)v0 * P.npix, w, P.eg.Nu, P.eg.Nv, rect ? rect + v0 : nullptr, out + (size_t)v0 * P.npix);
        RB_CUDA(cudaGetLastError());
    }
    return RECON_OK;
}

// The plan's ray rectangles from view `first` for `count` views, when those are
// plan views.
static const int4* view_rects_from(const Plan& P, unsigned first, unsigned count)
{
    return (P.d_view_rect && first + count <= P.nviews) ? P.d_view_rect + first : nullptr;
}

// The MLEM ratio of views [first, first+count).  For the gather back projector
// it is written [view][v][u] into the plan's staging buffer and transposed into
// the detector-column layout.
recon_status_t exact_fp_ratio(Plan& P, const float* vol, const void* g, void* ratio, cudaStream_t s,
                              unsigned first, unsigned count)
{
    const size_t off = (size_t)first * P.npix;
    using bf = __nv_bfloat16;
    if (P.fp_column) {  // straight into the layout the back projector reads
        const bool bf16 = P.opt.sino == RECON_SINO_BF16;
        const size_t es = bf16 ? sizeof(bf) : sizeof(float);
        const int layout = !mlem_ratio_in_columns(P) ? kLayoutRows : P.col_pairs ? kLayoutPairs : kLayoutColumns;
        const size_t roff = (size_t)first * (layout == kLayoutPairs ? column_view_elems(P) : P.npix);
        return exact_fp_column_ratio(P, vol, (const char*)g + off * es, (char*)ratio + roff * es, 1, layout, bf16,
                                     first, count, s);
    }
    if (P.opt.sino == RECON_SINO_BF16) {
        bf* r = mlem_ratio_in_columns(P) ? (bf*)P.d_ratio_rm : (bf*)ratio;
        RB_CHECK((launch_fp<1, bf, bf>(P, vol, first, count, (const bf*)g + off, r + off, s)));
        if (mlem_ratio_in_columns(P))
            return to_columns<bf>(P, r + off, nullptr, count, view_rects_from(P, first, count), (bf*)ratio + off, s);
        return RECON_OK;
    }
    float* r = mlem_ratio_in_columns(P) ? (float*)P.d_ratio_rm : (float*)ratio;
    RB_CHECK((launch_fp<1, float, float>(P, vol, first, count, (const float*)g + off, r + off, s)));
    if (mlem_ratio_in_columns(P))
        return to_columns<float>(P, r + off, nullptr, count, view_rects_from(P, first, count), (float*)ratio + off, s);
    return RECON_OK;
}

// Number of (ray, voxel) pairs with positive length: the forward walk with
// a counter in place of the accumulator.
namespace exact {
__global__ void __launch_bounds__(128) count_kernel(ExactGeom G, const float4* __restrict__ txy,
                                                     const int2* __restrict__ kxy, const ZParam* __restrict__ zp,
                                                     const uint2* __restrict__ tiles,
                                                     unsigned long long* __restrict__ total)
{
    const RayPos R = ray_pos(tiles, 0u);
    const int u = R.u, v = R.v;
    const unsigned view = R.view;
    unsigned cnt = 0;
    if (u < G.Nu && v < G.Nv) {
        const float4 T = txy[(size_t)view * G.Nu + u];
        const int2 K = kxy[(size_t)view * G.Nu + u];
        const ZParam Z = zp[v];
        float x0 = plane_t(0, T.x, T.y, K.x), x1 = plane_t(G.X, T.x, T.y, K.x);
        float y0 = plane_t(0, T.z, T.w, K.y), y1 = plane_t(G.Y, T.z, T.w, K.y);
        float z0 = plane_t(0, Z.S, Z.O, Z.kc), z1 = plane_t(G.Z, Z.S, Z.O, Z.kc);
        const float t_in = fmaxf(fmaxf(fminf(x0, x1), fminf(y0, y1)), fminf(z0, z1));
        const float t_out = fminf(fminf(fmaxf(x0, x1), fmaxf(y0, y1)), fmaxf(z0, z1));
        if (t_in < t_out) {
            const double ivx = 1.0 / (double)T.x, ivy = 1.0 / (double)T.z, ivz = 1.0 / (double)Z.S;
            int ix = locate<true>(t_in, T.x, T.y, K.x, G.X, ivx), ex = locate<false>(t_out, T.x, T.y, K.x, G.X, ivx);
            int iy = locate<true>(t_in, T.z, T.w, K.y, G.Y, ivy), ey = locate<false>(t_out, T.z, T.w, K.y, G.Y, ivy);
            int iz = locate<true>(t_in, Z.S, Z.O, Z.kc, G.Z, ivz), ez = locate<false>(t_out, Z.S, Z.O, Z.kc, G.Z, ivz);
            const int nsteps = abs(ex - ix) + abs(ey - iy) + abs(ez - iz) + 1;
            const int dx = T.x > 0.0f ? 1 : -1, dy = T.z > 0.0f ? 1 : -1, dz = Z.S > 0.0f ? 1 : -1;
            float kx = (float)((dx > 0 ? ix + 1 : ix) - K.x);
            float ky = (float)((dy > 0 ? iy + 1 : iy) - K.y);
            float kz = (float)((dz > 0 ? iz + 1 : iz) - Z.kc);
            float tx = fmaf(kx, T.x, T.y), ty = fmaf(ky, T.z, T.w), tz = fmaf(kz, Z.S, Z.O);
            float cur = t_in;
            for (int s = 0; s < nsteps; ++s) {
                const float m = fminf(tx, fminf(ty, tz));
                cnt += (m > cur) ? 1u : 0u;
                cur = m;
                if (tx == m) {
                    kx += (float)dx;
                    tx = fmaf(kx, T.x, T.y);
                } else if (ty == m) {
                    ky += (float)dy;
                    ty = fmaf(ky, T.z, T.w);
                } else {
                    kz += (float)dz;
                    tz = fmaf(kz, Z.S, Z.O);
                }
            }
        }
    }
    for (int o = 16; o > 0; o >>= 1) cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
    if ((threadIdx.x & 31) == 0 && cnt) atomicAdd(total, (unsigned long long)cnt);
}
}  // namespace exact

recon_status_t exact_count(Plan& P, unsigned long long* out)
{
    unsigned long long* d = nullptr;
    RB_CUDA(cudaMalloc(&d, sizeof(unsigned long long)));
    cudaError_t e = cudaMemset(d, 0, sizeof(unsigned long long));
    if (e == cudaSuccess && P.nviews) {
        dim3 grid;
        const uint2* tiles;
        unsigned n_launch;
        ray_launch(P, P.fp_tiles, 0, P.nviews, &grid, &tiles, &n_launch);
        if (n_launch) {
            exact::count_kernel<<<grid, fp_block()>>>(P.eg, P.d_txy, P.d_kxy, P.d_zp, tiles, d);
            e = cudaGetLastError();
        }
    }
    if (e == cudaSuccess) e = cudaMemcpy(out, d, sizeof(unsigned long long), cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (e != cudaSuccess) return cuda_fail(e, "intersection count");
    return RECON_OK;
}

recon_status_t exact_fp_plain_ratio(Plan& P, const float* vol, const float* g, float* ratio, cudaStream_t s)
{
    if (P.fp_column)
        return exact_fp_column_ratio(P, vol, g, ratio, 2, voxel_ratio_in_columns(P) ? kLayoutColumns : kLayoutRows,
                                     false, 0u, P.nviews, s);
    if (voxel_ratio_in_columns(P)) {
        float* r = (float*)P.d_ratio_rm;
        RB_CHECK((launch_fp<2, float, float>(P, vol, 0u, P.nviews, g, r, s)));
        return to_columns<float>(P, r, nullptr, P.nviews, view_rects_from(P, 0, P.nviews), ratio, s);
    }
    return launch_fp<2, float, float>(P, vol, 0u, P.nviews, g, ratio, s);
}

// Bound on the number of contributions one voxel receives from `nview`
// views, as bits: a voxel's projection is at most diag * Ry / depth_min
// detector pitches wide in u and in v, so at most floor(w) + 2 pixel centres
// per axis see it.
int bp_count_bits(const Plan& P, unsigned nview)
{
    const ExactGeom& E = P.eg;
    const double vx = E.vox[0], vy = E.vox[1], vz = E.vox[2];
    const double diag = std::sqrt(vx * vx + vy * vy + vz * vz);
    const double hx = 0.5 * E.X * vx, hy = 0.5 * E.Y * vy, hz = 0.5 * E.Z * vz;
    const double depth_min = std::max((double)E.Rf - std::sqrt(hx * hx + hy * hy + hz * hz), 1e-3);
    const double mag = std::fabs((double)E.Ry) / depth_min;
    const double fu = diag * mag / std::fabs((double)E.du), fv = diag * mag / std::fabs((double)E.dv);
    const double total = (double)std::max(nview, 1u) * (std::floor(fu) + 2.0) * (std::floor(fv) + 2.0);
    return (int)std::ceil(std::log2(total)) + 1;
}

// Longest segment in t: a segment's length in t is at most its length in
// mm (the source-to-pixel distance is at least R), at most a voxel diagonal.
float bp_max_len(const Plan& P)
{
    const ExactGeom& E = P.eg;
    return (float)(std::sqrt((double)E.vox[0] * E.vox[0] + (double)E.vox[1] * E.vox[1] +
                             (double)E.vox[2] * E.vox[2]) * 1.0001);
}

// z-slices per slab: both accumulators of a slab (16 bytes per voxel) in
// about 64 MiB, which stays resident in the 126 MB L2.
int bp_slab_depth(const Plan& P)
{
    const size_t per_slice = (size_t)P.eg.X * P.eg.Y * 2 * sizeof(unsigned long long);
    return (int)std::max<size_t>(1, std::min<size_t>((size_t)P.eg.Z, (size_t(64) << 20) / per_slice));
}

template <int MODE, bool WEIGHTED, class ST>
static recon_status_t launch_bp(Plan& P, const ST* sino, unsigned first, unsigned count, float* vol,
                                const float* sens, cudaStream_t s)
{
    // max |value| of this call's input, for the fixed-point scale
    RB_CUDA(cudaMemsetAsync(P.d_bpmax, 0, sizeof(unsigned), s));
    const size_t n = (MODE == 1) ? P.npix : (size_t)count * P.npix;
    const unsigned mblocks = (unsigned)std::min<size_t>((n + 255) / 256, (size_t)P.sm_count * 8);
    if (MODE == 1)
        exact::maxabs_kernel<float><<<mblocks, 256, 0, s>>>(P.d_w, n, nullptr, P.npix, P.d_bpmax);
    else
        exact::maxabs_kernel<ST><<<mblocks, 256, 0, s>>>(sino, n, WEIGHTED ? P.d_w : nullptr, P.npix, P.d_bpmax);
    RB_CUDA(cudaGetLastError());
    const float max_len = bp_max_len(P);
    const int cbits = bp_count_bits(P, count);
    const int depth = bp_slab_depth(P);
    const dim3 blk = fp_block();
    constexpr int RMODE = (MODE == 1) ? 1 : 0;
    const RayTiles none;
    for (int k0 = 0, slab = 0; k0 < P.eg.Z; k0 += depth, ++slab) {
        const int k1 = std::min(k0 + depth, P.eg.Z);
        dim3 grid;
        const uint2* tiles;
        unsigned n_launch;
        ray_launch(P, slab < (int)P.bp_tiles.size() ? P.bp_tiles[slab] : none, first, count, &grid, &tiles,
                   &n_launch);
        if (n_launch) {
            exact::bp_ray_kernel<RMODE, WEIGHTED, ST><<<grid, blk, 0, s>>>(P.eg, P.d_txy, P.d_kxy, P.d_cs, P.d_zp,
                                                                           P.d_w, tiles, first, sino, P.d_bpmax,
                                                                           max_len, cbits, k0, k1, P.d_bpacc,
                                                                           P.d_bpacc_t);
            RB_CUDA(cudaGetLastError());
        }
        const dim3 fgrid((P.eg.X + 31) / 32, (P.eg.Y + 31) / 32, k1 - k0);
        exact::bp_finish_kernel<MODE == 2 ? 2 : 0><<<fgrid, dim3(32, 8), 0, s>>>(P.eg, P.d_bpmax, max_len, cbits,
                                                                                 k0, P.d_bpacc, P.d_bpacc_t, vol,
                                                                                 sens);
        RB_CUDA(cudaGetLastError());
    }
    return RECON_OK;
}

// The gather back projector is the faster one where each voxel has about one
// candidate row per detector column and view: the rays of adjacent detector
// rows cross a column 1 to 1.4 voxels apart in z (at the depth nearest the
// source; closer rows give voxels several candidates, further ones leave many
// voxels without one while the gather still pays for them), a ray's piece of
// one column spans less than one voxel of z, and columns are at least 128
// voxels tall (shorter ones leave the per-view set-up unamortised).  Measured
// on one B200: 0.75x the ray design's time at 256^3 / 360 views / 512^2,
// 0.93x at 128^3; 0.90-0.97x on the generated problems inside these bounds and
// 1.1-2.2x outside them.
bool exact_bp_gather_suits(const Plan& P)
{
    const ExactGeom& E = P.eg;
    const double vx = E.vox[0], vy = E.vox[1], vz = E.vox[2];
    const double hx = 0.5 * E.X * vx, hy = 0.5 * E.Y * vy;
    const double d_min = (double)E.Rf - std::sqrt(hx * hx + hy * hy);
    if (!(d_min > 0.0) || !(vz > 0.0) || E.Ry == 0.0f) return false;
    const double ry = std::fabs((double)E.Ry), dv = std::fabs((double)E.dv);
    const double row_step = d_min * dv / (ry * vz);
    const double slope = (0.5 * E.Nv * dv + std::fabs((double)E.Dz)) / ry;  // max |dz / d(depth)| of a ray
    const double needle = std::sqrt(vx * vx + vy * vy) * slope / vz;
    return row_step >= 1.0 && row_step <= 1.4 && needle < 1.0 && E.Nv <= 3072 && E.Z >= 128;
}

// Both projectors pair mirrored rows / voxels (walk_rows_mirror,
// bp_gather_mirror_kernel) when the volume has an even number of slices and
// the plan's z table is exactly mirror-symmetric: row Nv-1-v has S = -S_v,
// O = O_v and kc = Z - kc_v, so that its plane Z-k is row v's plane k bit for
// bit, and the lower rows (v < Nv/2) descend along t.  That holds with no
// vertical detector offset (Dz = 0) and symmetric pixel centres; the table
// itself is checked (synchronous, at plan creation, before the culling that
// lays out the forward projector's tiles).
recon_status_t exact_check_mirror(Plan& P)
{
    P.z_mirror = false;
    if (P.eg.Z % 2 != 0 || P.eg.Z < 2) return RECON_OK;
    std::vector<ZParam> z(P.eg.Nv);
    RB_CUDA(cudaMemcpy(z.data(), P.d_zp, z.size() * sizeof(ZParam), cudaMemcpyDeviceToHost));
    const int n = P.eg.Nv;
    for (int v = 0; v < n; ++v) {
        const ZParam& a = z[v];
        const ZParam& b = z[n - 1 - v];
        if (!(b.S == -a.S && b.O == a.O && b.kc == P.eg.Z - a.kc)) return RECON_OK;
        if (v < n / 2 && !(a.S < 0.0f)) return RECON_OK;  // lower rows descend along t
    }
    P.z_mirror = true;
    return RECON_OK;
}

// RECON_SIDDON_BP_TUNED: the design a plan of this geometry (on this device)
// measured faster, kept for the process so that every plan of the geometry
// makes the same choice.
namespace {
std::mutex g_bp_tune_mutex;
std::map<std::string, bool> g_bp_tune_gather;
}  // namespace

// The geometry and device of a plan as a key of the tuning caches (floats
// written exactly, as hexadecimal).
std::string geometry_key(const Plan& P)
{
    const recon_geometry_t& g = P.geom;
    char buf[512];
    std::snprintf(buf, sizeof buf, "%d|%a %a %a %a %a %a|%u %u %a %a|%u %u %u %a %a %a|%u %a", P.device, g.cal.R,
                  g.cal.Rf, g.cal.Ry, g.cal.Dx, g.cal.Dz, g.cal.M, g.det.NumTAxPixels, g.det.NumAxPixels,
                  g.det.TAxPixDimMm, g.det.AxPixDimMm, g.vox.Xdim, g.vox.Ydim, g.vox.Zdim, g.vox.XVoxSize,
                  g.vox.YVoxSize, g.vox.ZVoxSize, g.scan.NumProj, g.scan.DeltaAng);
    return buf;
}

void plan_release(Plan& P, void* p, size_t bytes)
{
    if (!p) return;
    cudaFree(p);
    P.allocations.erase(std::find(P.allocations.begin(), P.allocations.end(), p));
    P.device_bytes -= bytes;
}

// Times the plan's sensitivity back projection (all views, both designs set up
// by the plan) with each design, CUDA events around the second of two runs on
// the legacy stream, and keeps the faster; the ray design's slab accumulators
// are released when the gather wins.  Synchronous (plan creation).
recon_status_t exact_tune_bp(Plan& P)
{
    const std::string key = geometry_key(P);
    bool known = false, gather = true;
    {
        std::lock_guard<std::mutex> lock(g_bp_tune_mutex);
        auto it = g_bp_tune_gather.find(key);
        if (it != g_bp_tune_gather.end()) {
            known = true;
            gather = it->second;
        }
    }
    if (!known && P.nviews > 0) {
        float* out = nullptr;
        RB_CUDA(cudaMalloc(&out, P.nvox * sizeof(float)));
        cudaEvent_t e0 = nullptr, e1 = nullptr;
        cudaError_t e = cudaEventCreate(&e0);
        if (e == cudaSuccess) e = cudaEventCreate(&e1);
        float ms[2] = {0.0f, 0.0f};
        recon_status_t st = RECON_OK;
        for (int d = 0; d < 2 && e == cudaSuccess && st == RECON_OK; ++d) {
            P.bp_gather = (d == 0);
            P.col_pairs = (d == 0) && P.d_wq_pairs != nullptr;  // as the plan will use the gather
            st = exact_bp(P, nullptr, false, false, 0, P.nviews, false, true, out, nullptr, nullptr, 0);
            if (st == RECON_OK) e = cudaEventRecord(e0, 0);
            if (e == cudaSuccess && st == RECON_OK)
                st = exact_bp(P, nullptr, false, false, 0, P.nviews, false, true, out, nullptr, nullptr, 0);
            if (e == cudaSuccess && st == RECON_OK) e = cudaEventRecord(e1, 0);
            if (e == cudaSuccess && st == RECON_OK) e = cudaEventSynchronize(e1);
            if (e == cudaSuccess && st == RECON_OK) e = cudaEventElapsedTime(&ms[d], e0, e1);
        }
        if (e0) cudaEventDestroy(e0);
        if (e1) cudaEventDestroy(e1);
        cudaFree(out);
        if (st != RECON_OK) return st;
        if (e != cudaSuccess) return cuda_fail(e, "back projector tuning");
        gather = ms[0] <= ms[1];
        std::lock_guard<std::mutex> lock(g_bp_tune_mutex);
        g_bp_tune_gather.emplace(key, gather);
    }
    P.bp_gather = gather;
    if (gather) {
        const size_t slab = (size_t)P.eg.X * P.eg.Y * bp_slab_depth(P) * sizeof(unsigned long long);
        plan_release(P, P.d_bpacc, slab);
        plan_release(P, P.d_bpacc_t, slab);
        plan_release(P, P.d_bpmax, sizeof(unsigned));
        P.d_bpacc = P.d_bpacc_t = nullptr;
        P.d_bpmax = nullptr;
    }
    return RECON_OK;
}

// Largest detector row count the gather back projector takes: its rows' z
// planes are held in shared memory, 16 bytes per row, beside 18 KB of per-warp
// arrays, within the 227 KB a block may use.
int exact_bp_gather_max_rows() { return 12288; }

static exact::GatherConst gather_const(const Plan& P, const float* vol, const float* sens)
{
    const ExactGeom& E = P.eg;
    exact::GatherConst C;
    C.eu = (float)((double)E.Ry / E.du);
    C.ou = (float)(-((double)E.Dx + E.ud0) / E.du);
    C.ez = (float)((double)E.Ry / E.dv);
    C.oz = (float)(-((double)E.Dz + E.vd0) / E.dv);
    C.vec4 = (E.X % 4 == 0) && (reinterpret_cast<uintptr_t>(vol) % 16 == 0) &&
             (reinterpret_cast<uintptr_t>(sens) % 16 == 0);
    return C;
}

// bp_gather_quarter_kernel's shared memory: the rows' z planes and its staging
// area (dynamic), the per-warp view set-up (static).
template <int PS>
static size_t quarter_dynamic_smem(const Plan& P)
{
    return (size_t)P.eg.Nv * sizeof(float4) + sizeof(float) * exact::kGatherWarps * 8 * PS * 32;
}
constexpr size_t kQuarterStaticSmem = sizeof(exact::GatherView) * 32 * exact::kGatherWarps;

// The quarter-turn gather serves this call: all of the plan's views, which
// come in exact quarter turns, in mirrored row pairs, within a block's shared
// memory.
template <int PS>
static bool quarter_gather_serves(const Plan& P, unsigned first, unsigned count)
{
    return P.quarter && P.col_pairs && P.z_mirror && first == 0 && count == P.nviews && count >= 4 &&
           quarter_dynamic_smem<PS>(P) + kQuarterStaticSmem <= 227 * 1024;
}

// The plan's MLEM back projection takes quarter sets of views
// (exact_bp_quarters): the quarter-turn gather is its back projector.
bool exact_quarter_sets(const Plan& P)
{
    return P.opt.arith == RECON_ARITH_EXACT && P.opt.bp == RECON_BP_SIDDON && P.bp_gather &&
           quarter_gather_serves<4>(P, 0, P.nviews);
}

// vals: view 0 of the plan's views; m0, mc: the base views of the quarter set
template <int EPI, class ST, int PS, bool SET = false>
static recon_status_t launch_gather_quarter(Plan& P, const ST* vals, size_t view_stride, float* vol,
                                            const float* sens, cudaStream_t s, unsigned long long* npairs,
                                            unsigned m0, unsigned mc)
{
    const ExactGeom& E = P.eg;
    const exact::GatherConst C = gather_const(P, vol, sens);
    const size_t smem = quarter_dynamic_smem<PS>(P);
    auto kernel = exact::bp_gather_quarter_kernel<EPI, ST, PS, SET>;
    if (smem + kQuarterStaticSmem > 48 * 1024)
        RB_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    constexpr int tx = exact::kGatherTileX, ty = exact::kGatherWarps / exact::kGatherTileX;
    const int H = E.X / 2;  // base columns: the quadrant x, y < X/2
    const dim3 grid((H + tx - 1) / tx, (H + ty - 1) / ty);
    kernel<<<grid, exact::kGatherWarps * 32, smem, s>>>(E, C, P.d_txy, P.d_kxy, P.d_cs, P.d_zp, P.nviews, m0, mc,
                                                         vals, view_stride, vol, sens, npairs);
    RB_CUDA(cudaGetLastError());
    return RECON_OK;
}

// SLOTS: voxels per lane for bp_gather_kernel, voxel pairs per lane for the
// mirror kernels (MIRROR).
template <int EPI, class ST, int SLOTS, bool MIRROR = false>
static recon_status_t launch_gather_slots(Plan& P, const ST* vals, size_t view_stride, unsigned first,
                                          unsigned count, float* vol, const float* sens, cudaStream_t s,
                                          unsigned long long* npairs = nullptr)
{
    const ExactGeom& E = P.eg;
    const exact::GatherConst C = gather_const(P, vol, sens);
    const size_t smem = (size_t)E.Nv * sizeof(float4);
    auto kernel = [&P] {
        if constexpr (MIRROR)
            return P.col_pairs ? exact::bp_gather_pairs_kernel<EPI, ST, SLOTS> : exact::bp_gather_mirror_kernel<EPI, ST, SLOTS>;
        else return exact::bp_gather_kernel<EPI, ST, SLOTS>;
    }();
    const size_t static_smem = sizeof(exact::GatherView) * 32 * exact::kGatherWarps +          // sview
                               sizeof(float) * exact::kGatherWarps * SLOTS * 32 * (MIRROR ? 2 : 1);  // sacc2
    if (smem + static_smem > 48 * 1024)
        RB_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    constexpr int tx = exact::kGatherTileX, ty = exact::kGatherWarps / exact::kGatherTileX;
    const dim3 grid((E.X + tx - 1) / tx, (E.Y + ty - 1) / ty);
    kernel<<<grid, exact::kGatherWarps * 32, smem, s>>>(E, C, P.d_txy, P.d_kxy, P.d_cs, P.d_zp, first, count, vals,
                                                         view_stride, vol, sens, npairs);
    RB_CUDA(cudaGetLastError());
    return RECON_OK;
}

// Voxels per lane: the volume's height in as few chunks of at most 8 x 32
// slices as possible, split evenly (a lane's slots beyond the volume cost
// as much as used ones).
int gather_slots(int Z)
{
    const int chunks = (Z + 255) / 256;
    return std::min(8, std::max(1, (Z + 32 * chunks - 1) / (32 * chunks)));
}

// Voxel pairs per lane for the mirror kernel: the lower half's height in as
// few chunks of at most 4 x 32 slices as possible, split evenly.
int gather_mirror_slots(int Z)
{
    const int half = Z / 2;
    const int chunks = (half + 127) / 128;
    return std::min(4, std::max(1, (half + 32 * chunks - 1) / (32 * chunks)));
}

// Voxel pairs per lane for the quarter-turn kernel: the lower half's height
// in as few chunks of at most kQuarterSlots x 32 slices as possible, split
// evenly.
constexpr int kQuarterSlots = 4;
static int gather_quarter_slots(int Z)
{
    const int half = Z / 2;
    const int chunks = (half + 32 * kQuarterSlots - 1) / (32 * kQuarterSlots);
    return std::min(kQuarterSlots, std::max(1, (half + 32 * chunks - 1) / (32 * chunks)));
}

template <int EPI, class ST>
static recon_status_t launch_gather(Plan& P, const ST* vals, size_t view_stride, unsigned first, unsigned count,
                                    float* vol, const float* sens, cudaStream_t s,
                                    unsigned long long* npairs = nullptr)
{
    if (P.z_mirror) {
        if (quarter_gather_serves<kQuarterSlots>(P, first, count)) {
            const unsigned q = P.nviews / 4;
            switch (gather_quarter_slots(P.eg.Z)) {
                case 1: return launch_gather_quarter<EPI, ST, 1>(P, vals, view_stride, vol, sens, s, npairs, 0u, q);
                case 2: return launch_gather_quarter<EPI, ST, 2>(P, vals, view_stride, vol, sens, s, npairs, 0u, q);
                case 3: return launch_gather_quarter<EPI, ST, 3>(P, vals, view_stride, vol, sens, s, npairs, 0u, q);
                default: return launch_gather_quarter<EPI, ST, 4>(P, vals, view_stride, vol, sens, s, npairs, 0u, q);
            }
        }
        switch (gather_mirror_slots(P.eg.Z)) {
            case 1: return launch_gather_slots<EPI, ST, 1, true>(P, vals, view_stride, first, count, vol, sens, s, npairs);
            case 2: return launch_gather_slots<EPI, ST, 2, true>(P, vals, view_stride, first, count, vol, sens, s, npairs);
            case 3: return launch_gather_slots<EPI, ST, 3, true>(P, vals, view_stride, first, count, vol, sens, s, npairs);
            default: return launch_gather_slots<EPI, ST, 4, true>(P, vals, view_stride, first, count, vol, sens, s, npairs);
        }
    }
#define RB_GATHER_SLOTS(n) \
    case n: return launch_gather_slots<EPI, ST, n>(P, vals, view_stride, first, count, vol, sens, s, npairs)
    switch (gather_slots(P.eg.Z)) {
        RB_GATHER_SLOTS(1);
        RB_GATHER_SLOTS(2);
        RB_GATHER_SLOTS(3);
        RB_GATHER_SLOTS(4);
        RB_GATHER_SLOTS(5);
        RB_GATHER_SLOTS(6);
        RB_GATHER_SLOTS(7);
        default: return launch_gather_slots<EPI, ST, 8>(P, vals, view_stride, first, count, vol, sens, s, npairs);
    }
#undef RB_GATHER_SLOTS
}

// The MLEM ratio's back projection over the quarter set of base views first ..
// first + count - 1 (first + count <= N/4) and their quarter turns, into vol
// (overwritten); the plan takes quarter sets (exact_quarter_sets).
recon_status_t exact_bp_quarters(Plan& P, unsigned first, unsigned count, float* vol, cudaStream_t s)
{
    if (!exact_quarter_sets(P)) return fail(RECON_ERR_UNSUPPORTED, "the plan's back projection takes no quarter sets");
    if ((size_t)first + count > P.nviews / 4) return fail(RECON_ERR_INVALID_ARGUMENT, "quarter range beyond NumProj/4");
    if (count == 0) return launch_fill(vol, 0.0f, P.nvox, s);
    const size_t qv = column_view_elems(P);
    auto run = [&](auto tag) -> recon_status_t {
        using ST = decltype(tag);
        const ST* vals = static_cast<const ST*>(P.d_ratio);
        switch (gather_quarter_slots(P.eg.Z)) {
            case 1: return launch_gather_quarter<0, ST, 1, true>(P, vals, qv, vol, nullptr, s, nullptr, first, count);
            case 2: return launch_gather_quarter<0, ST, 2, true>(P, vals, qv, vol, nullptr, s, nullptr, first, count);
            case 3: return launch_gather_quarter<0, ST, 3, true>(P, vals, qv, vol, nullptr, s, nullptr, first, count);
            default: return launch_gather_quarter<0, ST, 4, true>(P, vals, qv, vol, nullptr, s, nullptr, first, count);
        }
    };
    if (P.opt.sino == RECON_SINO_BF16) return run(__nv_bfloat16{});
    return run(float{});
}

// (ray, voxel) pairs the gather back projector gives a positive length, over
// all plan views (synchronous).  Its candidate rows and detector columns are
// found with margins; this count equals the forward walk's exactly when no
// pair is lost to them.
recon_status_t exact_bp_gather_count(Plan& P, unsigned long long* total)
{
    unsigned long long* d = nullptr;
    RB_CUDA(cudaMalloc(&d, sizeof(unsigned long long)));
    cudaError_t e = cudaMemset(d, 0, sizeof(unsigned long long));
    recon_status_t st = RECON_OK;
    if (e == cudaSuccess && P.nviews)
        st = launch_gather<2, float>(P, P.col_pairs ? P.d_wq_pairs : P.d_wq, 0, 0u, P.nviews, nullptr, nullptr, 0,
                                     d);  // the weights in the layout the kernel reads
    if (e == cudaSuccess && st == RECON_OK) e = cudaMemcpy(total, d, sizeof(unsigned long long), cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (st != RECON_OK) return st;
    if (e != cudaSuccess) return cuda_fail(e, "gather pair count");
    return RECON_OK;
}

// Scratch for `count` views in the detector-column layout (grown on demand).
static recon_status_t ensure_column_scratch(Plan& P, unsigned count)
{
    if (P.colsino_views >= count) return RECON_OK;
    if (P.d_colsino) {
        cudaFree(P.d_colsino);
        P.allocations.erase(std::find(P.allocations.begin(), P.allocations.end(), (void*)P.d_colsino));
        P.device_bytes -= (size_t)P.colsino_views * column_view_elems(P) * sizeof(float);
        P.d_colsino = nullptr;
        P.colsino_views = 0;
    }
    RB_CHECK(P.alloc(&P.d_colsino, (size_t)count * column_view_elems(P), "detector-column sinogram"));
    P.colsino_views = count;
    return RECON_OK;
}

// The MLEM ratio is stored in the detector-column layout [view][u][v] when the
// gather back projector reads it, else [view][v][u].
bool mlem_ratio_in_columns(const Plan& P)
{
    return P.bp_gather && P.opt.arith == RECON_ARITH_EXACT && P.opt.bp == RECON_BP_SIDDON;
}

// The voxel-driven back projector's ratio (no w) is in detector columns too
// for EXACT plans in GEOMETRIC mode (no detector tilt there), read by its
// gather kernel.
bool voxel_ratio_in_columns(const Plan& P)
{
    return P.opt.arith == RECON_ARITH_EXACT && P.opt.bp == RECON_BP_VOXEL && P.opt.voxel_mode == RECON_VOXEL_GEOMETRIC;
}

// The gather's inputs in mirrored row pairs (kLayoutPairs) where both projectors
// pair mirrored rows: the z table is mirror-symmetric, the forward projector
// walks detector columns, the detector has an even row count.  Builds the pair
// copy of w that the sensitivity reads; the plan sets col_pairs where the
// gather is its back projector.
bool exact_pairs_suit(const Plan& P)
{
    return P.z_mirror && P.fp_column && P.eg.Nv % 2 == 0 && P.opt.arith == RECON_ARITH_EXACT &&
           P.opt.bp == RECON_BP_SIDDON;
}

recon_status_t build_wq_pairs(Plan& P)
{
    if (P.d_wq_pairs) return RECON_OK;
    const size_t n = (size_t)P.eg.Nu * (P.eg.Nv / 2 + 1);
    RB_CHECK(P.alloc(&P.d_wq_pairs, 2 * n, "ray weights (mirrored row pairs)"));
    exact::wq_pairs_kernel<<<(unsigned)std::min<size_t>((n + 255) / 256, 148 * 8), 256>>>(P.d_wq, P.eg.Nu, P.eg.Nv,
                                                                                         P.d_wq_pairs);
    RB_CUDA(cudaGetLastError());
    return RECON_OK;
}

recon_status_t exact_bp(Plan& P, const void* sino, bool sino_is_rw, bool bf16, unsigned first, unsigned count,
                        bool scratch_slot, bool sens_mode, float* vol, const float* sens, float* f_update,
                        cudaStream_t s)
{
    if (scratch_slot) {
        first = P.nviews;
        count = 1;
    }
    if (count == 0) return launch_fill(f_update ? f_update : vol, 0.0f, P.nvox, s);
    using bf = __nv_bfloat16;
    if (P.bp_gather) {
        const size_t qv = column_view_elems(P);
        if (sens_mode)
            return launch_gather<false, float>(P, P.col_pairs ? P.d_wq_pairs : P.d_wq, 0, first, count, vol, nullptr, s);
        if (sino_is_rw) {  // the MLEM ratio: detector columns, carries w
            float* out = f_update ? f_update : vol;
            if (bf16) {
                if (f_update) return launch_gather<true, bf>(P, (const bf*)sino, qv, first, count, out, sens, s);
                return launch_gather<false, bf>(P, (const bf*)sino, qv, first, count, out, nullptr, s);
            }
            if (f_update) return launch_gather<true, float>(P, (const float*)sino, qv, first, count, out, sens, s);
            return launch_gather<false, float>(P, (const float*)sino, qv, first, count, out, nullptr, s);
        }
        // a sinogram [view][v][u]: weighted by w into the gather's layout first
        RB_CHECK(ensure_column_scratch(P, count));
        if (P.col_pairs) {
            const ExactGeom& E = P.eg;
            exact::to_pairs_kernel<float><<<dim3((E.Nu + 31) / 32, (E.Nv / 2 + 1 + 31) / 32, count), dim3(32, 8), 0, s>>>(
                (const float*)sino, P.d_wq, E.Nu, E.Nv, P.d_colsino);
            RB_CUDA(cudaGetLastError());
        } else {
            RB_CHECK(to_columns<float>(P, (const float*)sino, P.d_w, count, nullptr, P.d_colsino, s));
        }
        return launch_gather<false, float>(P, P.d_colsino, qv, first, count, vol, nullptr, s);
    }
    if (sens_mode) return launch_bp<1, false, float>(P, nullptr, first, count, vol, nullptr, s);
    if (f_update) {
        if (bf16) return launch_bp<2, false, bf>(P, (const bf*)sino, first, count, f_update, sens, s);
        return launch_bp<2, false, float>(P, (const float*)sino, first, count, f_update, sens, s);
    }
    if (sino_is_rw) {
        if (bf16) return launch_bp<0, false, bf>(P, (const bf*)sino, first, count, vol, nullptr, s);
        return launch_bp<0, false, float>(P, (const float*)sino, first, count, vol, nullptr, s);
    }
    return launch_bp<0, true, float>(P, (const float*)sino, first, count, vol, nullptr, s);
}

}  // namespace rb
