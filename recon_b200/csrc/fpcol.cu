// fpcol.cu -- EXACT forward projection by detector columns.
//
// With no detector tilt, every ray of one detector column (view, u) crosses the
// same (x, y) voxel columns at the same t: its x and y plane crossings depend on
// (view, u) only, its z crossings on the row v only.  A CTA therefore builds the
// column's xy path once -- piece j is the rays' stretch [t_{j-1}, t_j] inside one
// (x, y) voxel column, found by ranking every x crossing among the y crossings
// and the other way round (a thread-parallel merge, ties x first as in the ray
// walk) -- and each warp walks the path for 32 consecutive detector rows, one
// row per lane.  A lane tracks only its row's z planes: per piece it adds
//     (m - t_{j-1}) * f[layer] + (t_j - m) * f[next layer],   m = min(t_z, t_j),
// and steps to the next layer when its next z plane t_z falls inside the piece.
// The plan uses this kernel only where a piece spans less than a voxel of z
// (0.9 at most, from the steepest row and the column diagonal), so a piece
// holds at most one z crossing.  The volume is read from a z-fastest copy with
// a zero layer below and above every column: the 32 rows of a warp read
// neighbouring addresses, and a row outside the volume reads zeros, which
// spares the lanes any entry and exit tests except where a row leaves the
// volume through its top or bottom before the path ends.
//
// Every (ray, voxel) pair gets the length min(t_j, hi_z) - max(t_{j-1}, lo_z)
// from the plane values plane_t of the ray walk (exact_device.cuh) and of both
// back projectors, so the projector pair stays an exact transpose; only the
// order of the ray sum's additions differs from the walk.  Ray sums are
// compensated (Kahan) over blocks of pieces (8 per block, 16 in the mirrored
// walk): each block's products are summed in FP32 and the block sums
// Kahan-added.
#include "exact_device.cuh"
#include "internal.h"

#include <algorithm>
#include <climits>
#include <cmath>
#include <map>
#include <mutex>
#include <string>
#include <type_traits>

namespace rb {
namespace exact {

constexpr int kColRows = 128;  // at most this many detector rows per CTA (one warp per 32; the plan picks 32, 64 or 128)

// Number of b in [0, n) whose plane value fmaf(q0 + b*d, S, O) lies before t
// (strictly when LT, else at or before); the values increase with b (d has the
// sign of S).  Estimated from the first value and the step |S|, then corrected
// against the FP32 plane values themselves.
template <bool LT>
__device__ __forceinline__ int count_before(float t, int q0, int d, float S, float O, float inv_abs_S, int n)
{
    auto before = [&](int b) {
        const float tb = fmaf((float)(q0 + b * d), S, O);
        return LT ? (tb < t) : (tb <= t);
    };
    int c = (int)ceilf((t - fmaf((float)q0, S, O)) * inv_abs_S);
    c = min(max(c, 0), n);
    while (c < n && before(c)) ++c;
    while (c > 0 && !before(c - 1)) --c;
    return c;
}

// Smallest piece index j in [0, n) whose end spc[j].x is after t (STRICT) or at
// or after t; the last piece ends at the path's exit, which the callers' t
// never passes.
template <bool STRICT>
__device__ __forceinline__ int first_piece_ending(const float2* spc, int n, float t)
{
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        const float e = spc[mid].x;
        if (STRICT ? (e > t) : (e >= t)) hi = mid;
        else lo = mid + 1;
    }
    return lo;
}

__device__ __forceinline__ void kahan_add(float& acc, float& comp, float x)
{
    const float y = x - comp;
    const float t = acc + y;
    comp = (t - acc) - y;
    acc = t;
}

// One warp's rows over pieces jb..je.  Per lane: cur = start of the next
// piece, kaddr = offset of the row's current layer in a padded column (layer
// k at k + 1), kf = index of the next z plane minus kc as a float, tzn = that
// plane's t.  STEP = the layer step of every lane (+1 or -1), or 0 for a
// warp with rows of both directions (step then holds each lane's).  Unless
// FAST, a lane that leaves through the far face (kaddr reaching kexit) parks
// its next plane at infinity.  COUNT: no volume reads; the result is the
// number of pieces of positive length the row has inside the volume (its
// (ray, voxel) pairs).
template <bool KAHAN, bool FAST, int STEP, bool COUNT>
__device__ __forceinline__ float walk_rows(const float* __restrict__ volz, const float2* spc, int jb, int je, float cur,
                                           int kaddr, float kf, float tzn, float S, float O, int step, int kexit,
                                           int Z)
{
    const int st = STEP != 0 ? STEP : step;
    const float fst = (float)st;
    float acc = 0.0f, comp = 0.0f, f1 = 0.0f;
    auto piece = [&](int j, float& blk) {
        const float2 pc = spc[j];
        const float B = pc.x;
        const float* p = volz + (__float_as_int(pc.y) + kaddr);
        const bool cross = tzn < B;
        const float m = fminf(tzn, B);
        if (COUNT) {  // layers 0 .. Z-1 sit at kaddr 1 .. Z
            blk += (m - cur > 0.0f && (unsigned)(kaddr - 1) < (unsigned)Z) ? 1.0f : 0.0f;
            blk += (B - m > 0.0f && (unsigned)(kaddr + st - 1) < (unsigned)Z) ? 1.0f : 0.0f;
        } else {
            const float f0 = __ldg(p);
            if (cross) f1 = __ldg(p + st);
            blk = fmaf(m - cur, f0, blk);
            blk = fmaf(B - m, f1, blk);  // B - m = 0 without a crossing
        }
        if (cross) {
            kaddr += st;
            kf += fst;
            tzn = fmaf(kf, S, O);
            if (!FAST && kaddr == kexit) tzn = __int_as_float(0x7f800000);
        }
        cur = B;
    };
    int j = jb;
    for (; j + 7 <= je; j += 8) {
        float blk = 0.0f;
#pragma unroll
        for (int q = 0; q < 8; ++q) piece(j + q, blk);
        if (KAHAN && !COUNT) kahan_add(acc, comp, blk);
        else acc += blk;
    }
    float blk = 0.0f;
#pragma unroll 1
    for (; j <= je; ++j) piece(j, blk);
    if (KAHAN && !COUNT) {
        kahan_add(acc, comp, blk);
        return acc - comp;
    }
    return acc + blk;
}

// Sum over the voxels that detector row v's ray crosses of (t_exit - t_entry) *
// f[voxel] (the projection divided by w), for the column path in spc (n pieces
// from t_in to t_out), or with COUNT the row's number of (ray, voxel) pairs.
// Called by whole warps.
template <bool KAHAN, bool COUNT>
__device__ __forceinline__ float column_row_sum(const ExactGeom& G, const ZParam* __restrict__ zp,
                                                const float* __restrict__ volz, const float2* spc, int n, float t_in,
                                                float t_out, int v, bool valid)
{
    ZParam Z;
    Z.S = 0.0f;
    Z.O = 0.0f;
    Z.inv_S = 0.0f;
    Z.kc = 0;
    if (valid) Z = zp[v];
    // the volume's bottom and top planes along this row's ray
    const float z0 = plane_t(0, Z.S, Z.O, Z.kc), zZ = plane_t(G.Z, Z.S, Z.O, Z.kc);
    const float t_lo = fminf(z0, zZ), t_hi = fmaxf(z0, zZ);
    const float ta = fmaxf(t_in, t_lo), tb = fminf(t_out, t_hi);
    const bool hit = valid && ta < tb;
    int jb = INT_MAX, je = -1;
    if (hit) {
        jb = first_piece_ending<true>(spc, n, ta);
        je = first_piece_ending<false>(spc, n, tb);
    }
    jb = __reduce_min_sync(0xffffffffu, jb);
    je = __reduce_max_sync(0xffffffffu, je);
    if (jb > je) return 0.0f;  // no row of the warp crosses the volume
    const float t_start = (jb == 0) ? t_in : spc[jb - 1].x;
    const float t_end = spc[je].x;
    const int dk = Z.S > 0.0f ? 1 : -1;  // layer step along increasing t
    // rows that miss the volume read the zero layer below their column and never cross
    int kaddr = 0;
    float kf = 0.0f, tzn = __int_as_float(0x7f800000);
    if (hit) {
        int plane;  // the next z plane the row crosses
        if (t_start < t_lo) {  // outside, the volume ahead: the first plane is the near face
            kaddr = dk > 0 ? 0 : G.Z + 1;
            plane = dk > 0 ? 0 : G.Z;
        } else {  // inside (t_start <= ta < tb <= t_hi)
            const int k = locate<true>(t_start, Z.S, Z.O, Z.kc, G.Z, 1.0 / (double)Z.S);
            kaddr = k + 1;
            plane = dk > 0 ? k + 1 : k;
        }
        kf = (float)(plane - Z.kc);
        tzn = fmaf(kf, Z.S, Z.O);
    }
    const int kexit = dk > 0 ? G.Z + 1 : 0;
    const bool leaves = hit && t_start < t_hi && t_end > t_hi;  // crosses the far face within the pieces
    const bool fast = !__any_sync(0xffffffffu, leaves);
    const bool up = __all_sync(0xffffffffu, !hit || dk > 0);
    const bool down = __all_sync(0xffffffffu, !hit || dk < 0);
    if (fast) {
        if (up) return walk_rows<KAHAN, true, 1, COUNT>(volz, spc, jb, je, t_start, kaddr, kf, tzn, Z.S, Z.O, dk, kexit, G.Z);
        if (down) return walk_rows<KAHAN, true, -1, COUNT>(volz, spc, jb, je, t_start, kaddr, kf, tzn, Z.S, Z.O, dk, kexit, G.Z);
        return walk_rows<KAHAN, true, 0, COUNT>(volz, spc, jb, je, t_start, kaddr, kf, tzn, Z.S, Z.O, dk, kexit, G.Z);
    }
    if (up) return walk_rows<KAHAN, false, 1, COUNT>(volz, spc, jb, je, t_start, kaddr, kf, tzn, Z.S, Z.O, dk, kexit, G.Z);
    if (down) return walk_rows<KAHAN, false, -1, COUNT>(volz, spc, jb, je, t_start, kaddr, kf, tzn, Z.S, Z.O, dk, kexit, G.Z);
    return walk_rows<KAHAN, false, 0, COUNT>(volz, spc, jb, je, t_start, kaddr, kf, tzn, Z.S, Z.O, dk, kexit, G.Z);
}

// Rows mirrored about the source plane z = 0 (the plan's z table mirror-
// symmetric: row Nv-1-v's plane Z-k is row v's plane k, bit for bit) cross
// their z planes at the same t, so one lane walks lower row v (below z = 0,
// its layer falling along t) and its mirror Nv-1-v together: one crossing
// test and plane update, two loads and two sums.  The mirror's layer is
// Z-1-k, at offset Z + 1 - kaddr of its padded column.  Returns {row v, row
// Nv-1-v}.
template <bool KAHAN, bool FAST, bool COUNT, bool PAIRED>
__device__ __forceinline__ float2 walk_rows_mirror(const float* __restrict__ volz, const float2* spc, int jb, int je,
                                                   float cur, int kaddr, float kf, float tzn, float S, float O, int Z)
{
    int dm = Z + 1 - 2 * kaddr;  // the mirror row's offset from row v's in the same column
    float acc = 0.0f, comp = 0.0f, accm = 0.0f, compm = 0.0f, f1 = 0.0f, f1m = 0.0f;
    // piece {B, column}: B = where it ends, its column's offset in volz (int bits)
    auto piece_at = [&](float B, float cbits, float& blk, float& blkm) {
        const int cb = __float_as_int(cbits);
        const float* p = volz + (cb + kaddr);
        const float* pm = p + dm;
        const bool cross = tzn < B;
        const float m = fminf(tzn, B);
        if (COUNT) {  // layers 0 .. Z-1 sit at kaddr 1 .. Z, for both rows
            const float in0 = (m - cur > 0.0f && (unsigned)(kaddr - 1) < (unsigned)Z) ? 1.0f : 0.0f;
            const float in1 = (B - m > 0.0f && (unsigned)(kaddr - 2) < (unsigned)Z) ? 1.0f : 0.0f;
            blk += in0 + in1;
            blkm += in0 + in1;
        } else {
            const float f0 = __ldg(p), f0m = __ldg(pm);
            if (cross) {
                f1 = __ldg(p - 1);
                f1m = __ldg(pm + 1);
            }
            const float L0 = m - cur, L1 = B - m;  // L1 = 0 without a crossing
            blk = fmaf(L0, f0, blk);
            blk = fmaf(L1, f1, blk);
            blkm = fmaf(L0, f0m, blkm);
            blkm = fmaf(L1, f1m, blkm);
        }
        if (cross) {
            kaddr -= 1;
            dm += 2;
            kf -= 1.0f;
            tzn = fmaf(kf, S, O);
            if (!FAST && kaddr == 0) tzn = __int_as_float(0x7f800000);  // left through the bottom
        }
        cur = B;
    };
    auto piece = [&](int j, float& blk, float& blkm) {
        const float2 pc = spc[j];
        piece_at(pc.x, pc.y, blk, blkm);
    };
    const float4* spc4 = reinterpret_cast<const float4*>(spc);  // pieces 2i, 2i + 1
    int j = jb;
    // blocks of 16 pieces: the pair's loads of a block issue together; with
    // PAIRED the table is read two pieces per 16-byte load (j is the same for
    // the warp)
    for (; j + 15 <= je; j += 16) {
        float blk = 0.0f, blkm = 0.0f;
        if (!PAIRED) {
#pragma unroll
            for (int q = 0; q < 16; ++q) piece(j + q, blk, blkm);
        } else if ((j & 1) == 0) {
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                const float4 pp = spc4[(j >> 1) + q];
                piece_at(pp.x, pp.y, blk, blkm);
                piece_at(pp.z, pp.w, blk, blkm);
            }
        } else {
            piece(j, blk, blkm);
#pragma unroll
            for (int q = 0; q < 7; ++q) {
                const float4 pp = spc4[((j + 1) >> 1) + q];
                piece_at(pp.x, pp.y, blk, blkm);
                piece_at(pp.z, pp.w, blk, blkm);
            }
            piece(j + 15, blk, blkm);
        }
        if (KAHAN && !COUNT) {
            kahan_add(acc, comp, blk);
            kahan_add(accm, compm, blkm);
        } else {
            acc += blk;
            accm += blkm;
        }
    }
    float blk = 0.0f, blkm = 0.0f;
#pragma unroll 1
    for (; j <= je; ++j) piece(j, blk, blkm);
    if (KAHAN && !COUNT) {
        kahan_add(acc, comp, blk);
        kahan_add(accm, compm, blkm);
        return make_float2(acc - comp, accm - compm);
    }
    return make_float2(acc + blk, accm + blkm);
}

// column_row_sum for lower row v (v < Nv/2) and its mirror Nv-1-v.
template <bool KAHAN, bool COUNT, bool PAIRED>
__device__ __forceinline__ float2 column_row_sum_mirror(const ExactGeom& G, const ZParam* __restrict__ zp,
                                                        const float* __restrict__ volz, const float2* spc, int n,
                                                        float t_in, float t_out, int v, bool valid)
{
    ZParam Z;
    Z.S = 0.0f;
    Z.O = 0.0f;
    Z.inv_S = 0.0f;
    Z.kc = 0;
    if (valid) Z = zp[v];
    const float z0 = plane_t(0, Z.S, Z.O, Z.kc), zZ = plane_t(G.Z, Z.S, Z.O, Z.kc);
    const float t_lo = fminf(z0, zZ), t_hi = fmaxf(z0, zZ);  // the same for the mirror row
    const float ta = fmaxf(t_in, t_lo), tb = fminf(t_out, t_hi);
    const bool hit = valid && ta < tb;
    int jb = INT_MAX, je = -1;
    if (hit) {
        jb = first_piece_ending<true>(spc, n, ta);
        je = first_piece_ending<false>(spc, n, tb);
    }
    jb = __reduce_min_sync(0xffffffffu, jb);
    je = __reduce_max_sync(0xffffffffu, je);
    if (jb > je) return make_float2(0.0f, 0.0f);
    const float t_start = (jb == 0) ? t_in : spc[jb - 1].x;
    const float t_end = spc[je].x;
    // lower rows descend along t (S < 0): their next plane is the layer's own
    int kaddr = 0;
    float kf = 0.0f, tzn = __int_as_float(0x7f800000);
    if (hit) {
        int plane;
        if (t_start < t_lo) {  // above the volume: the first plane is the top face
            kaddr = G.Z + 1;
            plane = G.Z;
        } else {
            const int k = locate<true>(t_start, Z.S, Z.O, Z.kc, G.Z, 1.0 / (double)Z.S);
            kaddr = k + 1;
            plane = k;
        }
        kf = (float)(plane - Z.kc);
        tzn = fmaf(kf, Z.S, Z.O);
    }
    const bool leaves = hit && t_start < t_hi && t_end > t_hi;
    if (!__any_sync(0xffffffffu, leaves))
        return walk_rows_mirror<KAHAN, true, COUNT, PAIRED>(volz, spc, jb, je, t_start, kaddr, kf, tzn, Z.S, Z.O,
                                                            G.Z);
    return walk_rows_mirror<KAHAN, false, COUNT, PAIRED>(volz, spc, jb, je, t_start, kaddr, kf, tzn, Z.S, Z.O, G.Z);
}

// MODE 0: out = projection (w * sum); MODE 1 (MLEM): out = w * g / Hf (0 where
// Hf == 0), the Siddon back projector's input; MODE 2: out = g / Hf (the
// voxel-driven back projector's); MODE 3: the (ray, voxel) pairs of positive
// length are counted into out[0] (OT = unsigned long long); MODE 4: the sum is
// added to out (float, detector-column layout), one xy block's share of it;
// MODE 5: MODE 3 within one xy block.  MODES 4 and 5 take the column's stretch
// inside the xy block blk = {x planes blk.x .. blk.y, y planes blk.z .. blk.w},
// the others the whole volume's.
// g is read [view][v][u]; out is written in LAYOUT: rows [view][v][u],
// detector columns [view][u][v] (a warp's 32 rows store 128 contiguous bytes)
// or, with MIRROR, mirrored row pairs (a lane stores its pair at once).  A CTA
// takes detector column u of one view and rows vstart .. vstart + blockDim.x - 1:
// from the tile list {view, u | vstart << 16} (blockIdx.x indexes it) or,
// without one, u = blockIdx.x, vstart = blockIdx.y * blockDim.x, view = view0 +
// blockIdx.z.
// MIRROR: rows come in mirrored pairs (see walk_rows_mirror); the CTA's rows
// are lower rows (below Nv/2) and each lane also produces its mirror row.
template <bool KAHAN, int MODE, int LAYOUT, class GT, class OT, bool MIRROR = false>
__device__ __forceinline__ void column_kernel_body(ExactGeom G, const float4* __restrict__ txy, const int2* __restrict__ kxy, const ZParam* __restrict__ zp, const float* __restrict__ wq, const uint2* __restrict__ tiles, unsigned view0, int4 blk, const float* __restrict__ volz, const GT* __restrict__ g, OT* __restrict__ out)
{
    // piece j: {t where it ends, offset of its (x, y) voxel column in volz (int bits)}
    extern __shared__ float2 spc[];
    unsigned view;
    int u, vstart;
    if (tiles) {
        const uint2 t = tiles[blockIdx.x];
        view = t.x;
        u = (int)(t.y & 0xffffu);
        vstart = (int)(t.y >> 16);
    } else {
        view = view0 + blockIdx.z;
        u = (int)blockIdx.x;
        vstart = (int)(blockIdx.y * blockDim.x);
    }
    const int Zp = G.Z + 2;
    const float4 T = __ldg(txy + (size_t)view * G.Nu + u);
    const int2 K = __ldg(kxy + (size_t)view * G.Nu + u);
    constexpr bool COUNTING = MODE == 3 || MODE == 5;
    const int4 b = MODE >= 4 ? blk : make_int4(0, G.X, 0, G.Y);
    const float x0 = plane_t(b.x, T.x, T.y, K.x), x1 = plane_t(b.y, T.x, T.y, K.x);
    const float y0 = plane_t(b.z, T.z, T.w, K.y), y1 = plane_t(b.w, T.z, T.w, K.y);
    const float t_in = fmaxf(fminf(x0, x1), fminf(y0, y1));
    const float t_out = fminf(fmaxf(x0, x1), fmaxf(y0, y1));
    int n = 0;  // pieces; 0 when the column's rays miss the block's xy footprint
    if (t_in < t_out) {
        const double ivx = 1.0 / (double)T.x, ivy = 1.0 / (double)T.z;
        const int ix = locate_in<true>(t_in, T.x, T.y, K.x, b.x, b.y, ivx);
        const int ex = locate_in<false>(t_out, T.x, T.y, K.x, b.x, b.y, ivx);
        const int iy = locate_in<true>(t_in, T.z, T.w, K.y, b.z, b.w, ivy);
        const int ey = locate_in<false>(t_out, T.z, T.w, K.y, b.z, b.w, ivy);
        const int nx = abs(ex - ix), ny = abs(ey - iy);
        n = nx + ny + 1;
        const int dx = T.x > 0.0f ? 1 : -1, dy = T.z > 0.0f ? 1 : -1;
        // the first x and y planes crossed, relative to their kc
        const int qx = (dx > 0 ? ix + 1 : ix) - K.x, qy = (dy > 0 ? iy + 1 : iy) - K.y;
        const float isx = 1.0f / fabsf(T.x), isy = 1.0f / fabsf(T.z);
        for (int q = threadIdx.x; q < nx + ny; q += blockDim.x) {
            float t;
            int pos, cx, cy;
            if (q < nx) {  // x crossing q: after the y crossings strictly before it
                t = fmaf((float)(qx + q * dx), T.x, T.y);
                const int c = count_before<true>(t, qy, dy, T.z, T.w, isy, ny);
                pos = q + c;
                cx = ix + dx * (q + 1);
                cy = iy + dy * c;
            } else {  // y crossing b: after the x crossings at or before it
                const int b = q - nx;
                t = fmaf((float)(qy + b * dy), T.z, T.w);
                const int c = count_before<false>(t, qx, dx, T.x, T.y, isx, nx);
                pos = b + c;
                cx = ix + dx * c;
                cy = iy + dy * (b + 1);
            }
            spc[pos].x = t;                                        // piece pos ends here
            spc[pos + 1].y = __int_as_float((cy * G.X + cx) * Zp);  // piece pos + 1 lies in (cx, cy)
        }
        if (threadIdx.x == 0) {
            spc[0].y = __int_as_float((iy * G.X + ix) * Zp);
            // the last piece ends at the first x or y plane after the exit voxel
            spc[n - 1].x = fminf(fmaf((float)(qx + nx * dx), T.x, T.y), fmaf((float)(qy + ny * dy), T.z, T.w));
        }
    }
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int vend = MIRROR ? G.Nv / 2 : G.Nv;  // rows this kernel walks (mirrors come with them)
    if (vstart + warp * 32 >= vend) return;  // whole warps past them; no barrier follows
    const int v = vstart + warp * 32 + lane;
    const bool valid = v < vend;
    float2 sum = make_float2(0.0f, 0.0f);
    if (n > 0) {
        // the table read in pairs for whole-volume walks; the xy blocks' shorter
        // walks measured faster reading it piece by piece
        if (MIRROR) sum = column_row_sum_mirror<KAHAN, COUNTING, (MODE < 4)>(G, zp, volz, spc, n, t_in, t_out, v, valid);
        else sum.x = column_row_sum<KAHAN, COUNTING>(G, zp, volz, spc, n, t_in, t_out, v, valid);
    }
    if (COUNTING) {
        unsigned long long c = valid ? (unsigned long long)sum.x + (unsigned long long)sum.y : 0ull;
        for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
        if (lane == 0 && c) atomicAdd(reinterpret_cast<unsigned long long*>(out), c);
        return;
    }
    if (!valid) return;
    if constexpr (!COUNTING) {
        const size_t base = (size_t)(view - view0) * G.Nu * G.Nv;
        // row's output value (MODE 0..2)
        auto value = [&](int row, float acc) {
            const size_t pix_rm = (size_t)row * G.Nu + u, pix_col = (size_t)u * G.Nv + row;
            const float w = __ldg(wq + pix_col);
            const float hf = w * acc;
            if (MODE == 0) return hf;
            const float gv = load_val<GT>(g + base + pix_rm);
            const float ratio = (hf != 0.0f) ? __fdiv_rn(gv, hf) : 0.0f;
            return MODE == 1 ? ratio * w : ratio;
        };
        if constexpr (MODE == 4) {
            static_assert(LAYOUT == kLayoutColumns, "block sums are kept in the detector-column layout");
            out[base + (size_t)u * G.Nv + v] += sum.x;
            if (MIRROR) out[base + (size_t)u * G.Nv + (G.Nv - 1 - v)] += sum.y;
        } else if constexpr (LAYOUT == kLayoutPairs) {
            static_assert(MIRROR, "mirrored row pairs come from the mirror-paired walk");
            const int Np = G.Nv / 2 + 1;
            OT* const o = out + ((size_t)(view - view0) * G.Nu + u) * Np * 2;
            const float a = value(v, sum.x), b = value(G.Nv - 1 - v, sum.y);
            store_pair<OT>(o + 2 * v, a, b);
            if (v == G.Nv / 2 - 1) store_pair<OT>(o + 2 * (v + 1), b, a);  // entry Nv/2: rows Nv/2, Nv/2 - 1
        } else {
            auto emit = [&](int row, float acc) {
                const size_t pix = LAYOUT == kLayoutColumns ? (size_t)u * G.Nv + row : (size_t)row * G.Nu + u;
                store_val<OT>(out + base + pix, value(row, acc));
            };
            emit(v, sum.x);
            if (MIRROR) emit(G.Nv - 1 - v, sum.y);
        }
    }
}

// The whole-volume walks (MODES 0 .. 3) held at 32 registers, 16 CTAs per SM:
// 2.98 against 3.07 ms at 256^3 / 360 / 512^2.  The xy-block walks (MODES 4, 5)
// keep the compiler's own allocation, which measured faster for them.
template <bool KAHAN, int MODE, int LAYOUT, class GT, class OT, bool MIRROR = false>
__global__ void __launch_bounds__(kColRows, 16) fp_column_kernel(ExactGeom G, const float4* __restrict__ txy, const int2* __restrict__ kxy, const ZParam* __restrict__ zp, const float* __restrict__ wq, const uint2* __restrict__ tiles, unsigned view0, int4 blk, const float* __restrict__ volz, const GT* __restrict__ g, OT* __restrict__ out)
{
    column_kernel_body<KAHAN, MODE, LAYOUT, GT, OT, MIRROR>(G, txy, kxy, zp, wq, tiles, view0, blk, volz, g, out);
}
template <bool KAHAN, int MODE, int LAYOUT, class GT, class OT, bool MIRROR = false>
__global__ void __launch_bounds__(kColRows) fp_column_block_kernel(ExactGeom G, const float4* __restrict__ txy, const int2* __restrict__ kxy, const ZParam* __restrict__ zp, const float* __restrict__ wq, const uint2* __restrict__ tiles, unsigned view0, int4 blk, const float* __restrict__ volz, const GT* __restrict__ g, OT* __restrict__ out)
{
    column_kernel_body<KAHAN, MODE, LAYOUT, GT, OT, MIRROR>(G, txy, kxy, zp, wq, tiles, view0, blk, volz, g, out);
}
// the kernel of a MODE
template <int MODE, bool KAHAN, int LAYOUT, class GT, class OT, bool MIRROR>
constexpr auto fp_column_kernel_of()
{
    if constexpr (MODE >= 4) return fp_column_block_kernel<KAHAN, MODE, LAYOUT, GT, OT, MIRROR>;
    else return fp_column_kernel<KAHAN, MODE, LAYOUT, GT, OT, MIRROR>;
}

// f[z][y][x] -> volz[(y*X + x)*(Z + 2) + z + 1], 32 (x) x 32 (z) tiles of one y
// through shared memory; the zero layers (z = -1 and z = Z) are set once when
// the buffer is allocated and never written here.
__global__ void __launch_bounds__(256) to_zfast_kernel(const float* __restrict__ in, float* __restrict__ out, int X,
                                                       int Y, int Z)
{
    __shared__ float tile[32][33];
    const int x0 = blockIdx.x * 32, z0 = blockIdx.y * 32, y = blockIdx.z;
    for (int r = threadIdx.y; r < 32; r += 8) {
        const int x = x0 + threadIdx.x, z = z0 + r;
        if (x < X && z < Z) tile[r][threadIdx.x] = in[((size_t)z * Y + y) * X + x];
    }
    __syncthreads();
    const size_t Zp = (size_t)Z + 2;
    for (int r = threadIdx.y; r < 32; r += 8) {
        const int z = z0 + threadIdx.x, x = x0 + r;
        if (x < X && z < Z) out[((size_t)y * X + x) * Zp + z + 1] = tile[threadIdx.x][r];
    }
}

// Bit b of mask[view][u]: detector column u's rays cross xy block b (blocks of
// `side` voxels, nbx along x), by the column kernel's own test.
__global__ void __launch_bounds__(128) column_block_mask_kernel(ExactGeom G, const float4* __restrict__ txy,
                                                                const int2* __restrict__ kxy, unsigned nview, int side,
                                                                int nbx, int nby,
                                                                unsigned long long* __restrict__ mask)
{
    const size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (q >= (size_t)nview * G.Nu) return;
    const float4 T = txy[q];
    const int2 K = kxy[q];
    unsigned long long m = 0ull;
    for (int by = 0; by < nby; ++by)
        for (int bx = 0; bx < nbx; ++bx) {
            const float x0 = plane_t(bx * side, T.x, T.y, K.x), x1 = plane_t(min((bx + 1) * side, G.X), T.x, T.y, K.x);
            const float y0 = plane_t(by * side, T.z, T.w, K.y), y1 = plane_t(min((by + 1) * side, G.Y), T.z, T.w, K.y);
            if (fmaxf(fminf(x0, x1), fminf(y0, y1)) < fminf(fmaxf(x0, x1), fmaxf(y0, y1)))
                m |= 1ull << (by * nbx + bx);
        }
    mask[q] = m;
}

// The blocks' summed ray sums acc ([view][u][v], from view0) into the forward
// projector's output as fp_column_kernel's MODE writes it (0, 1 or 2), over
// 32 (u) x 32 (v) tiles: g is read along u and acc, w along v; a row-major out
// is written along u through the same tile.  acc may be out itself (float,
// detector-column layout): each thread reads its pixel before writing it.
template <int MODE, int LAYOUT, class GT, class OT>
__global__ void __launch_bounds__(256) column_finish_kernel(ExactGeom G, const float* acc,
                                                            const float* __restrict__ wq,
                                                            const GT* __restrict__ g, OT* out)
{
    __shared__ float tile[32][33];
    const int u0 = blockIdx.x * 32, v0 = blockIdx.y * 32;
    const size_t base = (size_t)blockIdx.z * G.Nu * G.Nv;
    if (MODE != 0) {
        for (int r = threadIdx.y; r < 32; r += 8) {
            const int u = u0 + threadIdx.x, v = v0 + r;
            if (u < G.Nu && v < G.Nv) tile[r][threadIdx.x] = load_val<GT>(g + base + (size_t)v * G.Nu + u);
        }
        __syncthreads();
    }
    float val[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const int u = u0 + threadIdx.y + 8 * q, v = v0 + threadIdx.x;
        val[q] = 0.0f;
        if (u < G.Nu && v < G.Nv) {
            const size_t pc = (size_t)u * G.Nv + v;
            const float w = __ldg(wq + pc);
            const float hf = w * acc[base + pc];
            if (MODE == 0) {
                val[q] = hf;
            } else {
                const float ratio = (hf != 0.0f) ? __fdiv_rn(tile[threadIdx.x][threadIdx.y + 8 * q], hf) : 0.0f;
                val[q] = MODE == 1 ? ratio * w : ratio;
            }
            if (LAYOUT == kLayoutColumns) store_val<OT>(out + base + pc, val[q]);
        }
    }
    if (LAYOUT == kLayoutRows) {
        __syncthreads();  // the g tile is read
#pragma unroll
        for (int q = 0; q < 4; ++q) tile[threadIdx.x][threadIdx.y + 8 * q] = val[q];
        __syncthreads();
        for (int r = threadIdx.y; r < 32; r += 8) {
            const int u = u0 + threadIdx.x, v = v0 + r;
            if (u < G.Nu && v < G.Nv) store_val<OT>(out + base + (size_t)v * G.Nu + u, tile[r][threadIdx.x]);
        }
    }
}

// column_finish_kernel for an output in mirrored row pairs: 32 (u) x 32 (pair)
// tiles, g of both rows of each pair read along u through shared memory, acc
// and w read along the pair index (rows p ascending, rows Nv-1-p descending),
// each pair stored at once.
template <int MODE, class GT, class OT>
__global__ void __launch_bounds__(256) column_finish_pairs_kernel(ExactGeom G, const float* __restrict__ acc,
                                                                  const float* __restrict__ wq,
                                                                  const GT* __restrict__ g, OT* __restrict__ out)
{
    __shared__ float lo[32][33], hi[32][33];
    const int Np = G.Nv / 2 + 1;
    const int u0 = blockIdx.x * 32, p0 = blockIdx.y * 32;
    const size_t base = (size_t)blockIdx.z * G.Nu * G.Nv;
    if (MODE != 0) {
        for (int r = threadIdx.y; r < 32; r += 8) {
            const int u = u0 + threadIdx.x, p = p0 + r;
            if (u < G.Nu && p < Np) {
                lo[r][threadIdx.x] = load_val<GT>(g + base + (size_t)p * G.Nu + u);
                hi[r][threadIdx.x] = load_val<GT>(g + base + (size_t)(G.Nv - 1 - p) * G.Nu + u);
            }
        }
        __syncthreads();
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const int u = u0 + threadIdx.y + 8 * q, p = p0 + threadIdx.x;
        if (u >= G.Nu || p >= Np) continue;
        auto value = [&](int row, float gv) {
            const size_t pc = (size_t)u * G.Nv + row;
            const float w = __ldg(wq + pc);
            const float hf = w * acc[base + pc];
            if (MODE == 0) return hf;
            const float ratio = (hf != 0.0f) ? __fdiv_rn(gv, hf) : 0.0f;
            return MODE == 1 ? ratio * w : ratio;
        };
        const float a = value(p, MODE ? lo[threadIdx.x][threadIdx.y + 8 * q] : 0.0f);
        const float b = value(G.Nv - 1 - p, MODE ? hi[threadIdx.x][threadIdx.y + 8 * q] : 0.0f);
        store_pair<OT>(out + (((size_t)blockIdx.z * G.Nu + u) * Np + p) * 2, a, b);
    }
}

}  // namespace exact

// ---- host side -----------------------------------------------------------------------------

// The column kernel needs every piece of a detector column's path to span less
// than a voxel of z (0.9 at most: the column diagonal times the steepest row's
// dz/dt, z being dz_v * (t + Rf) / R along row v's ray), int offsets into the
// padded volume, u and row starts that fit 16 bits, and the path in shared memory.
bool exact_fp_column_suits(const Plan& P)
{
    const ExactGeom& E = P.eg;
    const double vx = E.vox[0], vy = E.vox[1], vz = E.vox[2];
    if (!(vz > 0.0) || E.Ry == 0.0f) return false;
    const double diag = std::sqrt(vx * vx + vy * vy);
    const double slope = (0.5 * E.Nv * std::fabs((double)E.dv) + std::fabs((double)E.Dz)) / std::fabs((double)E.Ry);
    const double needle = diag * slope / vz;
    const double padded = (double)E.X * E.Y * (E.Z + 2.0);
    return needle < 0.9 && padded < 2147483647.0 && E.Nu <= 65535 && E.Nv <= 65535 && E.Y <= 65535 &&
           (size_t)(E.X + E.Y + 2) * sizeof(float2) <= 200 * 1024;
}

// Side of the xy blocks the column projector walks one at a time (0: the
// whole volume in one pass).  AUTO: blocks when the z-fastest copy is larger
// than 96 MiB, so that the CTAs in flight, which all take one block, read at
// most 40 MiB of it and the 126 MB L2 holds their reads across views; at most
// 64 blocks.  The option's n > 0 asks for n x n columns.
static int column_block_side(const Plan& P)
{
    const ExactGeom& E = P.eg;
    if (P.opt.fp_block < 0) return 0;
    const double col_bytes = 4.0 * (E.Z + 2.0);
    int side = P.opt.fp_block;
    if (side == 0) {
        if ((double)E.X * E.Y * col_bytes <= 96.0 * (1 << 20)) return 0;
        side = std::max(8, (int)std::sqrt(40.0 * (1 << 20) / col_bytes) / 8 * 8);
        side = std::max(side, (std::max(E.X, E.Y) + 7) / 8);
    }
    return (side >= E.X && side >= E.Y) ? 0 : side;
}

// The rows of view n's tiles: blocks of P.col_rows rows (from the first)
// inside its rectangle of rays; mirror plans take the lower rows of the
// rectangle and of its mirror image.
static void column_rows(const Plan& P, const int4& r, int* v0, int* v1)
{
    const int Nv = P.eg.Nv;
    *v0 = P.z_mirror ? std::min(r.z, Nv - 1 - r.w) : r.z;
    *v1 = P.z_mirror ? std::min(std::max(r.w, Nv - 1 - r.z), Nv / 2 - 1) : r.w;
}

// Rows per CTA before any measurement: the fewest of 32, 64 and 128 that cover
// the most rows a detector column walks in any view (so no warp of a CTA is
// idle), 128 beyond.
int exact_column_rows_default(const Plan& P, const std::vector<int4>& rect)
{
    int most = 0;
    for (const int4& r : rect) {
        if (r.y < r.x) continue;
        int v0, v1;
        column_rows(P, r, &v0, &v1);
        most = std::max(most, v1 - v0 + 1);
    }
    return most <= 32 ? 32 : most <= 64 ? 64 : exact::kColRows;
}

static void free_tiles(Plan& P, RayTiles& T)
{
    if (T.d && !T.prefix.empty()) plan_release(P, T.d, (size_t)T.prefix.back() * sizeof(uint2));
    T.d = nullptr;
    T.prefix.clear();
}

static recon_status_t upload_tiles(Plan& P, RayTiles& T, const std::vector<uint2>& tiles)
{
    if (tiles.empty()) return RECON_OK;
    RB_CHECK(P.alloc(&T.d, tiles.size(), "column tiles"));
    RB_CUDA(cudaMemcpy(T.d, tiles.data(), tiles.size() * sizeof(uint2), cudaMemcpyHostToDevice));
    return RECON_OK;
}

// Tiles {view, u | vstart << 16} of the column kernel: per view, the columns and
// row blocks inside the rectangle of rays that cross the volume (rect, per
// plan view {u_min, u_max, v_min, v_max}); with xy blocks, one list per block
// of the columns whose rays cross it.
recon_status_t build_column_tiles(Plan& P, const std::vector<int4>& rect)
{
    const unsigned nv = P.nviews;
    const ExactGeom& E = P.eg;
    free_tiles(P, P.col_tiles);
    for (RayTiles& T : P.col_btiles) free_tiles(P, T);
    P.col_block = column_block_side(P);
    P.col_btiles.clear();
    const int step = P.col_rows;
    if (P.col_block == 0) {
        P.col_tiles.prefix.assign(nv + 1, 0);
        std::vector<uint2> tiles;
        for (unsigned n = 0; n < nv; ++n) {
            P.col_tiles.prefix[n] = (unsigned)tiles.size();
            const int4 r = rect[n];
            if (r.y < r.x) continue;
            int v0, v1;
            column_rows(P, r, &v0, &v1);
            for (int u = r.x; u <= r.y; ++u)
                for (int vs = v0; vs <= v1; vs += step)
                    tiles.push_back(make_uint2(n, (unsigned)u | ((unsigned)vs << 16)));
        }
        P.col_tiles.prefix[nv] = (unsigned)tiles.size();
        return upload_tiles(P, P.col_tiles, tiles);
    }
    const int side = P.col_block;
    P.col_nbx = (E.X + side - 1) / side;
    P.col_nby = (E.Y + side - 1) / side;
    const int nb = P.col_nbx * P.col_nby;
    if (nb > 64) return fail(RECON_ERR_INVALID_ARGUMENT, "fp_block: more than 64 xy blocks");
    std::vector<unsigned long long> mask((size_t)nv * E.Nu, 0ull);
    if (nv) {
        unsigned long long* d_mask = nullptr;
        RB_CUDA(cudaMalloc(&d_mask, mask.size() * sizeof(unsigned long long)));
        const size_t nq = mask.size();
        exact::column_block_mask_kernel<<<(unsigned)((nq + 127) / 128), 128>>>(E, P.d_txy, P.d_kxy, nv, side,
                                                                             P.col_nbx, P.col_nby, d_mask);
        cudaError_t e = cudaGetLastError();
        if (e == cudaSuccess)
            e = cudaMemcpy(mask.data(), d_mask, nq * sizeof(unsigned long long), cudaMemcpyDeviceToHost);
        cudaFree(d_mask);
        if (e != cudaSuccess) return cuda_fail(e, "column block masks");
    }
    P.col_btiles.resize(nb);
    std::vector<std::vector<uint2>> tiles(nb);
    for (int b = 0; b < nb; ++b) P.col_btiles[b].prefix.assign(nv + 1, 0);
    for (unsigned n = 0; n < nv; ++n) {
        for (int b = 0; b < nb; ++b) P.col_btiles[b].prefix[n] = (unsigned)tiles[b].size();
        const int4 r = rect[n];
        if (r.y < r.x) continue;
        int v0, v1;
        column_rows(P, r, &v0, &v1);
        for (int u = r.x; u <= r.y; ++u)
            for (unsigned long long m = mask[(size_t)n * E.Nu + u]; m; m &= m - 1) {
                const int b = __builtin_ctzll(m);
                for (int vs = v0; vs <= v1; vs += step)
                    tiles[b].push_back(make_uint2(n, (unsigned)u | ((unsigned)vs << 16)));
            }
    }
    for (int b = 0; b < nb; ++b) {
        P.col_btiles[b].prefix[nv] = (unsigned)tiles[b].size();
        RB_CHECK(upload_tiles(P, P.col_btiles[b], tiles[b]));
    }
    return RECON_OK;
}

recon_status_t exact_to_zfast(const Plan& P, const float* vol, cudaStream_t s)
{
    const ExactGeom& E = P.eg;
    exact::to_zfast_kernel<<<dim3((E.X + 31) / 32, (E.Z + 31) / 32, E.Y), dim3(32, 8), 0, s>>>(vol, P.d_vol_z, E.X,
                                                                                             E.Y, E.Z);
    RB_CUDA(cudaGetLastError());
    return RECON_OK;
}

// Views [first, first + count) of table slots through the column kernel: the
// tile list for plan views, the full grid otherwise (the scratch slot).  The
// volume is copied to the z-fastest layout first.  For MODE 0 the pixels
// outside the tiles are zeroed; the MLEM ratio buffers are zero there from
// allocation on.
template <int MODE, int LAYOUT, class GT, class OT>
static auto column_kernel(const Plan& P)
{
    const bool kahan = P.opt.sum == RECON_SUM_KAHAN;
    if constexpr (LAYOUT == kLayoutPairs) {  // only from the mirror-paired walk
        return kahan ? exact::fp_column_kernel_of<MODE, true, LAYOUT, GT, OT, true>()
                     : exact::fp_column_kernel_of<MODE, false, LAYOUT, GT, OT, true>();
    } else {
        return P.z_mirror ? (kahan ? exact::fp_column_kernel_of<MODE, true, LAYOUT, GT, OT, true>()
                                   : exact::fp_column_kernel_of<MODE, false, LAYOUT, GT, OT, true>())
                          : (kahan ? exact::fp_column_kernel_of<MODE, true, LAYOUT, GT, OT, false>()
                                   : exact::fp_column_kernel_of<MODE, false, LAYOUT, GT, OT, false>());
    }
}

// Views [first, first + count) of plan views over the xy blocks: each block's
// tiles add their stretch of the ray sums into acc (in launch order, so the sums
// are deterministic), then column_finish_kernel forms the output; MODE 3 adds
// each block's pair count.  acc is the output itself where that is float in
// detector columns, else the plan's block-sum buffer.
template <int MODE, int LAYOUT, class GT, class OT>
static recon_status_t launch_column_blocks(Plan& P, const float* vol, unsigned first, unsigned count, const GT* g,
                                          OT* out, cudaStream_t s)
{
    const ExactGeom& E = P.eg;
    const size_t smem = (size_t)(E.X + E.Y + 2) * sizeof(float2);
    constexpr bool in_place = LAYOUT == kLayoutColumns && std::is_same<OT, float>::value;
    float* acc = nullptr;
    if (MODE != 3) {
        if (in_place) {
            acc = reinterpret_cast<float*>(out);
        } else {
            if (!P.d_col_acc) RB_CHECK(P.alloc(&P.d_col_acc, (size_t)P.nviews * P.npix, "column block sums"));
            acc = P.d_col_acc;
        }
        RB_CUDA(cudaMemsetAsync(acc, 0, (size_t)count * P.npix * sizeof(float), s));
        RB_CHECK(exact_to_zfast(P, vol, s));
    }
    constexpr int BMODE = MODE == 3 ? 5 : 4;
    using BOT = typename std::conditional<MODE == 3, OT, float>::type;
    auto kernel = column_kernel<BMODE, MODE == 3 ? LAYOUT : kLayoutColumns, float, BOT>(P);
    if (smem > 48 * 1024) RB_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    BOT* bout;
    if constexpr (MODE == 3) bout = out;
    else bout = acc;
    const int side = P.col_block;
    for (int by = 0; by < P.col_nby; ++by)
        for (int bx = 0; bx < P.col_nbx; ++bx) {
            const RayTiles& T = P.col_btiles[by * P.col_nbx + bx];
            const unsigned t0 = T.prefix[first], nt = T.prefix[first + count] - t0;
            if (nt == 0) continue;
            const int4 blk = make_int4(bx * side, std::min((bx + 1) * side, E.X), by * side,
                                       std::min((by + 1) * side, E.Y));
            kernel<<<nt, P.col_rows, smem, s>>>(E, P.d_txy, P.d_kxy, P.d_zp, P.d_wq, T.d + t0, first, blk,
                                                     P.d_vol_z, nullptr, bout);
            RB_CUDA(cudaGetLastError());
        }
    if constexpr (MODE != 3 && LAYOUT == kLayoutPairs) {
        const dim3 grid((E.Nu + 31) / 32, (E.Nv / 2 + 1 + 31) / 32, count);
        exact::column_finish_pairs_kernel<MODE, GT, OT><<<grid, dim3(32, 8), 0, s>>>(E, acc, P.d_wq, g, out);
        RB_CUDA(cudaGetLastError());
    } else if constexpr (MODE != 3) {
        const dim3 grid((E.Nu + 31) / 32, (E.Nv + 31) / 32, count);
        exact::column_finish_kernel<MODE, LAYOUT, GT, OT><<<grid, dim3(32, 8), 0, s>>>(E, acc, P.d_wq, g, out);
        RB_CUDA(cudaGetLastError());
    }
    return RECON_OK;
}

// Views [first, first + count) of table slots through the column kernel: the
// tile list for plan views, the full grid otherwise (the scratch slot).  The
// volume is copied to the z-fastest layout first.  For MODE 0 the pixels
// outside the tiles are zeroed; the MLEM ratio buffers are zero there from
// allocation on.  Plans with xy blocks take plan views block by block.
template <int MODE, int LAYOUT, class GT, class OT>
static recon_status_t launch_column(Plan& P, const float* vol, unsigned first, unsigned count, const GT* g, OT* out,
                                    cudaStream_t s)
{
    if (count == 0) return RECON_OK;
    const ExactGeom& E = P.eg;
    const bool plan_views = first + count <= P.nviews;
    if (plan_views && P.col_block > 0 && P.col_btiles.size() == (size_t)P.col_nbx * P.col_nby)
        return launch_column_blocks<MODE, LAYOUT, GT, OT>(P, vol, first, count, g, out, s);
    dim3 grid;
    const uint2* tiles = nullptr;
    if (plan_views && P.col_tiles.prefix.size() == P.nviews + 1) {
        const unsigned t0 = P.col_tiles.prefix[first], nt = P.col_tiles.prefix[first + count] - t0;
        if (MODE == 0) RB_CUDA(cudaMemsetAsync(out, 0, (size_t)count * P.npix * sizeof(OT), s));
        if (nt == 0) return RECON_OK;
        grid = dim3(nt, 1, 1);
        tiles = P.col_tiles.d + t0;
    } else {
        const int rows = P.z_mirror ? E.Nv / 2 : E.Nv;
        grid = dim3(E.Nu, (rows + P.col_rows - 1) / P.col_rows, count);
    }
    if (MODE != 3) RB_CHECK(exact_to_zfast(P, vol, s));
    const size_t smem = (size_t)(E.X + E.Y + 2) * sizeof(float2);
    auto kernel = column_kernel<MODE, LAYOUT, GT, OT>(P);
    if (smem > 48 * 1024) RB_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    kernel<<<grid, P.col_rows, smem, s>>>(E, P.d_txy, P.d_kxy, P.d_zp, P.d_wq, tiles, first,
                                               make_int4(0, E.X, 0, E.Y), P.d_vol_z, g, out);
    RB_CUDA(cudaGetLastError());
    return RECON_OK;
}

// (ray, voxel) pairs of positive length over all plan views, as the column
// kernel assigns them (synchronous; no volume is read).
recon_status_t exact_fp_column_count(Plan& P, unsigned long long* total)
{
    unsigned long long* d = nullptr;
    RB_CUDA(cudaMalloc(&d, sizeof(unsigned long long)));
    cudaError_t e = cudaMemset(d, 0, sizeof(unsigned long long));
    recon_status_t st = RECON_OK;
    if (e == cudaSuccess)
        st = launch_column<3, kLayoutRows, float, unsigned long long>(P, nullptr, 0u, P.nviews, nullptr, d, 0);
    if (e == cudaSuccess && st == RECON_OK) e = cudaMemcpy(total, d, sizeof(unsigned long long), cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (st != RECON_OK) return st;
    if (e != cudaSuccess) return cuda_fail(e, "column pair count");
    return RECON_OK;
}

recon_status_t exact_fp_column(Plan& P, const float* vol, unsigned first, unsigned count, float* out, cudaStream_t s)
{
    return launch_column<0, kLayoutRows, float, float>(P, vol, first, count, nullptr, out, s);
}

// RECON_SIDDON_BP_TUNED also measures the column forward projector's rows per
// CTA: each of 32, 64 and 128 (a warp per 32 rows; fewer rows leave no warp
// idle where a detector column has few rows to walk, more build the column's
// path once for more rows) is timed on a projection of up to 64 of the plan's
// views, CUDA events around the second of two runs on the legacy stream, and
// the fastest kept.  The choice is kept for the process per geometry and
// device, as the back projector's.  Synchronous (plan creation).
namespace {
std::mutex g_fp_tune_mutex;
std::map<std::string, int> g_fp_tune_rows;
}  // namespace

recon_status_t exact_tune_fp(Plan& P)
{
    if (!P.fp_column || P.nviews == 0 || P.view_rect_host.size() != P.nviews) return RECON_OK;
    const std::string key = geometry_key(P);
    int rows = 0;
    {
        std::lock_guard<std::mutex> lock(g_fp_tune_mutex);
        auto it = g_fp_tune_rows.find(key);
        if (it != g_fp_tune_rows.end()) rows = it->second;
    }
    if (rows == 0) {
        const unsigned nv = std::min(P.nviews, 64u);
        float *vol = nullptr, *out = nullptr;
        cudaError_t e = cudaMalloc(&vol, P.nvox * sizeof(float));
        if (e == cudaSuccess) e = cudaMalloc(&out, (size_t)nv * P.npix * sizeof(float));
        if (e == cudaSuccess) e = cudaMemset(vol, 0, P.nvox * sizeof(float));
        cudaEvent_t e0 = nullptr, e1 = nullptr;
        if (e == cudaSuccess) e = cudaEventCreate(&e0);
        if (e == cudaSuccess) e = cudaEventCreate(&e1);
        recon_status_t st = RECON_OK;
        float best = 0.0f;
        for (int r = 32; r <= exact::kColRows && e == cudaSuccess && st == RECON_OK; r *= 2) {
            P.col_rows = r;
            st = build_column_tiles(P, P.view_rect_host);
            if (st == RECON_OK) st = exact_fp_column(P, vol, 0, nv, out, 0);
            if (st == RECON_OK) e = cudaEventRecord(e0, 0);
            if (e == cudaSuccess && st == RECON_OK) st = exact_fp_column(P, vol, 0, nv, out, 0);
            if (e == cudaSuccess && st == RECON_OK) e = cudaEventRecord(e1, 0);
            if (e == cudaSuccess && st == RECON_OK) e = cudaEventSynchronize(e1);
            float ms = 0.0f;
            if (e == cudaSuccess && st == RECON_OK) e = cudaEventElapsedTime(&ms, e0, e1);
            if (e == cudaSuccess && st == RECON_OK && (rows == 0 || ms < best)) {
                best = ms;
                rows = r;
            }
        }
        if (e0) cudaEventDestroy(e0);
        if (e1) cudaEventDestroy(e1);
        cudaFree(vol);
        cudaFree(out);
        if (st != RECON_OK) return st;
        if (e != cudaSuccess) return cuda_fail(e, "forward projector tuning");
        std::lock_guard<std::mutex> lock(g_fp_tune_mutex);
        g_fp_tune_rows.emplace(key, rows);
    }
    if (P.col_rows != rows) {
        P.col_rows = rows;
        RB_CHECK(build_column_tiles(P, P.view_rect_host));
    }
    return RECON_OK;
}

// The MLEM ratio (MODE 1: times w, Siddon back projectors; MODE 2: without w,
// voxel-driven) of views [first, first+count), written straight into the
// layout its back projector reads (kLayoutRows, kLayoutColumns or, for MODE 1,
// kLayoutPairs).  g and ratio start at view `first`.
recon_status_t exact_fp_column_ratio(Plan& P, const float* vol, const void* g, void* ratio, int mode, int layout,
                                     bool bf16, unsigned first, unsigned count, cudaStream_t s)
{
    using bf = __nv_bfloat16;
    const float* gf = static_cast<const float*>(g);
    float* rf = static_cast<float*>(ratio);
    if (mode == 2) {
        if (layout == kLayoutColumns) return launch_column<2, kLayoutColumns, float, float>(P, vol, first, count, gf, rf, s);
        return launch_column<2, kLayoutRows, float, float>(P, vol, first, count, gf, rf, s);
    }
    if (bf16) {
        const bf* gb = static_cast<const bf*>(g);
        bf* rb = static_cast<bf*>(ratio);
        if (layout == kLayoutPairs) return launch_column<1, kLayoutPairs, bf, bf>(P, vol, first, count, gb, rb, s);
        if (layout == kLayoutColumns) return launch_column<1, kLayoutColumns, bf, bf>(P, vol, first, count, gb, rb, s);
        return launch_column<1, kLayoutRows, bf, bf>(P, vol, first, count, gb, rb, s);
    }
    if (layout == kLayoutPairs) return launch_column<1, kLayoutPairs, float, float>(P, vol, first, count, gf, rf, s);
    if (layout == kLayoutColumns) return launch_column<1, kLayoutColumns, float, float>(P, vol, first, count, gf, rf, s);
    return launch_column<1, kLayoutRows, float, float>(P, vol, first, count, gf, rf, s);
}

}  // namespace rb
