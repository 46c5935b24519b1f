// exact_device.cuh -- device functions of the EXACT projector pair, shared by
// the single-problem kernels (exact.cu) and the batched persistent kernels
// (batch.cu).  See exact.cu for the ray parameterisation.
#pragma once

#include <cuda_bf16.h>

#include "internal.h"

namespace rb {
namespace exact {

// ---- shared device helpers -------------------------------------------------------------

__device__ __forceinline__ float plane_t(int k, float S, float O, int kc) { return fmaf((float)(k - kc), S, O); }

// Voxel i along an axis with N voxels: the voxel whose t-interval [lo, hi)
// contains t (entry: lo <= t < hi) or (lo, hi] (exit: lo < t <= hi), found
// from an FP64 estimate and corrected against the FP32 plane values.
template <bool ENTRY>
__device__ __forceinline__ int locate(float t, float S, float O, int kc, int N, double invS)
{
    double kf = (double)kc + ((double)t - (double)O) * invS;
    int i = (int)floor(fmin(fmax(kf, -1.0), (double)N));
    i = min(max(i, 0), N - 1);
    const int up = (S > 0.0f) ? 1 : -1;  // index step toward larger t
#pragma unroll 1
    for (int it = 0; it < 6; ++it) {
        float t0 = plane_t(i, S, O, kc), t1 = plane_t(i + 1, S, O, kc);
        float lo = fminf(t0, t1), hi = fmaxf(t0, t1);
        bool before = ENTRY ? (t < lo) : (t <= lo);
        bool after = ENTRY ? (t >= hi) : (t > hi);
        int ni = before ? i - up : (after ? i + up : i);
        if (ni == i || ni < 0 || ni >= N) break;
        i = ni;
    }
    return i;
}

__device__ __forceinline__ float bf2f(__nv_bfloat16 x) { return __bfloat162float(x); }
template <class T>
__device__ __forceinline__ float load_val(const T* p);
template <>
__device__ __forceinline__ float load_val<float>(const float* p) { return __ldg(p); }
template <>
__device__ __forceinline__ float load_val<__nv_bfloat16>(const __nv_bfloat16* p) { return bf2f(*p); }
template <class T>
__device__ __forceinline__ void store_val(T* p, float v);
template <>
__device__ __forceinline__ void store_val<float>(float* p, float v) { *p = v; }
template <>
__device__ __forceinline__ void store_val<__nv_bfloat16>(__nv_bfloat16* p, float v) { *p = __float2bfloat16_rn(v); }

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
#pragma unroll 2
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

// Gather of views [view0, view0+nview) into the ZC accumulators of column
// (i, j), voxels k0..k1-1 (acc[(k-k0)*128 + tid] in shared memory).  sino holds
// the views' values, view vi at sino + vi*Nv*Nu; szb the mirrored z planes.
template <int ZC, int MODE, bool WEIGHTED, class ST>
__device__ __forceinline__ void bp_gather_column(const ExactGeom& G, const float4* __restrict__ txy,
                                                 const int2* __restrict__ kxy, const float2* __restrict__ cs,
                                                 const float* __restrict__ wtab, unsigned view0, unsigned nview,
                                                 const ST* __restrict__ sino, const float4* szb, float* acc,
                                                 int tid, int i, int j, int k0, int k1)
{
    const float Xa = G.P0[0] + i * G.vox[0], Xb = Xa + G.vox[0];
    const float Ya = G.P0[1] + j * G.vox[1], Yb = Ya + G.vox[1];
    const float Za = G.P0[2] + k0 * G.vox[2], Zb = G.P0[2] + k1 * G.vox[2];
    const float RyR = G.Ry / G.R;
    const float inv_du = 1.0f / G.du, inv_dv = 1.0f / G.dv;
    for (unsigned vi = 0; vi < nview; ++vi) {
        const unsigned view = view0 + vi;
        const float2 CS = __ldg(cs + view);
        // detector u range of the column: project its four corners
        float umin = 3.0e38f, umax = -3.0e38f;
#pragma unroll
        for (int c4 = 0; c4 < 4; ++c4) {
            const float X = (c4 & 1) ? Xb : Xa, Y = (c4 & 2) ? Yb : Ya;
            const float xv = X * CS.x - Y * CS.y, yv = X * CS.y + Y * CS.x;
            const float ud = __fdividef(G.R * xv, yv + G.Rf) * RyR - G.Dx;  // candidates only
            const float uf = (ud - G.ud0) * inv_du;
            umin = fminf(umin, uf);
            umax = fmaxf(umax, uf);
        }
        const int u_lo = max(0, (int)ceilf(umin - 2e-3f));
        const int u_hi = min(G.Nu - 1, (int)floorf(umax + 2e-3f));
        for (int u = u_lo; u <= u_hi; ++u) {
            const float4 T = __ldg(txy + (size_t)view * G.Nu + u);
            const int2 K = __ldg(kxy + (size_t)view * G.Nu + u);
            const float xa = plane_t(i, T.x, T.y, K.x), xb = plane_t(i + 1, T.x, T.y, K.x);
            const float ya = plane_t(j, T.z, T.w, K.y), yb = plane_t(j + 1, T.z, T.w, K.y);
            const float A = fmaxf(fminf(xa, xb), fminf(ya, yb));
            const float B = fminf(fmaxf(xa, xb), fmaxf(ya, yb));
            if (!(A < B)) continue;
            // rows v whose ray can cross the z-chunk inside [A, B]
            // (candidates only, with a margin): z = vd * (t + Rf) / R
            const float ra = __fdividef(G.R, A + G.Rf), rb = __fdividef(G.R, B + G.Rf);
            const float c1 = Za * ra, c2 = Za * rb, c3 = Zb * ra, c4 = Zb * rb;
            const float vdmin = fminf(fminf(c1, c2), fminf(c3, c4));
            const float vdmax = fmaxf(fmaxf(c1, c2), fmaxf(c3, c4));
            const float vfa = (vdmin * RyR - G.Dz - G.vd0) * inv_dv;
            const float vfb = (vdmax * RyR - G.Dz - G.vd0) * inv_dv;
            const int v_lo = max(0, (int)ceilf(fminf(vfa, vfb) - 2e-3f));
            const int v_hi = min(G.Nv - 1, (int)floorf(fmaxf(vfa, vfb) + 2e-3f));
            const ST* srow = sino + ((size_t)vi * G.Nv) * G.Nu + u;
            // Sweep the needles (the rays' pieces inside this column) in
            // increasing z together with the chunk's voxels.  The lowest
            // voxel a needle touches never decreases from one needle to
            // the next, so k carries over.  Each ray's z planes are
            // mirrored (t -> -t for rays going down, exact in IEEE) so
            // that T(k) increases with k for every ray:
            //   L(v, k) = min(B', T(k+1)) - max(A', T(k)).
            int k = k0;
            for (int v = v_lo; v <= v_hi; ++v) {
                const float4 Z = szb[v];  // {|S|, sign(S)*O, kc, sign(S)}
                float val;
                if (MODE == 1) val = __ldg(wtab + (size_t)v * G.Nu + u);
                else val = load_val<ST>(srow + (size_t)v * G.Nu);
                if (WEIGHTED && MODE != 1) val *= __ldg(wtab + (size_t)v * G.Nu + u);
                const float Ap = Z.w > 0.0f ? A : -B;
                const float Bp = Z.w > 0.0f ? B : -A;
                float kf = (float)k;
                float T1 = fmaf(kf + 1.0f - Z.z, Z.x, Z.y);
                while (T1 <= Ap && k < k1) {  // voxel k lies wholly before the needle
                    ++k;
                    kf += 1.0f;
                    T1 = fmaf(kf + 1.0f - Z.z, Z.x, Z.y);
                }
                if (k >= k1) break;  // this and every later needle lie above the chunk
                float T0 = fmaf(kf - Z.z, Z.x, Z.y);
                float* a = acc + (k - k0) * 128 + tid;
#pragma unroll 1
                for (int kk = k;;) {
                    const float L = fminf(Bp, T1) - fmaxf(Ap, T0);
                    if (L > 0.0f) *a = fmaf(L, val, *a);
                    if (T1 >= Bp || ++kk >= k1) break;
                    a += 128;
                    T0 = T1;
                    T1 = fmaf((float)kk + 1.0f - Z.z, Z.x, Z.y);
                }
            }
        }
    }
}

}  // namespace exact
}  // namespace rb
