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
// the step count known before the loop (no exit test on planes).  Back
// projection: a gather, one thread per (x, y) column and z-chunk; for every
// view it enumerates the rays crossing its column and accumulates
// L * value into per-thread shared-memory accumulators in a fixed order
// (views, then u, then v), so results are bit-reproducible; the MLEM update
// f <- f * Ht / sens is applied in the epilogue.
#include "internal.h"

#include <cmath>

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

__global__ void w_table_kernel(GeomD G, float* __restrict__ w)
{
    const int u = blockIdx.x * blockDim.x + threadIdx.x;
    const int v = blockIdx.y;
    if (u >= G.Nu) return;
    const double det_x = G.R / G.Ry * (pixel_center_d(G.Nu, G.du, u) + G.Dx);
    const double det_z = G.R / G.Ry * (pixel_center_d(G.Nv, G.dv, v) + G.Dz);
    w[(size_t)v * G.Nu + u] = (float)(sqrt(det_x * det_x + G.R * G.R + det_z * det_z) / G.R);
}

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

// MODE 0: out = projection (w * sum L_t * f).  MODE 1 (MLEM): out = w * ratio
// with ratio = g / Hf (0 where Hf == 0), the Siddon back projector's input.
// MODE 2: out = ratio (input of the voxel-driven back projector).
template <bool KAHAN, int MODE, class GT, class OT>
__global__ void __launch_bounds__(128) fp_kernel(ExactGeom G, const float4* __restrict__ txy,
                                                  const int2* __restrict__ kxy, const ZParam* __restrict__ zp,
                                                  const float* __restrict__ wtab, unsigned view0,
                                                  const float* __restrict__ vol, const GT* __restrict__ g,
                                                  OT* __restrict__ out)
{
    const int u = blockIdx.x * blockDim.x + threadIdx.x;
    const int v = blockIdx.y * blockDim.y + threadIdx.y;
    const unsigned view = view0 + blockIdx.z;
    if (u >= G.Nu || v >= G.Nv) return;
    const size_t pix = (size_t)u + (size_t)v * G.Nu;
    const size_t n = (size_t)blockIdx.z * G.Nu * G.Nv + pix;
    const float4 T = __ldg(txy + (size_t)view * G.Nu + u);
    const int2 K = __ldg(kxy + (size_t)view * G.Nu + u);
    const ZParam Z = zp[v];
    const float w = __ldg(wtab + pix);

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
        const int sx = dx, sy = dy * G.X, sz = dz * G.X * G.Y;
        const unsigned vmax = (unsigned)(G.X * G.Y * G.Z - 1);
        int idx = ix + iy * G.X + iz * G.X * G.Y;
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
    const float hf = w * acc;
    if (MODE == 0) {
        store_val<OT>(out + n, hf);
    } else {
        const float gv = load_val<GT>(g + n);
        const float ratio = (hf != 0.0f) ? __fdiv_rn(gv, hf) : 0.0f;
        store_val<OT>(out + n, MODE == 1 ? ratio * w : ratio);
    }
}

// ---- back projection (gather) ------------------------------------------------------------

// MODE 0: vol = Ht (back projection of the sinogram)
// MODE 1: vol = sensitivity (back projection of ones)
// MODE 2: f = (sens != 0) ? f*Ht/sens : 0 (MLEM update, in place)
// WEIGHTED: sinogram values are plain (multiply by w); otherwise they already
// carry w (the MLEM ratio written by the forward kernel).
template <int ZC, int MODE, bool WEIGHTED, class ST>
__global__ void __launch_bounds__(128) bp_kernel(ExactGeom G, const float4* __restrict__ txy,
                                                  const int2* __restrict__ kxy, const float2* __restrict__ cs,
                                                  const ZParam* __restrict__ zp, const float* __restrict__ wtab,
                                                  unsigned view0, unsigned nview, const ST* __restrict__ sino,
                                                  float* __restrict__ vol, const float* __restrict__ sens)
{
    extern __shared__ float smem[];
    float* acc = smem;                                         // [ZC][128]
    float4* szb = reinterpret_cast<float4*>(smem + ZC * 128);  // [Nv] mirrored z planes
    const int tid = threadIdx.x + threadIdx.y * 32;
    for (int q = tid; q < G.Nv; q += 128) {
        const ZParam z = zp[q];
        const bool pos = z.S > 0.0f;
        szb[q] = make_float4(fabsf(z.S), pos ? z.O : -z.O, (float)z.kc, pos ? 1.0f : -1.0f);
    }
#pragma unroll
    for (int q = 0; q < ZC; ++q) acc[q * 128 + tid] = 0.0f;
    __syncthreads();

    const int i = blockIdx.x * 32 + threadIdx.x;
    const int j = blockIdx.y * 4 + threadIdx.y;
    const int k0 = blockIdx.z * ZC;
    const int k1 = min(k0 + ZC, G.Z);
    const bool active = (i < G.X) && (j < G.Y);
    if (active) {
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
        // epilogue
        for (int k = k0; k < k1; ++k) {
            const size_t vox = (size_t)i + (size_t)j * G.X + (size_t)k * G.X * G.Y;
            const float ht = acc[(k - k0) * 128 + tid];
            if (MODE == 2) {
                const float s = sens[vox];
                const float f = vol[vox];
                vol[vox] = (s != 0.0f) ? __fdiv_rn(__fmul_rn(f, ht), s) : 0.0f;
            } else {
                vol[vox] = ht;
            }
        }
    }
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

recon_status_t build_exact_tables(Plan& P, cudaStream_t s)
{
    exact::GeomD G = geom_d(P);
    if (P.nviews) {
        exact::xy_table_kernel<<<dim3((G.Nu + 127) / 128, P.nviews), 128, 0, s>>>(G, P.d_angles, 0u, P.nviews,
                                                                                 P.d_txy, P.d_kxy, P.d_cs);
        RB_CUDA(cudaGetLastError());
    }
    exact::z_table_kernel<<<(G.Nv + 127) / 128, 128, 0, s>>>(G, P.d_zp);
    RB_CUDA(cudaGetLastError());
    exact::w_table_kernel<<<dim3((G.Nu + 127) / 128, G.Nv), 128, 0, s>>>(G, P.d_w);
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

recon_status_t exact_fp(Plan& P, const float* vol, unsigned first, unsigned count, bool scratch_slot, float* out,
                        cudaStream_t s)
{
    if (scratch_slot) {
        first = P.nviews;
        count = 1;
    }
    if (count == 0) return RECON_OK;
    if (P.opt.sum == RECON_SUM_KAHAN)
        exact::fp_kernel<true, 0, float, float><<<fp_grid(P, count), fp_block(), 0, s>>>(
            P.eg, P.d_txy, P.d_kxy, P.d_zp, P.d_w, first, vol, nullptr, out);
    else
        exact::fp_kernel<false, 0, float, float><<<fp_grid(P, count), fp_block(), 0, s>>>(
            P.eg, P.d_txy, P.d_kxy, P.d_zp, P.d_w, first, vol, nullptr, out);
    RB_CUDA(cudaGetLastError());
    return RECON_OK;
}

recon_status_t exact_fp_ratio(Plan& P, const float* vol, const void* g, void* ratio, cudaStream_t s,
                              unsigned first, unsigned count)
{
    if (count == 0) return RECON_OK;
    const bool kahan = P.opt.sum == RECON_SUM_KAHAN;
    const bool bf16 = P.opt.sino == RECON_SINO_BF16;
    const dim3 grid = fp_grid(P, count), blk = fp_block();
    const size_t off = (size_t)first * P.npix;
    using bf = __nv_bfloat16;
    if (bf16) {
        const bf* gb = (const bf*)g + off;
        bf* rb = (bf*)ratio + off;
        if (kahan)
            exact::fp_kernel<true, 1, bf, bf><<<grid, blk, 0, s>>>(P.eg, P.d_txy, P.d_kxy, P.d_zp, P.d_w, first, vol,
                                                                   gb, rb);
        else
            exact::fp_kernel<false, 1, bf, bf><<<grid, blk, 0, s>>>(P.eg, P.d_txy, P.d_kxy, P.d_zp, P.d_w, first, vol,
                                                                    gb, rb);
    } else {
        const float* gf = (const float*)g + off;
        float* rf = (float*)ratio + off;
        if (kahan)
            exact::fp_kernel<true, 1, float, float><<<grid, blk, 0, s>>>(P.eg, P.d_txy, P.d_kxy, P.d_zp, P.d_w, first,
                                                                         vol, gf, rf);
        else
            exact::fp_kernel<false, 1, float, float><<<grid, blk, 0, s>>>(P.eg, P.d_txy, P.d_kxy, P.d_zp, P.d_w,
                                                                          first, vol, gf, rf);
    }
    RB_CUDA(cudaGetLastError());
    return RECON_OK;
}

// Number of (ray, voxel) pairs with positive length: the forward walk with
// a counter in place of the accumulator.
namespace exact {
__global__ void __launch_bounds__(128) count_kernel(ExactGeom G, const float4* __restrict__ txy,
                                                     const int2* __restrict__ kxy, const ZParam* __restrict__ zp,
                                                     unsigned long long* __restrict__ total)
{
    const int u = blockIdx.x * blockDim.x + threadIdx.x;
    const int v = blockIdx.y * blockDim.y + threadIdx.y;
    const unsigned view = blockIdx.z;
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
        exact::count_kernel<<<fp_grid(P, P.nviews), fp_block()>>>(P.eg, P.d_txy, P.d_kxy, P.d_zp, d);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(out, d, sizeof(unsigned long long), cudaMemcpyDeviceToHost);
    cudaFree(d);
    if (e != cudaSuccess) return cuda_fail(e, "intersection count");
    return RECON_OK;
}

recon_status_t exact_fp_plain_ratio(Plan& P, const float* vol, const float* g, float* ratio, cudaStream_t s)
{
    if (P.opt.sum == RECON_SUM_KAHAN)
        exact::fp_kernel<true, 2, float, float><<<fp_grid(P, P.nviews), fp_block(), 0, s>>>(
            P.eg, P.d_txy, P.d_kxy, P.d_zp, P.d_w, 0u, vol, g, ratio);
    else
        exact::fp_kernel<false, 2, float, float><<<fp_grid(P, P.nviews), fp_block(), 0, s>>>(
            P.eg, P.d_txy, P.d_kxy, P.d_zp, P.d_w, 0u, vol, g, ratio);
    RB_CUDA(cudaGetLastError());
    return RECON_OK;
}

template <int ZC, int MODE, bool WEIGHTED, class ST>
static recon_status_t launch_bp(Plan& P, const ST* sino, unsigned first, unsigned count, float* vol,
                                const float* sens, cudaStream_t s)
{
    const size_t smem = (size_t)ZC * 128 * sizeof(float) + (size_t)P.eg.Nv * sizeof(ZParam);
    auto kern = exact::bp_kernel<ZC, MODE, WEIGHTED, ST>;
    RB_CUDA(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    dim3 grid((P.eg.X + 31) / 32, (P.eg.Y + 3) / 4, (P.eg.Z + ZC - 1) / ZC);
    kern<<<grid, dim3(32, 4, 1), smem, s>>>(P.eg, P.d_txy, P.d_kxy, P.d_cs, P.d_zp, P.d_w, first, count, sino, vol,
                                             sens);
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
    constexpr int ZC = 32;
    using bf = __nv_bfloat16;
    if (sens_mode) return launch_bp<ZC, 1, false, float>(P, nullptr, first, count, vol, nullptr, s);
    if (f_update) {
        if (bf16) return launch_bp<ZC, 2, false, bf>(P, (const bf*)sino, first, count, f_update, sens, s);
        return launch_bp<ZC, 2, false, float>(P, (const float*)sino, first, count, f_update, sens, s);
    }
    if (sino_is_rw) return launch_bp<ZC, 0, false, float>(P, (const float*)sino, first, count, vol, nullptr, s);
    return launch_bp<ZC, 0, true, float>(P, (const float*)sino, first, count, vol, nullptr, s);
}

}  // namespace rb
