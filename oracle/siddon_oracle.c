/*
 * siddon_oracle.c -- CPU oracle for the MLEM / Siddon cone-beam path.
 *
 * TEST INFRASTRUCTURE ONLY: the checker the CUDA product is compared against.
 * It is never linked into the product.  See siddon_oracle.h for the three
 * restatements held here and the geometry conventions they share.
 *
 * Every function names the reference file:line it restates (paths relative to
 * the reference project root).  Build: oracle/build_oracle.py (gcc -O2
 * -ffp-contract=off -fopenmp; no FMA contraction, SSE float arithmetic, so the
 * FP32 restatement evaluates every operation with one IEEE rounding).
 */
#include "siddon_oracle.h"

#include <float.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_PI 3.14159265358979323846

/* ------------------------------------------------------------------------- */
/* Host stand-ins for the GPU intrinsics the reference calls.                 */
/* ------------------------------------------------------------------------- */

/* __fdividef(a,b): approximate on the GPU; the host uses IEEE a/b.  Bit
 * agreement with the GPU is therefore not expected through this op. */
static inline float h_fdividef(float a, float b) { return a / b; }

/* __fdiv_rz(a,b): IEEE single division rounded toward zero.  The double
 * quotient of two floats is never within 2^-53 (relative) of a float it does
 * not equal, so truncating the correctly rounded double quotient toward zero
 * gives the correctly rounded-toward-zero float quotient. */
static float h_fdiv_rz(float a, float b)
{
    double q = (double)a / (double)b;
    if (isnan(q) || isinf(q)) return (float)q;
    float r = (float)q;
    if (isinf(r)) return copysignf(FLT_MAX, r);
    if (fabs((double)r) > fabs(q)) r = nextafterf(r, 0.0f);
    return r;
}

/* sin(pi*x) / cos(pi*x) in double after reduction to the nearest half
 * integer, so that integer and half-integer arguments give exact 0 and +-1
 * (as cospif / sinpif do), then rounded to float. */
static double h_sinpi_d(double x)
{
    if (!isfinite(x)) return NAN;
    double n = rint(2.0 * x);
    double f = x - 0.5 * n;
    double s = sin(ORC_PI * f), c = cos(ORC_PI * f);
    long q = (long)fmod(n, 4.0);
    if (q < 0) q += 4;
    double r = (q == 0) ? s : (q == 1) ? c : (q == 2) ? -s : -c;
    return r + 0.0;
}
static double h_cospi_d(double x)
{
    if (!isfinite(x)) return NAN;
    double n = rint(2.0 * x);
    double f = x - 0.5 * n;
    double s = sin(ORC_PI * f), c = cos(ORC_PI * f);
    long q = (long)fmod(n, 4.0);
    if (q < 0) q += 4;
    double r = (q == 0) ? c : (q == 1) ? -s : (q == 2) ? -c : s;
    return r + 0.0;
}
static inline float h_sinpif(float x) { return (float)h_sinpi_d((double)x); }
static inline float h_cospif(float x) { return (float)h_cospi_d((double)x); }

/* float -> unsigned as the GPU converts (cvt.rzi.u32.f32): NaN -> 0,
 * negative -> 0, saturating above.  Used wherever the reference assigns a
 * float (including CUDART_NAN_F) to an unsigned. */
static inline uint32_t h_f2u(float x)
{
    if (x != x) return 0u;
    if (x <= 0.0f) return 0u;
    if (x >= 4294967296.0f) return 0xFFFFFFFFu;
    return (uint32_t)x;
}
/* __float2int_rz: truncation, NaN -> 0, saturating. */
static inline int32_t h_f2i_rz(float x)
{
    if (x != x) return 0;
    if (x >= 2147483648.0f) return INT32_MAX;
    if (x <= -2147483648.0f) return INT32_MIN;
    return (int32_t)x;
}
/* __float2uint_rd: floor, NaN -> 0, saturating. */
static inline uint32_t h_f2u_rd(float x)
{
    if (x != x) return 0u;
    float f = floorf(x);
    if (f <= 0.0f) return 0u;
    if (f >= 4294967296.0f) return 0xFFFFFFFFu;
    return (uint32_t)f;
}
/* CUDART_NAN_F (siddon_device_kernelsMLEM.cuh:10): the reference's NaN bit
 * pattern, so NaN-valued outputs match bit for bit. */
static const union {
    uint32_t u;
    float f;
} kNaN_bits = {0x7FFFFFFFu};
#define kNaN (kNaN_bits.f)

/* Two arithmetic models of the reference's FP32 kernels.
 *   host (default): every operation rounded on its own and CUDART_NAN_F
 *     stored into an unsigned mask as 0 -- what the reference's kernel
 *     sources compute when compiled by a host compiler
 *     (oracle/_ref/libref_cpu.so), against which this file is pinned bit for
 *     bit;
 *   device: what the reference's sm_100a build computes -- the
 *     multiply-adds nvcc contracts are fused (fmaf) and the stores of
 *     CUDART_NAN_F into unsigned masks are absent, so every mask stays 1.
 *     Converting NaN to an integer is undefined behaviour in C++ and nvcc's
 *     optimizer drops those stores (measured on oracle/_ref/libref_gpu.so:
 *     mask = 1 for every ray of every geometry tested).  __fdividef remains
 *     IEEE division here, so agreement with the device is close but not
 *     bitwise. */
static int g_device_model = 0;
void orc_c_set_device_model(int on) { g_device_model = on ? 1 : 0; }
#define MAD(a, b, c) (g_device_model ? fmaf((a), (b), (c)) : ((a) * (b) + (c)))
#define MASK_CLEAR(m) do { if (!g_device_model) (m) = h_f2u(kNaN); } while (0)

/* ------------------------------------------------------------------------- */
/* Geometry shared by the FP32 restatement                                    */
/* ------------------------------------------------------------------------- */

/* rotation_matrix3D (CT_Recon/hf_cuda_functions.cuh:66-88): float trig of the
 * float misalignment angles, float products. */
void orc_rotation_matrix(float tx, float ty, float tz, float RM[9])
{
    RM[0] = cosf(ty) * cosf(tz) - sinf(ty) * sinf(tx) * sinf(tz);
    RM[1] = -cosf(tx) * sinf(tz);
    RM[2] = -cosf(tz) * sinf(ty) - cosf(ty) * sinf(tx) * sinf(tz);
    RM[3] = cosf(tz) * sinf(ty) * sinf(tx) + cosf(ty) * sinf(tz);
    RM[4] = cosf(tx) * cosf(tz);
    RM[5] = cosf(ty) * cosf(tz) * sinf(tx) - sinf(ty) * sinf(tz);
    RM[6] = cosf(tx) * sinf(ty);
    RM[7] = -sinf(tx);
    RM[8] = cosf(ty) * cosf(tx);
}

/* pixel_iterate2 (CT_Recon/hf_cuda_kernels.cuh:92-97): pixel centre rounded
 * to 1e-5 mm. */
float orc_c_pixel_iterate2(float NumPixels, float PixelsDimMm, float Mag, int iterator)
{
    float result = MAD(h_fdividef(-(NumPixels - 1.0f), 2.0f) * PixelsDimMm, Mag,
                       h_fdividef((float)iterator, NumPixels) * NumPixels * PixelsDimMm * Mag);
    return h_fdiv_rz(rintf(result * 100000.0f), 100000.0f);
}

/* pixel_iterate (CT_Recon/hf_cuda_kernels.cuh:83-87): unrounded centre. */
static float c_pixel_iterate(float NumPixels, float PixelsDimMm, float Mag, int iterator)
{
    return -(NumPixels - 1.0f) / 2.0f * PixelsDimMm * Mag + (float)iterator * PixelsDimMm * Mag;
}

typedef struct {
    float Pi[3], Pf[3], Pd[3], Xs[3];
} c_planes;

/* siddon_commons::a1_initiate (CT_Recon/hf_siddon_class.hpp:43-61). */
static void c_planes_init(const orc_geom* g, c_planes* p)
{
    p->Pi[0] = -(float)g->Xdim / 2.0f * (float)g->XVoxSize;
    p->Pi[1] = -(float)g->Ydim / 2.0f * (float)g->YVoxSize;
    p->Pi[2] = -(float)g->Zdim / 2.0f * (float)g->ZVoxSize;
    p->Pf[0] = (float)g->Xdim / 2.0f * (float)g->XVoxSize;
    p->Pf[1] = (float)g->Ydim / 2.0f * (float)g->YVoxSize;
    p->Pf[2] = (float)g->Zdim / 2.0f * (float)g->ZVoxSize;
    p->Pd[0] = g->XVoxSize;
    p->Pd[1] = g->YVoxSize;
    p->Pd[2] = g->ZVoxSize;
    p->Xs[0] = 0.0f;
    p->Xs[1] = -g->Rf;
    p->Xs[2] = 0.0f;
}

/* calc_points12 (CT_Recon/siddon_device_kernelsMLEM.cuh:305-331), including
 * the overwrite of detector.x at :315 before its use at :316. */
static void c_points12(const orc_geom* g, const float RM[9], const c_planes* P, int u, int v,
                       float angle, float p1[3], float p2[3])
{
    float dx = orc_c_pixel_iterate2((float)g->NumAxPixels, g->AxPixDimMm, g->M, u);
    float dy = g->R - g->Rf;
    float dz = orc_c_pixel_iterate2((float)g->NumTAxPixels, g->TAxPixDimMm, g->M, v);
    dx = h_fdividef(g->R, MAD(RM[5], dz, MAD(RM[3], dx, g->Ry))) * (MAD(RM[0], dx, RM[2] * dz) + g->Dx);
    dz = h_fdividef(g->R, MAD(RM[5], dz, MAD(RM[3], dx, g->Ry))) * (MAD(RM[6], dx, RM[8] * dz) + g->Dz);
    float c = h_cospif(h_fdividef(angle, 180.0f));
    float s = h_sinpif(h_fdividef(angle, 180.0f));
    p1[0] = MAD(P->Xs[0], c, P->Xs[1] * s);
    p1[1] = MAD(-P->Xs[0], s, P->Xs[1] * c);
    p1[2] = P->Xs[2];
    p2[0] = MAD(dx, c, dy * s);
    p2[1] = MAD(-dx, s, dy * c);
    p2[2] = dz;
}

/* calc_alpha_1N (siddon_device_kernelsMLEM.cuh:71-85) */
static void c_alpha_1N(float p1, float p2, float plane1, float plane2, float a[2])
{
    if ((p2 - p1) != 0) {
        a[0] = h_fdividef(plane1 - p1, p2 - p1);
        a[1] = h_fdividef(plane2 - p1, p2 - p1);
    } else {
        a[0] = kNaN;
        a[1] = kNaN;
    }
}

/* find_index (siddon_device_kernelsMLEM.cuh:151-185) */
static float c_find_index(float index, float amin, float amax, float p1, float p2, float plane1,
                          float dplane)
{
    if (index > 0.0f) {
        float low = floorf(index), high = ceilf(index);
        float plane_low = MAD(dplane, (low - 1.0f), plane1);
        float plane_high = MAD(dplane, (high - 1.0f), plane1);
        float alow = h_fdividef(plane_low - p1, p2 - p1);
        float ahigh = h_fdividef(plane_high - p1, p2 - p1);
        if (alow >= amin && alow <= amax) return low;
        else if (ahigh >= amin && ahigh <= amax) return high;
        else return kNaN;
    }
    return kNaN;
}

/* bound_index (siddon_device_kernelsMLEM.cuh:50-58) */
static void c_bound_index(float* imin, float* imax, uint32_t* mask)
{
    if ((*imax - *imin) < 0 && *imin <= 1 && *imax <= 1) {
        *imin = 0;
        *imax = 0;
        MASK_CLEAR(*mask);
    }
}

/* alpha_float (siddon_device_kernelsMLEM.cuh:218-237): the plane indices
 * arrive as unsigned, the "> 0" test is on their unsigned difference. */
static float c_alpha_float(uint32_t mn, uint32_t mx, float p1, float p2, float plane1,
                           float dplane)
{
    float plane;
    if ((p2 - p1) > 0 && (mx - mn) > 0) {
        plane = MAD(dplane, ((float)mn - 1.0f), plane1);
        return h_fdividef(plane - p1, p2 - p1);
    } else if ((p2 - p1) < 0 && (mx - mn) > 0) {
        plane = MAD(dplane, ((float)mx - 1.0f), plane1);
        return h_fdividef(plane - p1, p2 - p1);
    }
    return kNaN;
}

/* siddon_calc_indices (siddon_device_kernelsMLEM.cuh:240-270) */
static uint32_t c_calc_indices(float* ai, float* af, uint32_t* mask, float p1, float p2,
                               float plane1, float plane2, float Nplanes, float amin, float amax,
                               float dplane)
{
    float ix, iy;
    if ((p2 - p1) > 0) {
        ix = Nplanes - h_fdividef((MAD(-amin, (p2 - p1), plane2) - p1), dplane);
        iy = 1.0f + h_fdividef((MAD(amax, (p2 - p1), p1) - plane1), dplane);
    } else if ((p2 - p1) < 0) {
        ix = Nplanes - h_fdividef((MAD(-amax, (p2 - p1), plane2) - p1), dplane);
        iy = 1.0f + h_fdividef((MAD(amin, (p2 - p1), p1) - plane1), dplane);
    } else {
        ix = 0;
        iy = 0;
        MASK_CLEAR(*mask);
    }
    ix = (float)*mask * c_find_index(ix, amin, amax, p1, p2, plane1, dplane);
    iy = (float)*mask * c_find_index(iy, amin, amax, p1, p2, plane1, dplane);
    c_bound_index(&ix, &iy, mask);
    *ai = (float)*mask * c_alpha_float(h_f2u(ix), h_f2u(iy), p1, p2, plane1, dplane);
    *af = (float)*mask * c_alpha_float(h_f2u(iy), h_f2u(ix), p1, p2, plane1, dplane);
    return h_f2u(iy - ix);
}

/* siddon_alpha_limits (CT_Recon/siddon_kernelsMLEM.cuh:103-149) for one ray. */
static void c_ray_setup(const orc_geom* g, const float RM[9], const c_planes* P, float angle,
                        int u, int v, orc_c_ray* r)
{
    float* p1 = r->p1;
    float* p2 = r->p2;
    c_points12(g, RM, P, u, v, angle, p1, p2);
    r->d12 = sqrtf(MAD((p2[2] - p1[2]), (p2[2] - p1[2]),
                       MAD((p2[0] - p1[0]), (p2[0] - p1[0]), (p2[1] - p1[1]) * (p2[1] - p1[1]))));
    float ax[2], ay[2], az[2];
    c_alpha_1N(p1[0], p2[0], P->Pi[0], P->Pf[0], ax);
    c_alpha_1N(p1[1], p2[1], P->Pi[1], P->Pf[1], ay);
    c_alpha_1N(p1[2], p2[2], P->Pi[2], P->Pf[2], az);
    float amin = fmaxf(fmaxf(fmaxf(0, fminf(ax[0], ax[1])), fminf(ay[0], ay[1])), fminf(az[0], az[1]));
    float amax = fminf(fminf(fminf(1, fmaxf(ax[0], ax[1])), fmaxf(ay[0], ay[1])), fmaxf(az[0], az[1]));
    uint32_t mask = (amax <= amin && !g_device_model) ? h_f2u(kNaN) : 1u; /* calc_mask :88-98 */
    amin = (float)mask * amin;
    amax = (float)mask * amax;
    uint32_t idx[3];
    const unsigned dims[3] = {g->Xdim, g->Ydim, g->Zdim};
    for (int a = 0; a < 3; ++a)
        idx[a] = c_calc_indices(&r->alpha_i[a], &r->alpha_f[a], &mask, p1[a], p2[a], P->Pi[a],
                                P->Pf[a], (float)dims[a] + 1.0f, amin, amax, P->Pd[a]);
    r->delta_index = idx[0] + 1 + idx[1] + 1 + idx[2] + 1 + 1;
    /* delta_alpha (siddon_device_kernelsMLEM.cuh:100-113): its NaN guards
     * compare against NaN and are always true. */
    for (int a = 0; a < 3; ++a) r->delta_alpha[a] = fabsf(h_fdividef(P->Pd[a], p2[a] - p1[a]));
    r->mask = mask;
    r->alpha_min = amin;
    r->alpha_max = amax;
}

void orc_c_ray_setup(const orc_geom* g, const float RM[9], float angle_deg, int u, int v,
                     orc_c_ray* out)
{
    c_planes P;
    c_planes_init(g, &P);
    c_ray_setup(g, RM, &P, angle_deg, u, v, out);
}

/* siddon_alpha_limits over every ray of a view, in the array layout of
 * siddon_commons (hf_siddon_class.hpp:20-34); float3 arrays are [n][3].
 * Returns max(delta_index) = loopN (hf_siddon_class.hpp:103-104). */
uint32_t orc_c_setup_view(const orc_geom* g, const float RM[9], float angle_deg, float* alpha_min,
                          float* alpha_max, float* d12, uint32_t* mask, float* alpha_i,
                          float* alpha_f, float* delta_alpha, float* p1, float* p2,
                          uint32_t* delta_index)
{
    c_planes P;
    c_planes_init(g, &P);
    uint32_t mx = 0;
    const unsigned Nu = g->NumAxPixels, Nv = g->NumTAxPixels;
    for (unsigned v = 0; v < Nv; ++v)
        for (unsigned u = 0; u < Nu; ++u) {
            size_t n = u + (size_t)v * Nu;
            orc_c_ray r;
            c_ray_setup(g, RM, &P, angle_deg, (int)u, (int)v, &r);
            alpha_min[n] = r.alpha_min;
            alpha_max[n] = r.alpha_max;
            d12[n] = r.d12;
            mask[n] = r.mask;
            delta_index[n] = r.delta_index;
            for (int k = 0; k < 3; ++k) {
                alpha_i[3 * n + k] = r.alpha_i[k];
                alpha_f[3 * n + k] = r.alpha_f[k];
                delta_alpha[3 * n + k] = r.delta_alpha[k];
                p1[3 * n + k] = r.p1[k];
                p2[3 * n + k] = r.p2[k];
            }
            if (r.delta_index > mx) mx = r.delta_index;
        }
    return mx;
}

uint32_t orc_c_loopN(const orc_geom* g, const float RM[9], float angle_deg)
{
    c_planes P;
    c_planes_init(g, &P);
    uint32_t mx = 0;
    for (unsigned v = 0; v < g->NumTAxPixels; ++v)
        for (unsigned u = 0; u < g->NumAxPixels; ++u) {
            orc_c_ray r;
            c_ray_setup(g, RM, &P, angle_deg, (int)u, (int)v, &r);
            if (r.delta_index > mx) mx = r.delta_index;
        }
    return mx;
}

/* ---- traversal state machine ---- */
typedef struct {
    float a[3];
    float cur, next;
} c_state;

static inline int same_f(float x, float y) { return (x == y) || (x != x && y != y); }

/* siddon_begin (siddon_kernelsMLEM.cuh:283-303) */
static void c_begin(const orc_c_ray* r, c_state* s)
{
    for (int k = 0; k < 3; ++k) s->a[k] = (float)r->mask * r->alpha_i[k];
    s->next = fminf(fminf(r->alpha_i[0], r->alpha_i[1]), r->alpha_i[2]);
    s->cur = kNaN;
}

/* alpha_bound (siddon_device_kernelsMLEM.cuh:134-148) */
static inline float c_alpha_bound(float a, float ai, float af, float amax)
{
    if (a >= ai && a <= af) return a;
    else if (a > af) return amax;
    return kNaN;
}

/* siddon_sort_alpha (siddon_kernelsMLEM.cuh:153-190).  Returns 1 when the
 * state after the step equals the state before it with next == current, i.e.
 * every later step repeats it and contributes a zero-length segment. */
static int c_sort(const orc_c_ray* r, c_state* s)
{
    float a0 = s->a[0], a1 = s->a[1], a2 = s->a[2], n0 = s->next;
    s->cur = s->next;
    if (s->cur == s->a[0]) {
        s->a[0] = s->a[0] + r->delta_alpha[0];
        s->a[0] = c_alpha_bound(s->a[0], r->alpha_i[0], r->alpha_f[0], r->alpha_max);
    } else if (s->cur == s->a[1]) {
        s->a[1] = s->a[1] + r->delta_alpha[1];
        s->a[1] = c_alpha_bound(s->a[1], r->alpha_i[1], r->alpha_f[1], r->alpha_max);
    } else if (s->cur == s->a[2]) {
        s->a[2] = s->a[2] + r->delta_alpha[2];
        s->a[2] = c_alpha_bound(s->a[2], r->alpha_i[2], r->alpha_f[2], r->alpha_max);
    }
    s->next = fminf(fminf(s->a[0], s->a[1]), s->a[2]);
    return same_f(a0, s->a[0]) && same_f(a1, s->a[1]) && same_f(a2, s->a[2]) &&
           same_f(n0, s->next) && same_f(s->next, s->cur);
}

/* Segment evaluation shared by siddon_fp_calc_ray_path (:193-233),
 * siddon_fp_end (:238-279), siddon_bp_calc_ray_path (:307-352) and
 * siddon_bp_end (:367-411): the midpoint voxel index and the ray length. The
 * mask / NaN guards there compare against NaN and are always true. */
static int32_t c_segment(const orc_geom* g, const c_planes* P, const orc_c_ray* r, float a_hi,
                         float a_lo, float* len)
{
    int32_t ix = -1, iy = -1, iz = -1;
    float rl = 0.0f;
    if (a_hi > a_lo) {
        float mid = h_fdividef((a_hi + a_lo), 2.0f);
        rl = r->d12 * (a_hi - a_lo);
        ix = h_f2i_rz((h_fdividef((MAD(mid, (r->p2[0] - r->p1[0]), r->p1[0]) - P->Pi[0]), P->Pd[0])));
        iy = h_f2i_rz((h_fdividef((MAD(mid, (r->p2[1] - r->p1[1]), r->p1[1]) - P->Pi[1]), P->Pd[1])));
        iz = h_f2i_rz((h_fdividef((MAD(mid, (r->p2[2] - r->p1[2]), r->p1[2]) - P->Pi[2]), P->Pd[2])));
    }
    *len = rl;
    if (ix >= 0 && ix < (int32_t)g->Xdim && iy >= 0 && iy < (int32_t)g->Ydim && iz >= 0 &&
        iz < (int32_t)g->Zdim)
        return (int32_t)((uint32_t)iz * (g->Ydim * g->Xdim) + (uint32_t)iy * g->Xdim + (uint32_t)ix);
    return -1;
}

int orc_c_trace(const orc_geom* g, const float RM[9], float angle_deg, int u, int v,
                uint32_t loopN, int32_t* idx, float* len, int cap)
{
    c_planes P;
    c_planes_init(g, &P);
    orc_c_ray r;
    c_ray_setup(g, RM, &P, angle_deg, u, v, &r);
    c_state s;
    c_begin(&r, &s);
    int n = 0;
    for (uint32_t k = 0; k < loopN; ++k) {
        int fixed = c_sort(&r, &s);
        float l;
        int32_t id = c_segment(g, &P, &r, s.next, s.cur, &l);
        if (n >= cap) return -1;
        idx[n] = id;
        len[n] = (id >= 0) ? l : 0.0f;
        ++n;
        if (fixed) break;
    }
    float l;
    int32_t id = c_segment(g, &P, &r, r.alpha_max, s.cur, &l);
    if (n >= cap) return -1;
    idx[n] = id;
    len[n] = (id >= 0) ? l : 0.0f;
    return n + 1;
}

/* forward::a2_fp_per_angle (CT_Recon/hf_siddon_class.hpp:195-225): the image
 * is the sum over steps, in step order, of len*f[idx] (one product rounding,
 * then one add rounding via siddon_add). */
void orc_c_fp_view(const orc_geom* g, const float RM[9], float angle_deg, const float* vol,
                   float* img)
{
    c_planes P;
    c_planes_init(g, &P);
    const unsigned Nu = g->NumAxPixels, Nv = g->NumTAxPixels;
    uint32_t loopN = orc_c_loopN(g, RM, angle_deg);
    for (unsigned v = 0; v < Nv; ++v)
        for (unsigned u = 0; u < Nu; ++u) {
            orc_c_ray r;
            c_ray_setup(g, RM, &P, angle_deg, (int)u, (int)v, &r);
            c_state s;
            c_begin(&r, &s);
            float acc = 0.0f, l;
            for (uint32_t k = 0; k < loopN; ++k) {
                int fixed = c_sort(&r, &s);
                int32_t id = c_segment(g, &P, &r, s.next, s.cur, &l);
                float t = (id >= 0) ? l * vol[id] : 0.0f;
                acc = acc + t;
                if (fixed) break;
            }
            int32_t id = c_segment(g, &P, &r, r.alpha_max, s.cur, &l);
            float t = (id >= 0) ? l * vol[id] : 0.0f;
            acc = acc + t;
            img[u + v * Nu] = acc;
        }
}

/* backward::a2_bp_per_angle (CT_Recon/hf_siddon_class.hpp:313-347): per step
 * the contributions len*img[n] of all rays are summed into a temporary volume
 * (float atomics in the reference; ray order here), then the temporary is
 * added to the output.  Rays advance in lock step as the step kernels do. */
void orc_c_bp_view(const orc_geom* g, const float RM[9], float angle_deg, const float* img,
                   float* vol_out)
{
    c_planes P;
    c_planes_init(g, &P);
    const unsigned Nu = g->NumAxPixels, Nv = g->NumTAxPixels;
    const size_t Npix = (size_t)Nu * Nv;
    const size_t V = (size_t)g->Xdim * g->Ydim * g->Zdim;
    uint32_t loopN = orc_c_loopN(g, RM, angle_deg);
    orc_c_ray* rays = (orc_c_ray*)malloc(Npix * sizeof(orc_c_ray));
    c_state* st = (c_state*)malloc(Npix * sizeof(c_state));
    uint32_t* active = (uint32_t*)malloc(Npix * sizeof(uint32_t));
    float* temp = (float*)calloc(V, sizeof(float));
    uint8_t* touched = (uint8_t*)calloc(V, 1);
    uint32_t* tlist = (uint32_t*)malloc(Npix * sizeof(uint32_t));
    size_t nact = 0;
    for (size_t n = 0; n < Npix; ++n) {
        c_ray_setup(g, RM, &P, angle_deg, (int)(n % Nu), (int)(n / Nu), &rays[n]);
        c_begin(&rays[n], &st[n]);
        active[nact++] = (uint32_t)n;
    }
    memset(vol_out, 0, V * sizeof(float));
    for (uint32_t k = 0; k < loopN && nact > 0; ++k) {
        size_t nt = 0, keep = 0;
        for (size_t q = 0; q < nact; ++q) {
            uint32_t n = active[q];
            int fixed = c_sort(&rays[n], &st[n]);
            float l;
            int32_t id = c_segment(g, &P, &rays[n], st[n].next, st[n].cur, &l);
            if (id >= 0) {
                float c = l * img[n];
                temp[id] = temp[id] + c;
                if (!touched[id]) {
                    touched[id] = 1;
                    tlist[nt++] = (uint32_t)id;
                }
            }
            if (!fixed) active[keep++] = n;
        }
        nact = keep;
        for (size_t q = 0; q < nt; ++q) {
            uint32_t id = tlist[q];
            vol_out[id] = vol_out[id] + temp[id];
            temp[id] = 0.0f;
            touched[id] = 0;
        }
    }
    /* siddon_bp_end for every ray (fixed-point rays keep their current) */
    {
        size_t nt = 0;
        for (size_t n = 0; n < Npix; ++n) {
            float l;
            int32_t id = c_segment(g, &P, &rays[n], rays[n].alpha_max, st[n].cur, &l);
            if (id >= 0) {
                float c = l * img[n];
                temp[id] = temp[id] + c;
                if (!touched[id]) {
                    touched[id] = 1;
                    tlist[nt++] = (uint32_t)id;
                }
            }
        }
        for (size_t q = 0; q < nt; ++q) {
            uint32_t id = tlist[q];
            vol_out[id] = vol_out[id] + temp[id];
            temp[id] = 0.0f;
            touched[id] = 0;
        }
    }
    free(rays);
    free(st);
    free(active);
    free(temp);
    free(touched);
    free(tlist);
}

/* m_calc_sensitivity + m_mlem_all_iterations + m_mlem_single_iteration
 * (CT_Recon/hf_siddon_recon.hpp:388-415, 437-511): sensitivity = sum over
 * views of BP(ones); f0 = 1; per iteration Ht = sum over views of
 * BP(divide1(g, FP(f))); then f = f*Ht; f = divide1(f, sens). */
void orc_c_mlem(const orc_geom* g, unsigned int NumProj, float DeltaAng, const float* g_sino,
                unsigned int iters, float* f, float* sens_out, float* f_history)
{
    float RM[9];
    orc_rotation_matrix(g->xangle, g->yangle, g->zangle, RM);
    const size_t Npix = (size_t)g->NumAxPixels * g->NumTAxPixels;
    const size_t V = (size_t)g->Xdim * g->Ydim * g->Zdim;
    float* ones = (float*)malloc(Npix * sizeof(float));
    float* bp = (float*)malloc(V * sizeof(float));
    float* Ht = (float*)malloc(V * sizeof(float));
    float* hf = (float*)malloc(Npix * sizeof(float));
    float* sens = sens_out ? sens_out : (float*)malloc(V * sizeof(float));
    for (size_t i = 0; i < Npix; ++i) ones[i] = 1.0f;
    memset(sens, 0, V * sizeof(float));
    for (unsigned n = 0; n < NumProj; ++n) {
        float ang = DeltaAng * (float)n;
        orc_c_bp_view(g, RM, ang, ones, bp);
        for (size_t i = 0; i < V; ++i) sens[i] = sens[i] + bp[i];
    }
    for (size_t i = 0; i < V; ++i) f[i] = 1.0f;
    for (unsigned it = 0; it < iters; ++it) {
        memset(Ht, 0, V * sizeof(float));
        for (unsigned n = 0; n < NumProj; ++n) {
            float ang = (float)n * DeltaAng;
            orc_c_fp_view(g, RM, ang, f, hf);
            const float* gv = g_sino + (size_t)n * Npix;
            for (size_t i = 0; i < Npix; ++i) hf[i] = (hf[i] != 0) ? h_fdividef(gv[i], hf[i]) : 0.0f;
            orc_c_bp_view(g, RM, ang, hf, bp);
            for (size_t i = 0; i < V; ++i) Ht[i] = Ht[i] + bp[i];
        }
        for (size_t i = 0; i < V; ++i) f[i] = f[i] * Ht[i];
        for (size_t i = 0; i < V; ++i) f[i] = (sens[i] != 0) ? h_fdividef(f[i], sens[i]) : 0.0f;
        if (f_history) memcpy(f_history + (size_t)it * V, f, V * sizeof(float));
    }
    free(ones);
    free(bp);
    free(Ht);
    free(hf);
    if (!sens_out) free(sens);
}

/* ------------------------------------------------------------------------- */
/* FP64 exact Siddon                                                          */
/* ------------------------------------------------------------------------- */

/* Scanner geometry of calc_points12 (siddon_device_kernelsMLEM.cuh:305-331)
 * evaluated in double: detector pixel centres -(N-1)/2*d*M + i*d*M rounded to
 * the 1e-5 mm grid as pixel_iterate2 intends (hf_cuda_kernels.cuh:92-97),
 * misalignment with the same overwrite order, rotation by the view angle. */
static double x_pixel_center(unsigned N, float d, float M, int i)
{
    double c = -((double)N - 1.0) / 2.0 * (double)d * (double)M + (double)i * (double)d * (double)M;
    return rint(c * 1e5) / 1e5;
}

void orc_x_ray_geom(const orc_geom* g, float angle_deg, int u, int v, orc_x_ray* r)
{
    double tx = g->xangle, ty = g->yangle, tz = g->zangle;
    double RM[9];
    RM[0] = cos(ty) * cos(tz) - sin(ty) * sin(tx) * sin(tz);
    RM[2] = -cos(tz) * sin(ty) - cos(ty) * sin(tx) * sin(tz);
    RM[3] = cos(tz) * sin(ty) * sin(tx) + cos(ty) * sin(tz);
    RM[5] = cos(ty) * cos(tz) * sin(tx) - sin(ty) * sin(tz);
    RM[6] = cos(tx) * sin(ty);
    RM[8] = cos(ty) * cos(tx);
    double dx = x_pixel_center(g->NumAxPixels, g->AxPixDimMm, g->M, u);
    double dy = (double)g->R - (double)g->Rf;
    double dz = x_pixel_center(g->NumTAxPixels, g->TAxPixDimMm, g->M, v);
    double R = g->R, Ry = g->Ry;
    dx = R / (Ry + RM[3] * dx + RM[5] * dz) * (RM[0] * dx + RM[2] * dz + (double)g->Dx);
    dz = R / (Ry + RM[3] * dx + RM[5] * dz) * (RM[6] * dx + RM[8] * dz + (double)g->Dz);
    double t = (double)angle_deg / 180.0;
    double c = h_cospi_d(t), s = h_sinpi_d(t);
    double Rf = g->Rf;
    r->p1[0] = -Rf * s;
    r->p1[1] = -Rf * c;
    r->p1[2] = 0.0;
    r->p2[0] = dx * c + dy * s;
    r->p2[1] = -dx * s + dy * c;
    r->p2[2] = dz;
    double a = r->p2[0] - r->p1[0], b = r->p2[1] - r->p1[1], e = r->p2[2] - r->p1[2];
    r->d12 = sqrt(a * a + b * b + e * e);
}

typedef void (*x_emit_fn)(void* ctx, int64_t voxel, double len);

/* Exact traversal: every voxel the segment p1->p2 crosses with positive
 * length, in order along the ray; tied plane crossings advance together. */
static void x_traverse(const orc_geom* g, const orc_x_ray* r, x_emit_fn emit, void* ctx)
{
    const unsigned dims[3] = {g->Xdim, g->Ydim, g->Zdim};
    const double vox[3] = {g->XVoxSize, g->YVoxSize, g->ZVoxSize};
    double P0[3], d[3];
    double ain = 0.0, aout = 1.0;
    for (int k = 0; k < 3; ++k) {
        P0[k] = -(double)dims[k] / 2.0 * vox[k];
        d[k] = r->p2[k] - r->p1[k];
        double PN = P0[k] + dims[k] * vox[k];
        if (d[k] == 0.0) {
            if (r->p1[k] < P0[k] || r->p1[k] >= PN) return;
        } else {
            double a0 = (P0[k] - r->p1[k]) / d[k], a1 = (PN - r->p1[k]) / d[k];
            double lo = a0 < a1 ? a0 : a1, hi = a0 < a1 ? a1 : a0;
            if (lo > ain) ain = lo;
            if (hi < aout) aout = hi;
        }
    }
    if (!(ain < aout)) return;
    int64_t i[3];
    double anext[3];
    int step[3];
    for (int k = 0; k < 3; ++k) {
        double x = r->p1[k] + ain * d[k];
        double fidx = (x - P0[k]) / vox[k];
        int64_t ii;
        if (d[k] > 0) ii = (int64_t)floor(fidx);
        else if (d[k] < 0) ii = (int64_t)ceil(fidx) - 1;
        else ii = (int64_t)floor(fidx);
        if (ii < 0) ii = 0;
        if (ii >= (int64_t)dims[k]) ii = dims[k] - 1;
        i[k] = ii;
        if (d[k] > 0) {
            step[k] = 1;
            anext[k] = (P0[k] + (ii + 1) * vox[k] - r->p1[k]) / d[k];
        } else if (d[k] < 0) {
            step[k] = -1;
            anext[k] = (P0[k] + ii * vox[k] - r->p1[k]) / d[k];
        } else {
            step[k] = 0;
            anext[k] = INFINITY;
        }
    }
    double cur = ain;
    for (;;) {
        double m = anext[0];
        if (anext[1] < m) m = anext[1];
        if (anext[2] < m) m = anext[2];
        if (aout < m) m = aout;
        double L = (m - cur) * r->d12;
        if (L > 0.0)
            emit(ctx, i[0] + i[1] * (int64_t)dims[0] + i[2] * (int64_t)dims[0] * dims[1], L);
        cur = m;
        if (m >= aout) return;
        for (int k = 0; k < 3; ++k) {
            if (anext[k] == m) {
                i[k] += step[k];
                if (i[k] < 0 || i[k] >= (int64_t)dims[k]) return;
                double pl = (step[k] > 0) ? P0[k] + (i[k] + 1) * vox[k] : P0[k] + i[k] * vox[k];
                anext[k] = (pl - r->p1[k]) / d[k];
            }
        }
    }
}

typedef struct {
    int64_t* idx;
    double* len;
    int n, cap;
} x_trace_ctx;
static void x_emit_trace(void* c, int64_t vox, double len)
{
    x_trace_ctx* t = (x_trace_ctx*)c;
    if (t->n < t->cap) {
        t->idx[t->n] = vox;
        t->len[t->n] = len;
    }
    t->n++;
}
int orc_x_trace(const orc_geom* g, float angle_deg, int u, int v, int64_t* idx, double* len,
                int cap)
{
    orc_x_ray r;
    orc_x_ray_geom(g, angle_deg, u, v, &r);
    x_trace_ctx t = {idx, len, 0, cap};
    x_traverse(g, &r, x_emit_trace, &t);
    return t.n <= cap ? t.n : -1;
}

typedef struct {
    const double* vol;
    double acc;
} x_fp_ctx;
static void x_emit_fp(void* c, int64_t vox, double len)
{
    x_fp_ctx* t = (x_fp_ctx*)c;
    t->acc += len * t->vol[vox];
}

void orc_x_fp_view(const orc_geom* g, float angle_deg, const double* vol, double* img)
{
    const unsigned Nu = g->NumAxPixels, Nv = g->NumTAxPixels;
    for (unsigned v = 0; v < Nv; ++v)
        for (unsigned u = 0; u < Nu; ++u) {
            orc_x_ray r;
            orc_x_ray_geom(g, angle_deg, (int)u, (int)v, &r);
            x_fp_ctx c = {vol, 0.0};
            x_traverse(g, &r, x_emit_fp, &c);
            img[u + (size_t)v * Nu] = c.acc;
        }
}

static int set_threads(int threads)
{
#ifdef _OPENMP
    if (threads > 0) return threads;
    return omp_get_max_threads();
#else
    (void)threads;
    return 1;
#endif
}

/* Views first .. first+count-1 (view n at (float)n * DeltaAng) into sino
 * (count images back to back). */
static void x_fp_views(const orc_geom* g, unsigned int first, unsigned int count, float DeltaAng,
                       const double* vol, double* sino, int threads)
{
    const size_t Npix = (size_t)g->NumAxPixels * g->NumTAxPixels;
    int nt = set_threads(threads);
    (void)nt;
#pragma omp parallel for schedule(dynamic, 1) num_threads(nt)
    for (long n = 0; n < (long)count; ++n)
        orc_x_fp_view(g, (float)(first + (unsigned)n) * DeltaAng, vol, sino + (size_t)n * Npix);
}

void orc_x_fp_all(const orc_geom* g, unsigned int NumProj, float DeltaAng, const double* vol,
                  double* sino, int threads)
{
    x_fp_views(g, 0, NumProj, DeltaAng, vol, sino, threads);
}

typedef struct {
    double* vol;
    double val;
} x_bp_ctx;
static void x_emit_bp(void* c, int64_t vox, double len)
{
    x_bp_ctx* t = (x_bp_ctx*)c;
    t->vol[vox] += len * t->val;
}

/* Ray-driven FP64 back projection, deterministic for a given thread count:
 * views are split statically over threads, each thread owns a partial
 * volume, partials are summed in thread order. */
static void x_bp_views(const orc_geom* g, unsigned int first, unsigned int NumProj, float DeltaAng,
                       const double* sino, double* vol, int threads);

void orc_x_bp_all(const orc_geom* g, unsigned int NumProj, float DeltaAng, const double* sino,
                  double* vol, int threads)
{
    x_bp_views(g, 0, NumProj, DeltaAng, sino, vol, threads);
}

/* Views first .. first+NumProj-1 of sino (NumProj images back to back). */
static void x_bp_views(const orc_geom* g, unsigned int first, unsigned int NumProj, float DeltaAng,
                       const double* sino, double* vol, int threads)
{
    const unsigned Nu = g->NumAxPixels, Nv = g->NumTAxPixels;
    const size_t Npix = (size_t)Nu * Nv;
    const size_t V = (size_t)g->Xdim * g->Ydim * g->Zdim;
    int nt = set_threads(threads);
    if ((unsigned)nt > NumProj) nt = (int)NumProj;
    if (nt < 1) nt = 1;
    double* part = (double*)calloc((size_t)nt * V, sizeof(double));
#pragma omp parallel num_threads(nt)
    {
        int t = 0;
#ifdef _OPENMP
        t = omp_get_thread_num();
#endif
        double* pv = part + (size_t)t * V;
        for (unsigned n = (unsigned)t; n < NumProj; n += (unsigned)nt) {
            float ang = (float)(first + n) * DeltaAng;
            const double* img = sino + (size_t)n * Npix;
            for (unsigned v = 0; v < Nv; ++v)
                for (unsigned u = 0; u < Nu; ++u) {
                    double val = img[u + (size_t)v * Nu];
                    orc_x_ray r;
                    orc_x_ray_geom(g, ang, (int)u, (int)v, &r);
                    x_bp_ctx c = {pv, val};
                    x_traverse(g, &r, x_emit_bp, &c);
                }
        }
    }
    memset(vol, 0, V * sizeof(double));
    for (int t = 0; t < nt; ++t) {
        const double* pv = part + (size_t)t * V;
        for (size_t i = 0; i < V; ++i) vol[i] += pv[i];
    }
    free(part);
}

/* MLEM in FP64 with the reference's update rule (hf_siddon_recon.hpp:437-511)
 * and zero guards (divide1, hf_cuda_kernels.cuh:370-387). */
void orc_x_mlem(const orc_geom* g, unsigned int NumProj, float DeltaAng, const float* g_sino,
                unsigned int iters, double* f, double* sens_out, int threads)
{
    const size_t Npix = (size_t)g->NumAxPixels * g->NumTAxPixels;
    const size_t P = Npix * NumProj;
    const size_t V = (size_t)g->Xdim * g->Ydim * g->Zdim;
    double* sino = (double*)malloc(P * sizeof(double));
    double* Ht = (double*)malloc(V * sizeof(double));
    double* sens = sens_out ? sens_out : (double*)malloc(V * sizeof(double));
    for (size_t i = 0; i < P; ++i) sino[i] = 1.0;
    orc_x_bp_all(g, NumProj, DeltaAng, sino, sens, threads);
    for (size_t i = 0; i < V; ++i) f[i] = 1.0;
    for (unsigned it = 0; it < iters; ++it) {
        orc_x_fp_all(g, NumProj, DeltaAng, f, sino, threads);
        for (size_t i = 0; i < P; ++i) sino[i] = (sino[i] != 0.0) ? (double)g_sino[i] / sino[i] : 0.0;
        orc_x_bp_all(g, NumProj, DeltaAng, sino, Ht, threads);
        for (size_t i = 0; i < V; ++i) f[i] = (sens[i] != 0.0) ? f[i] * Ht[i] / sens[i] : 0.0;
    }
    free(sino);
    free(Ht);
    if (!sens_out) free(sens);
}

/* OSEM in FP64 with N_subsets contiguous subsets of NumProj / N_subsets
 * views (the subset layout of osem_input_values / check_recon_inputs,
 * hf_cpp_functions.hpp:298-375, where the reference stops): per subset s,
 * f <- f * BP_s(g / FP_s(f)) / BP_s(1) with the zero guards of MLEM.
 * Returns 0, or -1 when N_subsets does not divide NumProj. */
int orc_x_osem(const orc_geom* g, unsigned int NumProj, float DeltaAng, const float* g_sino, unsigned int iters,
               unsigned int N_subsets, double* f, int threads)
{
    if (N_subsets == 0 || NumProj % N_subsets != 0) return -1;
    const unsigned n = NumProj / N_subsets;
    const size_t Npix = (size_t)g->NumAxPixels * g->NumTAxPixels;
    const size_t Ps = Npix * n;
    const size_t V = (size_t)g->Xdim * g->Ydim * g->Zdim;
    double* sino = (double*)malloc(Ps * sizeof(double));
    double* Ht = (double*)malloc(V * sizeof(double));
    double* sens = (double*)malloc((size_t)N_subsets * V * sizeof(double));
    for (size_t i = 0; i < Ps; ++i) sino[i] = 1.0;
    for (unsigned s = 0; s < N_subsets; ++s) x_bp_views(g, s * n, n, DeltaAng, sino, sens + (size_t)s * V, threads);
    for (size_t i = 0; i < V; ++i) f[i] = 1.0;
    for (unsigned it = 0; it < iters; ++it)
        for (unsigned s = 0; s < N_subsets; ++s) {
            const double* ss = sens + (size_t)s * V;
            const float* gs = g_sino + (size_t)s * Ps;
            x_fp_views(g, s * n, n, DeltaAng, f, sino, threads);
            for (size_t i = 0; i < Ps; ++i) sino[i] = (sino[i] != 0.0) ? (double)gs[i] / sino[i] : 0.0;
            x_bp_views(g, s * n, n, DeltaAng, sino, Ht, threads);
            for (size_t i = 0; i < V; ++i) f[i] = (ss[i] != 0.0) ? f[i] * Ht[i] / ss[i] : 0.0;
        }
    free(sino);
    free(Ht);
    free(sens);
    return 0;
}

/* One MLEM update of the slab z in [z0, z1) of a large volume, in FP64, from
 * an FP32 image f and FP32 data: for every ray that crosses the slab, its full
 * line integral Hf through f, the ratio g/Hf (0 where Hf = 0) and the back
 * projection of the ratio and of 1 into the slab's voxels; then
 * out = f * Ht / sens over the slab (0 where sens = 0) -- the update of
 * hf_siddon_recon.hpp:437-476 for the slab, with the sensitivity of all
 * views.  Views are split over threads, each with its own slab partials,
 * summed in thread order.  Returns 0, or -1 on a bad slab or allocation
 * failure. */
typedef struct {
    const float* f;
    double sum;
    int64_t lo, hi;  /* slab voxel range [lo, hi) */
    int64_t* idx;
    double* len;
    int n;
} x_slab_ctx;
static void x_emit_slab(void* c, int64_t vox, double len)
{
    x_slab_ctx* t = (x_slab_ctx*)c;
    t->sum += len * (double)t->f[vox];
    if (vox >= t->lo && vox < t->hi) {
        t->idx[t->n] = vox - t->lo;
        t->len[t->n] = len;
        t->n++;
    }
}

int orc_x_slab_update(const orc_geom* g, unsigned int NumProj, float DeltaAng, const float* f,
                      const float* g_meas, unsigned int z0, unsigned int z1, double* out, int threads)
{
    if (z0 >= z1 || z1 > g->Zdim) return -1;
    const unsigned Nu = g->NumAxPixels, Nv = g->NumTAxPixels;
    const size_t Npix = (size_t)Nu * Nv;
    const size_t plane = (size_t)g->Xdim * g->Ydim;
    const size_t S = plane * (z1 - z0);
    const int64_t lo = (int64_t)(plane * z0), hi = (int64_t)(plane * z1);
    const double zlo = -(double)g->Zdim / 2.0 * g->ZVoxSize + z0 * (double)g->ZVoxSize;
    const double zhi = -(double)g->Zdim / 2.0 * g->ZVoxSize + z1 * (double)g->ZVoxSize;
    int nt = set_threads(threads);
    if ((unsigned)nt > NumProj) nt = (int)NumProj;
    if (nt < 1) nt = 1;
    double* part = (double*)calloc((size_t)nt * 2 * S, sizeof(double));
    if (!part) return -1;
    const int cap = (int)(g->Xdim + g->Ydim + g->Zdim + 4);
#pragma omp parallel num_threads(nt)
    {
        int t = 0;
#ifdef _OPENMP
        t = omp_get_thread_num();
#endif
        double* ht = part + (size_t)t * 2 * S;
        double* sn = ht + S;
        int64_t* idx = (int64_t*)malloc((size_t)cap * sizeof(int64_t));
        double* len = (double*)malloc((size_t)cap * sizeof(double));
        for (unsigned n = (unsigned)t; n < NumProj; n += (unsigned)nt) {
            const float ang = (float)n * DeltaAng;
            for (unsigned v = 0; v < Nv; ++v)
                for (unsigned u = 0; u < Nu; ++u) {
                    orc_x_ray r;
                    orc_x_ray_geom(g, ang, (int)u, (int)v, &r);
                    /* the ray's z over its length: skip rays that never reach the slab */
                    const double za = r.p1[2] < r.p2[2] ? r.p1[2] : r.p2[2];
                    const double zb = r.p1[2] < r.p2[2] ? r.p2[2] : r.p1[2];
                    if (zb < zlo || za > zhi) continue;
                    x_slab_ctx c = {f, 0.0, lo, hi, idx, len, 0};
                    x_traverse(g, &r, x_emit_slab, &c);
                    if (c.n == 0) continue;
                    const double gm = (double)g_meas[(size_t)n * Npix + u + (size_t)v * Nu];
                    const double ratio = (c.sum != 0.0) ? gm / c.sum : 0.0;
                    for (int k = 0; k < c.n; ++k) {
                        ht[c.idx[k]] += c.len[k] * ratio;
                        sn[c.idx[k]] += c.len[k];
                    }
                }
        }
        free(idx);
        free(len);
    }
    for (size_t i = 0; i < S; ++i) {
        double h = 0.0, s = 0.0;
        for (int t = 0; t < nt; ++t) {
            h += part[(size_t)t * 2 * S + i];
            s += part[(size_t)t * 2 * S + S + i];
        }
        out[i] = (s != 0.0) ? (double)f[lo + (int64_t)i] * h / s : 0.0;
    }
    free(part);
    return 0;
}

typedef struct {
    int64_t n;
} x_count_ctx;
static void x_emit_count(void* c, int64_t vox, double len)
{
    (void)vox;
    (void)len;
    ((x_count_ctx*)c)->n++;
}

int64_t orc_x_count_isects(const orc_geom* g, unsigned int NumProj, float DeltaAng, int threads)
{
    const unsigned Nu = g->NumAxPixels, Nv = g->NumTAxPixels;
    int nt = set_threads(threads);
    (void)nt;
    int64_t total = 0;
#pragma omp parallel for schedule(dynamic, 1) reduction(+ : total) num_threads(nt)
    for (long n = 0; n < (long)NumProj; ++n) {
        float ang = (float)n * DeltaAng;
        x_count_ctx c = {0};
        for (unsigned v = 0; v < Nv; ++v)
            for (unsigned u = 0; u < Nu; ++u) {
                orc_x_ray r;
                orc_x_ray_geom(g, ang, (int)u, (int)v, &r);
                x_traverse(g, &r, x_emit_count, &c);
            }
        total += c.n;
    }
    return total;
}

/* Intersection length of one ray with one voxel box (slab method, FP64). */
static double x_ray_box(const orc_geom* g, const orc_x_ray* r, int64_t voxel)
{
    const unsigned dims[3] = {g->Xdim, g->Ydim, g->Zdim};
    const double vox[3] = {g->XVoxSize, g->YVoxSize, g->ZVoxSize};
    int64_t ii[3] = {voxel % dims[0], (voxel / dims[0]) % dims[1], voxel / ((int64_t)dims[0] * dims[1])};
    double lo = 0.0, hi = 1.0;
    for (int k = 0; k < 3; ++k) {
        double P0 = -(double)dims[k] / 2.0 * vox[k];
        double b0 = P0 + ii[k] * vox[k], b1 = P0 + (ii[k] + 1) * vox[k];
        double d = r->p2[k] - r->p1[k];
        if (d == 0.0) {
            if (r->p1[k] < b0 || r->p1[k] >= b1) return 0.0;
            continue;
        }
        double a0 = (b0 - r->p1[k]) / d, a1 = (b1 - r->p1[k]) / d;
        double l = a0 < a1 ? a0 : a1, h = a0 < a1 ? a1 : a0;
        if (l > lo) lo = l;
        if (h < hi) hi = h;
    }
    return (hi > lo) ? (hi - lo) * r->d12 : 0.0;
}

/* One column of the FP64 system matrix: every (view, pixel, length) with
 * positive length for the given voxel.  Candidate pixels come from
 * projecting the voxel's corners (no misalignment) with a one-pixel margin;
 * each candidate's length is evaluated exactly. */
int orc_x_voxel_column(const orc_geom* g, unsigned int NumProj, float DeltaAng, int64_t voxel,
                       int32_t* view, int32_t* pixel, double* len, int cap)
{
    const unsigned dims[3] = {g->Xdim, g->Ydim, g->Zdim};
    const double vox[3] = {g->XVoxSize, g->YVoxSize, g->ZVoxSize};
    int64_t ii[3] = {voxel % dims[0], (voxel / dims[0]) % dims[1], voxel / ((int64_t)dims[0] * dims[1])};
    const unsigned Nu = g->NumAxPixels, Nv = g->NumTAxPixels;
    const double dM = (double)g->AxPixDimMm * g->M, dvM = (double)g->TAxPixDimMm * g->M;
    int n = 0;
    for (unsigned vw = 0; vw < NumProj; ++vw) {
        float ang = (float)vw * DeltaAng;
        double t = (double)ang / 180.0, c = h_cospi_d(t), s = h_sinpi_d(t);
        double umin = 1e300, umax = -1e300, vmin = 1e300, vmax = -1e300;
        for (int corner = 0; corner < 8; ++corner) {
            double P[3];
            for (int k = 0; k < 3; ++k) {
                double P0 = -(double)dims[k] / 2.0 * vox[k];
                P[k] = P0 + (ii[k] + ((corner >> k) & 1)) * vox[k];
            }
            double xv = P[0] * c - P[1] * s, yv = P[0] * s + P[1] * c;
            double X = (double)g->R * xv / (yv + g->Rf), Z = (double)g->R * P[2] / (yv + g->Rf);
            double uf = (X * g->Ry / g->R - g->Dx) / dM + (Nu - 1) / 2.0;
            double vf = (Z * g->Ry / g->R - g->Dz) / dvM + (Nv - 1) / 2.0;
            if (uf < umin) umin = uf;
            if (uf > umax) umax = uf;
            if (vf < vmin) vmin = vf;
            if (vf > vmax) vmax = vf;
        }
        long u0 = (long)floor(umin) - 1, u1 = (long)ceil(umax) + 1;
        long v0 = (long)floor(vmin) - 1, v1 = (long)ceil(vmax) + 1;
        if (u0 < 0) u0 = 0;
        if (v0 < 0) v0 = 0;
        if (u1 > (long)Nu - 1) u1 = (long)Nu - 1;
        if (v1 > (long)Nv - 1) v1 = (long)Nv - 1;
        for (long v = v0; v <= v1; ++v)
            for (long u = u0; u <= u1; ++u) {
                orc_x_ray r;
                orc_x_ray_geom(g, ang, (int)u, (int)v, &r);
                double L = x_ray_box(g, &r, voxel);
                if (L > 0.0) {
                    if (n < cap) {
                        view[n] = (int32_t)vw;
                        pixel[n] = (int32_t)(u + v * (long)Nu);
                        len[n] = L;
                    }
                    ++n;
                }
            }
    }
    return n <= cap ? n : -1;
}

/* ------------------------------------------------------------------------- */
/* Voxel-driven bilinear back projection                                     */
/* ------------------------------------------------------------------------- */

/* mode 0 ("reference"): backward_projection2 (CT_Recon/hf_cuda_kernels.cuh:
 *   240-284) as written: the voxel is rotated with the same matrix Siddon uses
 *   for rays, the detector coordinate is in millimetres and used directly as
 *   a texel coordinate, the bounds are inclusive, and the bilinear taps read
 *   the image as a flat array (a tap beyond the image end reads 0 here).
 * mode 1 ("geometric"): the rotation is the transpose (the angle sense of the
 *   Siddon projector), the coordinate is converted to pixel units
 *   (mm / (pitch*M) + (N-1)/2), taps are clamped inside the image and points
 *   outside [0, N-1] contribute nothing.
 * Both add value/Nproj to vol_accum. */
void orc_v_bp_view(const orc_geom* g, const float RM[9], float angle_deg, const float* img,
                   unsigned int Nproj, int mode, float* vol_accum)
{
    const unsigned X = g->Xdim, Y = g->Ydim, Z = g->Zdim;
    const unsigned Nu = g->NumAxPixels, Nv = g->NumTAxPixels;
    const size_t Npix = (size_t)Nu * Nv;
    const float R = g->R, Rf = g->Rf, Ry = g->Ry, M = g->M;
    float s, c;
    if (mode == 0) {
        const float PI_REF = (float)3.1415927; /* #define M_PI, hf_cuda_kernels.cuh:23 */
        s = sinf(angle_deg * PI_REF / 180.0f);
        c = cosf(angle_deg * PI_REF / 180.0f);
    } else {
        c = h_cospif(angle_deg / 180.0f);
        s = h_sinpif(angle_deg / 180.0f);
    }
    for (unsigned z = 0; z < Z; ++z)
        for (unsigned y = 0; y < Y; ++y)
            for (unsigned x = 0; x < X; ++x) {
                size_t n = x + (size_t)y * X + (size_t)z * X * Y;
                float xo = c_pixel_iterate((float)X, g->XVoxSize, 1.0f, (int)x);
                float yo = c_pixel_iterate((float)Y, g->YVoxSize, 1.0f, (int)y);
                float zo = c_pixel_iterate((float)Z, g->ZVoxSize, 1.0f, (int)z);
                float xa, ya;
                if (mode == 0) {
                    xa = xo * c + yo * s;
                    ya = -xo * s + yo * c;
                } else {
                    xa = xo * c - yo * s;
                    ya = xo * s + yo * c;
                }
                float u_id = h_fdividef(R * xa, ya + Rf);
                float v_id = h_fdividef(R * zo, ya + Rf);
                float detQ = (RM[0] - RM[3] * u_id / R) * (RM[8] - RM[5] * v_id / R) -
                             (RM[2] - RM[5] * u_id / R) * (RM[6] - RM[3] * v_id / R);
                float uu = h_fdividef(1, detQ) * ((RM[8] - RM[5] * v_id / R) * (Ry / R * u_id - g->Dx) -
                                                  (RM[2] - RM[5] * u_id / R) * (Ry / R * v_id - g->Dz));
                float vv = h_fdividef(1, detQ) * (-(RM[6] - RM[3] * v_id / R) * (Ry / R * u_id - g->Dx) +
                                                  (RM[0] - RM[3] * u_id / R) * (Ry / R * v_id - g->Dz));
                if (mode == 0) {
                    float u_pix = uu + (float)(Nu - 1) / 2.0f * g->AxPixDimMm * M;
                    float v_pix = vv + (float)(Nv - 1) / 2.0f * g->TAxPixDimMm * M;
                    uint32_t ui = h_f2u_rd(u_pix), vi = h_f2u_rd(v_pix);
                    float uw = (u_pix - (float)ui), vw = (v_pix - (float)vi);
                    if (u_pix >= 0.0 && u_pix <= (float)(Nu - 1) * g->AxPixDimMm * M && v_pix >= 0.0f &&
                        v_pix <= (float)(Nv - 1) * g->TAxPixDimMm * M) {
                        size_t i00 = ui + (size_t)vi * Nu, i10 = ui + 1 + (size_t)vi * Nu;
                        size_t i01 = ui + (size_t)(vi + 1) * Nu, i11 = ui + 1 + (size_t)(vi + 1) * Nu;
                        float t00 = i00 < Npix ? img[i00] : 0.0f, t10 = i10 < Npix ? img[i10] : 0.0f;
                        float t01 = i01 < Npix ? img[i01] : 0.0f, t11 = i11 < Npix ? img[i11] : 0.0f;
                        vol_accum[n] = vol_accum[n] +
                                       h_fdividef((t00 * (1 - uw) + t10 * uw) * (1 - vw) +
                                                      (t01 * (1 - uw) + t11 * uw) * vw,
                                                  (float)Nproj);
                    }
                } else {
                    float u_pix = uu / (g->AxPixDimMm * M) + (float)(Nu - 1) * 0.5f;
                    float v_pix = vv / (g->TAxPixDimMm * M) + (float)(Nv - 1) * 0.5f;
                    if (u_pix >= 0.0f && u_pix <= (float)(Nu - 1) && v_pix >= 0.0f &&
                        v_pix <= (float)(Nv - 1)) {
                        float uf = floorf(u_pix), vf = floorf(v_pix);
                        int ui = (int)uf, vi = (int)vf;
                        if (ui > (int)Nu - 2) ui = (int)Nu - 2;
                        if (vi > (int)Nv - 2) vi = (int)Nv - 2;
                        if (ui < 0) ui = 0;
                        if (vi < 0) vi = 0;
                        float uw = u_pix - (float)ui, vw = v_pix - (float)vi;
                        const float* r0 = img + (size_t)vi * Nu + ui;
                        const float* r1 = r0 + Nu;
                        float val = (r0[0] * (1.0f - uw) + r0[1] * uw) * (1.0f - vw) +
                                    (r1[0] * (1.0f - uw) + r1[1] * uw) * vw;
                        vol_accum[n] = vol_accum[n] + val / (float)Nproj;
                    }
                }
            }
}

/* ---- ray-marching forward projection ----------------------------------------
 * forward_projection (CT_Recon/hf_cuda_kernels.cuh:126-180): a pixel's ray
 * (pixel_iterate, :83-87, and the misalignment matrix, :140-141) is followed to
 * depth y0 of the view's frame, rotated into the volume (:158-159) and sampled;
 * each sample is weighted by distance_traveled (:78-81).  The reference has no
 * caller, so the depths and the sampling follow recon_march_fp_view:
 *   mode 0 (REFERENCE): depths at the texel centres of the normalised y
 *     coordinate, y0 = L*((k + 1/2)/Ydim - 1/2) (k < Ydim, L =
 *     (Ydim-1)*YVoxSize), coordinates normalised by L for every axis (:161-163),
 *     point sampling of a normalised, border-addressed texture (texel
 *     floor(c*size) inside [0,1), 0 outside; hf_texture_helper.hpp:113-121);
 *   mode 1 (GEOMETRIC): depths y0 = -r + (k + 1/2)*YVoxSize spanning the
 *     volume's bounding circle (r = half diagonal of the xy extent), trilinear
 *     interpolation at voxel centres, 0 outside.
 * All in FP64, except the REFERENCE angle's sine and cosine (FP32, as the GPU
 * path computes them). */
void orc_m_fp_view(const orc_geom* g, const float RM[9], float angle_deg, int mode, const float* vol,
                   double* img)
{
    const int X = (int)g->Xdim, Y = (int)g->Ydim, Z = (int)g->Zdim;
    const int Nu = (int)g->NumAxPixels, Nv = (int)g->NumTAxPixels;
    const double vx = g->XVoxSize, vy = g->YVoxSize, vz = g->ZVoxSize;
    const double P0x = -X / 2.0 * vx, P0y = -Y / 2.0 * vy, P0z = -Z / 2.0 * vz;
    const double R = g->R, Rf = g->Rf, Ry = g->Ry, M = g->M;
    const double du = g->AxPixDimMm, dv = g->TAxPixDimMm;
    const double L = (Y - 1.0) * vy;
    const size_t plane = (size_t)X * Y;
    double c, s;
    int nplanes;
    double y_first;
    if (mode == 0) {
        const float a = angle_deg * 3.1415927f / 180.0f; /* #define M_PI, hf_cuda_kernels.cuh:23 */
        c = (double)cosf(a);
        s = (double)sinf(a);
        nplanes = Y;
        y_first = L * (0.5 / Y - 0.5);
    } else {
        const double pi = 3.14159265358979323846;
        c = cos(pi * (double)angle_deg / 180.0);
        s = sin(pi * (double)angle_deg / 180.0);
        const double hx = 0.5 * X * vx, hy = 0.5 * Y * vy, r = sqrt(hx * hx + hy * hy);
        nplanes = (int)ceil(2.0 * r / vy);
        y_first = -r + 0.5 * vy;
    }
    for (int v = 0; v < Nv; ++v)
        for (int u = 0; u < Nu; ++u) {
            const double pu = -(Nu - 1.0) / 2.0 * du * M + u * du * M;
            const double pv = -(Nv - 1.0) / 2.0 * dv * M + v * dv * M;
            const double den = Ry + RM[3] * pu + RM[5] * pv;
            const double u_id = R / den * (RM[0] * pu + RM[2] * pv + g->Dx);
            const double v_id = R / den * (RM[6] * pu + RM[8] * pv + g->Dz);
            const double w = sqrt(v_id * v_id + u_id * u_id + R * R) / R * vy;
            double acc = 0.0;
            const double y_step = (mode == 0) ? L / Y : vy;
            for (int k = 0; k < nplanes; ++k) {
                const double y0 = y_first + k * y_step;
                const double x0 = (y0 + Rf) * u_id / R, z0 = (y0 + Rf) * v_id / R;
                const double xa = x0 * c + y0 * s, ya = -x0 * s + y0 * c;
                if (mode == 0) {
                    const double xn = xa / L + 0.5, yn = ya / L + 0.5, zn = z0 / L + 0.5;
                    if (!(xn >= 0.0 && xn < 1.0 && yn >= 0.0 && yn < 1.0 && zn >= 0.0 && zn < 1.0)) continue;
                    int ix = (int)floor(xn * X), iy = (int)floor(yn * Y), iz = (int)floor(zn * Z);
                    if (ix > X - 1) ix = X - 1;
                    if (iy > Y - 1) iy = Y - 1;
                    if (iz > Z - 1) iz = Z - 1;
                    acc += vol[(size_t)ix + (size_t)iy * X + (size_t)iz * plane] * w;
                } else {
                    const double fx = (xa - P0x) / vx - 0.5, fy = (ya - P0y) / vy - 0.5, fz = (z0 - P0z) / vz - 0.5;
                    if (!(fx > -1.0 && fx < X && fy > -1.0 && fy < Y && fz > -1.0 && fz < Z)) continue;
                    const double gx = floor(fx), gy = floor(fy), gz = floor(fz);
                    const int ix = (int)gx, iy = (int)gy, iz = (int)gz;
                    const double ax = fx - gx, ay = fy - gy, az = fz - gz;
                    double sample = 0.0;
                    for (int t = 0; t < 8; ++t) {
                        const int jx = ix + (t & 1), jy = iy + ((t >> 1) & 1), jz = iz + (t >> 2);
                        if (jx < 0 || jx >= X || jy < 0 || jy >= Y || jz < 0 || jz >= Z) continue;
                        const double wt = ((t & 1) ? ax : 1.0 - ax) * (((t >> 1) & 1) ? ay : 1.0 - ay) *
                                          ((t >> 2) ? az : 1.0 - az);
                        sample += wt * vol[(size_t)jx + (size_t)jy * X + (size_t)jz * plane];
                    }
                    acc += sample * w;
                }
            }
            img[(size_t)u + (size_t)v * Nu] = acc;
        }
}
