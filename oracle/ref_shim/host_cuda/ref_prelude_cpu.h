/* Forced-include prelude for compiling the reference's kernel sources
 * (CT_Recon/siddon_kernelsMLEM.cuh, siddon_device_kernelsMLEM.cuh,
 * hf_cuda_kernels.cuh) with the host C++ compiler.  Checker shim: it makes the
 * reference's own kernel bodies callable as host functions so that they can
 * be (a) compared bit for bit with the FP32 restatement in
 * oracle/siddon_oracle.c and (b) timed as the reference's CPU path.
 *
 * __global__/__device__ become ordinary functions; the launch indices become
 * thread-local variables set by the launcher in ref_cpu_harness.cpp.  The GPU
 * intrinsics are replaced by IEEE host arithmetic, identical to the
 * replacements the oracle uses (see oracle/siddon_oracle.c for why each is
 * chosen):  __fdividef -> a/b; __fdiv_rz -> division rounded toward zero;
 * cospif/sinpif -> half-integer-exact double routine rounded to float;
 * __float2int_rz / __float2uint_rd -> truncation / floor with NaN -> 0 and
 * saturation. */
#pragma once
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>

#define __global__
#define __device__
#define __host__
#define __forceinline__ inline

struct uint3 { unsigned int x, y, z; };
struct int3 { int x, y, z; };
struct float2 { float x, y; };
struct float3 { float x, y, z; };
struct dim3 {
    unsigned int x, y, z;
    dim3(unsigned int a = 1, unsigned int b = 1, unsigned int c = 1) : x(a), y(b), z(c) {}
};
extern thread_local uint3 threadIdx;
extern thread_local uint3 blockIdx;
extern thread_local dim3 blockDim;
extern thread_local dim3 gridDim;

typedef int cudaError_t;
static const int cudaSuccess = 0;
static inline const char* cudaGetErrorString(cudaError_t) { return "host build"; }

static inline float __int_as_float(int i) { float f; std::memcpy(&f, &i, 4); return f; }
static inline float __fdividef(float a, float b) { return a / b; }
static inline float __fdiv_rz(float a, float b)
{
    double q = (double)a / (double)b;
    if (std::isnan(q) || std::isinf(q)) return (float)q;
    float r = (float)q;
    if (std::isinf(r)) return std::copysign(FLT_MAX, r);
    if (std::fabs((double)r) > std::fabs(q)) r = std::nextafter(r, 0.0f);
    return r;
}
static inline int __float2int_rz(float x)
{
    if (x != x) return 0;
    if (x >= 2147483648.0f) return INT32_MAX;
    if (x <= -2147483648.0f) return INT32_MIN;
    return (int)x;
}
static inline unsigned int __float2uint_rd(float x)
{
    if (x != x) return 0u;
    float f = std::floor(x);
    if (f <= 0.0f) return 0u;
    if (f >= 4294967296.0f) return 0xFFFFFFFFu;
    return (unsigned int)f;
}
static inline double recon_ref_sinpi_d(double x)
{
    if (!std::isfinite(x)) return NAN;
    double n = std::rint(2.0 * x), f = x - 0.5 * n;
    double s = std::sin(3.14159265358979323846 * f), c = std::cos(3.14159265358979323846 * f);
    long q = (long)std::fmod(n, 4.0);
    if (q < 0) q += 4;
    return ((q == 0) ? s : (q == 1) ? c : (q == 2) ? -s : -c) + 0.0;
}
static inline double recon_ref_cospi_d(double x)
{
    if (!std::isfinite(x)) return NAN;
    double n = std::rint(2.0 * x), f = x - 0.5 * n;
    double s = std::sin(3.14159265358979323846 * f), c = std::cos(3.14159265358979323846 * f);
    long q = (long)std::fmod(n, 4.0);
    if (q < 0) q += 4;
    return ((q == 0) ? c : (q == 1) ? -s : (q == 2) ? -c : s) + 0.0;
}
static inline float sinpif(float x) { return (float)recon_ref_sinpi_d((double)x); }
static inline float cospif(float x) { return (float)recon_ref_cospi_d((double)x); }

/* float atomicAdd: the launcher runs the scatter kernel with one thread per
 * element in element order, so a plain add reproduces a deterministic order;
 * under OpenMP it is an atomic update. */
static inline float atomicAdd(float* p, float v)
{
    float old;
#pragma omp atomic capture
    { old = *p; *p += v; }
    return old;
}

/* CT_Recon/hf_texture_helper.hpp needs the Ruijters library and legacy
 * texture references; skip it (include guard) and give the three texture
 * kernels inert stand-ins.  They are never launched. */
#define TEXTURE_HELPER_HF_HPP_ 1
struct recon_ref_texture_standin { int unused; };
static recon_ref_texture_standin tex2_float, tex3_float;
static inline float tex3D(const recon_ref_texture_standin&, float, float, float) { return 0.0f; }
static inline float cubicTex2D(const recon_ref_texture_standin&, float, float) { return 0.0f; }
