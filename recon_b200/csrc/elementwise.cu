// elementwise.cu -- the MLEM elementwise steps of the reference
// (set_ones, divide1, multiply1, siddon_add_bp; CT_Recon/hf_cuda_kernels.cuh:25-35,
// 370-421, siddon_kernelsMLEM.cuh:46-74) as 128-bit vectorised grid-stride
// kernels over any length (the reference's 4-wide grids need multiples of 4
// and have no bounds checks).
#include "internal.h"

namespace rb {

enum { OP_ADD = 0, OP_MUL = 1, OP_DIV1 = 2 };

template <int OP>
__device__ __forceinline__ float apply(float a, float b)
{
    if (OP == OP_ADD) return __fadd_rn(a, b);
    if (OP == OP_MUL) return __fmul_rn(a, b);
    return (b != 0.0f) ? __fdividef(a, b) : 0.0f;  // divide1
}

template <int OP>
__global__ void binary_kernel(float* __restrict__ a, const float* __restrict__ b, size_t n)
{
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    const size_t n4 = n / 4;
    const bool aligned = ((reinterpret_cast<uintptr_t>(a) | reinterpret_cast<uintptr_t>(b)) & 15) == 0;
    size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (aligned) {
        float4* a4 = reinterpret_cast<float4*>(a);
        const float4* b4 = reinterpret_cast<const float4*>(b);
        for (size_t q = i; q < n4; q += stride) {
            float4 x = a4[q];
            const float4 y = __ldg(b4 + q);
            x.x = apply<OP>(x.x, y.x);
            x.y = apply<OP>(x.y, y.y);
            x.z = apply<OP>(x.z, y.z);
            x.w = apply<OP>(x.w, y.w);
            a4[q] = x;
        }
        for (size_t q = n4 * 4 + i; q < n; q += stride) a[q] = apply<OP>(a[q], b[q]);
    } else {
        for (size_t q = i; q < n; q += stride) a[q] = apply<OP>(a[q], b[q]);
    }
}

__global__ void fill_kernel(float* __restrict__ a, float v, size_t n)
{
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n; q += stride) a[q] = v;
}

// f = f * Ht; f = divide1(f, sens) (hf_siddon_recon.hpp:473-474), two roundings
// in that order.  fast_div: the reference's __fdividef; else IEEE division.
template <bool FAST>
__device__ __forceinline__ float update_one(float f, float ht, float s)
{
    const float p = __fmul_rn(f, ht);
    return (s != 0.0f) ? (FAST ? __fdividef(p, s) : __fdiv_rn(p, s)) : 0.0f;
}

// 128-bit loads and stores where all three arrays are 16-byte aligned.
template <bool FAST>
__global__ void update_kernel(float* __restrict__ f, const float* __restrict__ ht, const float* __restrict__ sens,
                              size_t n)
{
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    const bool aligned =
        ((reinterpret_cast<uintptr_t>(f) | reinterpret_cast<uintptr_t>(ht) | reinterpret_cast<uintptr_t>(sens)) & 15) == 0;
    size_t q0 = 0;
    if (aligned) {
        const size_t n4 = n / 4;
        float4* f4 = reinterpret_cast<float4*>(f);
        const float4* h4 = reinterpret_cast<const float4*>(ht);
        const float4* s4 = reinterpret_cast<const float4*>(sens);
        for (size_t q = i; q < n4; q += stride) {
            float4 x = f4[q];
            const float4 h = __ldg(h4 + q), sv = __ldg(s4 + q);
            x.x = update_one<FAST>(x.x, h.x, sv.x);
            x.y = update_one<FAST>(x.y, h.y, sv.y);
            x.z = update_one<FAST>(x.z, h.z, sv.z);
            x.w = update_one<FAST>(x.w, h.w, sv.w);
            f4[q] = x;
        }
        q0 = n4 * 4;
    }
    for (size_t q = q0 + i; q < n; q += stride) f[q] = update_one<FAST>(f[q], ht[q], sens[q]);
}

static unsigned blocks_for(size_t n)
{
    size_t b = (n + 1023) / 1024;
    if (b < 1) b = 1;
    if (b > 148 * 8) b = 148 * 8;
    return (unsigned)b;
}

recon_status_t launch_elementwise(int op, float* a, const float* b, size_t n, cudaStream_t s)
{
    if (n == 0) return RECON_OK;
    if (op == OP_ADD) binary_kernel<OP_ADD><<<blocks_for(n), 256, 0, s>>>(a, b, n);
    else if (op == OP_MUL) binary_kernel<OP_MUL><<<blocks_for(n), 256, 0, s>>>(a, b, n);
    else binary_kernel<OP_DIV1><<<blocks_for(n), 256, 0, s>>>(a, b, n);
    RB_CUDA(cudaGetLastError());
    return RECON_OK;
}

recon_status_t launch_fill(float* a, float v, size_t n, cudaStream_t s)
{
    if (n == 0) return RECON_OK;
    fill_kernel<<<blocks_for(n), 256, 0, s>>>(a, v, n);
    RB_CUDA(cudaGetLastError());
    return RECON_OK;
}

recon_status_t launch_update(float* f, const float* ht, const float* sens, size_t n, bool fast_div, cudaStream_t s)
{
    if (n == 0) return RECON_OK;
    if (fast_div) update_kernel<true><<<blocks_for(n), 256, 0, s>>>(f, ht, sens, n);
    else update_kernel<false><<<blocks_for(n), 256, 0, s>>>(f, ht, sens, n);
    RB_CUDA(cudaGetLastError());
    return RECON_OK;
}

}  // namespace rb
