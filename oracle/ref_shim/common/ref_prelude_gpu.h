/* Forced-include prelude for building the reference's CUDA sources with
 * nvcc 12.9 for sm_100a (checker build, output in oracle/_ref/).
 *
 * CT_Recon/hf_texture_helper.hpp declares legacy texture references
 * (texture<float,2,...>), which CUDA 12 removed, and includes the Ruijters
 * cubic B-spline library, which is not part of the reference.  Defining that
 * header's include guard skips it; the three kernels that sample those
 * textures (rotate_volume_3D, forward_projection, backward_projection in
 * CT_Recon/hf_cuda_kernels.cuh) then compile against the stand-ins below.
 * Nothing on the Siddon path touches them.
 *
 * tex3D samples a volume the checker binds (recon_ref_tex3_data / _dims, set
 * with cudaMemcpyToSymbol), so that the reference's own forward_projection can
 * run: its coordinates are normalised over each axis (hf_cuda_kernels.cuh:
 * 161-163) and are taken as normalised texture coordinates with point
 * filtering and border addressing (hf_texture_helper.hpp:107-122): texel
 * floor(c * size), clamped to the last texel, for c in [0, 1) on every axis,
 * 0 outside.  texture_helper3D itself sets normalized = false (:112), under
 * which every coordinate in [0, 1) would read texel 0.  cubicTex2D (the
 * absent library) stays inert. */
#pragma once
#include <cuda_runtime.h>
#define TEXTURE_HELPER_HF_HPP_ 1
struct recon_ref_texture_standin { int unused; };
__device__ recon_ref_texture_standin tex2_float;
__device__ recon_ref_texture_standin tex3_float;
__device__ const float* recon_ref_tex3_data;
__device__ int recon_ref_tex3_dims[3];
__device__ inline float tex3D(const recon_ref_texture_standin&, float x, float y, float z)
{
    const float* d = recon_ref_tex3_data;
    if (!d) return 0.0f;
    if (!(x >= 0.0f && x < 1.0f && y >= 0.0f && y < 1.0f && z >= 0.0f && z < 1.0f)) return 0.0f;
    const int X = recon_ref_tex3_dims[0], Y = recon_ref_tex3_dims[1], Z = recon_ref_tex3_dims[2];
    int ix = (int)(x * (float)X), iy = (int)(y * (float)Y), iz = (int)(z * (float)Z);
    ix = ix < X - 1 ? ix : X - 1;
    iy = iy < Y - 1 ? iy : Y - 1;
    iz = iz < Z - 1 ? iz : Z - 1;
    return d[(size_t)ix + (size_t)iy * X + (size_t)iz * X * Y];
}
__device__ inline float cubicTex2D(const recon_ref_texture_standin&, float, float) { return 0.0f; }
