/* Forced-include prelude for building the reference's CUDA sources with
 * nvcc 12.9 for sm_100a (checker build, output in oracle/_ref/).
 *
 * CT_Recon/hf_texture_helper.hpp declares legacy texture references
 * (texture<float,2,...>), which CUDA 12 removed, and includes the Ruijters
 * cubic B-spline library, which is not part of the reference.  Defining that
 * header's include guard skips it; the three kernels that sample those
 * textures (rotate_volume_3D, forward_projection, backward_projection in
 * CT_Recon/hf_cuda_kernels.cuh) then compile against the inert stand-ins
 * below and return 0 -- they are never launched by the checker (their
 * parity cannot be pinned without the absent library).  Nothing on the
 * Siddon path touches them. */
#pragma once
#include <cuda_runtime.h>
#define TEXTURE_HELPER_HF_HPP_ 1
struct recon_ref_texture_standin { int unused; };
__device__ recon_ref_texture_standin tex2_float;
__device__ recon_ref_texture_standin tex3_float;
__device__ inline float tex3D(const recon_ref_texture_standin&, float, float, float) { return 0.0f; }
__device__ inline float cubicTex2D(const recon_ref_texture_standin&, float, float) { return 0.0f; }
