/*
 * ref_gpu_harness.cu -- the reference's own CUDA implementation, built for
 * sm_100a, driven through its own classes.
 *
 * CHECKER INFRASTRUCTURE.  Built by oracle/build_ref.py from the reference
 * sources where they lie (no copies) with oracle/ref_shim/common on the
 * include path and ref_prelude_gpu.h forced in, into
 * oracle/_ref/libref_gpu.so.  The tests use it on the GPU as the parity
 * anchor: per-ray setup arrays and per-step (voxel, length) records must match
 * the CUDA product bit for bit in compat mode, and FP / BP / MLEM outputs
 * within tolerance.
 *
 * Everything here calls the reference's siddon_commons / forward / backward /
 * siddon_recon classes (CT_Recon/hf_siddon_class.hpp, hf_siddon_recon.hpp) or
 * launches its kernels with its own launch shapes (hf_siddon_recon.hpp:
 * 366-386).  Inputs and outputs are host arrays.
 */
#include "hf_siddon_recon.hpp"

#include <cmath>
#include <cstdint>
#include <vector>

#include "siddon_oracle.h"

namespace {

struct RefGeom {
    CalibrationParam cp;
    Detector det;
    VoxVolParam vox;
    dim3 bimg, timg, bobj, tobj, batom, tatom;
    explicit RefGeom(const orc_geom* g)
    {
        cp.R = g->R; cp.Rf = g->Rf; cp.Ry = g->Ry; cp.Dx = g->Dx; cp.Dz = g->Dz;
        cp.xangle = g->xangle; cp.yangle = g->yangle; cp.zangle = g->zangle; cp.M = g->M;
        det.NumTAxPixels = g->NumTAxPixels; det.NumAxPixels = g->NumAxPixels;
        det.TAxPixDimMm = g->TAxPixDimMm; det.AxPixDimMm = g->AxPixDimMm;
        vox.Xdim = g->Xdim; vox.Ydim = g->Ydim; vox.Zdim = g->Zdim;
        vox.XVoxSize = g->XVoxSize; vox.YVoxSize = g->YVoxSize; vox.ZVoxSize = g->ZVoxSize;
        /* m_calc_kernel_threads (hf_siddon_recon.hpp:366-386) */
        timg = dim3(4, 4);
        bimg = dim3(det.NumAxPixels / 4, det.NumTAxPixels / 4);
        tobj = dim3(4, 4, 4);
        bobj = dim3(vox.Xdim / 4, vox.Ydim / 4, vox.Zdim / 4);
        cudaDeviceProp prop;
        cudaGetDeviceProperties(&prop, 0);
        tatom = dim3(256);
        batom = dim3(2 * prop.multiProcessorCount);
    }
};

}  // namespace

extern "C" {

/* siddon_commons::a_calc_initial_limits and its per-ray arrays. */
unsigned ref_gpu_setup(const orc_geom* g, float angle, float* alpha_min, float* alpha_max, float* d12,
                       unsigned* mask, float* alpha_i, float* alpha_f, float* delta_alpha, float* p1,
                       float* p2, unsigned* delta_index)
{
    RefGeom G(g);
    siddon_commons sc;
    sc.a1_initiate(G.cp, G.det, G.vox);
    sc.a2_allocate();
    unsigned loopN = sc.a_calc_initial_limits(angle, G.bimg, G.timg);
    const size_t n = sc.N_image_pixels;
    CUDA_SAFE_CALL(cudaMemcpy(alpha_min, sc.d_alpha_min, n * 4, cudaMemcpyDeviceToHost));
    CUDA_SAFE_CALL(cudaMemcpy(alpha_max, sc.d_alpha_max, n * 4, cudaMemcpyDeviceToHost));
    CUDA_SAFE_CALL(cudaMemcpy(d12, sc.d_d12, n * 4, cudaMemcpyDeviceToHost));
    CUDA_SAFE_CALL(cudaMemcpy(mask, sc.d_mask, n * 4, cudaMemcpyDeviceToHost));
    CUDA_SAFE_CALL(cudaMemcpy(alpha_i, sc.d_alpha_i, n * 12, cudaMemcpyDeviceToHost));
    CUDA_SAFE_CALL(cudaMemcpy(alpha_f, sc.d_alpha_f, n * 12, cudaMemcpyDeviceToHost));
    CUDA_SAFE_CALL(cudaMemcpy(delta_alpha, sc.d_delta_alpha, n * 12, cudaMemcpyDeviceToHost));
    CUDA_SAFE_CALL(cudaMemcpy(p1, sc.p1, n * 12, cudaMemcpyDeviceToHost));
    CUDA_SAFE_CALL(cudaMemcpy(p2, sc.p2, n * 12, cudaMemcpyDeviceToHost));
    CUDA_SAFE_CALL(cudaMemcpy(delta_index, sc.d_delta_index, n * 4, cudaMemcpyDeviceToHost));
    sc.a3_deallocate();
    CUDA_SAFE_CALL(cudaFree(sc.p1));
    CUDA_SAFE_CALL(cudaFree(sc.p2));
    return loopN;
}

/* forward::a2_fp_per_angle for one view; returns loopN. */
unsigned ref_gpu_fp_view(const orc_geom* g, float angle, const float* vol, float* img)
{
    RefGeom G(g);
    siddon_commons sc;
    sc.a1_initiate(G.cp, G.det, G.vox);
    sc.a2_allocate();
    float* d_vol;
    CUDA_SAFE_CALL(cudaMalloc((void**)&d_vol, (size_t)sc.N_object_voxels * 4));
    CUDA_SAFE_CALL(cudaMemcpy(d_vol, vol, (size_t)sc.N_object_voxels * 4, cudaMemcpyHostToDevice));
    unsigned loopN = sc.a_calc_initial_limits(angle, G.bimg, G.timg);
    {
        forward fw;
        fw.a1_Finitiate(sc.N_image_pixels);
        fw.a2_fp_per_angle(d_vol, sc, G.bimg, G.timg);
        CUDA_SAFE_CALL(cudaMemcpy(img, fw.a_Fdevicepointer(), (size_t)sc.N_image_pixels * 4,
                                  cudaMemcpyDeviceToHost));
    }
    CUDA_SAFE_CALL(cudaFree(d_vol));
    sc.a3_deallocate();
    CUDA_SAFE_CALL(cudaFree(sc.p1));
    CUDA_SAFE_CALL(cudaFree(sc.p2));
    return loopN;
}

/* backward::a2_bp_per_angle for one view (float atomics: nondeterministic
 * summation order). */
unsigned ref_gpu_bp_view(const orc_geom* g, float angle, const float* img, float* vol)
{
    RefGeom G(g);
    siddon_commons sc;
    sc.a1_initiate(G.cp, G.det, G.vox);
    sc.a2_allocate();
    float* d_img;
    CUDA_SAFE_CALL(cudaMalloc((void**)&d_img, (size_t)sc.N_image_pixels * 4));
    CUDA_SAFE_CALL(cudaMemcpy(d_img, img, (size_t)sc.N_image_pixels * 4, cudaMemcpyHostToDevice));
    unsigned loopN = sc.a_calc_initial_limits(angle, G.bimg, G.timg);
    {
        backward bw;
        bw.a1_Binitiate(sc.N_object_voxels, sc.N_image_pixels);
        bw.a2_bp_per_angle(d_img, sc, G.bimg, G.timg, G.bobj, G.tobj, G.batom, G.tatom);
        CUDA_SAFE_CALL(cudaMemcpy(vol, bw.a_bpdevicepointer(), (size_t)sc.N_object_voxels * 4,
                                  cudaMemcpyDeviceToHost));
    }
    CUDA_SAFE_CALL(cudaFree(d_img));
    sc.a3_deallocate();
    CUDA_SAFE_CALL(cudaFree(sc.p1));
    CUDA_SAFE_CALL(cudaFree(sc.p2));
    return loopN;
}

/* Per-step records of the back projection step kernels with an all-ones
 * image (value = ray length; pad index V -> -1), for a list of rays:
 * out[ray][step], loopN steps then the end segment.  Returns loopN; when
 * loopN + 1 > cap_steps nothing is written and 0 is returned. */
unsigned ref_gpu_trace(const orc_geom* g, float angle, int nrays, const int* rays, int cap_steps,
                       int* idx_out, float* val_out)
{
    RefGeom G(g);
    siddon_commons sc;
    sc.a1_initiate(G.cp, G.det, G.vox);
    sc.a2_allocate();
    const int Npix = sc.N_image_pixels, V = sc.N_object_voxels;
    unsigned loopN = sc.a_calc_initial_limits(angle, G.bimg, G.timg);
    if ((int)loopN + 1 > cap_steps) {
        sc.a3_deallocate();
        CUDA_SAFE_CALL(cudaFree(sc.p1));
        CUDA_SAFE_CALL(cudaFree(sc.p2));
        return 0;
    }
    float *d_ones, *d_val;
    int* d_idx;
    CUDA_SAFE_CALL(cudaMalloc((void**)&d_ones, (size_t)Npix * 4));
    CUDA_SAFE_CALL(cudaMalloc((void**)&d_val, (size_t)Npix * 4));
    CUDA_SAFE_CALL(cudaMalloc((void**)&d_idx, (size_t)Npix * 4));
    set_ones<<<G.bimg, G.timg>>>(d_ones);
    std::vector<int> hidx(Npix);
    std::vector<float> hval(Npix);
    auto grab = [&](int k) {
        CUDA_SAFE_CALL(cudaMemcpy(hidx.data(), d_idx, (size_t)Npix * 4, cudaMemcpyDeviceToHost));
        CUDA_SAFE_CALL(cudaMemcpy(hval.data(), d_val, (size_t)Npix * 4, cudaMemcpyDeviceToHost));
        for (int r = 0; r < nrays; ++r) {
            int n = rays[r];
            idx_out[(size_t)r * cap_steps + k] = hidx[n] >= V ? -1 : hidx[n];
            val_out[(size_t)r * cap_steps + k] = hval[n];
        }
    };
    siddon_begin<<<G.bimg, G.timg>>>(sc.d_alpha_min, sc.d_alpha, sc.d_alpha_i, sc.d_mask, sc.d_next_alpha);
    for (unsigned i = 0; i < loopN; ++i) {
        siddon_sort_alpha<<<G.bimg, G.timg>>>(sc.d_alpha, sc.d_alpha_i, sc.d_alpha_f, sc.d_delta_alpha,
                                              sc.d_current_alpha, sc.d_next_alpha, sc.d_alpha_max, sc.d_alpha_min);
        siddon_bp_calc_ray_path<<<G.bimg, G.timg>>>(sc.system, sc.p1, sc.p2, sc.d_index, d_idx,
                                                    sc.d_current_alpha, sc.d_next_alpha, sc.d_d12, sc.d_mask,
                                                    d_ones, d_val);
        grab((int)i);
    }
    siddon_bp_end<<<G.bimg, G.timg>>>(sc.d_alpha_max, sc.d_d12, sc.d_mask, sc.system, sc.p1, sc.p2, sc.d_index,
                                      d_idx, sc.d_current_alpha, d_ones, d_val);
    grab((int)loopN);
    CUDA_SAFE_CALL(cudaFree(d_ones));
    CUDA_SAFE_CALL(cudaFree(d_val));
    CUDA_SAFE_CALL(cudaFree(d_idx));
    sc.a3_deallocate();
    CUDA_SAFE_CALL(cudaFree(sc.p1));
    CUDA_SAFE_CALL(cudaFree(sc.p2));
    return loopN;
}

/* The reference's own end-to-end MLEM from a configuration file
 * (siddon_recon::a0_RECON_MLEM, hf_siddon_recon.hpp:91-108): reads the
 * per-view projection files, writes <ReconFileNameRoot>_<it><suffix> per
 * iteration and the .info file.  Returns the elapsed device+host time in ms
 * measured with CUDA events around the call. */
float ref_gpu_mlem_cfg(const char* folder, const char* cfg)
{
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    cudaEventRecord(a, 0);
    {
        siddon_recon recon;
        recon.a0_RECON_MLEM(std::string(folder), std::string(cfg));
    }
    cudaEventRecord(b, 0);
    cudaEventSynchronize(b);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    return ms;
}

/* siddon_recon::a1_FORWARD_PROJECTION (hf_siddon_recon.hpp:146-163). */
void ref_gpu_forward_projection_cfg(const char* folder, const char* cfg)
{
    siddon_recon recon;
    recon.a1_FORWARD_PROJECTION(std::string(folder), std::string(cfg));
}

/* siddon_recon::a1_BACKWARD_PROJECTION (hf_siddon_recon.hpp:165-182).  Its total
 * image accumulates into md_f, which m_recon_initiate allocates without
 * clearing (hf_siddon_recon.hpp:425, 568); the per-view images
 * (write_per_angle) start from cleared memory (hf_siddon_class.hpp:318). */
void ref_gpu_backward_projection_cfg(const char* folder, const char* cfg, int write_per_angle)
{
    siddon_recon recon;
    recon.a1_BACKWARD_PROJECTION(std::string(folder), std::string(cfg), write_per_angle != 0);
}

/* backward_projection2 (hf_cuda_kernels.cuh:240-284) for one view, added
 * into vol.  The device image is padded by two rows and two pixels so the
 * kernel's inclusive upper-edge taps stay inside the allocation (they read
 * zeros there). */
void ref_gpu_voxel_bp2_view(const orc_geom* g, float angle, const float* img, unsigned Nproj, float* vol)
{
    RefGeom G(g);
    const size_t Npix = (size_t)g->NumAxPixels * g->NumTAxPixels;
    const size_t pad = 2 * (size_t)g->NumAxPixels + 2;
    const size_t V = (size_t)g->Xdim * g->Ydim * g->Zdim;
    float *d_img, *d_vol, *d_RM;
    CUDA_SAFE_CALL(cudaMalloc((void**)&d_img, (Npix + pad) * 4));
    CUDA_SAFE_CALL(cudaMemset(d_img, 0, (Npix + pad) * 4));
    CUDA_SAFE_CALL(cudaMemcpy(d_img, img, Npix * 4, cudaMemcpyHostToDevice));
    CUDA_SAFE_CALL(cudaMalloc((void**)&d_vol, V * 4));
    CUDA_SAFE_CALL(cudaMemcpy(d_vol, vol, V * 4, cudaMemcpyHostToDevice));
    CUDA_SAFE_CALL(cudaMalloc((void**)&d_RM, 9 * 4));
    rotation_matrix3D(d_RM, G.cp.xangle, G.cp.yangle, G.cp.zangle); /* hf_cuda_functions.cuh:66-88 */
    ObjectParam op;
    op.ObjX = op.ObjY = op.ObjZ = op.ObjXangle = op.ObjYangle = op.ObjZangle = 0.f;
    backward_projection2<<<G.bobj, G.tobj>>>(d_vol, d_img, G.cp, G.det, op, G.vox, d_RM, angle, Nproj);
    CUDA_SAFE_CALL(cudaGetLastError());
    CUDA_SAFE_CALL(cudaMemcpy(vol, d_vol, V * 4, cudaMemcpyDeviceToHost));
    CUDA_SAFE_CALL(cudaFree(d_img));
    CUDA_SAFE_CALL(cudaFree(d_vol));
    CUDA_SAFE_CALL(cudaFree(d_RM));
}

/* forward_projection (hf_cuda_kernels.cuh:126-180), the reference's texture
 * ray-marching projector, for one view: the reference gives no loop over
 * depths, so it is launched once per depth y0 = L((k + 1/2)/Ydim - 1/2),
 * k < Ydim, L = (Ydim - 1) YVoxSize (the normalised texel centres along y),
 * adding into a cleared image, with the volume bound to the tex3D stand-in of
 * ref_prelude_gpu.h.  Launch shape as its other image kernels (4 x 4 threads,
 * hf_siddon_recon.hpp:368-371). */
void ref_gpu_march_fp_view(const orc_geom* g, float angle, const float* vol, float* img)
{
    RefGeom G(g);
    const size_t V = (size_t)g->Xdim * g->Ydim * g->Zdim;
    const size_t N = (size_t)g->NumAxPixels * g->NumTAxPixels;
    float *d_vol, *d_img, *d_RM;
    CUDA_SAFE_CALL(cudaMalloc((void**)&d_vol, V * 4));
    CUDA_SAFE_CALL(cudaMemcpy(d_vol, vol, V * 4, cudaMemcpyHostToDevice));
    CUDA_SAFE_CALL(cudaMalloc((void**)&d_img, N * 4));
    CUDA_SAFE_CALL(cudaMemset(d_img, 0, N * 4));
    CUDA_SAFE_CALL(cudaMalloc((void**)&d_RM, 9 * 4));
    rotation_matrix3D(d_RM, G.cp.xangle, G.cp.yangle, G.cp.zangle); /* hf_cuda_functions.cuh:66-88 */
    const int dims[3] = {(int)g->Xdim, (int)g->Ydim, (int)g->Zdim};
    const float* bound = d_vol;
    CUDA_SAFE_CALL(cudaMemcpyToSymbol(recon_ref_tex3_dims, dims, sizeof dims));
    CUDA_SAFE_CALL(cudaMemcpyToSymbol(recon_ref_tex3_data, &bound, sizeof bound));
    ObjectParam op;
    op.ObjX = op.ObjY = op.ObjZ = op.ObjXangle = op.ObjYangle = op.ObjZangle = 0.f;
    const float L = ((float)g->Ydim - 1.0f) * g->YVoxSize;
    const float step = L / (float)g->Ydim, first = L * (0.5f / (float)g->Ydim - 0.5f);
    for (unsigned k = 0; k < g->Ydim; ++k) {
        const float y0 = std::fma((float)k, step, first);
        forward_projection<<<G.bimg, G.timg>>>(d_img, G.cp, G.det, op, G.vox, d_RM, y0, angle);
    }
    CUDA_SAFE_CALL(cudaGetLastError());
    CUDA_SAFE_CALL(cudaMemcpy(img, d_img, N * 4, cudaMemcpyDeviceToHost));
    bound = nullptr;
    CUDA_SAFE_CALL(cudaMemcpyToSymbol(recon_ref_tex3_data, &bound, sizeof bound));
    CUDA_SAFE_CALL(cudaFree(d_vol));
    CUDA_SAFE_CALL(cudaFree(d_img));
    CUDA_SAFE_CALL(cudaFree(d_RM));
}

}  // extern "C"
