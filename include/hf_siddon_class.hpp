// hf_siddon_class.hpp -- drop-in for the reference's projector classes
// (CT_Recon/hf_siddon_class.hpp:18-417) over librecon_b200.
//
// Same class names, public members and method signatures; the dim3 launch
// arguments are accepted and ignored (the library picks its own launch
// shapes).  Output pointers are borrowed device buffers owned by the object,
// valid until its next call, exactly as in the reference.  The arithmetic
// defaults to RECON_ARITH_COMPAT, which reproduces the reference's FP32
// traversal bit for bit per ray; set `options.arith = RECON_ARITH_EXACT`
// before a2_allocate() for the exact Siddon projector pair.  Failures throw
// recon_b200::config_error (the reference prints and exits on CUDA errors).
#pragma once

#include <cuda_runtime.h>

#include <vector>

#include "CTSystemElements_HF.h"
#include "recon_b200.h"

namespace recon_b200 {
inline void check(recon_status_t s)
{
    if (s != RECON_OK) throw config_error(s, recon_last_error());
}
inline void check_cuda(cudaError_t e)
{
    if (e != cudaSuccess) throw config_error(RECON_ERR_CUDA, cudaGetErrorString(e));
}
}  // namespace recon_b200

// siddon_commons (hf_siddon_class.hpp:18-133)
struct siddon_commons {
    unsigned int loopN = 0;
    float angle_degree = 0.0f;
    int N_image_pixels = 0;
    int N_object_voxels = 0;
    int check = 0;
    recon_options_t options;
    recon_plan_t plan = nullptr;
    recon_geometry_t geom;

    siddon_commons()
    {
        recon_default_options(&options);
        options.arith = RECON_ARITH_COMPAT;
    }
    ~siddon_commons() { a3_deallocate(); }
    siddon_commons(const siddon_commons&) = delete;
    siddon_commons& operator=(const siddon_commons&) = delete;

    void a1_initiate(CalibrationParam params, Detector det, VoxVolParam vox)
    {
        geom = recon_b200::make_geometry(params, det, vox);
        N_image_pixels = (int)(det.NumAxPixels * det.NumTAxPixels);
        N_object_voxels = (int)(vox.Xdim * vox.Ydim * vox.Zdim);
        check = 1;
    }
    void a2_allocate()
    {
        if (check != 1) return;
        recon_b200::check(recon_plan_create(&geom, &options, &plan));
        check = 2;
    }
    // The device-side step count replaces the reference's blocking copy of
    // every ray's delta_index; the value returned is the same loopN.
    unsigned int a_calc_initial_limits(float angle, dim3 = dim3(), dim3 = dim3())
    {
        angle_degree = angle;
        recon_b200::check(recon_view_step_count(plan, angle, &loopN));
        return loopN;
    }
    void a3_deallocate()
    {
        if (plan) recon_plan_destroy(plan);
        plan = nullptr;
        if (check == 2) check = 1;
    }
};

// forward (hf_siddon_class.hpp:136-244)
class forward {
public:
    void a1_Finitiate(int N_image_pixels)
    {
        pN_pixels = N_image_pixels;
        recon_b200::check_cuda(cudaMalloc((void**)&md_fp_image, (size_t)pN_pixels * sizeof(float)));
        pcheck = true;
    }
    void a2_fp_per_angle(float* d_object, siddon_commons& siddon_var, dim3 = dim3(), dim3 = dim3())
    {
        recon_b200::check(recon_fp_view(siddon_var.plan, d_object, siddon_var.angle_degree, md_fp_image, nullptr));
    }
    float* a_Fdevicepointer() { return md_fp_image; }
    ~forward()
    {
        if (pcheck) cudaFree(md_fp_image);
    }

protected:
    float* md_fp_image = nullptr;

private:
    int pN_pixels = 0;
    bool pcheck = false;
};

// backward (hf_siddon_class.hpp:247-368)
class backward {
public:
    void a1_Binitiate(int N_object_voxels, int N_image_pixels)
    {
        pN_voxels = N_object_voxels;
        pN_voxels_pad = N_object_voxels + 1;
        (void)N_image_pixels;
        recon_b200::check_cuda(cudaMalloc((void**)&md_bp_object, (size_t)pN_voxels_pad * sizeof(float)));
        recon_b200::check_cuda(cudaMemset(md_bp_object, 0, (size_t)pN_voxels_pad * sizeof(float)));
        pcheck = true;
    }
    void a2_bp_per_angle(float* d_image, siddon_commons& siddon_var, dim3 = dim3(), dim3 = dim3(), dim3 = dim3(),
                         dim3 = dim3(), dim3 = dim3(), dim3 = dim3())
    {
        recon_b200::check(recon_bp_view(siddon_var.plan, d_image, siddon_var.angle_degree, md_bp_object, nullptr));
    }
    float* a_bpdevicepointer() { return md_bp_object; }
    ~backward()
    {
        if (pcheck) cudaFree(md_bp_object);
    }

protected:
    float* md_bp_object = nullptr;
    int pN_voxels = 0;
    int pN_voxels_pad = 0;

private:
    bool pcheck = false;
};

// sensitivity (hf_siddon_class.hpp:371-417): back projection of ones summed
// over 360 views at integer degrees, as the reference class does.
class sensitivity : public backward {
public:
    void a1_Sinitiate(int N_object_voxels, int N_image_pixels)
    {
        a1_Binitiate(N_object_voxels, N_image_pixels);
        recon_b200::check_cuda(cudaMalloc((void**)&pd_ones, (size_t)N_image_pixels * sizeof(float)));
        recon_b200::check_cuda(cudaMalloc((void**)&pd_sensitivity, (size_t)N_object_voxels * sizeof(float)));
        recon_b200::check_cuda(cudaMemset(pd_sensitivity, 0, (size_t)N_object_voxels * sizeof(float)));
        npix = N_image_pixels;
        nvox = N_object_voxels;
    }
    void a3S_calculate(siddon_commons& siddon_var, dim3 = dim3(), dim3 = dim3(), dim3 = dim3(), dim3 = dim3(),
                       dim3 = dim3(), dim3 = dim3())
    {
        recon_b200::check(recon_set_ones(pd_ones, (size_t)npix, nullptr));
        for (int n = 0; n < 360; n++) {
            siddon_var.a_calc_initial_limits((float)n);
            a2_bp_per_angle(pd_ones, siddon_var);
            recon_b200::check(recon_add(pd_sensitivity, md_bp_object, (size_t)nvox, nullptr));
        }
    }
    float* a_dsensitivitypointer() { return pd_sensitivity; }
    ~sensitivity()
    {
        cudaFree(pd_ones);
        cudaFree(pd_sensitivity);
    }

private:
    float* pd_ones = nullptr;
    float* pd_sensitivity = nullptr;
    int npix = 0, nvox = 0;
};
