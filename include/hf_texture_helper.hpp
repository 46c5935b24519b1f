// hf_texture_helper.hpp -- drop-in for the reference's texture glue and its
// voxel-driven back projector (CT_Recon/hf_texture_helper.hpp:31-87,
// hf_cuda_kernels.cuh:183-237) over librecon_b200.
//
// texture_helper2D keeps the reference's three calls.  a2_input copies the
// view image (host or device, per the cudaMemcpyKind) into a device buffer
// the library samples through a texture object; the reference instead binds
// a process-global legacy texture reference (removed in CUDA 12).  The
// reference's optional cubic B-spline prefilter comes from a library that is
// not part of the reference and is not reproduced: pre_filter must be false.
// The reference launches backward_projection<<<blocks, threads>>>(...); here
// backward_projection(...) is a host function with the same arguments that
// adds value / Nprojections into md_Obj for the image last given to a2_input.
#pragma once

#include <cuda_runtime.h>

#include <cstring>

#include "hf_siddon_class.hpp"

namespace recon_b200 {
// The COMPAT plan backward_projection samples through, kept between calls: a
// reference-style caller back projects view after view with one geometry, and
// building a plan (tables, accumulators) per call would dominate.  A new
// geometry or device replaces it.  Like the reference's process-global
// texture binding, this is one per process and not for concurrent use.
struct voxel_bp_plan_cache {
    recon_geometry_t geom{};
    int device = -1;
    recon_plan_t plan = nullptr;
    ~voxel_bp_plan_cache()
    {
        if (plan) recon_plan_destroy(plan);
    }
    recon_plan_t get(const recon_geometry_t& g)
    {
        int dev = 0;
        check_cuda(cudaGetDevice(&dev));
        if (plan && dev == device && std::memcmp(&geom, &g, sizeof g) == 0) return plan;
        if (plan) recon_plan_destroy(plan);
        plan = nullptr;
        recon_options_t o;
        recon_default_options(&o);
        o.arith = RECON_ARITH_COMPAT;
        o.device = dev;
        check(recon_plan_create(&g, &o, &plan));
        geom = g;
        device = dev;
        return plan;
    }
    static voxel_bp_plan_cache& instance()
    {
        static voxel_bp_plan_cache c;
        return c;
    }
};
}  // namespace recon_b200

struct texture_helper2D {
    float* m_image = nullptr;
    unsigned m_width = 0, m_height = 0;

    int a1_allocate(unsigned width, unsigned height)
    {
        m_width = width;
        m_height = height;
        recon_b200::check_cuda(cudaMalloc((void**)&m_image, (size_t)width * height * sizeof(float)));
        current() = this;
        return 0;
    }
    int a2_input(float* data, unsigned width, unsigned height, bool pre_filter, cudaMemcpyKind kind)
    {
        if (pre_filter)
            throw recon_b200::config_error(RECON_ERR_UNSUPPORTED,
                                           "cubic B-spline prefiltering is not available (the library it needs is "
                                           "not part of the reference)");
        if (width != m_width || height != m_height)
            throw recon_b200::config_error(RECON_ERR_INVALID_ARGUMENT, "image size differs from a1_allocate");
        recon_b200::check_cuda(cudaMemcpy(m_image, data, (size_t)width * height * sizeof(float), kind));
        current() = this;
        return 0;
    }
    int a3_destroy()
    {
        if (m_image) cudaFree(m_image);
        m_image = nullptr;
        if (current() == this) current() = nullptr;
        return 0;
    }
    static texture_helper2D*& current()
    {
        static texture_helper2D* bound = nullptr;
        return bound;
    }
};

// backward_projection (hf_cuda_kernels.cuh:183-237) for the image bound by the
// last texture_helper2D::a2_input.  RM (the device rotation matrix) is taken
// from the misalignment angles in CalParam.  `mode` selects the reference's
// geometry (default) or the Siddon-consistent one.  Asynchronous on the
// legacy default stream, like the reference's kernel launch; the plan it runs
// on is built on the first call for a geometry and kept (voxel_bp_plan_cache).
inline void backward_projection(float* md_Obj, CalibrationParam CalParam, Detector Det, ObjectParam ObjParam,
                                VoxVolParam voxparam, float* RM, float alpha, unsigned int Nprojections,
                                int mode = RECON_VOXEL_REFERENCE)
{
    (void)ObjParam;
    (void)RM;
    texture_helper2D* t = texture_helper2D::current();
    if (!t || !t->m_image)
        throw recon_b200::config_error(RECON_ERR_INVALID_ARGUMENT, "no image bound (texture_helper2D::a2_input)");
    const recon_geometry_t g = recon_b200::make_geometry(CalParam, Det, voxparam);
    recon_plan_t plan = recon_b200::voxel_bp_plan_cache::instance().get(g);
    recon_b200::check(recon_voxel_bp_view(plan, t->m_image, alpha, Nprojections, mode, md_Obj, nullptr));
}
