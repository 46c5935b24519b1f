// hf_siddon_recon.hpp -- drop-in for the reference's reconstruction driver
// class siddon_recon (CT_Recon/hf_siddon_recon.hpp:18-608) over librecon_b200.
//
// Same entry points: a0_RECON_MLEM (three overloads), a1_FORWARD_PROJECTION,
// a1_BACKWARD_PROJECTION, a_pull_recon_pointer, a_dsensitivity_pointer,
// a_pull_kernel_threads.  The file formats are the reference's: a
// `key = value` configuration, one raw float32 file per view
// <ProjFileFolder><ProjFileNameRoot>_<n><ProjFileSuffix>, one raw float32
// volume per iteration <ReconFileFolder><ReconFileNameRoot>_<it><suffix>.
// On a configuration or file error the reference prints
// "Encountered error, so did nothing" and returns; so does this class (the
// library's message is printed first).  The optional `options` member picks
// the arithmetic (COMPAT by default, the reference's FP32 traversal).
#pragma once

#include <cuda_runtime.h>

#include <cstdio>
#include <iostream>
#include <string>
#include <vector>

#include "hf_siddon_class.hpp"

class siddon_recon : public forward, public backward {
public:
    // Declared (configurationfilename, outputparameterfilename) in the
    // reference but defined and used as (folder, file name)
    // (hf_siddon_recon.hpp:91-108, mlem.cu:32); the definition is what runs.
    void a0_RECON_MLEM(std::string configurationfilefolder, std::string configurationfilename)
    {
        run_mlem(configurationfilefolder, configurationfilename);
    }
    void a0_RECON_MLEM(std::string configurationfilename) { run_mlem("", configurationfilename); }
    void a0_RECON_MLEM(std::string configurationfilefolder, std::string configurationfilename,
                       std::string outputparameterfilename)
    {
        (void)outputparameterfilename;
        run_mlem(configurationfilefolder, configurationfilename);
    }
    void a1_FORWARD_PROJECTION(std::string folder, std::string cfg)
    {
        report(recon_forward_projection_from_cfg(folder.c_str(), cfg.c_str(), &options), "Do forward projection");
    }
    void a1_BACKWARD_PROJECTION(std::string folder, std::string cfg, bool write_files_per_angle)
    {
        report(recon_backward_projection_from_cfg(folder.c_str(), cfg.c_str(), write_files_per_angle ? 1 : 0,
                                                  &options),
               "do m_backward_projection()");
    }

    // host copy of the last reconstruction (the reference returns &m_object[0])
    float* a_pull_recon_pointer() { return m_object.empty() ? nullptr : &m_object[0]; }
    float* a_dsensitivity_pointer() { return pd_sensitivity; }
    void a_pull_kernel_threads()
    {
        a_pull_kernel_threads(b_blocks_image, b_threads_image, b_blocks_object, b_threads_object, b_blocks_atomic,
                              b_threads_atomic);
    }
    // the reference's launch shapes (m_calc_kernel_threads, :366-386), for callers that read them
    void a_pull_kernel_threads(dim3& blocks_image, dim3& threads_image, dim3& blocks_object, dim3& threads_object,
                               dim3& blocks_atomic, dim3& threads_atomic)
    {
        threads_image = dim3(4, 4);
        blocks_image = dim3(m_det.NumAxPixels / 4, m_det.NumTAxPixels / 4);
        threads_object = dim3(4, 4, 4);
        blocks_object = dim3(m_vox.Xdim / 4, m_vox.Ydim / 4, m_vox.Zdim / 4);
        int sms = 0;
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, 0);
        threads_atomic = dim3(256);
        blocks_atomic = dim3(2 * sms);
    }

    dim3 b_blocks_image, b_threads_image;
    dim3 b_blocks_object, b_threads_object;
    dim3 b_blocks_atomic, b_threads_atomic;
    int b_N_image_pixels = 0;
    int b_N_object_voxels = 0;
    recon_options_t options = default_options();

    ~siddon_recon()
    {
        if (pd_sensitivity) cudaFree(pd_sensitivity);
    }

protected:
    Detector m_det{};
    VoxVolParam m_vox{};
    std::vector<float> m_object;
    float* pd_sensitivity = nullptr;

private:
    static recon_options_t default_options()
    {
        recon_options_t o;
        recon_default_options(&o);
        o.arith = RECON_ARITH_COMPAT;
        return o;
    }
    static void report(recon_status_t s, const char* ok)
    {
        if (s == RECON_OK) {
            std::cout << ok << std::endl;
        } else {
            std::cout << recon_last_error() << std::endl;
            std::cout << "Encountered error, so did nothing" << std::endl;
        }
    }
    void run_mlem(const std::string& folder, const std::string& cfg)
    {
        recon_status_t s = recon_mlem_from_cfg(folder.c_str(), cfg.c_str(), &options);
        if (s == RECON_OK) load_last(folder, cfg);
        report(s, "Do reconstruction");
    }
    // keep the host image and the device sensitivity the reference exposes
    void load_last(const std::string& folder, const std::string& cfg)
    {
        std::string dir = folder;
        for (char& c : dir)
            if (c == '\\') c = '/';
        if (!dir.empty() && dir.back() != '/') dir.push_back('/');
        recon_geometry_t g;
        recon_filepaths_t p;
        if (recon_geometry_from_cfg((dir + cfg).c_str(), &g, &p) != RECON_OK) return;
        m_det = {g.det.NumTAxPixels, g.det.NumAxPixels, g.det.TAxPixDimMm, g.det.AxPixDimMm};
        m_vox = {g.vox.Xdim, g.vox.Ydim, g.vox.Zdim, g.vox.XVoxSize, g.vox.YVoxSize, g.vox.ZVoxSize};
        b_N_image_pixels = (int)(g.det.NumAxPixels * g.det.NumTAxPixels);
        b_N_object_voxels = (int)(g.vox.Xdim * g.vox.Ydim * g.vox.Zdim);
        std::string rf = p.ReconFileFolder[0] ? p.ReconFileFolder : p.ProjFileFolder;
        if (!p.ReconFileFolder[0] && !rf.empty() && rf.back() != '/') rf.push_back('/');
        if (g.scan.N_iteration == 0) return;
        std::string last = rf + p.ReconFileNameRoot + "_" + std::to_string(g.scan.N_iteration - 1) + p.ReconFileSuffix;
        m_object.assign((size_t)b_N_object_voxels, 0.0f);
        if (FILE* f = std::fopen(last.c_str(), "rb")) {
            size_t got = std::fread(m_object.data(), sizeof(float), m_object.size(), f);
            (void)got;
            std::fclose(f);
        }
        recon_plan_t plan = nullptr;
        if (recon_plan_create(&g, &options, &plan) == RECON_OK) {
            if (!pd_sensitivity) cudaMalloc((void**)&pd_sensitivity, (size_t)b_N_object_voxels * sizeof(float));
            recon_sensitivity(plan, pd_sensitivity, nullptr);
            cudaDeviceSynchronize();
            recon_plan_destroy(plan);
        }
    }
};
