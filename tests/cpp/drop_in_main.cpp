// A caller written against the reference's class interface (the way
// CT_Recon/mlem.cu and mlem.cu.orig use it), compiled against the drop-in
// headers in include/ and linked with librecon_b200.so.
//
//   drop_in_main <folder> <cfg> <out_folder>
//
// 1. siddon_recon::a0_RECON_MLEM(folder, cfg)               (mlem.cu:30-32)
// 2. per view: a_calc_initial_limits + a2_fp_per_angle and
//    a2_bp_per_angle of the projection, written to out_folder (mlem.cu.orig:49-104)
// 3. texture_helper2D + backward_projection of view 0       (hf_cuda_kernels.cuh:183-237)
#include <cstdio>
#include <string>
#include <vector>

#include "hf_siddon_recon.hpp"
#include "hf_texture_helper.hpp"

static void save(const std::string& path, const float* d, size_t n, bool device)
{
    std::vector<float> h(n);
    if (device) cudaMemcpy(h.data(), d, n * sizeof(float), cudaMemcpyDeviceToHost);
    else std::copy(d, d + n, h.begin());
    FILE* f = std::fopen(path.c_str(), "wb");
    std::fwrite(h.data(), sizeof(float), n, f);
    std::fclose(f);
}

int main(int argc, char** argv)
{
    if (argc < 4) return 2;
    std::string folder = argv[1], cfg = argv[2], out = argv[3];
    std::string path = folder + "/" + cfg;

    siddon_recon recon;
    recon.a0_RECON_MLEM(folder, cfg);
    if (!recon.a_pull_recon_pointer()) return 3;

    CalibrationParam cp;
    Detector det;
    VoxVolParam vox;
    ScanParameters sp;
    FilePaths fpth;
    cp.LoadFromConfigFile(path);
    det.LoadFromConfigFile(path);
    vox.LoadFromConfigFile(path);
    sp.LoadFromConfigFile(path);
    fpth.LoadFromconfigFile(path);

    siddon_commons sc;
    sc.a1_initiate(cp, det, vox);
    sc.a2_allocate();
    forward fw;
    fw.a1_Finitiate(sc.N_image_pixels);
    backward bw;
    bw.a1_Binitiate(sc.N_object_voxels, sc.N_image_pixels);
    dim3 bi, ti, bo, to, ba, ta;
    recon.a_pull_kernel_threads(bi, ti, bo, to, ba, ta);

    std::vector<float> obj(sc.N_object_voxels), img(sc.N_image_pixels);
    FILE* f = std::fopen((folder + "/object.bin").c_str(), "rb");
    if (!f || std::fread(obj.data(), sizeof(float), obj.size(), f) != obj.size()) return 4;
    std::fclose(f);
    float *d_obj, *d_img;
    cudaMalloc((void**)&d_obj, obj.size() * sizeof(float));
    cudaMalloc((void**)&d_img, img.size() * sizeof(float));
    cudaMemcpy(d_obj, obj.data(), obj.size() * sizeof(float), cudaMemcpyHostToDevice);
    for (unsigned n = 0; n < sp.NumProj; ++n) {
        float angle = (float)n * sp.DeltaAng;
        unsigned loopN = sc.a_calc_initial_limits(angle, bi, ti);
        if (loopN == 0) return 5;
        fw.a2_fp_per_angle(d_obj, sc, bi, ti);
        save(out + "/fp_" + std::to_string(n) + ".bin", fw.a_Fdevicepointer(), img.size(), true);
        bw.a2_bp_per_angle(fw.a_Fdevicepointer(), sc, bi, ti, bo, to, ba, ta);
        save(out + "/bp_" + std::to_string(n) + ".bin", bw.a_bpdevicepointer(), obj.size(), true);
    }

    texture_helper2D th;
    th.a1_allocate(det.NumAxPixels, det.NumTAxPixels);
    cudaMemcpy(img.data(), fw.a_Fdevicepointer(), img.size() * sizeof(float), cudaMemcpyDeviceToHost);
    th.a2_input(img.data(), det.NumAxPixels, det.NumTAxPixels, false, cudaMemcpyHostToDevice);
    float* d_vol;
    cudaMalloc((void**)&d_vol, obj.size() * sizeof(float));
    cudaMemset(d_vol, 0, obj.size() * sizeof(float));
    ObjectParam op{};
    backward_projection(d_vol, cp, det, op, vox, nullptr, (float)(sp.NumProj - 1) * sp.DeltaAng, sp.NumProj);
    save(out + "/voxel_bp.bin", d_vol, obj.size(), true);
    th.a3_destroy();
    cudaFree(d_obj);
    cudaFree(d_img);
    cudaFree(d_vol);
    std::printf("drop-in ok\n");
    return 0;
}
