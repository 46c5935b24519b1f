/*
 * siddon_oracle.h -- CPU oracle for the MLEM / Siddon cone-beam path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker that the CUDA
 * product is compared against.  Only tests/, __graft_entry__.smoke() and the
 * cpu_baseline leg of bench.py may load it.  Nothing in recon_b200/ links or
 * calls it.
 *
 * Three restatements of the reference algorithm live here:
 *
 *   orc_c_*  FP32 "compat" restatement of the reference kernels, op by op and
 *            in the reference's evaluation order, with the GPU intrinsics
 *            replaced by IEEE host arithmetic (__fdividef -> a/b,
 *            __fdiv_rz -> division rounded toward zero, cospif/sinpif -> a
 *            half-integer-exact host routine, float->unsigned conversions
 *            saturating with NaN -> 0 as the GPU does).  Pinned bit-exact
 *            against the reference's own kernel sources compiled for the host
 *            (oracle/_ref/libref_cpu.so).
 *   orc_x_*  FP64 exact Siddon: the true intersection length of every ray with
 *            every voxel, in the reference's scanner geometry.  This is the
 *            accuracy oracle that every result's error is stated against.
 *   orc_v_*  voxel-driven bilinear back projector (reference
 *            CT_Recon/hf_cuda_kernels.cuh:240-284) in FP32.
 *
 * Geometry conventions (all from the reference):
 *   volume index n = x + y*Xdim + z*Xdim*Ydim, planes at -dim/2*vox + k*vox
 *     (CT_Recon/hf_siddon_class.hpp:51-53)
 *   source (0,-Rf,0) (hf_siddon_class.hpp:54), detector plane y = R-Rf
 *     (siddon_device_kernelsMLEM.cuh:311)
 *   view image [TAxPixels rows v][AxPixels cols u], pixel n = u + v*AxPixels
 *     (siddon_kernelsMLEM.cuh:110-112)
 *   view n is at angle (float)n * DeltaAng degrees (hf_siddon_recon.hpp:443)
 */
#ifndef RECON_SIDDON_ORACLE_H
#define RECON_SIDDON_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* CalibrationParam + Detector + VoxVolParam (CT_Recon/CTSystemElements_HF.h:13-99) */
typedef struct {
    float R, Rf, Ry, Dx, Dz, xangle, yangle, zangle, M;
    unsigned int NumTAxPixels, NumAxPixels;
    float TAxPixDimMm, AxPixDimMm;
    unsigned int Xdim, Ydim, Zdim;
    float XVoxSize, YVoxSize, ZVoxSize;
} orc_geom;

/* Per-ray state written by siddon_alpha_limits (siddon_kernelsMLEM.cuh:103-149). */
typedef struct {
    float p1[3], p2[3];
    float d12;
    float alpha_min, alpha_max;
    uint32_t mask;
    float alpha_i[3], alpha_f[3], delta_alpha[3];
    uint32_t delta_index;
} orc_c_ray;

/* ---- FP32 compat restatement ---- */
void orc_rotation_matrix(float xangle, float yangle, float zangle, float RM[9]);
/* 0: host model (default), 1: device model -- see siddon_oracle.c */
void orc_c_set_device_model(int on);
float orc_c_pixel_iterate2(float NumPixels, float PixelsDimMm, float Mag, int iterator);
void orc_c_ray_setup(const orc_geom* g, const float RM[9], float angle_deg, int u, int v,
                     orc_c_ray* out);
uint32_t orc_c_setup_view(const orc_geom* g, const float RM[9], float angle_deg, float* alpha_min,
                          float* alpha_max, float* d12, uint32_t* mask, float* alpha_i,
                          float* alpha_f, float* delta_alpha, float* p1, float* p2,
                          uint32_t* delta_index);
uint32_t orc_c_loopN(const orc_geom* g, const float RM[9], float angle_deg);
/* Per-step trace of one ray: for every traversal step k < loopN (stopping early
 * once the state is a fixed point) and then the end segment, the voxel index
 * used (-1 when no segment) and the ray length.  Returns the number of records,
 * or -1 when cap is too small. */
int orc_c_trace(const orc_geom* g, const float RM[9], float angle_deg, int u, int v,
                uint32_t loopN, int32_t* idx, float* len, int cap);
void orc_c_fp_view(const orc_geom* g, const float RM[9], float angle_deg, const float* vol,
                   float* img);
void orc_c_bp_view(const orc_geom* g, const float RM[9], float angle_deg, const float* img,
                   float* vol_out);
void orc_c_mlem(const orc_geom* g, unsigned int NumProj, float DeltaAng, const float* g_sino,
                unsigned int iters, float* f, float* sens_out, float* f_history);

/* ---- FP64 exact Siddon ---- */
typedef struct {
    double p1[3], p2[3];
    double d12;
} orc_x_ray;
void orc_x_ray_geom(const orc_geom* g, float angle_deg, int u, int v, orc_x_ray* r);
int orc_x_trace(const orc_geom* g, float angle_deg, int u, int v, int64_t* idx, double* len,
                int cap);
void orc_x_fp_view(const orc_geom* g, float angle_deg, const double* vol, double* img);
void orc_x_fp_all(const orc_geom* g, unsigned int NumProj, float DeltaAng, const double* vol,
                  double* sino, int threads);
void orc_x_bp_all(const orc_geom* g, unsigned int NumProj, float DeltaAng, const double* sino,
                  double* vol, int threads);
void orc_x_mlem(const orc_geom* g, unsigned int NumProj, float DeltaAng, const float* g_sino,
                unsigned int iters, double* f, double* sens_out, int threads);
int orc_x_osem(const orc_geom* g, unsigned int NumProj, float DeltaAng, const float* g_sino, unsigned int iters,
               unsigned int N_subsets, double* f, int threads);
int orc_x_slab_update(const orc_geom* g, unsigned int NumProj, float DeltaAng, const float* f,
                      const float* g_meas, unsigned int z0, unsigned int z1, double* out, int threads);
int64_t orc_x_count_isects(const orc_geom* g, unsigned int NumProj, float DeltaAng, int threads);
/* column of the system matrix for one voxel: every (view, pixel, length) */
int orc_x_voxel_column(const orc_geom* g, unsigned int NumProj, float DeltaAng, int64_t voxel,
                       int32_t* view, int32_t* pixel, double* len, int cap);

/* ---- voxel-driven bilinear BP (FP32) ---- */
void orc_v_bp_view(const orc_geom* g, const float RM[9], float angle_deg, const float* img,
                   unsigned int Nproj, int mode, float* vol_accum);

/* ---- ray-marching forward projection (plane samples, FP64) ---- */
void orc_m_fp_view(const orc_geom* g, const float RM[9], float angle_deg, int mode, const float* vol,
                   double* img);

#ifdef __cplusplus
}
#endif
#endif
