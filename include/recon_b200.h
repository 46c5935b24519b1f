/*
 * recon_b200.h -- C ABI of the B200 MLEM / Siddon cone-beam library
 * (librecon_b200.so).
 *
 * Plain C types only: device buffers are `float*` (or `void*` for BF16
 * sinograms) in CUDA device memory, streams are `void*` holding a
 * cudaStream_t (NULL = legacy default stream), sizes are integers.  No call
 * exits the process or reads stdin; every call returns a recon_status_t and
 * recon_last_error() gives the message of the last failure on the calling
 * thread.
 *
 * Data layout (the reference's, unchanged):
 *   volume  f[x + y*Xdim + z*Xdim*Ydim], float32
 *   view    img[u + v*AxPixels]: TAxPixels rows (v, world z) of AxPixels
 *           columns (u); views are stored back to back, view n at angle
 *           (float)n * DeltaAng degrees.
 *
 * Each declaration names the reference interface it replaces (file:line in
 * the reference project hfan36/recon).
 */
#ifndef RECON_B200_H
#define RECON_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define RECON_B200_ABI_VERSION 4

typedef enum {
    RECON_OK = 0,
    RECON_ERR_INVALID_ARGUMENT = 1, /* bad size / pointer / option */
    RECON_ERR_UNSUPPORTED = 2,      /* geometry or option combination not handled */
    RECON_ERR_CUDA = 3,             /* CUDA runtime error (message has the detail) */
    RECON_ERR_OUT_OF_MEMORY = 4,
    RECON_ERR_FILE_NOT_FOUND = 5,   /* ConfigFile::file_not_found (ConfigFile.h:108-111) */
    RECON_ERR_KEY_NOT_FOUND = 6,    /* ConfigFile::key_not_found (ConfigFile.h:112-115) */
    RECON_ERR_SIZE_MISMATCH = 7,    /* check_projection_files (hf_cpp_functions.hpp:247-270) */
    RECON_ERR_IO = 8,               /* short read / write */
    RECON_ERR_NO_DEVICE = 9
} recon_status_t;

/* CalibrationParam (CT_Recon/CTSystemElements_HF.h:13-40) */
typedef struct {
    float R, Rf, Ry, Dx, Dz, xangle, yangle, zangle, M;
} recon_calibration_t;
/* Detector (CTSystemElements_HF.h:42-58) */
typedef struct {
    unsigned int NumTAxPixels, NumAxPixels;
    float TAxPixDimMm, AxPixDimMm;
} recon_detector_t;
/* VoxVolParam (CTSystemElements_HF.h:78-99) */
typedef struct {
    unsigned int Xdim, Ydim, Zdim;
    float XVoxSize, YVoxSize, ZVoxSize;
} recon_volume_t;
/* ScanParameters (CTSystemElements_HF.h:60-76) */
typedef struct {
    unsigned int N_iteration, NumProj;
    float DeltaAng;
} recon_scan_t;

typedef struct {
    recon_calibration_t cal;
    recon_detector_t det;
    recon_volume_t vox;
    recon_scan_t scan;
} recon_geometry_t;

/* FilePaths (CTSystemElements_HF.h:123-151) */
#define RECON_PATH_MAX 1024
typedef struct {
    char ProjFileFolder[RECON_PATH_MAX];
    char ProjFileNameRoot[RECON_PATH_MAX];
    char ProjFileSuffix[RECON_PATH_MAX];
    char ReconFileFolder[RECON_PATH_MAX];
    char ReconFileNameRoot[RECON_PATH_MAX];
    char ReconFileSuffix[RECON_PATH_MAX];
    char ObjFileFolder[RECON_PATH_MAX];
    char ObjFileName[RECON_PATH_MAX];
    char BpFileNameRoot[RECON_PATH_MAX];
    char BpFileSuffix[RECON_PATH_MAX];
} recon_filepaths_t;

/* Arithmetic of the Siddon projector pair.
 *   RECON_ARITH_EXACT  -- true Siddon: every ray-voxel intersection length,
 *     plane crossings set up in FP64 and traversed in FP32, forward and back
 *     projectors exact transposes of each other (the same length for every
 *     ray-voxel pair), back projection deterministic (recon_siddon_bp_t).
 *     Detector tilt angles (xangle/yangle/zangle) must be zero.
 *   RECON_ARITH_COMPAT -- the reference's FP32 traversal reproduced operation
 *     for operation (siddon_kernelsMLEM.cuh), including its quirks; per-ray
 *     voxel/length sequences are bit-identical to the reference's kernels on
 *     the same GPU.  Back projection is ray driven with exact (integer
 *     fixed-point) accumulation, so it is deterministic. */
typedef enum { RECON_ARITH_EXACT = 0, RECON_ARITH_COMPAT = 1 } recon_arith_t;
/* Ray-sum accumulation: compensated (Kahan) or plain FP32. */
typedef enum { RECON_SUM_KAHAN = 0, RECON_SUM_PLAIN = 1 } recon_sum_t;
/* Storage of the measured and ratio sinograms inside recon_mlem. */
typedef enum { RECON_SINO_F32 = 0, RECON_SINO_BF16 = 1 } recon_sino_t;
/* Back projector used by recon_mlem. */
typedef enum { RECON_BP_SIDDON = 0, RECON_BP_VOXEL = 1 } recon_bp_t;
/* Voxel-driven back projector geometry.
 *   REFERENCE -- backward_projection / backward_projection2
 *     (hf_cuda_kernels.cuh:183-284) as written: view angle mirrored relative
 *     to the Siddon projector, detector coordinate in millimetres used as the
 *     texel coordinate.
 *   GEOMETRIC -- angle sense of the Siddon projector, coordinate converted to
 *     pixels (mm / (pitch*M)). */
typedef enum { RECON_VOXEL_REFERENCE = 0, RECON_VOXEL_GEOMETRIC = 1 } recon_voxel_mode_t;
/* Design of the EXACT Siddon back projector (the same lengths either way; the
 * forward projector is unchanged).
 *   GATHER -- one warp per (x, y) column of voxels gathers every ray that
 *     crosses it, summing in FP32 in a fixed order (views, detector columns,
 *     rows), so results are deterministic; no atomics.  Fastest where the rays
 *     of adjacent detector rows cross a column at least one voxel apart.
 *   RAY    -- one thread per ray walks it through L2-resident z-slabs and adds
 *     into 64-bit fixed-point accumulators (exact, order-independent sums).
 *   AUTO   -- GATHER where the rays of adjacent rows cross a voxel column 1 to
 *     1.4 voxels apart (at the depth nearest the source), a ray's piece of one
 *     column spans less than a voxel of z, the volume is at least 128 voxels
 *     tall and the detector has at most 3072 rows; RAY otherwise.
 *   TUNED  -- measured: plan creation times a back projection with each
 *     design on the plan's own geometry and keeps the faster, and times the
 *     detector-column forward projector with 32, 64 and 128 detector rows per
 *     CTA and keeps the fastest.  The choices are kept for the process per
 *     geometry and device, so every plan of that geometry (a batch's and a
 *     plain one alike) makes the same choices and gives the same bits.
 *     recon_plan_siddon_bp and recon_plan_column_rows report them. */
typedef enum {
    RECON_SIDDON_BP_AUTO = 0,
    RECON_SIDDON_BP_GATHER = 1,
    RECON_SIDDON_BP_RAY = 2,
    RECON_SIDDON_BP_TUNED = 3
} recon_siddon_bp_t;

typedef struct {
    int arith;      /* recon_arith_t, default EXACT */
    int sum;        /* recon_sum_t, default KAHAN */
    int sino;       /* recon_sino_t, default F32 */
    int bp;         /* recon_bp_t, default SIDDON */
    int voxel_mode; /* recon_voxel_mode_t, default GEOMETRIC */
    int device;     /* CUDA device ordinal, default 0 */
    int siddon_bp;  /* recon_siddon_bp_t, default AUTO (EXACT arithmetic only) */
    int fp_block;   /* detector-column forward projector over xy blocks of
                     * fp_block x fp_block voxel columns, one block at a time
                     * (at most 64 blocks): 0 = AUTO (blocks where the volume's
                     * z-fastest copy exceeds 96 MiB, each block's share at most
                     * 40 MiB, so the views in flight reuse it from L2), -1 =
                     * never, n > 0 = n.  Same lengths; the ray sums add the
                     * blocks' shares in block order. */
    int fp_rows;    /* detector rows per CTA of the detector-column forward
                     * projector: 0 = AUTO (the fewest of 32, 64, 128 that
                     * cover a column's rows; measured with
                     * RECON_SIDDON_BP_TUNED), or 32, 64 or 128.  Results do not
                     * depend on it. */
} recon_options_t;

typedef struct recon_plan* recon_plan_t;

int recon_abi_version(void);
const char* recon_last_error(void);
recon_status_t recon_default_options(recon_options_t* opt);

/* ---- configuration files --------------------------------------------- */

/* Reads a `key = value  # comment` file and fills the geometry and (if not
 * NULL) the file paths.  Replaces CalibrationParam / Detector / VoxVolParam /
 * ScanParameters / FilePaths ::LoadFromConfigFile
 * (CTSystemElements_HF.h:25-39, 49-57, 67-75, 87-98, 136-150) over the
 * ConfigFile parser (ConfigFile.cpp:67-141): every key is required. */
recon_status_t recon_geometry_from_cfg(const char* cfg_path, recon_geometry_t* geom,
                                       recon_filepaths_t* paths);

/* ---- plans ------------------------------------------------------------ */

/* Validates the geometry, selects the device and builds the per-plan tables
 * (ray plane parameters in FP64 for EXACT, per-view step counts for COMPAT).
 * Replaces siddon_commons::a1_initiate + a2_allocate
 * (hf_siddon_class.hpp:43-91) and the buffer set-up of
 * siddon_recon::m_recon_initiate (hf_siddon_recon.hpp:417-435).  Dimensions
 * need not be multiples of 4. */
recon_status_t recon_plan_create(const recon_geometry_t* geom, const recon_options_t* opt,
                                 recon_plan_t* plan);
/* Replaces siddon_commons::a3_deallocate and the class destructors
 * (hf_siddon_class.hpp:109-132, 232-244, 354-368; hf_siddon_recon.hpp:594-606). */
void recon_plan_destroy(recon_plan_t plan);
/* Device bytes held by the plan. */
size_t recon_plan_device_bytes(recon_plan_t plan);
/* The Siddon back projector an EXACT plan uses (RECON_SIDDON_BP_GATHER or
 * RECON_SIDDON_BP_RAY, after the AUTO choice).  No counterpart in the
 * reference, which has one back projector. */
recon_status_t recon_plan_siddon_bp(recon_plan_t plan, int* design);
/* The forward projector an EXACT plan uses: RECON_FP_COLUMNS (the rays of one
 * detector column share their (x, y) path, walked once per column; used where
 * a ray's stretch in one (x, y) voxel column spans less than 0.9 voxel of z)
 * or RECON_FP_RAY_WALK (one thread walks each ray).  Both give every (ray,
 * voxel) pair the same length.  No counterpart in the reference, which has
 * one forward projector. */
#define RECON_FP_RAY_WALK 0
#define RECON_FP_COLUMNS 1
#define RECON_FP_COLUMN_BLOCKS 2 /* detector columns, volume walked in xy blocks (fp_block) */
recon_status_t recon_plan_forward_projector(recon_plan_t plan, int* design);
/* *paired = 1 when the plan's EXACT projectors take detector rows (and, in
 * the gather back projector, voxels) in pairs mirrored about the source plane
 * z = 0, computing each pair's shared lengths once: where the volume has an
 * even slice count and the FP64-built z table is exactly mirror-symmetric
 * (no vertical detector offset Dz).  Results are the same either way.  No
 * counterpart in the reference. */
recon_status_t recon_plan_mirror_pairs(recon_plan_t plan, int* paired);
/* *quarter = 1 when an EXACT plan's views come in quarter turns about a
 * square volume (Xdim = Ydim, even, XVoxSize = YVoxSize, NumProj a multiple
 * of 4 with view n + NumProj/4 at exactly angle(n) + 90 degrees).  The plan
 * then derives the ray tables of views NumProj/4 .. NumProj-1 from the first
 * quarter's by exact quarter turns, so both projectors give column (x, y) at
 * view n + NumProj/4 exactly the lengths of column (Xdim-1-y, x) at view n,
 * and the mirror-paired gather back projector finds each set of lengths once
 * for four columns.  *quarter = 2 when, besides, that gather is the plan's
 * MLEM back projector, so recon_mlem_backward_quarters serves it.  0
 * otherwise.  No counterpart in the reference. */
recon_status_t recon_plan_quarter_turns(recon_plan_t plan, int* quarter);
/* *rows = the detector rows per CTA of the plan's detector-column forward
 * projector (32, 64 or 128: the fewest that cover a column's rows, or the
 * fastest measured with RECON_SIDDON_BP_TUNED), 0 for other forward
 * projectors.  No counterpart in the reference. */
recon_status_t recon_plan_column_rows(recon_plan_t plan, int* rows);

/* ---- projectors (device pointers, asynchronous on `stream`) ----------- */

/* Forward projection of one view at an arbitrary angle (degrees): img is
 * overwritten.  Replaces siddon_commons::a_calc_initial_limits +
 * forward::a2_fp_per_angle + a_Fdevicepointer (hf_siddon_class.hpp:93-106,
 * 195-230); no host synchronisation. */
recon_status_t recon_fp_view(recon_plan_t plan, const float* d_vol, float angle_deg, float* d_img,
                             void* stream);
/* Forward projection of views first..first+count-1 (view n at
 * (float)n*DeltaAng) into d_sino (count views, back to back). */
recon_status_t recon_fp_views(recon_plan_t plan, const float* d_vol, unsigned int first,
                              unsigned int count, float* d_sino, void* stream);
/* Back projection of one view: d_vol is overwritten with the view's
 * contribution.  Replaces backward::a2_bp_per_angle + a_bpdevicepointer
 * (hf_siddon_class.hpp:313-352). */
recon_status_t recon_bp_view(recon_plan_t plan, const float* d_img, float angle_deg, float* d_vol,
                             void* stream);
/* Sum over views first..first+count-1 of the back projections of d_sino,
 * which holds those count views back to back; d_vol is overwritten. */
recon_status_t recon_bp_views(recon_plan_t plan, const float* d_sino, unsigned int first,
                              unsigned int count, float* d_vol, void* stream);
/* Sensitivity image: back projection of an all-ones sinogram over all views.
 * Replaces siddon_recon::m_calc_sensitivity (hf_siddon_recon.hpp:388-415)
 * and sensitivity::a3S_calculate (hf_siddon_class.hpp:393-405). */
recon_status_t recon_sensitivity(recon_plan_t plan, float* d_sens, void* stream);

/* Voxel-driven back projection of one view, added into d_vol_accum:
 * value/Nproj per voxel, bilinear from the view image through a texture
 * object.  Replaces texture_helper2D::a1_allocate / a2_input / a3_destroy +
 * backward_projection (hf_texture_helper.hpp:38-85, hf_cuda_kernels.cuh:
 * 183-237); `mode` is a recon_voxel_mode_t. */
recon_status_t recon_voxel_bp_view(recon_plan_t plan, const float* d_img, float angle_deg,
                                   unsigned int Nproj, int mode, float* d_vol_accum, void* stream);

/* Ray-marching forward projection of one view at an arbitrary angle: each
 * pixel's ray sampled on depth planes of the view's frame, every sample times
 * the ray length per plane spacing, summed into d_img (overwritten).
 * Replaces texture_helper3D::a1_allocate / a2_input / a3_destroy +
 * forward_projection (hf_texture_helper.hpp:99-178, hf_cuda_kernels.cuh:
 * 126-180), which the reference leaves without a caller.  `mode` is a
 * recon_voxel_mode_t: REFERENCE = the kernel's arithmetic (coordinates
 * normalised by L = (Ydim-1)*YVoxSize, point sampling with zero outside, planes
 * at the normalised texel centres y0 = L*((k+1/2)/Ydim - 1/2), k < Ydim);
 * GEOMETRIC = trilinear sampling at
 * voxel centres on planes YVoxSize apart spanning the volume's bounding
 * circle.  Any arithmetic; the view angle sense is the Siddon projector's. */
recon_status_t recon_march_fp_view(recon_plan_t plan, const float* d_vol, float angle_deg, int mode,
                                   float* d_img, void* stream);

/* ---- MLEM --------------------------------------------------------------- */

/* `iters` MLEM iterations over all NumProj views of the measured sinogram
 * d_g (float32, or bf16 when the plan uses RECON_SINO_BF16; NumProj views
 * back to back).  d_f holds the starting image on entry (pass
 * init_ones = 1 to start from f = 1 as the reference does) and the result on
 * return.  The sensitivity image is computed once per plan and cached.
 * Replaces siddon_recon::m_mlem_all_iterations / m_mlem_single_iteration
 * (hf_siddon_recon.hpp:437-511) without the per-view disk reads and host
 * synchronisations. */
recon_status_t recon_mlem(recon_plan_t plan, const void* d_g, unsigned int iters, float* d_f,
                          int init_ones, void* stream);
/* As recon_mlem for one iteration, capturable in a CUDA graph once the
 * plan's sensitivity is cached (call recon_mlem_prepare first). */
recon_status_t recon_mlem_prepare(recon_plan_t plan, void* stream);
recon_status_t recon_mlem_iteration(recon_plan_t plan, const void* d_g, float* d_f, void* stream);

/* Copies views [first, first + count) of a measured sinogram [view][v][u]
 * (element type as the plan's `sino` option) from host memory h_g to device
 * memory d_g, both holding all NumProj views: for EXACT plans only detector
 * rows v_min..v_max, the rows some ray crossing the volume reaches in some
 * view, as one strided copy; the other rows of d_g are left as they are (no
 * projector or MLEM call of the plan reads a value there: their rays miss the
 * volume, so their ratio is 0 whatever g holds).  COMPAT plans copy whole
 * views.  *bytes (may be NULL) receives the bytes copied.  Asynchronous on
 * `stream`; pinned host memory lets the copy overlap compute.  No counterpart
 * in the reference, which reads every view from disk every iteration
 * (hf_siddon_recon.hpp:437-476). */
recon_status_t recon_upload_sinogram(recon_plan_t plan, const void* h_g, void* d_g, unsigned first,
                                     unsigned count, size_t* bytes, void* stream);

/* The two halves of an iteration over a range of views, for callers that
 * split the views between devices (sum the partial Ht across devices, then
 * apply recon_mlem_update everywhere).  EXACT arithmetic, Siddon back
 * projector; recon_mlem_prepare first.
 *   forward:  ratio(views) = g / FP(f)   (the reference's divide1(g, Hf),
 *             hf_siddon_recon.hpp:455-458), kept inside the plan; d_g holds
 *             all NumProj views.
 *   backward: d_ht = sum over the views of BP(ratio) (overwritten).
 *   update:   f = (sens != 0) ? f * Ht / sens : 0 (hf_siddon_recon.hpp:473-474). */
recon_status_t recon_mlem_forward(recon_plan_t plan, const void* d_g, const float* d_f,
                                  unsigned int first, unsigned int count, void* stream);
recon_status_t recon_mlem_backward(recon_plan_t plan, unsigned int first, unsigned int count,
                                   float* d_ht, void* stream);
recon_status_t recon_mlem_update(recon_plan_t plan, float* d_f, const float* d_ht, void* stream);
/* The two halves over a quarter set of views: views first .. first+count-1
 * and the same views of the other three quarters (view n + k*NumProj/4,
 * k = 1, 2, 3), first + count <= NumProj/4, for plans whose views come in
 * quarter turns (recon_plan_quarter_turns).  A split of the views between
 * devices by quarter sets keeps the quarter-turn gather on every device,
 * where a split into contiguous view ranges gives it up.  forward: as
 * recon_mlem_forward over the four ranges (d_g holds all NumProj views);
 * backward: d_ht = sum over the set of BP(ratio) (overwritten), plans with
 * recon_plan_quarter_turns = 2 only (RECON_ERR_UNSUPPORTED otherwise).  No
 * counterpart in the reference. */
recon_status_t recon_mlem_forward_quarters(recon_plan_t plan, const void* d_g, const float* d_f,
                                           unsigned int first, unsigned int count, void* stream);
recon_status_t recon_mlem_backward_quarters(recon_plan_t plan, unsigned int first, unsigned int count,
                                            float* d_ht, void* stream);
/* backward over all views with the update fused into it (no Ht buffer):
 * recon_mlem_forward(all views) followed by this is one recon_mlem_iteration. */
recon_status_t recon_mlem_backward_update(recon_plan_t plan, float* d_f, void* stream);

/* OSEM (ordered-subset EM) from d_f (or f = 1 with init_ones): `iters` full
 * passes over n_subsets contiguous subsets of NumProj / n_subsets views each;
 * per subset s, f <- f * BP_s(g / FP_s(f)) / BP_s(1) with MLEM's zero guards.
 * The reference stops at the parameter structs osem_input_values /
 * osem_subset_inputs and their check check_recon_inputs
 * (hf_cpp_functions.hpp:298-375): n_subsets must divide NumProj
 * (RECON_ERR_INVALID_ARGUMENT otherwise) and a subset is a contiguous arc of
 * views.  With n_subsets = 1 this is recon_mlem, bit for bit.  EXACT
 * arithmetic, Siddon back projector; the per-subset sensitivities are
 * computed on the first call for a subset count and cached in the plan. */
recon_status_t recon_osem(recon_plan_t plan, const void* d_g, unsigned int iters, unsigned int n_subsets,
                          float* d_f, int init_ones, void* stream);

/* ---- batches of independent reconstructions ------------------------------ */

/* Many MLEM problems (each its own geometry) run together: one iteration of
 * every problem is captured once as a CUDA graph whose parallel branches share
 * the problems out (largest first), and replayed once per iteration.  The
 * reference has no batch entry point; it is the loop a user writes around
 * siddon_recon::a0_RECON_MLEM (hf_siddon_recon.hpp:91-108) over many scans.
 * Each problem's result is bit-identical to recon_mlem on a plan of the same
 * geometry and options.  EXACT arithmetic, Siddon back projector, FP32
 * sinograms only. */
typedef struct recon_batch* recon_batch_t;
recon_status_t recon_batch_create(const recon_geometry_t* geoms, int n, const recon_options_t* opt,
                                  recon_batch_t* batch);
void recon_batch_destroy(recon_batch_t batch);
/* d_g[p] / d_f[p]: problem p's sinogram [NumProj][Nv][Nu] and image
 * [Z][Y][X] on the batch's device.  The first call times graphs of 1, 2, 4
 * and 8 branches on the caller's data (the images are restored) and
 * synchronises; later calls are asynchronous on `stream` (a call with other
 * buffers than the previous one captures the graph again). */
recon_status_t recon_batch_mlem(recon_batch_t batch, const float* const* d_g, float* const* d_f,
                                unsigned int iters, int init_ones, void* stream);

/* Number of (ray, voxel) pairs with positive intersection length over all
 * NumProj views (EXACT arithmetic): the I of the throughput figure
 * "ray-voxel intersections per second".  Synchronous. */
recon_status_t recon_count_intersections(recon_plan_t plan, unsigned long long* count);
/* The same count as one projector of the plan produces it: the (ray, voxel)
 * pairs that the forward projector (projector = RECON_PROJECTOR_FORWARD) or
 * the Siddon back projector (RECON_PROJECTOR_BACK) gives a positive length.
 * Equal to recon_count_intersections when no projector drops or adds a pair;
 * where a projector is the ray walk itself (the ray-driven back projector, or
 * the forward walk where the detector-column forward projector does not
 * apply) it is that count.  EXACT arithmetic, synchronous.  A parity check
 * with no counterpart in the reference. */
#define RECON_PROJECTOR_FORWARD 0
#define RECON_PROJECTOR_BACK 1
recon_status_t recon_count_projector_pairs(recon_plan_t plan, int projector, unsigned long long* count);

/* ---- elementwise drop-ins (hf_cuda_kernels.cuh) -------------------------- */

/* set_ones (hf_cuda_kernels.cuh:25-35) */
recon_status_t recon_set_ones(float* d, size_t n, void* stream);
/* divide1<float> (hf_cuda_kernels.cuh:370-387): num = den != 0 ? num/den : 0 */
recon_status_t recon_divide1(float* d_num, const float* d_den, size_t n, void* stream);
/* multiply1<float> (hf_cuda_kernels.cuh:409-421): a = a*b */
recon_status_t recon_multiply1(float* d_a, const float* d_b, size_t n, void* stream);
/* siddon_add_bp / siddon_add (siddon_kernelsMLEM.cuh:46-74): a = a + b */
recon_status_t recon_add(float* d_a, const float* d_b, size_t n, void* stream);

/* ---- parity / diagnostics (COMPAT arithmetic) ---------------------------- */

/* Per-ray state after siddon_alpha_limits (siddon_kernelsMLEM.cuh:103-149)
 * for every ray of a view, copied to host arrays laid out like
 * siddon_commons (hf_siddon_class.hpp:20-34); float3 arrays are [n][3].
 * Returns loopN (max delta_index) in *loopN. */
recon_status_t recon_compat_setup_view(recon_plan_t plan, float angle_deg, float* alpha_min,
                                       float* alpha_max, float* d12, unsigned int* mask,
                                       float* alpha_i, float* alpha_f, float* delta_alpha,
                                       float* p1, float* p2, unsigned int* delta_index,
                                       unsigned int* loopN);
/* Per-step (voxel index, length) records of rays[0..nrays-1] (pixel indices
 * u + v*AxPixels) at one view: records[ray][step] for steps 0..cap_steps-1;
 * steps past the ray's fixed point and past loopN hold (-1, 0); the record
 * after the last traversal step is the end segment (siddon_bp_end).  The
 * record layout matches the reference's back-projection step kernels driven
 * with an all-ones image. */
recon_status_t recon_compat_trace(recon_plan_t plan, float angle_deg, int nrays, const int* rays,
                                  int cap_steps, int* idx_out, float* len_out,
                                  unsigned int* loopN);

/* loopN of a view: the largest per-ray step count delta_index of the
 * reference's set-up (siddon_commons::a_calc_initial_limits,
 * hf_siddon_class.hpp:93-106), for any plan.  Synchronous. */
recon_status_t recon_view_step_count(recon_plan_t plan, float angle_deg, unsigned int* loopN);

/* ---- allocation-free back projection ------------------------------------ */

/* COMPAT back projection of one view without any device allocation, for
 * callers that may not allocate device memory (no plan is needed): d_vol =
 * BP(d_img) at angle_deg, bit-identical to recon_bp_view on a COMPAT plan of
 * the same geometry.  No reference counterpart: the reference's backward
 * class allocates its buffers in a1_Binitiate (hf_siddon_class.hpp).
 * Device state lives in one static scratch array per device (about 16 MiB):
 *  - volumes above RECON_NOALLOC_MAX_VOXELS voxels return RECON_ERR_UNSUPPORTED;
 *  - overlapping calls on one device (other streams or host threads) share
 *    the scratch and corrupt each other; calls in one stream are safe;
 *  - the first call on a device looks up the scratch address and keeps it for
 *    the life of the process: make it before capturing a stream into a CUDA
 *    graph, and do not call this entry point after a cudaDeviceReset of that
 *    device (the kept address no longer belongs to the new context).
 * Uses the current device; asynchronous on `stream`. */
#define RECON_NOALLOC_MAX_VOXELS 2097152
recon_status_t recon_compat_bp_view_noalloc(const recon_geometry_t* geom, const float* d_img,
                                            float angle_deg, float* d_vol, void* stream);

/* ---- file-driven drivers (the reference's siddon_recon entry points) ------ */

/* siddon_recon::a0_RECON_MLEM(folder, cfg) (hf_siddon_recon.hpp:91-108):
 * reads the configuration, checks every projection file's size, runs
 * N_iteration MLEM iterations from f = 1 and writes
 * <ReconFileFolder><ReconFileNameRoot>_<it><ReconFileSuffix> after every
 * iteration plus the .info parameter echo.  `folder` may be NULL/"" (then
 * cfg is a full path).  opt may be NULL (defaults).  Two optional keys resume
 * a run (no reference counterpart): InitialVolume = <raw float32 image> starts
 * from that image instead of f = 1, StartIteration = k numbers the first
 * iteration run k (iterations k .. N_iteration-1 run). */
recon_status_t recon_mlem_from_cfg(const char* folder, const char* cfg,
                                   const recon_options_t* opt);
/* siddon_recon::a1_FORWARD_PROJECTION (hf_siddon_recon.hpp:146-163,
 * 515-544): projects <ObjFileFolder><ObjFileName> and writes
 * <ProjFileFolder><ProjFileNameRoot>_<n><ProjFileSuffix> per view. */
recon_status_t recon_forward_projection_from_cfg(const char* folder, const char* cfg,
                                                 const recon_options_t* opt);
/* siddon_recon::a1_BACKWARD_PROJECTION (hf_siddon_recon.hpp:165-182,
 * 546-592): back projects every view file and writes
 * <ProjFileFolder><BpFileNameRoot><BpFileSuffix> (and per view
 * <ProjFileFolder><BpFileNameRoot>_<n><BpFileSuffix> when write_per_angle). */
recon_status_t recon_backward_projection_from_cfg(const char* folder, const char* cfg,
                                                  int write_per_angle,
                                                  const recon_options_t* opt);

#ifdef __cplusplus
}
#endif
#endif
