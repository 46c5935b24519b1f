// internal.h -- shared declarations of librecon_b200 (not part of the ABI).
#pragma once

#include <cuda_runtime.h>
#include <cuda_bf16.h>

#include <cstdint>
#include <string>
#include <vector>

#include "../../include/recon_b200.h"

namespace rb {

// ---- error plumbing -------------------------------------------------------

void set_error(const std::string& msg);
recon_status_t fail(recon_status_t code, const std::string& msg);
recon_status_t cuda_fail(cudaError_t e, const char* what);

#define RB_CUDA(call)                                            \
    do {                                                         \
        cudaError_t rb_e_ = (call);                              \
        if (rb_e_ != cudaSuccess) return ::rb::cuda_fail(rb_e_, #call); \
    } while (0)
#define RB_CHECK(call)                                   \
    do {                                                 \
        recon_status_t rb_s_ = (call);                   \
        if (rb_s_ != RECON_OK) return rb_s_;             \
    } while (0)

inline cudaStream_t as_stream(void* s) { return reinterpret_cast<cudaStream_t>(s); }

// ---- geometry passed to kernels by value ----------------------------------

// COMPAT arithmetic: the reference's XraySystem (siddon_device_kernelsMLEM.cuh:27-48)
// flattened, plus the 3x3 detector rotation.
struct CompatGeom {
    float R, Rf, Ry, Dx, Dz, M;
    float NumAxPixels_f, NumTAxPixels_f, AxPixDimMm, TAxPixDimMm;
    float Pi[3], Pf[3], Pd[3], Xs[3];
    float RM[9];
    int dims[3];
    int Nu, Nv;
};

// EXACT arithmetic: plane crossings along a ray are parameterised by
// t = R*alpha - Rf, the depth along the view's central axis in mm (alpha is
// the ray parameter from source (0) to detector pixel (1)).  Plane k of an
// axis sits at t(k) = fmaf(float(k - kc), S, O), with S, O, kc set up in FP64
// per ray so that |t| is small where planes cross the volume.  The segment
// length in mm is (t1 - t0) * w with w = |p2 - p1| / R.
struct AxisT {
    float S, O;
    int kc;
};
struct ZParam {  // per detector row v (z planes)
    float S, O, inv_S;
    int kc;
};
struct ExactGeom {
    int X, Y, Z;        // voxels
    int Nu, Nv;         // detector columns (u) / rows (v)
    float vox[3];       // voxel size per axis
    float P0[3];        // first plane per axis (-dim/2*vox)
    float R, Rf, Ry, Dx, Dz;
    float ud0, du;      // detector u coordinate of pixel 0 and pitch (mm, before R/Ry)
    float vd0, dv;
};

// ---- plan -------------------------------------------------------------------

struct DeviceBuf {
    void* p = nullptr;
    size_t bytes = 0;
};

// Blocks of 32 x 4 rays that can cross a box of the volume: tiles
// {view, tu | tv << 16} in view order, prefix[n] = index of view n's first
// tile (prefix has nviews + 1 entries).
// Layouts of a sinogram on the device: rows [view][v][u] (the reference's),
// detector columns [view][u][v], or mirrored row pairs [view][u][p][2] holding
// {row p, row Nv-1-p} for p = 0 .. Nv/2 (even Nv; entry Nv/2 repeats the last
// pair swapped), which the mirror-paired gather reads with one load per pair.
enum : int { kLayoutRows = 0, kLayoutColumns = 1, kLayoutPairs = 2 };

struct RayTiles {
    uint2* d = nullptr;
    std::vector<unsigned> prefix;
};

// Texture objects over a sinogram's views, kept between voxel-driven back
// projections of the same buffer (MLEM reuses its ratio sinogram).
struct TexCache {
    const float* base = nullptr;
    unsigned count = 0;
    cudaTextureObject_t* d_handles = nullptr;
    std::vector<cudaTextureObject_t> handles;
};

struct Plan {
    recon_geometry_t geom{};
    recon_options_t opt{};
    int device = 0;
    int sm_count = 148;
    size_t npix = 0, nvox = 0;
    unsigned nviews = 0;
    std::vector<float> view_angles;  // (float)n * DeltaAng
    float RM[9];

    CompatGeom cg{};
    ExactGeom eg{};

    // EXACT tables (device)
    float4* d_txy = nullptr;   // [view][u] {Sx, Ox, Sy, Oy}
    int2* d_kxy = nullptr;     // [view][u] {kcx, kcy}
    float2* d_cs = nullptr;    // [view] {cos, sin} of the view angle
    ZParam* d_zp = nullptr;    // [v]
    float* d_w = nullptr;      // [v][u] |p2-p1| / R
    float* d_wq = nullptr;     // the same in the detector-column layout [u][v]
    float* d_colsino = nullptr;  // a sinogram in the detector-column layout (gather back projector input)
    unsigned colsino_views = 0;   // views d_colsino holds
    bool bp_gather = false;    // Siddon back projection by the column gather (else ray-driven slabs)
    bool z_mirror = false;     // z table mirror-symmetric about z = 0: both projectors pair mirrored rows/voxels
    bool quarter = false;      // views n + N/4 a quarter turn from view n about a square volume, their xy
                               // tables exact rotations of view n's (the gather serves four columns a warp)
    float* d_vol_t = nullptr;  // xy-transposed copy of the projected volume [z][x][y] (ray-walk forward projector)
    bool fp_column = false;    // forward projection by detector columns (fpcol.cu), else the ray walk
    float* d_vol_z = nullptr;  // z-fastest copy of the projected volume with a zero layer at each end:
                               // voxel (x, y, z) at [(y*X + x)*(Z + 2) + z + 1] (column forward projector)
    // back projection: fixed-point accumulators of one z-slab, image layout
    // and xy-transposed, and the max |value| of the call's input (float bits)
    unsigned long long* d_bpacc = nullptr;
    unsigned long long* d_bpacc_t = nullptr;
    unsigned* d_bpmax = nullptr;
    // ray blocks crossing the volume (forward projection) and each
    // back-projection z-slab; rays outside them contribute nothing
    RayTiles fp_tiles;
    RayTiles col_tiles;           // column forward projector: {view, u | vstart << 16} per CTA
    // column forward projector over xy blocks (volumes larger than L2): block
    // side in voxels (0: one pass over the whole volume), the blocks' tiles,
    // and block sums [nviews][u][v] where the output cannot hold them
    int col_rows = 128;            // detector rows per CTA of the column forward projector (32, 64, 128)
    bool col_pairs = false;        // the gather's inputs in mirrored row pairs (kLayoutPairs)
    float* d_wq_pairs = nullptr;   // d_wq in mirrored row pairs (the sensitivity's input)
    int col_block = 0;
    int col_nbx = 1, col_nby = 1;
    std::vector<RayTiles> col_btiles;
    float* d_col_acc = nullptr;
    int4* d_view_rect = nullptr;  // [view] {u_min, u_max, v_min, v_max} of the rays crossing the volume
    std::vector<int4> view_rect_host;  // the same on the host
    int sino_v0 = 0, sino_v1 = -1;  // rows some ray crossing the volume reaches, over all views
    bool sino_rows_known = false;   // EXACT culling ran: sino_v0..sino_v1 bound every row the plan reads
    std::vector<RayTiles> bp_tiles;
    TexCache tex;  // voxel-driven back projection
    // scratch view slot for arbitrary-angle single-view calls (index nviews)
    float* d_angles = nullptr;    // [view] (float)n*DeltaAng, + 1 scratch slot
    // COMPAT tables
    unsigned* d_loopN = nullptr;  // [view] (+1 scratch slot)
    // workspaces
    float* d_sens = nullptr;      // cached sensitivity
    float* d_osem_sens = nullptr; // OSEM: per-subset sensitivities [osem_subsets][nvox]
    unsigned osem_subsets = 0;
    bool sens_valid = false;
    void* d_ratio = nullptr;      // ratio sinogram (float or bf16) [nviews][npix]
    void* d_ratio_rm = nullptr;   // EXACT gather plans: the ratio as the forward projector writes it,
                                  // [view][v][u], before its transpose into d_ratio
    float* d_ht = nullptr;        // COMPAT: Ht accumulator [nvox]
    unsigned long long* d_fix = nullptr;  // COMPAT: fixed-point accumulator [nvox]
    unsigned* d_maxabs = nullptr; // COMPAT: per-view max |value| bits [nviews+1]
    float* d_view_img = nullptr;  // scratch image [npix]
    size_t device_bytes = 0;
    std::vector<void*> allocations;

    template <class T>
    recon_status_t alloc(T** p, size_t count, const char* what);
    ~Plan();
};

template <class T>
recon_status_t Plan::alloc(T** p, size_t count, const char* what)
{
    void* q = nullptr;
    cudaError_t e = cudaMalloc(&q, count * sizeof(T) > 0 ? count * sizeof(T) : 16);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return fail(e == cudaErrorMemoryAllocation ? RECON_ERR_OUT_OF_MEMORY : RECON_ERR_CUDA,
                    std::string("cudaMalloc(") + what + "): " + cudaGetErrorString(e));
    }
    allocations.push_back(q);
    device_bytes += count * sizeof(T);
    *p = static_cast<T*>(q);
    return RECON_OK;
}

// Elements one view of the gather's input occupies: Nu*Nv in detector columns,
// Nu*(Nv/2 + 1)*2 in mirrored row pairs.
inline size_t column_view_elems(const Plan& P)
{
    if (!P.col_pairs) return P.npix;
    return (size_t)P.geom.det.NumAxPixels * (P.geom.det.NumTAxPixels / 2 + 1) * 2;
}

// ---- entry points implemented in the .cu files --------------------------------

recon_status_t build_compat_tables(Plan& P, cudaStream_t s);
recon_status_t build_exact_tables(Plan& P, cudaStream_t s);
recon_status_t exact_view_table(Plan& P, float angle, cudaStream_t s);  // into slot nviews
recon_status_t compat_view_loopN(Plan& P, float angle, unsigned slot, cudaStream_t s);

// FP: views [first, first+count) (angles from the plan) or the scratch slot.
// mode 0: write projections; mode 1: MLEM ratio (g/Hf, times w for EXACT)
recon_status_t exact_fp(Plan& P, const float* vol, unsigned first, unsigned count, bool scratch_slot,
                        float* out, cudaStream_t s);
recon_status_t exact_fp_ratio(Plan& P, const float* vol, const void* g, void* ratio, cudaStream_t s,
                              unsigned first, unsigned count);
recon_status_t exact_count(Plan& P, unsigned long long* out);
recon_status_t exact_bp_gather_count(Plan& P, unsigned long long* total);
recon_status_t exact_fp_column_count(Plan& P, unsigned long long* total);
// BP gather over views [first, first+count) of `sino` (weighted by w) into vol (overwrite);
// sens_mode: back project ones; update: f = f*Ht/sens in the epilogue.
recon_status_t exact_bp(Plan& P, const void* sino, bool sino_is_rw, bool bf16, unsigned first,
                        unsigned count, bool scratch_slot, bool sens_mode, float* vol,
                        const float* sens, float* f_update, cudaStream_t s);

recon_status_t compat_fp(Plan& P, const float* vol, unsigned first, unsigned count, bool scratch_slot,
                         float angle_scratch, float* out, cudaStream_t s);
recon_status_t compat_bp_view(Plan& P, const float* img, unsigned view, bool scratch_slot,
                              float angle_scratch, float* out_or_accum, bool accumulate,
                              cudaStream_t s);
recon_status_t compat_mlem_iteration(Plan& P, const float* g, float* f, cudaStream_t s);
recon_status_t compat_sensitivity(Plan& P, float* sens, cudaStream_t s);

recon_status_t voxel_bp(Plan& P, const float* sino, unsigned first, unsigned count, bool scratch_slot,
                        float angle_scratch, unsigned Nproj, int mode, bool ones, float* vol_accum,
                        const float* sens, float* f_update, cudaStream_t s, bool columns = false);
recon_status_t plain_fp_ratio(Plan& P, const float* vol, const float* g, float* ratio, cudaStream_t s);
recon_status_t exact_fp_plain_ratio(Plan& P, const float* vol, const float* g, float* ratio, cudaStream_t s);
recon_status_t compat_fp_ratio_all(Plan& P, const float* vol, const float* g, float* ratio, cudaStream_t s);
void release_plan_textures(Plan* P);
recon_status_t ensure_mlem_buffers(Plan& P);
recon_status_t compute_sensitivity(Plan& P, float* sens, cudaStream_t s);
recon_status_t describe_compat_geometry(const recon_geometry_t& g, Plan& P);
recon_status_t exact_transpose(const float* vol, float* vol_t, int X, int Y, int Z, cudaStream_t s);
int bp_count_bits(const Plan& P, unsigned nview);
float bp_max_len(const Plan& P);
int bp_slab_depth(const Plan& P);
bool exact_bp_gather_suits(const Plan& P);
recon_status_t march_fp_view(Plan& P, const float* vol, float angle_deg, int mode, float* img, cudaStream_t s);
int exact_bp_gather_max_rows();
bool voxel_ratio_in_columns(const Plan& P);
int gather_slots(int Z);
// Sinograms read by the gather back projectors are in the detector-column
// layout [view][u][v].
bool mlem_ratio_in_columns(const Plan& P);
recon_status_t build_exact_culling(Plan& P);
bool exact_quarter_sets(const Plan& P);
recon_status_t exact_bp_quarters(Plan& P, unsigned first, unsigned count, float* vol, cudaStream_t s);
recon_status_t exact_check_mirror(Plan& P);
recon_status_t exact_tune_bp(Plan& P);
// forward projection by detector columns (fpcol.cu)
bool exact_fp_column_suits(const Plan& P);
bool exact_pairs_suit(const Plan& P);
recon_status_t exact_tune_fp(Plan& P);
int exact_column_rows_default(const Plan& P, const std::vector<int4>& rect);
std::string geometry_key(const Plan& P);
void plan_release(Plan& P, void* p, size_t bytes);
recon_status_t build_wq_pairs(Plan& P);
recon_status_t build_column_tiles(Plan& P, const std::vector<int4>& rect);
recon_status_t exact_fp_column(Plan& P, const float* vol, unsigned first, unsigned count, float* out, cudaStream_t s);
recon_status_t exact_fp_column_ratio(Plan& P, const float* vol, const void* g, void* ratio, int mode, int layout,
                                     bool bf16, unsigned first, unsigned count, cudaStream_t s);

recon_status_t launch_elementwise(int op, float* a, const float* b, size_t n, cudaStream_t s);
recon_status_t launch_update(float* f, const float* ht, const float* sens, size_t n, bool fast_div,
                             cudaStream_t s);
recon_status_t launch_fill(float* a, float v, size_t n, cudaStream_t s);

}  // namespace rb

// The opaque handle of the C ABI is the plan itself.
struct recon_plan : rb::Plan {};
