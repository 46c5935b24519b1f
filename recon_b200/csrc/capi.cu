// capi.cu -- the C ABI (include/recon_b200.h): plans, projectors, MLEM,
// elementwise drop-ins and the parity entry points.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>

#include "internal.h"

namespace rb {

static thread_local std::string g_last_error;

void set_error(const std::string& msg) { g_last_error = msg; }
recon_status_t fail(recon_status_t code, const std::string& msg)
{
    set_error(msg);
    return code;
}
recon_status_t cuda_fail(cudaError_t e, const char* what)
{
    std::string m = std::string(what) + ": " + cudaGetErrorString(e);
    // clear the sticky-free error state so the next call starts clean
    cudaGetLastError();
    return fail(e == cudaErrorMemoryAllocation ? RECON_ERR_OUT_OF_MEMORY : RECON_ERR_CUDA, m);
}

Plan::~Plan()
{
    int cur = -1;
    cudaGetDevice(&cur);
    if (cur != device) cudaSetDevice(device);
    release_plan_textures(this);
    for (void* p : allocations) cudaFree(p);
    if (cur >= 0 && cur != device) cudaSetDevice(cur);
}

recon_status_t compat_setup_dump(Plan& P, float angle, float* h[10], unsigned* loopN);
recon_status_t compat_trace(Plan& P, float angle, int nrays, const int* rays, int cap, int* idx, float* len,
                            unsigned* loopN_out);

static bool finite_pos(float x) { return std::isfinite(x) && x > 0.0f; }

static recon_status_t validate(const recon_geometry_t& g, const recon_options_t& o)
{
    const auto& c = g.cal;
    const auto& d = g.det;
    const auto& v = g.vox;
    if (!finite_pos(c.R) || !finite_pos(c.Rf) || !finite_pos(c.Ry) || !finite_pos(c.M))
        return fail(RECON_ERR_INVALID_ARGUMENT, "R, Rf, Ry and M must be finite and positive");
    if (!std::isfinite(c.Dx) || !std::isfinite(c.Dz) || !std::isfinite(c.xangle) || !std::isfinite(c.yangle) ||
        !std::isfinite(c.zangle))
        return fail(RECON_ERR_INVALID_ARGUMENT, "misalignment parameters must be finite");
    if (d.NumAxPixels < 2 || d.NumTAxPixels < 2 || !finite_pos(d.AxPixDimMm) || !finite_pos(d.TAxPixDimMm))
        return fail(RECON_ERR_INVALID_ARGUMENT, "detector needs at least 2x2 pixels of positive pitch");
    if (v.Xdim < 1 || v.Ydim < 1 || v.Zdim < 1 || !finite_pos(v.XVoxSize) || !finite_pos(v.YVoxSize) ||
        !finite_pos(v.ZVoxSize))
        return fail(RECON_ERR_INVALID_ARGUMENT, "volume needs at least one voxel of positive size per axis");
    if ((double)v.Xdim * v.Ydim * v.Zdim >= 2147483647.0)
        return fail(RECON_ERR_UNSUPPORTED, "volumes of 2^31 voxels or more are not supported");
    if ((double)d.NumAxPixels * d.NumTAxPixels >= 2147483647.0)
        return fail(RECON_ERR_UNSUPPORTED, "detectors of 2^31 pixels or more are not supported");
    if (g.scan.NumProj > 0 && !std::isfinite(g.scan.DeltaAng))
        return fail(RECON_ERR_INVALID_ARGUMENT, "DeltaAng must be finite");
    if (o.arith != RECON_ARITH_EXACT && o.arith != RECON_ARITH_COMPAT)
        return fail(RECON_ERR_INVALID_ARGUMENT, "unknown arith option");
    if (o.sum != RECON_SUM_KAHAN && o.sum != RECON_SUM_PLAIN) return fail(RECON_ERR_INVALID_ARGUMENT, "unknown sum option");
    if (o.sino != RECON_SINO_F32 && o.sino != RECON_SINO_BF16)
        return fail(RECON_ERR_INVALID_ARGUMENT, "unknown sino option");
    if (o.bp != RECON_BP_SIDDON && o.bp != RECON_BP_VOXEL) return fail(RECON_ERR_INVALID_ARGUMENT, "unknown bp option");
    if (o.voxel_mode != RECON_VOXEL_REFERENCE && o.voxel_mode != RECON_VOXEL_GEOMETRIC)
        return fail(RECON_ERR_INVALID_ARGUMENT, "unknown voxel_mode option");
    if (o.siddon_bp != RECON_SIDDON_BP_AUTO && o.siddon_bp != RECON_SIDDON_BP_GATHER &&
        o.siddon_bp != RECON_SIDDON_BP_RAY && o.siddon_bp != RECON_SIDDON_BP_TUNED)
        return fail(RECON_ERR_INVALID_ARGUMENT, "unknown siddon_bp option");
    if (o.fp_block < -1) return fail(RECON_ERR_INVALID_ARGUMENT, "fp_block must be -1, 0 or a block side");
    if (o.fp_rows != 0 && o.fp_rows != 32 && o.fp_rows != 64 && o.fp_rows != 128)
        return fail(RECON_ERR_INVALID_ARGUMENT, "fp_rows must be 0, 32, 64 or 128");
    if (o.fp_block > 0 && ((v.Xdim + o.fp_block - 1) / o.fp_block) * ((v.Ydim + o.fp_block - 1) / o.fp_block) > 64)
        return fail(RECON_ERR_INVALID_ARGUMENT, "fp_block: more than 64 xy blocks");
    if (o.arith == RECON_ARITH_EXACT) {
        if (c.xangle != 0.0f || c.yangle != 0.0f || c.zangle != 0.0f)
            return fail(RECON_ERR_UNSUPPORTED,
                        "EXACT arithmetic needs zero detector tilt (xangle, yangle, zangle); use COMPAT");
        const double hx = 0.5 * v.Xdim * (double)v.XVoxSize, hy = 0.5 * v.Ydim * (double)v.YVoxSize;
        const double hz = 0.5 * v.Zdim * (double)v.ZVoxSize;
        const double rad = std::sqrt(hx * hx + hy * hy + hz * hz);
        if (rad >= 0.999 * c.Rf || rad >= 0.999 * ((double)c.R - c.Rf))
            return fail(RECON_ERR_UNSUPPORTED, "EXACT arithmetic needs source and detector outside the volume");
        if (o.sino == RECON_SINO_BF16 && o.bp == RECON_BP_VOXEL)
            return fail(RECON_ERR_UNSUPPORTED, "BF16 sinograms are used with the Siddon back projector only");
    } else if (o.sino == RECON_SINO_BF16) {
        return fail(RECON_ERR_UNSUPPORTED, "BF16 sinograms are used with EXACT arithmetic only");
    }
    return RECON_OK;
}

static void host_rotation_matrix(float tx, float ty, float tz, float RM[9])
{
    // rotation_matrix3D (CT_Recon/hf_cuda_functions.cuh:66-88), float trig
    RM[0] = cosf(ty) * cosf(tz) - sinf(ty) * sinf(tx) * sinf(tz);
    RM[1] = -cosf(tx) * sinf(tz);
    RM[2] = -cosf(tz) * sinf(ty) - cosf(ty) * sinf(tx) * sinf(tz);
    RM[3] = cosf(tz) * sinf(ty) * sinf(tx) + cosf(ty) * sinf(tz);
    RM[4] = cosf(tx) * cosf(tz);
    RM[5] = cosf(ty) * cosf(tz) * sinf(tx) - sinf(ty) * sinf(tz);
    RM[6] = cosf(tx) * sinf(ty);
    RM[7] = -sinf(tx);
    RM[8] = cosf(ty) * cosf(tx);
}

static void fill_geoms(Plan& P)
{
    const recon_geometry_t& g = P.geom;
    CompatGeom& C = P.cg;
    C.R = g.cal.R;
    C.Rf = g.cal.Rf;
    C.Ry = g.cal.Ry;
    C.Dx = g.cal.Dx;
    C.Dz = g.cal.Dz;
    C.M = g.cal.M;
    C.NumAxPixels_f = (float)g.det.NumAxPixels;
    C.NumTAxPixels_f = (float)g.det.NumTAxPixels;
    C.AxPixDimMm = g.det.AxPixDimMm;
    C.TAxPixDimMm = g.det.TAxPixDimMm;
    // siddon_commons::a1_initiate (hf_siddon_class.hpp:51-54)
    C.Pi[0] = -(float)g.vox.Xdim / 2.0f * (float)g.vox.XVoxSize;
    C.Pi[1] = -(float)g.vox.Ydim / 2.0f * (float)g.vox.YVoxSize;
    C.Pi[2] = -(float)g.vox.Zdim / 2.0f * (float)g.vox.ZVoxSize;
    C.Pf[0] = (float)g.vox.Xdim / 2.0f * (float)g.vox.XVoxSize;
    C.Pf[1] = (float)g.vox.Ydim / 2.0f * (float)g.vox.YVoxSize;
    C.Pf[2] = (float)g.vox.Zdim / 2.0f * (float)g.vox.ZVoxSize;
    C.Pd[0] = g.vox.XVoxSize;
    C.Pd[1] = g.vox.YVoxSize;
    C.Pd[2] = g.vox.ZVoxSize;
    C.Xs[0] = 0.0f;
    C.Xs[1] = -g.cal.Rf;
    C.Xs[2] = 0.0f;
    for (int k = 0; k < 9; ++k) C.RM[k] = P.RM[k];
    C.dims[0] = (int)g.vox.Xdim;
    C.dims[1] = (int)g.vox.Ydim;
    C.dims[2] = (int)g.vox.Zdim;
    C.Nu = (int)g.det.NumAxPixels;
    C.Nv = (int)g.det.NumTAxPixels;

    ExactGeom& E = P.eg;
    E.X = C.dims[0];
    E.Y = C.dims[1];
    E.Z = C.dims[2];
    E.Nu = C.Nu;
    E.Nv = C.Nv;
    E.vox[0] = g.vox.XVoxSize;
    E.vox[1] = g.vox.YVoxSize;
    E.vox[2] = g.vox.ZVoxSize;
    for (int k = 0; k < 3; ++k) E.P0[k] = (float)(-(double)C.dims[k] / 2.0 * (double)E.vox[k]);
    E.R = g.cal.R;
    E.Rf = g.cal.Rf;
    E.Ry = g.cal.Ry;
    E.Dx = g.cal.Dx;
    E.Dz = g.cal.Dz;
    const double du = (double)g.det.AxPixDimMm * g.cal.M, dv = (double)g.det.TAxPixDimMm * g.cal.M;
    E.du = (float)du;
    E.dv = (float)dv;
    E.ud0 = (float)(-((double)C.Nu - 1.0) / 2.0 * du);
    E.vd0 = (float)(-((double)C.Nv - 1.0) / 2.0 * dv);
}

static recon_status_t use_device(const Plan& P)
{
    int cur = -1;
    RB_CUDA(cudaGetDevice(&cur));
    if (cur != P.device) RB_CUDA(cudaSetDevice(P.device));
    return RECON_OK;
}

// Index of a plan view whose angle equals `angle` exactly, else -1.
static int view_of_angle(const Plan& P, float angle)
{
    for (unsigned n = 0; n < P.nviews; ++n)
        if (P.view_angles[n] == angle) return (int)n;
    return -1;
}

recon_status_t ensure_mlem_buffers(Plan& P)
{
    if (!P.d_sens) RB_CHECK(P.alloc(&P.d_sens, P.nvox, "sensitivity"));
    if (!P.d_ratio) {
        const size_t es = (P.opt.sino == RECON_SINO_BF16) ? 2 : 4;
        const size_t n = (size_t)P.nviews * column_view_elems(P);
        char* q = nullptr;
        RB_CHECK(P.alloc(&q, n * es, "ratio sinogram"));
        // zero outside the ray blocks the forward projector writes (EXACT culling)
        RB_CUDA(cudaMemset(q, 0, n * es));
        P.d_ratio = q;
        if (P.opt.arith == RECON_ARITH_EXACT && !P.fp_column && (mlem_ratio_in_columns(P) || voxel_ratio_in_columns(P))) {
            RB_CHECK(P.alloc(&q, n * es, "ratio sinogram (staging)"));
            RB_CUDA(cudaMemset(q, 0, n * es));
            P.d_ratio_rm = q;
        }
    }
    // block sums of the column forward projector where the ratio cannot hold
    // them (allocated here, before any graph capture of an iteration)
    if (P.opt.arith == RECON_ARITH_EXACT && P.fp_column && P.col_block > 0 && !P.d_col_acc) {
        const bool in_place = P.opt.sino == RECON_SINO_F32 && !P.col_pairs &&
                              (mlem_ratio_in_columns(P) || voxel_ratio_in_columns(P));
        if (!in_place) RB_CHECK(P.alloc(&P.d_col_acc, (size_t)P.nviews * P.npix, "column block sums"));
    }
    return RECON_OK;
}

recon_status_t plain_fp_ratio(Plan& P, const float* vol, const float* g, float* ratio, cudaStream_t s)
{
    if (P.opt.arith == RECON_ARITH_COMPAT) return compat_fp_ratio_all(P, vol, g, ratio, s);
    return exact_fp_plain_ratio(P, vol, g, ratio, s);
}

recon_status_t compute_sensitivity(Plan& P, float* sens, cudaStream_t s)
{
    if (P.opt.bp == RECON_BP_VOXEL)
        return voxel_bp(P, nullptr, 0, P.nviews, false, 0.0f, P.nviews, P.opt.voxel_mode, true, sens, nullptr,
                        nullptr, s);
    if (P.opt.arith == RECON_ARITH_COMPAT) return compat_sensitivity(P, sens, s);
    return exact_bp(P, nullptr, false, false, 0, P.nviews, false, true, sens, nullptr, nullptr, s);
}

}  // namespace rb

using namespace rb;

extern "C" {

int recon_abi_version(void) { return RECON_B200_ABI_VERSION; }

const char* recon_last_error(void) { return g_last_error.c_str(); }

recon_status_t recon_default_options(recon_options_t* opt)
{
    if (!opt) return fail(RECON_ERR_INVALID_ARGUMENT, "opt is NULL");
    opt->arith = RECON_ARITH_EXACT;
    opt->sum = RECON_SUM_KAHAN;
    opt->sino = RECON_SINO_F32;
    opt->bp = RECON_BP_SIDDON;
    opt->voxel_mode = RECON_VOXEL_GEOMETRIC;
    opt->device = 0;
    opt->siddon_bp = RECON_SIDDON_BP_AUTO;
    opt->fp_block = 0;
    opt->fp_rows = 0;
    return RECON_OK;
}

recon_status_t recon_plan_create(const recon_geometry_t* geom, const recon_options_t* opt_in, recon_plan_t* out)
{
    if (!geom || !out) return fail(RECON_ERR_INVALID_ARGUMENT, "geom and plan must not be NULL");
    *out = nullptr;
    recon_options_t opt;
    if (opt_in) opt = *opt_in;
    else recon_default_options(&opt);
    RB_CHECK(validate(*geom, opt));
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev == 0) {
        cudaGetLastError();
        return fail(RECON_ERR_NO_DEVICE, std::string("no CUDA device: ") + cudaGetErrorString(e));
    }
    if (opt.device < 0 || opt.device >= ndev) return fail(RECON_ERR_INVALID_ARGUMENT, "device ordinal out of range");
    recon_plan* P = new recon_plan();
    P->geom = *geom;
    P->opt = opt;
    P->device = opt.device;
    recon_status_t st = [&]() -> recon_status_t {
        RB_CUDA(cudaSetDevice(P->device));
        RB_CUDA(cudaDeviceGetAttribute(&P->sm_count, cudaDevAttrMultiProcessorCount, P->device));
        P->npix = (size_t)geom->det.NumAxPixels * geom->det.NumTAxPixels;
        P->nvox = (size_t)geom->vox.Xdim * geom->vox.Ydim * geom->vox.Zdim;
        P->nviews = geom->scan.NumProj;
        P->view_angles.resize(P->nviews + 1);
        for (unsigned n = 0; n < P->nviews; ++n) P->view_angles[n] = (float)n * geom->scan.DeltaAng;
        P->view_angles[P->nviews] = 0.0f;
        host_rotation_matrix(geom->cal.xangle, geom->cal.yangle, geom->cal.zangle, P->RM);
        fill_geoms(*P);
        const size_t nv1 = P->nviews + 1;
        RB_CHECK(P->alloc(&P->d_angles, nv1, "angles"));
        RB_CUDA(cudaMemcpy(P->d_angles, P->view_angles.data(), nv1 * sizeof(float), cudaMemcpyHostToDevice));
        RB_CHECK(P->alloc(&P->d_view_img, P->npix, "view image"));
        RB_CHECK(P->alloc(&P->d_loopN, nv1, "loopN"));
        if (opt.arith == RECON_ARITH_EXACT) {
            RB_CHECK(P->alloc(&P->d_txy, nv1 * geom->det.NumAxPixels, "ray table xy"));
            RB_CHECK(P->alloc(&P->d_kxy, nv1 * geom->det.NumAxPixels, "ray table kc"));
            RB_CHECK(P->alloc(&P->d_cs, nv1, "view trig"));
            RB_CHECK(P->alloc(&P->d_zp, geom->det.NumTAxPixels, "ray table z"));
            RB_CHECK(P->alloc(&P->d_w, P->npix, "ray weights"));
            // TUNED: both designs are set up, timed below and the slower one's
            // accumulators released (exact_tune_bp)
            const bool tuned = opt.siddon_bp == RECON_SIDDON_BP_TUNED && P->eg.Nv <= exact_bp_gather_max_rows();
            P->bp_gather = opt.siddon_bp == RECON_SIDDON_BP_GATHER || tuned ||
                           (opt.siddon_bp == RECON_SIDDON_BP_AUTO && exact_bp_gather_suits(*P));
            RB_CHECK(P->alloc(&P->d_wq, P->npix, "ray weights (detector columns)"));
            RB_CUDA(cudaMemset(P->d_wq, 0, P->npix * sizeof(float)));
            if (P->bp_gather && P->eg.Nv > exact_bp_gather_max_rows())
                return fail(RECON_ERR_UNSUPPORTED, "the gather back projector takes at most 12288 detector rows");
            P->fp_column = exact_fp_column_suits(*P);
            if (P->fp_column) {
                const size_t nz = (size_t)P->eg.X * P->eg.Y * (P->eg.Z + 2);
                RB_CHECK(P->alloc(&P->d_vol_z, nz, "z-fastest volume"));
                RB_CUDA(cudaMemset(P->d_vol_z, 0, nz * sizeof(float)));  // the zero layers stay zero
            } else {
                RB_CHECK(P->alloc(&P->d_vol_t, P->nvox, "transposed volume"));
            }
            if (!P->bp_gather || tuned) {  // the ray-driven back projector's slab accumulators
                const size_t slab = (size_t)P->eg.X * P->eg.Y * bp_slab_depth(*P);
                RB_CHECK(P->alloc(&P->d_bpacc, slab, "back projection accumulator"));
                RB_CHECK(P->alloc(&P->d_bpacc_t, slab, "back projection accumulator (transposed)"));
                RB_CHECK(P->alloc(&P->d_bpmax, 1, "back projection max"));
                RB_CUDA(cudaMemset(P->d_bpacc, 0, slab * sizeof(unsigned long long)));
                RB_CUDA(cudaMemset(P->d_bpacc_t, 0, slab * sizeof(unsigned long long)));
            }
            RB_CHECK(build_exact_tables(*P, 0));
            RB_CHECK(exact_check_mirror(*P));
            if (tuned) P->bp_gather = false;  // the culling builds the ray design's slab tiles too
            RB_CHECK(build_exact_culling(*P));
            const bool pairs = exact_pairs_suit(*P) && (P->bp_gather || tuned);
            if (pairs) RB_CHECK(build_wq_pairs(*P));
            if (tuned) RB_CHECK(exact_tune_bp(*P));
            P->col_pairs = pairs && P->bp_gather;
            if (tuned && opt.fp_rows == 0) RB_CHECK(exact_tune_fp(*P));
        } else {
            RB_CHECK(P->alloc(&P->d_maxabs, nv1 + 1, "maxabs"));  // per view, scratch slot, all views
            RB_CHECK(P->alloc(&P->d_fix, P->nvox, "fixed-point accumulator"));
            RB_CHECK(P->alloc(&P->d_ht, P->nvox, "Ht"));
            RB_CUDA(cudaMemset(P->d_fix, 0, P->nvox * sizeof(unsigned long long)));
            RB_CHECK(build_compat_tables(*P, 0));
        }
        // the set-up ran on the legacy stream; waiting for that stream alone (not the
        // device) leaves alone other threads' graph captures, which a device-wide
        // synchronisation would invalidate
        RB_CUDA(cudaStreamSynchronize(cudaStreamLegacy));
        return RECON_OK;
    }();
    if (st != RECON_OK) {
        delete P;
        return st;
    }
    *out = P;
    return RECON_OK;
}

void recon_plan_destroy(recon_plan_t plan) { delete plan; }

size_t recon_plan_device_bytes(recon_plan_t plan) { return plan ? plan->device_bytes : 0; }

recon_status_t recon_plan_forward_projector(recon_plan_t plan, int* design)
{
    if (!plan || !design) return fail(RECON_ERR_INVALID_ARGUMENT, "NULL argument");
    if (plan->opt.arith != RECON_ARITH_EXACT)
        return fail(RECON_ERR_UNSUPPORTED, "COMPAT plans have a single forward projector");
    *design = !plan->fp_column ? RECON_FP_RAY_WALK : plan->col_block > 0 ? RECON_FP_COLUMN_BLOCKS : RECON_FP_COLUMNS;
    return RECON_OK;
}

recon_status_t recon_plan_column_rows(recon_plan_t plan, int* rows)
{
    if (!plan || !rows) return fail(RECON_ERR_INVALID_ARGUMENT, "NULL argument");
    *rows = (plan->opt.arith == RECON_ARITH_EXACT && plan->fp_column) ? plan->col_rows : 0;
    return RECON_OK;
}

recon_status_t recon_plan_mirror_pairs(recon_plan_t plan, int* paired)
{
    if (!plan || !paired) return fail(RECON_ERR_INVALID_ARGUMENT, "NULL argument");
    *paired = (plan->opt.arith == RECON_ARITH_EXACT && plan->z_mirror) ? 1 : 0;
    return RECON_OK;
}

recon_status_t recon_plan_quarter_turns(recon_plan_t plan, int* quarter)
{
    if (!plan || !quarter) return fail(RECON_ERR_INVALID_ARGUMENT, "NULL argument");
    *quarter = (plan->opt.arith == RECON_ARITH_EXACT && plan->quarter) ? (exact_quarter_sets(*plan) ? 2 : 1) : 0;
    return RECON_OK;
}

recon_status_t recon_plan_siddon_bp(recon_plan_t plan, int* design)
{
    if (!plan || !design) return fail(RECON_ERR_INVALID_ARGUMENT, "NULL argument");
    if (plan->opt.arith != RECON_ARITH_EXACT)
        return fail(RECON_ERR_UNSUPPORTED, "COMPAT plans have a single back projector");
    *design = plan->bp_gather ? RECON_SIDDON_BP_GATHER : RECON_SIDDON_BP_RAY;
    return RECON_OK;
}

recon_status_t recon_fp_view(recon_plan_t P, const float* d_vol, float angle, float* d_img, void* stream)
{
    if (!P || !d_vol || !d_img) return fail(RECON_ERR_INVALID_ARGUMENT, "NULL argument");
    if (!std::isfinite(angle)) return fail(RECON_ERR_INVALID_ARGUMENT, "angle must be finite");
    RB_CHECK(use_device(*P));
    cudaStream_t s = as_stream(stream);
    const int vw = view_of_angle(*P, angle);
    if (P->opt.arith == RECON_ARITH_COMPAT) {
        if (vw >= 0) return compat_fp(*P, d_vol, (unsigned)vw, 1, false, 0.0f, d_img, s);
        return compat_fp(*P, d_vol, 0, 1, true, angle, d_img, s);
    }
    if (vw >= 0) return exact_fp(*P, d_vol, (unsigned)vw, 1, false, d_img, s);
    RB_CHECK(exact_view_table(*P, angle, s));
    return exact_fp(*P, d_vol, 0, 1, true, d_img, s);
}

recon_status_t recon_fp_views(recon_plan_t P, const float* d_vol, unsigned first, unsigned count, float* d_sino,
                              void* stream)
{
    if (!P || !d_vol || !d_sino) return fail(RECON_ERR_INVALID_ARGUMENT, "NULL argument");
    if ((size_t)first + count > P->nviews) return fail(RECON_ERR_INVALID_ARGUMENT, "view range beyond NumProj");
    RB_CHECK(use_device(*P));
    cudaStream_t s = as_stream(stream);
    if (P->opt.arith == RECON_ARITH_COMPAT) return compat_fp(*P, d_vol, first, count, false, 0.0f, d_sino, s);
    return exact_fp(*P, d_vol, first, count, false, d_sino, s);
}

recon_status_t recon_bp_view(recon_plan_t P, const float* d_img, float angle, float* d_vol, void* stream)
{
    if (!P || !d_img || !d_vol) return fail(RECON_ERR_INVALID_ARGUMENT, "NULL argument");
    if (!std::isfinite(angle)) return fail(RECON_ERR_INVALID_ARGUMENT, "angle must be finite");
    RB_CHECK(use_device(*P));
    cudaStream_t s = as_stream(stream);
    const int vw = view_of_angle(*P, angle);
    if (P->opt.arith == RECON_ARITH_COMPAT) {
        if (vw >= 0) return compat_bp_view(*P, d_img, (unsigned)vw, false, 0.0f, d_vol, false, s);
        return compat_bp_view(*P, d_img, 0, true, angle, d_vol, false, s);
    }
    if (vw >= 0) return exact_bp(*P, d_img, false, false, (unsigned)vw, 1, false, false, d_vol, nullptr, nullptr, s);
    RB_CHECK(exact_view_table(*P, angle, s));
    return exact_bp(*P, d_img, false, false, 0, 1, true, false, d_vol, nullptr, nullptr, s);
}

recon_status_t recon_bp_views(recon_plan_t P, const float* d_sino, unsigned first, unsigned count, float* d_vol,
                              void* stream)
{
    if (!P || !d_sino || !d_vol) return fail(RECON_ERR_INVALID_ARGUMENT, "NULL argument");
    if ((size_t)first + count > P->nviews) return fail(RECON_ERR_INVALID_ARGUMENT, "view range beyond NumProj");
    RB_CHECK(use_device(*P));
    cudaStream_t s = as_stream(stream);
    if (count == 0) return launch_fill(d_vol, 0.0f, P->nvox, s);
    if (P->opt.arith == RECON_ARITH_COMPAT) {
        for (unsigned n = 0; n < count; ++n)
            RB_CHECK(compat_bp_view(*P, d_sino + (size_t)n * P->npix, first + n, false, 0.0f, d_vol, n > 0, s));
        return RECON_OK;
    }
    return exact_bp(*P, d_sino, false, false, first, count, false, false, d_vol, nullptr, nullptr, s);
}

recon_status_t recon_sensitivity(recon_plan_t P, float* d_sens, void* stream)
{
    if (!P || !d_sens) return fail(RECON_ERR_INVALID_ARGUMENT, "NULL argument");
    RB_CHECK(use_device(*P));
    return compute_sensitivity(*P, d_sens, as_stream(stream));
}

recon_status_t recon_voxel_bp_view(recon_plan_t P, const float* d_img, float angle, unsigned Nproj, int mode,
                                   float* d_vol_accum, void* stream)
{
    if (!P || !d_img || !d_vol_accum) return fail(RECON_ERR_INVALID_ARGUMENT, "NULL argument");
    if (mode != RECON_VOXEL_REFERENCE && mode != RECON_VOXEL_GEOMETRIC)
        return fail(RECON_ERR_INVALID_ARGUMENT, "unknown voxel mode");
    if (Nproj == 0) return fail(RECON_ERR_INVALID_ARGUMENT, "Nproj must be positive");
    RB_CHECK(use_device(*P));
    return voxel_bp(*P, d_img, 0, 1, true, angle, Nproj, mode, false, d_vol_accum, nullptr, nullptr,
                    as_stream(stream));
}

recon_status_t recon_march_fp_view(recon_plan_t P, const float* d_vol, float angle, int mode, float* d_img,
                                   void* stream)
{
    if (!P || !d_vol || !d_img) return fail(RECON_ERR_INVALID_ARGUMENT, "NULL argument");
    if (mode != RECON_VOXEL_REFERENCE && mode != RECON_VOXEL_GEOMETRIC)
        return fail(RECON_ERR_INVALID_ARGUMENT, "unknown sampling mode");
    if (!std::isfinite(angle)) return fail(RECON_ERR_INVALID_ARGUMENT, "angle must be finite");
    if (mode == RECON_VOXEL_REFERENCE && P->geom.vox.Ydim < 2)
        return fail(RECON_ERR_INVALID_ARGUMENT, "REFERENCE sampling normalises by (Ydim-1)*YVoxSize: Ydim must be at least 2");
    RB_CHECK(use_device(*P));
    return march_fp_view(*P, d_vol, angle, mode, d_img, as_stream(stream));
}

recon_status_t recon_mlem_prepare(recon_plan_t P, void* stream)
{
    if (!P) return fail(RECON_ERR_INVALID_ARGUMENT, "NULL plan");
    RB_CHECK(use_device(*P));
    RB_CHECK(ensure_mlem_buffers(*P));
    if (!P->sens_valid) {
        RB_CHECK(compute_sensitivity(*P, P->d_sens, as_stream(stream)));
        P->sens_valid = true;
    }
    return RECON_OK;
}

recon_status_t recon_mlem_iteration(recon_plan_t P, const void* d_g, float* d_f, void* stream)
{
    if (!P || !d_g || !d_f) return fail(RECON_ERR_INVALID_ARGUMENT, "NULL argument");
    if (!P->sens_valid || !P->d_ratio) return fail(RECON_ERR_INVALID_ARGUMENT, "call recon_mlem_prepare first");
    RB_CHECK(use_device(*P));
    cudaStream_t s = as_stream(stream);
    if (P->opt.bp == RECON_BP_VOXEL) {
        RB_CHECK(plain_fp_ratio(*P, d_f, static_cast<const float*>(d_g), static_cast<float*>(P->d_ratio), s));
        return voxel_bp(*P, static_cast<const float*>(P->d_ratio), 0, P->nviews, false, 0.0f, P->nviews,
                        P->opt.voxel_mode, false, nullptr, P->d_sens, d_f, s, voxel_ratio_in_columns(*P));
    }
    if (P->opt.arith == RECON_ARITH_COMPAT) return compat_mlem_iteration(*P, static_cast<const float*>(d_g), d_f, s);
    RB_CHECK(exact_fp_ratio(*P, d_f, d_g, P->d_ratio, s, 0, P->nviews));
    return exact_bp(*P, P->d_ratio, true, P->opt.sino == RECON_SINO_BF16, 0, P->nviews, false, false, nullptr,
                    P->d_sens, d_f, s);
}

recon_status_t recon_upload_sinogram(recon_plan_t P, const void* h_g, void* d_g, unsigned first, unsigned count,
                                     size_t* bytes, void* stream)
{
    if (bytes) *bytes = 0;
    if (!P || !h_g || !d_g) return fail(RECON_ERR_INVALID_ARGUMENT, "NULL argument");
    if ((size_t)first + count > P->nviews) return fail(RECON_ERR_INVALID_ARGUMENT, "view range beyond NumProj");
    if (count == 0) return RECON_OK;
    RB_CHECK(use_device(*P));
    const size_t es = P->opt.sino == RECON_SINO_BF16 ? 2 : 4;
    const size_t Nu = P->geom.det.NumAxPixels, Nv = P->geom.det.NumTAxPixels;
    size_t row0 = 0, rows = Nv;
    if (P->opt.arith == RECON_ARITH_EXACT && P->sino_rows_known) {
        if (P->sino_v1 < P->sino_v0) return RECON_OK;  // no ray crosses the volume
        row0 = (size_t)P->sino_v0;
        rows = (size_t)(P->sino_v1 - P->sino_v0 + 1);
    }
    const size_t pitch = Nu * Nv * es, width = rows * Nu * es, off = ((size_t)first * Nv + row0) * Nu * es;
    RB_CUDA(cudaMemcpy2DAsync(static_cast<char*>(d_g) + off, pitch, static_cast<const char*>(h_g) + off, pitch, width,
                              count, cudaMemcpyHostToDevice, as_stream(stream)));
    if (bytes) *bytes = width * count;
    return RECON_OK;
}

static recon_status_t split_ok(recon_plan_t P, unsigned first, unsigned count)
{
    if (!P) return fail(RECON_ERR_INVALID_ARGUMENT, "NULL plan");
    if (P->opt.arith != RECON_ARITH_EXACT || P->opt.bp != RECON_BP_SIDDON)
        return fail(RECON_ERR_UNSUPPORTED, "split iterations need EXACT arithmetic and the Siddon back projector");
    if (!P->sens_valid || !P->d_ratio) return fail(RECON_ERR_INVALID_ARGUMENT, "call recon_mlem_prepare first");
    if ((size_t)first + count > P->nviews) return fail(RECON_ERR_INVALID_ARGUMENT, "view range beyond NumProj");
    return RECON_OK;
}

recon_status_t recon_mlem_forward(recon_plan_t P, const void* d_g, const float* d_f, unsigned first, unsigned count,
                                  void* stream)
{
    RB_CHECK(split_ok(P, first, count));
    if (!d_g || !d_f) return fail(RECON_ERR_INVALID_ARGUMENT, "NULL argument");
    RB_CHECK(use_device(*P));
    return exact_fp_ratio(*P, d_f, d_g, P->d_ratio, as_stream(stream), first, count);
}

recon_status_t recon_mlem_backward(recon_plan_t P, unsigned first, unsigned count, float* d_ht, void* stream)
{
    RB_CHECK(split_ok(P, first, count));
    if (!d_ht) return fail(RECON_ERR_INVALID_ARGUMENT, "NULL argument");
    RB_CHECK(use_device(*P));
    cudaStream_t s = as_stream(stream);
    if (count == 0) return launch_fill(d_ht, 0.0f, P->nvox, s);
    const size_t es = P->opt.sino == RECON_SINO_BF16 ? 2 : 4;
    const void* r = static_cast<const char*>(P->d_ratio) + (size_t)first * column_view_elems(*P) * es;
    return exact_bp(*P, r, true, P->opt.sino == RECON_SINO_BF16, first, count, false, false, d_ht, nullptr, nullptr,
                    s);
}

// Quarter sets: base views first .. first + count - 1 (first + count <= N/4) and
// their turns by one, two and three quarters.
static recon_status_t quarters_ok(recon_plan_t P, unsigned first, unsigned count)
{
    RB_CHECK(split_ok(P, 0, P ? P->nviews : 0));
    if (!P->quarter) return fail(RECON_ERR_UNSUPPORTED, "the plan's views do not come in quarter turns");
    if ((size_t)first + count > P->nviews / 4) return fail(RECON_ERR_INVALID_ARGUMENT, "quarter range beyond NumProj/4");
    return RECON_OK;
}

recon_status_t recon_mlem_forward_quarters(recon_plan_t P, const void* d_g, const float* d_f, unsigned first,
                                           unsigned count, void* stream)
{
    RB_CHECK(quarters_ok(P, first, count));
    if (!d_g || !d_f) return fail(RECON_ERR_INVALID_ARGUMENT, "NULL argument");
    RB_CHECK(use_device(*P));
    const unsigned q = P->nviews / 4;
    for (unsigned r = 0; r < 4 && count > 0; ++r)
        RB_CHECK(exact_fp_ratio(*P, d_f, d_g, P->d_ratio, as_stream(stream), first + r * q, count));
    return RECON_OK;
}

recon_status_t recon_mlem_backward_quarters(recon_plan_t P, unsigned first, unsigned count, float* d_ht,
                                            void* stream)
{
    RB_CHECK(quarters_ok(P, first, count));
    if (!d_ht) return fail(RECON_ERR_INVALID_ARGUMENT, "NULL argument");
    RB_CHECK(use_device(*P));
    return exact_bp_quarters(*P, first, count, d_ht, as_stream(stream));
}

recon_status_t recon_mlem_update(recon_plan_t P, float* d_f, const float* d_ht, void* stream)
{
    if (!P || !d_f || !d_ht) return fail(RECON_ERR_INVALID_ARGUMENT, "NULL argument");
    if (!P->sens_valid) return fail(RECON_ERR_INVALID_ARGUMENT, "call recon_mlem_prepare first");
    RB_CHECK(use_device(*P));
    return launch_update(d_f, d_ht, P->d_sens, P->nvox, P->opt.arith == RECON_ARITH_COMPAT, as_stream(stream));
}

recon_status_t recon_mlem_backward_update(recon_plan_t P, float* d_f, void* stream)
{
    RB_CHECK(split_ok(P, 0, P ? P->nviews : 0));
    if (!d_f) return fail(RECON_ERR_INVALID_ARGUMENT, "NULL argument");
    RB_CHECK(use_device(*P));
    return exact_bp(*P, P->d_ratio, true, P->opt.sino == RECON_SINO_BF16, 0, P->nviews, false, false, nullptr,
                    P->d_sens, d_f, as_stream(stream));
}

recon_status_t recon_osem(recon_plan_t P, const void* d_g, unsigned iters, unsigned n_subsets, float* d_f,
                          int init_ones, void* stream)
{
    if (!P || !d_g || !d_f) return fail(RECON_ERR_INVALID_ARGUMENT, "NULL argument");
    if (P->opt.arith != RECON_ARITH_EXACT || P->opt.bp != RECON_BP_SIDDON)
        return fail(RECON_ERR_UNSUPPORTED, "OSEM needs EXACT arithmetic and the Siddon back projector");
    // check_recon_inputs (hf_cpp_functions.hpp:358-375): the subsets must split the views evenly
    if (n_subsets == 0 || P->nviews == 0 || P->nviews % n_subsets != 0)
        return fail(RECON_ERR_INVALID_ARGUMENT, "The input values does not agree with each other: "
                                                "N_subsets must divide NumProj");
    RB_CHECK(use_device(*P));
    cudaStream_t s = as_stream(stream);
    RB_CHECK(ensure_mlem_buffers(*P));
    const unsigned n = P->nviews / n_subsets;
    if (P->osem_subsets != n_subsets) {
        // per-subset sensitivities BP_s(1), computed once per subset count
        if (P->d_osem_sens) {
            cudaFree(P->d_osem_sens);
            P->allocations.erase(std::find(P->allocations.begin(), P->allocations.end(), (void*)P->d_osem_sens));
            P->device_bytes -= (size_t)P->osem_subsets * P->nvox * sizeof(float);
            P->d_osem_sens = nullptr;
            P->osem_subsets = 0;
        }
        RB_CHECK(P->alloc(&P->d_osem_sens, (size_t)n_subsets * P->nvox, "OSEM subset sensitivities"));
        for (unsigned k = 0; k < n_subsets; ++k)
            RB_CHECK(exact_bp(*P, nullptr, false, false, k * n, n, false, true, P->d_osem_sens + (size_t)k * P->nvox,
                              nullptr, nullptr, s));
        P->osem_subsets = n_subsets;
    }
    if (init_ones) RB_CHECK(launch_fill(d_f, 1.0f, P->nvox, s));
    const bool bf16 = P->opt.sino == RECON_SINO_BF16;
    const size_t es = bf16 ? 2 : 4;
    for (unsigned it = 0; it < iters; ++it)
        for (unsigned k = 0; k < n_subsets; ++k) {
            const unsigned first = k * n;
            RB_CHECK(exact_fp_ratio(*P, d_f, d_g, P->d_ratio, s, first, n));
            const void* r = static_cast<const char*>(P->d_ratio) + (size_t)first * column_view_elems(*P) * es;
            RB_CHECK(exact_bp(*P, r, true, bf16, first, n, false, false, nullptr,
                              P->d_osem_sens + (size_t)k * P->nvox, d_f, s));
        }
    return RECON_OK;
}

recon_status_t recon_view_step_count(recon_plan_t P, float angle, unsigned* loopN)
{
    if (!P || !loopN) return fail(RECON_ERR_INVALID_ARGUMENT, "NULL argument");
    RB_CHECK(use_device(*P));
    RB_CHECK(compat_view_loopN(*P, angle, P->nviews, 0));
    RB_CUDA(cudaMemcpy(loopN, P->d_loopN + P->nviews, sizeof(unsigned), cudaMemcpyDeviceToHost));
    return RECON_OK;
}

recon_status_t recon_count_intersections(recon_plan_t P, unsigned long long* count)
{
    if (!P || !count) return fail(RECON_ERR_INVALID_ARGUMENT, "NULL argument");
    if (P->opt.arith != RECON_ARITH_EXACT) return fail(RECON_ERR_UNSUPPORTED, "counting uses EXACT arithmetic");
    RB_CHECK(use_device(*P));
    return exact_count(*P, count);
}

recon_status_t recon_count_projector_pairs(recon_plan_t P, int projector, unsigned long long* count)
{
    if (!P || !count) return fail(RECON_ERR_INVALID_ARGUMENT, "NULL argument");
    if (P->opt.arith != RECON_ARITH_EXACT) return fail(RECON_ERR_UNSUPPORTED, "counting uses EXACT arithmetic");
    if (projector != RECON_PROJECTOR_FORWARD && projector != RECON_PROJECTOR_BACK)
        return fail(RECON_ERR_INVALID_ARGUMENT, "projector must be RECON_PROJECTOR_FORWARD or RECON_PROJECTOR_BACK");
    RB_CHECK(use_device(*P));
    if (projector == RECON_PROJECTOR_FORWARD && P->fp_column) return exact_fp_column_count(*P, count);
    if (projector == RECON_PROJECTOR_BACK && P->bp_gather) return exact_bp_gather_count(*P, count);
    return exact_count(*P, count);  // the ray walk, which these projectors run
}

recon_status_t recon_mlem(recon_plan_t P, const void* d_g, unsigned iters, float* d_f, int init_ones, void* stream)
{
    if (!P || !d_g || !d_f) return fail(RECON_ERR_INVALID_ARGUMENT, "NULL argument");
    if (P->nviews == 0) return fail(RECON_ERR_INVALID_ARGUMENT, "plan has no views (NumProj = 0)");
    RB_CHECK(recon_mlem_prepare(P, stream));
    cudaStream_t s = as_stream(stream);
    if (init_ones) RB_CHECK(launch_fill(d_f, 1.0f, P->nvox, s));
    for (unsigned it = 0; it < iters; ++it) RB_CHECK(recon_mlem_iteration(P, d_g, d_f, stream));
    return RECON_OK;
}

recon_status_t recon_set_ones(float* d, size_t n, void* stream)
{
    if (!d && n) return fail(RECON_ERR_INVALID_ARGUMENT, "NULL pointer");
    return launch_fill(d, 1.0f, n, as_stream(stream));
}
recon_status_t recon_divide1(float* num, const float* den, size_t n, void* stream)
{
    if ((!num || !den) && n) return fail(RECON_ERR_INVALID_ARGUMENT, "NULL pointer");
    return launch_elementwise(2, num, den, n, as_stream(stream));
}
recon_status_t recon_multiply1(float* a, const float* b, size_t n, void* stream)
{
    if ((!a || !b) && n) return fail(RECON_ERR_INVALID_ARGUMENT, "NULL pointer");
    return launch_elementwise(1, a, b, n, as_stream(stream));
}
recon_status_t recon_add(float* a, const float* b, size_t n, void* stream)
{
    if ((!a || !b) && n) return fail(RECON_ERR_INVALID_ARGUMENT, "NULL pointer");
    return launch_elementwise(0, a, b, n, as_stream(stream));
}

recon_status_t recon_compat_setup_view(recon_plan_t P, float angle, float* alpha_min, float* alpha_max, float* d12,
                                       unsigned* mask, float* alpha_i, float* alpha_f, float* delta_alpha, float* p1,
                                       float* p2, unsigned* delta_index, unsigned* loopN)
{
    if (!P || !alpha_min || !alpha_max || !d12 || !mask || !alpha_i || !alpha_f || !delta_alpha || !p1 || !p2 ||
        !delta_index || !loopN)
        return fail(RECON_ERR_INVALID_ARGUMENT, "NULL argument");
    RB_CHECK(use_device(*P));
    float* h[10] = {alpha_min, alpha_max, d12, (float*)mask, alpha_i, alpha_f, delta_alpha, p1, p2, (float*)delta_index};
    return compat_setup_dump(*P, angle, h, loopN);
}

recon_status_t recon_compat_trace(recon_plan_t P, float angle, int nrays, const int* rays, int cap_steps, int* idx_out,
                                  float* len_out, unsigned* loopN)
{
    if (!P || (!rays && nrays) || !idx_out || !len_out || !loopN || nrays < 0 || cap_steps < 1)
        return fail(RECON_ERR_INVALID_ARGUMENT, "bad argument");
    for (int q = 0; q < nrays; ++q)
        if (rays[q] < 0 || (size_t)rays[q] >= P->npix) return fail(RECON_ERR_INVALID_ARGUMENT, "ray index out of range");
    if (P->opt.arith != RECON_ARITH_COMPAT)
        return fail(RECON_ERR_UNSUPPORTED, "per-step traces are defined for COMPAT arithmetic");
    RB_CHECK(use_device(*P));
    return compat_trace(*P, angle, nrays, rays, cap_steps, idx_out, len_out, loopN);
}

}  // extern "C"

namespace rb {

// Host-side description of a COMPAT geometry in a Plan that owns no device
// memory (sizes, rotation matrix and the CompatGeom kernel parameters), for
// callers that point its device fields at buffers of their own.
recon_status_t describe_compat_geometry(const recon_geometry_t& g, Plan& P)
{
    recon_options_t o;
    recon_default_options(&o);
    o.arith = RECON_ARITH_COMPAT;
    RB_CHECK(validate(g, o));
    P.geom = g;
    P.opt = o;
    P.npix = (size_t)g.det.NumAxPixels * g.det.NumTAxPixels;
    P.nvox = (size_t)g.vox.Xdim * g.vox.Ydim * g.vox.Zdim;
    P.nviews = 0;
    host_rotation_matrix(g.cal.xangle, g.cal.yangle, g.cal.zangle, P.RM);
    fill_geoms(P);
    return RECON_OK;
}

}  // namespace rb
