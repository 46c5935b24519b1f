/*
 * ref_cpu_harness.cpp -- host build of the reference's own Siddon kernels.
 *
 * CHECKER / BASELINE INFRASTRUCTURE.  Built by oracle/build_oracle.py from the
 * reference sources where they lie (no copies), with the prelude
 * oracle/ref_shim/host_cuda/ref_prelude_cpu.h forced in, into
 * oracle/_ref/libref_cpu.so.  Two uses:
 *   - pins the FP32 restatement in siddon_oracle.c (bit-exact, 1 thread);
 *   - is the reference's CPU path that bench.py times (OpenMP threads).
 *
 * The kernels are the reference's (CT_Recon/siddon_kernelsMLEM.cuh,
 * hf_cuda_kernels.cuh).  The per-view orchestration restates
 * forward::a2_fp_per_angle / backward::a2_bp_per_angle
 * (CT_Recon/hf_siddon_class.hpp:195-225, 313-347) and the MLEM driver
 * m_mlem_single_iteration / m_mlem_all_iterations / m_calc_sensitivity
 * (CT_Recon/hf_siddon_recon.hpp:388-511), because those files use the
 * <<< >>> launch syntax a host compiler cannot parse.  Launch shapes follow
 * m_calc_kernel_threads (hf_siddon_recon.hpp:366-386).
 *
 * loopN is passed in by the caller: the reference derives it by converting
 * negative float differences to unsigned (siddon_device_kernelsMLEM.cuh:269),
 * which saturates to 0 on the GPU but wraps on x86; the caller supplies the
 * GPU-semantics value (oracle orc_c_loopN) so the host run performs the same
 * number of steps as the device would.
 */
#include "siddon_kernelsMLEM.cuh"

#include <cstdlib>
#include <vector>

#include "siddon_oracle.h"

thread_local uint3 threadIdx;
thread_local uint3 blockIdx;
thread_local dim3 blockDim;
thread_local dim3 gridDim;

static int g_threads = 1;

template <class F>
static void launch(dim3 grid, dim3 block, F&& body)
{
    const long nb = (long)grid.x * grid.y * grid.z;
#pragma omp parallel for schedule(static) num_threads(g_threads) if (g_threads > 1)
    for (long b = 0; b < nb; ++b) {
        gridDim = grid;
        blockDim = block;
        blockIdx.x = (unsigned)(b % grid.x);
        blockIdx.y = (unsigned)((b / grid.x) % grid.y);
        blockIdx.z = (unsigned)(b / ((long)grid.x * grid.y));
        for (unsigned tz = 0; tz < block.z; ++tz)
            for (unsigned ty = 0; ty < block.y; ++ty)
                for (unsigned tx = 0; tx < block.x; ++tx) {
                    threadIdx.x = tx;
                    threadIdx.y = ty;
                    threadIdx.z = tz;
                    body();
                }
    }
}

namespace {

/* siddon_commons (CT_Recon/hf_siddon_class.hpp:18-133) state, host-resident. */
struct RefState {
    XraySystem sys;
    int Npix = 0, V = 0;
    dim3 bimg, timg, bobj, tobj, batom, tatom;
    std::vector<float> alpha_min, alpha_max, d12, current, next, RM;
    std::vector<unsigned int> mask, delta_index;
    std::vector<float3> alpha_i, alpha_f, alpha, delta_alpha, p1, p2;
    std::vector<int3> index;

    explicit RefState(const orc_geom* g)
    {
        CalibrationParam cp;
        cp.R = g->R; cp.Rf = g->Rf; cp.Ry = g->Ry; cp.Dx = g->Dx; cp.Dz = g->Dz;
        cp.xangle = g->xangle; cp.yangle = g->yangle; cp.zangle = g->zangle; cp.M = g->M;
        Detector det;
        det.NumTAxPixels = g->NumTAxPixels; det.NumAxPixels = g->NumAxPixels;
        det.TAxPixDimMm = g->TAxPixDimMm; det.AxPixDimMm = g->AxPixDimMm;
        VoxVolParam vox;
        vox.Xdim = g->Xdim; vox.Ydim = g->Ydim; vox.Zdim = g->Zdim;
        vox.XVoxSize = g->XVoxSize; vox.YVoxSize = g->YVoxSize; vox.ZVoxSize = g->ZVoxSize;
        /* siddon_commons::a1_initiate (hf_siddon_class.hpp:43-61) */
        Planes Pi, Pf, Pd, Xs;
        Pi.fill(-(float)vox.Xdim / 2.0f * (float)vox.XVoxSize, -(float)vox.Ydim / 2.0f * (float)vox.YVoxSize,
                -(float)vox.Zdim / 2.0f * (float)vox.ZVoxSize);
        Pf.fill((float)vox.Xdim / 2.0f * (float)vox.XVoxSize, (float)vox.Ydim / 2.0f * (float)vox.YVoxSize,
                (float)vox.Zdim / 2.0f * (float)vox.ZVoxSize);
        Pd.fill(vox.XVoxSize, vox.YVoxSize, vox.ZVoxSize);
        Xs.fill(0.0f, (-cp.Rf), 0.0f);
        sys.create(cp, det, vox, Pi, Pf, Pd, Xs);
        Npix = (int)(det.NumAxPixels * det.NumTAxPixels);
        V = (int)(vox.Xdim * vox.Ydim * vox.Zdim);
        alpha_min.resize(Npix); alpha_max.resize(Npix); d12.resize(Npix);
        current.resize(Npix); next.resize(Npix); mask.resize(Npix); delta_index.resize(Npix);
        alpha_i.resize(Npix); alpha_f.resize(Npix); alpha.resize(Npix); delta_alpha.resize(Npix);
        p1.resize(Npix); p2.resize(Npix); index.resize(Npix);
        RM.resize(9);
        orc_rotation_matrix(cp.xangle, cp.yangle, cp.zangle, RM.data());
        /* m_calc_kernel_threads (hf_siddon_recon.hpp:366-386); the scatter
         * grid holds one thread per element so the host order is the
         * element order. */
        timg = dim3(4, 4);
        bimg = dim3(det.NumAxPixels / 4, det.NumTAxPixels / 4);
        tobj = dim3(4, 4, 4);
        bobj = dim3(vox.Xdim / 4, vox.Ydim / 4, vox.Zdim / 4);
        tatom = dim3(256);
        batom = dim3((unsigned)((Npix + 255) / 256));
    }

    unsigned limits(float angle)
    {
        /* siddon_commons::a_calc_initial_limits (hf_siddon_class.hpp:93-106) */
        float* RMp = RM.data();
        XraySystem s = sys;
        launch(bimg, timg, [&] {
            siddon_alpha_limits(alpha_min.data(), alpha_max.data(), mask.data(), d12.data(),
                                alpha_i.data(), alpha_f.data(), delta_alpha.data(),
                                delta_index.data(), RMp, angle, s, p1.data(), p2.data());
        });
        unsigned mx = 0;
        for (unsigned d : delta_index) mx = std::max(mx, d);
        return mx;
    }
};

}  // namespace

extern "C" {

void ref_cpu_set_threads(int n) { g_threads = n > 0 ? n : 1; }

/* Per-ray setup arrays after siddon_alpha_limits; returns the reference's
 * own max(delta_index) (host conversion semantics). */
unsigned ref_cpu_setup(const orc_geom* g, float angle, float* alpha_min, float* alpha_max,
                       float* d12, unsigned* mask, float* alpha_i, float* alpha_f,
                       float* delta_alpha, float* p1, float* p2, unsigned* delta_index)
{
    RefState st(g);
    unsigned mx = st.limits(angle);
    for (int n = 0; n < st.Npix; ++n) {
        alpha_min[n] = st.alpha_min[n];
        alpha_max[n] = st.alpha_max[n];
        d12[n] = st.d12[n];
        mask[n] = st.mask[n];
        delta_index[n] = st.delta_index[n];
        const float3* src[5] = {&st.alpha_i[n], &st.alpha_f[n], &st.delta_alpha[n], &st.p1[n], &st.p2[n]};
        float* dst[5] = {alpha_i, alpha_f, delta_alpha, p1, p2};
        for (int k = 0; k < 5; ++k) {
            dst[k][3 * n + 0] = src[k]->x;
            dst[k][3 * n + 1] = src[k]->y;
            dst[k][3 * n + 2] = src[k]->z;
        }
    }
    return mx;
}

/* forward::a2_fp_per_angle (hf_siddon_class.hpp:195-225) */
void ref_cpu_fp_view(const orc_geom* g, float angle, unsigned loopN, const float* vol_in, float* img)
{
    RefState st(g);
    st.limits(angle);
    std::vector<float> vol(vol_in, vol_in + st.V);
    std::vector<float> tmp(st.Npix, 0.0f), out(st.Npix, 0.0f);
    XraySystem s = st.sys;
    launch(st.bimg, st.timg, [&] {
        siddon_begin(st.alpha_min.data(), st.alpha.data(), st.alpha_i.data(), st.mask.data(), st.next.data());
    });
    for (unsigned i = 0; i < loopN; ++i) {
        std::fill(tmp.begin(), tmp.end(), 0.0f);
        launch(st.bimg, st.timg, [&] {
            siddon_sort_alpha(st.alpha.data(), st.alpha_i.data(), st.alpha_f.data(), st.delta_alpha.data(),
                              st.current.data(), st.next.data(), st.alpha_max.data(), st.alpha_min.data());
        });
        launch(st.bimg, st.timg, [&] {
            siddon_fp_calc_ray_path(s, st.p1.data(), st.p2.data(), st.index.data(), st.current.data(),
                                    st.next.data(), st.d12.data(), st.mask.data(), tmp.data(), vol.data());
        });
        launch(st.bimg, st.timg, [&] { siddon_add(out.data(), tmp.data()); });
    }
    std::fill(tmp.begin(), tmp.end(), 0.0f);
    launch(st.bimg, st.timg, [&] {
        siddon_fp_end(st.alpha_max.data(), st.d12.data(), st.mask.data(), s, st.p1.data(), st.p2.data(),
                      st.index.data(), st.current.data(), tmp.data(), vol.data());
    });
    launch(st.bimg, st.timg, [&] { siddon_add(out.data(), tmp.data()); });
    std::copy(out.begin(), out.end(), img);
}

static void bp_view(RefState& st, unsigned loopN, float* img, std::vector<float>& obj)
{
    /* backward::a2_bp_per_angle (hf_siddon_class.hpp:313-347) */
    XraySystem s = st.sys;
    std::vector<float> tmp(st.V + 1, 0.0f);
    std::vector<int> oidx(st.Npix);
    std::vector<float> oval(st.Npix);
    obj.assign(st.V + 1, 0.0f);
    launch(st.bimg, st.timg, [&] {
        siddon_begin(st.alpha_min.data(), st.alpha.data(), st.alpha_i.data(), st.mask.data(), st.next.data());
    });
    for (unsigned i = 0; i < loopN; ++i) {
        std::fill(tmp.begin(), tmp.end(), 0.0f);
        launch(st.bimg, st.timg, [&] {
            siddon_sort_alpha(st.alpha.data(), st.alpha_i.data(), st.alpha_f.data(), st.delta_alpha.data(),
                              st.current.data(), st.next.data(), st.alpha_max.data(), st.alpha_min.data());
        });
        launch(st.bimg, st.timg, [&] {
            siddon_bp_calc_ray_path(s, st.p1.data(), st.p2.data(), st.index.data(), oidx.data(), st.current.data(),
                                    st.next.data(), st.d12.data(), st.mask.data(), img, oval.data());
        });
        launch(st.batom, st.tatom, [&] { kernel(tmp.data(), oidx.data(), oval.data(), st.Npix); });
        launch(st.bobj, st.tobj, [&] { siddon_add_bp(obj.data(), tmp.data()); });
    }
    std::fill(tmp.begin(), tmp.end(), 0.0f);
    launch(st.bimg, st.timg, [&] {
        siddon_bp_end(st.alpha_max.data(), st.d12.data(), st.mask.data(), s, st.p1.data(), st.p2.data(),
                      st.index.data(), oidx.data(), st.current.data(), img, oval.data());
    });
    launch(st.batom, st.tatom, [&] { kernel(tmp.data(), oidx.data(), oval.data(), st.Npix); });
    launch(st.bobj, st.tobj, [&] { siddon_add_bp(obj.data(), tmp.data()); });
}

void ref_cpu_bp_view(const orc_geom* g, float angle, unsigned loopN, const float* img_in, float* vol_out)
{
    RefState st(g);
    st.limits(angle);
    std::vector<float> img(img_in, img_in + st.Npix), obj;
    bp_view(st, loopN, img.data(), obj);
    std::copy(obj.begin(), obj.begin() + st.V, vol_out);
}

/* Per-step (voxel index, value) of the back projection step kernels with an
 * all-ones image (so value = ray length), for a list of rays.  Records are
 * [ray][step], loopN steps then the end segment; index V (pad) -> -1. */
void ref_cpu_trace(const orc_geom* g, float angle, unsigned loopN, int nrays, const int* rays,
                   int* idx_out, float* val_out)
{
    RefState st(g);
    st.limits(angle);
    XraySystem s = st.sys;
    std::vector<float> ones(st.Npix, 1.0f), oval(st.Npix);
    std::vector<int> oidx(st.Npix);
    const int rec = (int)loopN + 1;
    launch(st.bimg, st.timg, [&] {
        siddon_begin(st.alpha_min.data(), st.alpha.data(), st.alpha_i.data(), st.mask.data(), st.next.data());
    });
    auto grab = [&](int k) {
        for (int r = 0; r < nrays; ++r) {
            int n = rays[r];
            idx_out[(size_t)r * rec + k] = (oidx[n] >= st.V) ? -1 : oidx[n];
            val_out[(size_t)r * rec + k] = oval[n];
        }
    };
    for (unsigned i = 0; i < loopN; ++i) {
        launch(st.bimg, st.timg, [&] {
            siddon_sort_alpha(st.alpha.data(), st.alpha_i.data(), st.alpha_f.data(), st.delta_alpha.data(),
                              st.current.data(), st.next.data(), st.alpha_max.data(), st.alpha_min.data());
        });
        launch(st.bimg, st.timg, [&] {
            siddon_bp_calc_ray_path(s, st.p1.data(), st.p2.data(), st.index.data(), oidx.data(), st.current.data(),
                                    st.next.data(), st.d12.data(), st.mask.data(), ones.data(), oval.data());
        });
        grab((int)i);
    }
    launch(st.bimg, st.timg, [&] {
        siddon_bp_end(st.alpha_max.data(), st.d12.data(), st.mask.data(), s, st.p1.data(), st.p2.data(),
                      st.index.data(), oidx.data(), st.current.data(), ones.data(), oval.data());
    });
    grab((int)loopN);
}

/* m_calc_sensitivity + m_mlem_all_iterations (hf_siddon_recon.hpp:388-511)
 * on in-memory projections g[view][pixel]; loopN[view] per view.  f_history
 * (optional) receives f after every iteration, as the reference writes it. */
void ref_cpu_mlem(const orc_geom* g, unsigned NumProj, float DeltaAng, const unsigned* loopN,
                  const float* gsino, unsigned iters, float* f_out, float* sens_out, float* f_history)
{
    RefState st(g);
    const int V = st.V, Npix = st.Npix;
    std::vector<float> f(V), Ht(V), sens(V, 0.0f), gdata(Npix), obj;
    launch(st.bimg, st.timg, [&] { set_ones(gdata.data()); });
    for (unsigned n = 0; n < NumProj; ++n) {
        float angle = DeltaAng * (float)n;
        st.limits(angle);
        bp_view(st, loopN[n], gdata.data(), obj);
        launch(st.bobj, st.tobj, [&] { siddon_add_bp(sens.data(), obj.data()); });
    }
    launch(st.bobj, st.tobj, [&] { set_ones(f.data()); });
    std::vector<float> img(Npix), tmp(Npix);
    XraySystem s = st.sys;
    for (unsigned it = 0; it < iters; ++it) {
        std::fill(Ht.begin(), Ht.end(), 0.0f);
        for (unsigned n = 0; n < NumProj; ++n) {
            float angle = (float)n * DeltaAng;
            std::copy(gsino + (size_t)n * Npix, gsino + (size_t)(n + 1) * Npix, gdata.begin());
            st.limits(angle);
            /* forward::a2_fp_per_angle */
            std::fill(img.begin(), img.end(), 0.0f);
            launch(st.bimg, st.timg, [&] {
                siddon_begin(st.alpha_min.data(), st.alpha.data(), st.alpha_i.data(), st.mask.data(), st.next.data());
            });
            for (unsigned i = 0; i < loopN[n]; ++i) {
                std::fill(tmp.begin(), tmp.end(), 0.0f);
                launch(st.bimg, st.timg, [&] {
                    siddon_sort_alpha(st.alpha.data(), st.alpha_i.data(), st.alpha_f.data(), st.delta_alpha.data(),
                                      st.current.data(), st.next.data(), st.alpha_max.data(), st.alpha_min.data());
                });
                launch(st.bimg, st.timg, [&] {
                    siddon_fp_calc_ray_path(s, st.p1.data(), st.p2.data(), st.index.data(), st.current.data(),
                                            st.next.data(), st.d12.data(), st.mask.data(), tmp.data(), f.data());
                });
                launch(st.bimg, st.timg, [&] { siddon_add(img.data(), tmp.data()); });
            }
            std::fill(tmp.begin(), tmp.end(), 0.0f);
            launch(st.bimg, st.timg, [&] {
                siddon_fp_end(st.alpha_max.data(), st.d12.data(), st.mask.data(), s, st.p1.data(), st.p2.data(),
                              st.index.data(), st.current.data(), tmp.data(), f.data());
            });
            launch(st.bimg, st.timg, [&] { siddon_add(img.data(), tmp.data()); });
            launch(st.bimg, st.timg, [&] { divide1<float>(gdata.data(), img.data()); });
            bp_view(st, loopN[n], gdata.data(), obj);
            launch(st.bobj, st.tobj, [&] { siddon_add_bp(Ht.data(), obj.data()); });
        }
        launch(st.bobj, st.tobj, [&] { multiply1<float>(f.data(), Ht.data()); });
        launch(st.bobj, st.tobj, [&] { divide1<float>(f.data(), sens.data()); });
        if (f_history) std::copy(f.begin(), f.end(), f_history + (size_t)it * V);
    }
    std::copy(f.begin(), f.end(), f_out);
    if (sens_out) std::copy(sens.begin(), sens.end(), sens_out);
}

/* The first `steps` traversal steps of one view of one MLEM iteration (FP
 * and BP each run `steps` of their loopN step launches, then their end
 * segment), for timing: every step launches the same kernels over all rays
 * and the full volume, so the time of a view scales as (loopN + 1) / (steps
 * + 1) of this. */
void ref_cpu_mlem_view_steps(const orc_geom* g, float angle, unsigned steps, const float* f_in,
                             const float* gview, float* Ht_accum)
{
    RefState st(g);
    st.limits(angle);
    std::vector<float> img(st.Npix), gd(gview, gview + st.Npix), obj;
    ref_cpu_fp_view(g, angle, steps, f_in, img.data());
    launch(st.bimg, st.timg, [&] { divide1<float>(gd.data(), img.data()); });
    bp_view(st, steps, gd.data(), obj);
    launch(st.bobj, st.tobj, [&] { siddon_add_bp(Ht_accum, obj.data()); });
}

/* One view of one MLEM iteration (FP, ratio, BP, accumulate), the unit the
 * CPU baseline is timed on. */
void ref_cpu_mlem_view(const orc_geom* g, float angle, unsigned loopN, const float* f_in,
                       const float* gview, float* Ht_accum)
{
    RefState st(g);
    st.limits(angle);
    std::vector<float> img(st.Npix), gd(gview, gview + st.Npix), obj;
    ref_cpu_fp_view(g, angle, loopN, f_in, img.data());
    launch(st.bimg, st.timg, [&] { divide1<float>(gd.data(), img.data()); });
    bp_view(st, loopN, gd.data(), obj);
    launch(st.bobj, st.tobj, [&] { siddon_add_bp(Ht_accum, obj.data()); });
}

}  // extern "C"
