// batch.cu -- many independent MLEM reconstructions, one CUDA graph per iteration.
//
// Every problem keeps its own plan (tables, culled ray blocks, ratio buffer,
// back-projection accumulators), so problems share no device state.  One
// MLEM iteration of every problem -- the forward projection with the ratio
// fused in, then the back projection with the update fused in, exactly the
// kernels of recon_mlem_forward / recon_mlem_backward_update -- is captured
// once into a CUDA graph whose K parallel branches each run a share of the
// problems; problems go to branches longest first, each to the branch with the
// least work so far, so the branches end together.  Replaying the graph costs
// one launch per iteration for all problems, and small problems, whose kernels
// cannot fill the GPU alone, run concurrently with others.  Each problem's
// image is bit-identical to recon_mlem on its own plan (same kernels, exact
// back-projection sums).  K is picked by timing graph replays on the first
// call (cached per set of shapes for the process); the graph is captured
// again when the caller's buffers change.
#include <algorithm>
#include <map>
#include <memory>
#include <mutex>
#include <numeric>
#include <string>
#include <vector>

#include "internal.h"

using namespace rb;

struct recon_batch {
    std::vector<recon_plan_t> plans;
    std::vector<double> work;  // ray-voxel work estimate per problem
    int device = 0;
    std::string key;
    int branches = 0;  // chosen K
    std::vector<const float*> g;
    std::vector<float*> f;
    std::vector<cudaStream_t> streams;  // origin + branches
    std::vector<cudaEvent_t> events;    // fork / join events of the capture
    cudaEvent_t sync = nullptr;         // orders the caller's stream and the origin
    cudaGraphExec_t exec = nullptr;
    int exec_branches = 0;
    std::vector<const float*> exec_g;
    std::vector<float*> exec_f;

    ~recon_batch()
    {
        if (exec) cudaGraphExecDestroy(exec);
        for (auto e : events) cudaEventDestroy(e);
        if (sync) cudaEventDestroy(sync);
        for (auto s : streams) cudaStreamDestroy(s);
        for (auto p : plans) recon_plan_destroy(p);
    }
};

namespace {

const int kMaxBranches = 8;

// Branch counts picked so far, per set of shapes (process-wide, guarded).
std::mutex g_tune_mutex;
std::map<std::string, int> g_tune_cache;

bool tuned_branches(const std::string& key, int* k)
{
    std::lock_guard<std::mutex> lock(g_tune_mutex);
    auto it = g_tune_cache.find(key);
    if (it == g_tune_cache.end()) return false;
    *k = it->second;
    return true;
}

void remember_branches(const std::string& key, int k)
{
    std::lock_guard<std::mutex> lock(g_tune_mutex);
    g_tune_cache[key] = k;
}

// one MLEM iteration of problem p on stream s
recon_status_t problem_iteration(recon_batch& b, size_t p, cudaStream_t s)
{
    Plan& P = *b.plans[p];
    RB_CHECK(exact_fp_ratio(P, b.f[p], b.g[p], P.d_ratio, s, 0, P.nviews));
    return exact_bp(P, P.d_ratio, true, false, 0, P.nviews, false, false, nullptr, P.d_sens, b.f[p], s);
}

// Problems per branch: longest first, each to the least-loaded branch.
std::vector<std::vector<size_t>> assign(const recon_batch& b, int k)
{
    std::vector<size_t> order(b.plans.size());
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](size_t a, size_t c) { return b.work[a] > b.work[c]; });
    std::vector<std::vector<size_t>> out(k);
    std::vector<double> load(k, 0.0);
    for (size_t p : order) {
        const int j = (int)(std::min_element(load.begin(), load.end()) - load.begin());
        out[j].push_back(p);
        load[j] += b.work[p];
    }
    return out;
}

recon_status_t capture(recon_batch& b, int k)
{
    if (b.exec) {
        cudaGraphExecDestroy(b.exec);
        b.exec = nullptr;
    }
    const auto groups = assign(b, k);
    cudaStream_t origin = b.streams[0];
    cudaGraph_t graph = nullptr;
    RB_CUDA(cudaStreamBeginCapture(origin, cudaStreamCaptureModeThreadLocal));
    recon_status_t st = RECON_OK;
    cudaError_t e = cudaEventRecord(b.events[0], origin);
    for (int j = 0; j < k && e == cudaSuccess && st == RECON_OK; ++j) {
        cudaStream_t s = b.streams[1 + j];
        e = cudaStreamWaitEvent(s, b.events[0], 0);
        for (size_t q = 0; q < groups[j].size() && e == cudaSuccess && st == RECON_OK; ++q)
            st = problem_iteration(b, groups[j][q], s);
        if (e == cudaSuccess && st == RECON_OK) e = cudaEventRecord(b.events[1 + j], s);
        if (e == cudaSuccess && st == RECON_OK) e = cudaStreamWaitEvent(origin, b.events[1 + j], 0);
    }
    const cudaError_t e_end = cudaStreamEndCapture(origin, &graph);
    if (st != RECON_OK || e != cudaSuccess || e_end != cudaSuccess) {
        if (graph) cudaGraphDestroy(graph);
        if (st != RECON_OK) return st;
        return cuda_fail(e != cudaSuccess ? e : e_end, "batch graph capture");
    }
    e = cudaGraphInstantiate(&b.exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) return cuda_fail(e, "batch graph instantiate");
    b.exec_branches = k;
    b.exec_g = b.g;
    b.exec_f = b.f;
    return RECON_OK;
}

// Time two graph replays for each K on the caller's data, restoring the
// images afterwards.
recon_status_t autotune(recon_batch& b)
{
    if (tuned_branches(b.key, &b.branches)) return RECON_OK;
    cudaStream_t origin = b.streams[0];
    size_t total = 0;
    for (auto P : b.plans) total += P->nvox;
    float* save = nullptr;
    RB_CUDA(cudaMalloc(&save, total * sizeof(float)));
    for (size_t p = 0, off = 0; p < b.plans.size(); off += b.plans[p]->nvox, ++p)
        cudaMemcpyAsync(save + off, b.f[p], b.plans[p]->nvox * sizeof(float), cudaMemcpyDeviceToDevice, origin);
    cudaEvent_t e0, e1;
    RB_CUDA(cudaEventCreate(&e0));
    RB_CUDA(cudaEventCreate(&e1));
    float best = 1e30f;
    int pick = 1;
    for (int k = 1; k <= kMaxBranches && k <= (int)b.plans.size(); k *= 2) {
        if (capture(b, k) != RECON_OK) continue;
        cudaGraphLaunch(b.exec, origin);
        cudaEventRecord(e0, origin);
        cudaGraphLaunch(b.exec, origin);
        cudaGraphLaunch(b.exec, origin);
        cudaEventRecord(e1, origin);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (ms < best) {
            best = ms;
            pick = k;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    for (size_t p = 0, off = 0; p < b.plans.size(); off += b.plans[p]->nvox, ++p)
        cudaMemcpyAsync(b.f[p], save + off, b.plans[p]->nvox * sizeof(float), cudaMemcpyDeviceToDevice, origin);
    cudaStreamSynchronize(origin);
    cudaFree(save);
    RB_CUDA(cudaGetLastError());
    b.branches = pick;
    remember_branches(b.key, pick);
    return RECON_OK;
}

}  // namespace

extern "C" {

recon_status_t recon_batch_create(const recon_geometry_t* geoms, int n, const recon_options_t* opt_in,
                                  recon_batch_t* out)
{
    if (!geoms || n <= 0 || !out) return fail(RECON_ERR_INVALID_ARGUMENT, "need at least one geometry");
    *out = nullptr;
    recon_options_t opt;
    if (opt_in) opt = *opt_in;
    else recon_default_options(&opt);
    if (opt.arith != RECON_ARITH_EXACT || opt.bp != RECON_BP_SIDDON || opt.sino != RECON_SINO_F32)
        return fail(RECON_ERR_UNSUPPORTED, "batches use EXACT arithmetic, the Siddon back projector and FP32 sinograms");
    std::unique_ptr<recon_batch> b(new recon_batch());
    b->device = opt.device;
    std::string key = std::to_string(n) + (opt.sum == RECON_SUM_KAHAN ? "k" : "p") + std::to_string(opt.siddon_bp) +
                      "b" + std::to_string(opt.fp_block) + "r" + std::to_string(opt.fp_rows);
    for (int p = 0; p < n; ++p) {
        if (geoms[p].scan.NumProj == 0) return fail(RECON_ERR_INVALID_ARGUMENT, "every problem needs views");
        recon_plan_t plan = nullptr;
        RB_CHECK(recon_plan_create(&geoms[p], &opt, &plan));
        b->plans.push_back(plan);
        RB_CHECK(recon_mlem_prepare(plan, nullptr));
        const recon_geometry_t& g = geoms[p];
        b->work.push_back((double)g.scan.NumProj * g.det.NumAxPixels * g.det.NumTAxPixels *
                          (double)(g.vox.Xdim + g.vox.Ydim + g.vox.Zdim));
        key += "|" + std::to_string(g.vox.Xdim) + "x" + std::to_string(g.vox.Ydim) + "x" + std::to_string(g.vox.Zdim) +
               "/" + std::to_string(g.scan.NumProj) + "/" + std::to_string(g.det.NumAxPixels) + "x" +
               std::to_string(g.det.NumTAxPixels);
    }
    b->key = key;
    b->g.assign(n, nullptr);
    b->f.assign(n, nullptr);
    RB_CUDA(cudaSetDevice(b->device));
    for (int j = 0; j <= kMaxBranches; ++j) {
        cudaStream_t s = nullptr;
        cudaEvent_t e = nullptr;
        RB_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
        b->streams.push_back(s);
        RB_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        b->events.push_back(e);
    }
    RB_CUDA(cudaEventCreateWithFlags(&b->sync, cudaEventDisableTiming));
    // plans are set up on the legacy stream; a device-wide synchronisation here
    // would invalidate another thread's batch graph capture
    RB_CUDA(cudaStreamSynchronize(cudaStreamLegacy));
    *out = b.release();
    return RECON_OK;
}

void recon_batch_destroy(recon_batch_t b)
{
    if (!b) return;
    cudaSetDevice(b->device);
    delete b;
}

recon_status_t recon_batch_mlem(recon_batch_t b, const float* const* d_g, float* const* d_f, unsigned iters,
                                int init_ones, void* stream)
{
    if (!b || !d_g || !d_f) return fail(RECON_ERR_INVALID_ARGUMENT, "NULL argument");
    const size_t n = b->plans.size();
    for (size_t p = 0; p < n; ++p)
        if (!d_g[p] || !d_f[p]) return fail(RECON_ERR_INVALID_ARGUMENT, "NULL problem buffer");
    RB_CUDA(cudaSetDevice(b->device));
    cudaStream_t s = as_stream(stream), origin = b->streams[0];
    // the work runs on the graph's stream, ordered after the caller's stream
    cudaEvent_t ev = b->sync;
    RB_CUDA(cudaEventRecord(ev, s));
    RB_CUDA(cudaStreamWaitEvent(origin, ev, 0));
    for (size_t p = 0; p < n; ++p) {
        b->g[p] = d_g[p];
        b->f[p] = d_f[p];
        if (init_ones) RB_CHECK(launch_fill(d_f[p], 1.0f, b->plans[p]->nvox, origin));
    }
    if (b->branches == 0) RB_CHECK(autotune(*b));
    if (!b->exec || b->exec_branches != b->branches || b->exec_g != b->g || b->exec_f != b->f)
        RB_CHECK(capture(*b, b->branches));
    for (unsigned it = 0; it < iters; ++it) RB_CUDA(cudaGraphLaunch(b->exec, origin));
    RB_CUDA(cudaEventRecord(ev, origin));
    RB_CUDA(cudaStreamWaitEvent(s, ev, 0));
    return RECON_OK;
}

}  // extern "C"
