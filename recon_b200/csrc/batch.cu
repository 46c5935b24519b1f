// batch.cu -- many independent MLEM reconstructions per launch.
//
// Every iteration of all problems is two persistent kernels (after a
// transpose of every image, which the forward walk reads for some views): the forward
// projection with the ratio fused in, over 32x4-ray tiles of every view of
// every problem, and the gather back projection with the update fused in,
// over (32x4 column block, z-chunk) tiles of every problem.  CTAs pull tile
// indices from an atomic counter; back-projection tiles are ordered by
// decreasing cost (views x rows per chunk), longest first, so the last wave
// is short.  The per-ray and per-column work is the same device code as the
// single-problem kernels (exact_device.cuh), so each problem's result is
// bit-identical to recon_mlem on its own plan.  One iteration (counter reset
// + two launches) is captured once in a CUDA graph and replayed.  The z-chunk
// size and the number of resident CTAs are picked by timing graph replays on
// the first call (cached per shape class for the process).
#include <algorithm>
#include <map>
#include <memory>
#include <numeric>
#include <string>
#include <vector>

#include "exact_device.cuh"
#include "internal.h"

namespace rb {

struct BatchProb {
    ExactGeom G;
    const float4* txy;
    const int2* kxy;
    const float2* cs;
    const ZParam* zp;
    const float* w;
    const float* sens;
    float* ratio;
    const float* g;
    float* f;
    float* f_t;  // xy-transposed copy of f, made before each forward projection
    unsigned nviews;
    unsigned fp_tx, fp_ty;
    unsigned bp_bx, bp_by, bp_bz;
};

namespace batch {

// largest p in [0, n) with prefix[p] <= t
__device__ __forceinline__ int find_problem(const unsigned long long* prefix, int n, unsigned long long t)
{
    int lo = 0, hi = n - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (prefix[mid] <= t) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

template <bool KAHAN>
__global__ void __launch_bounds__(128) fp_kernel(const BatchProb* __restrict__ probs,
                                                  const unsigned long long* __restrict__ prefix, int nprob,
                                                  unsigned long long* __restrict__ counter)
{
    __shared__ unsigned long long s_tile;
    const int tid = threadIdx.x + threadIdx.y * 32;
    const unsigned long long total = prefix[nprob];
    for (;;) {
        if (tid == 0) s_tile = atomicAdd(counter, 1ull);
        __syncthreads();
        const unsigned long long t = s_tile;
        __syncthreads();
        if (t >= total) return;
        const int p = find_problem(prefix, nprob, t);
        const BatchProb& B = probs[p];
        const ExactGeom G = B.G;
        const unsigned per_view = B.fp_tx * B.fp_ty;
        const unsigned long long local = t - prefix[p];
        const unsigned view = (unsigned)(local / per_view);
        const unsigned r = (unsigned)(local % per_view);
        const int u = (int)(r % B.fp_tx) * 32 + threadIdx.x;
        const int v = (int)(r / B.fp_tx) * 4 + threadIdx.y;
        if (u >= G.Nu || v >= G.Nv) continue;
        const size_t pix = (size_t)u + (size_t)v * G.Nu;
        const float4 T = __ldg(B.txy + (size_t)view * G.Nu + u);
        const int2 K = __ldg(B.kxy + (size_t)view * G.Nu + u);
        const ZParam Z = B.zp[v];
        const float w = __ldg(B.w + pix);
        const exact::VolView V = exact::vol_view_for(__ldg(B.cs + view), B.f, B.f_t, G.X, G.Y);
        const float hf = w * exact::fp_ray_sum<KAHAN>(G, T, K, Z, V);
        const size_t n = (size_t)view * G.Nu * G.Nv + pix;
        const float gv = __ldg(B.g + n);
        const float ratio = (hf != 0.0f) ? __fdiv_rn(gv, hf) : 0.0f;
        B.ratio[n] = ratio * w;
    }
}

// f -> f_t of every problem, 32x32 tiles (one z slice each) spread over a
// grid-stride loop; prefix[p] counts the tiles of problems before p.
__global__ void __launch_bounds__(256) transpose_kernel(const BatchProb* __restrict__ probs,
                                                         const unsigned long long* __restrict__ prefix, int nprob)
{
    __shared__ float tile[32][33];
    const unsigned long long total = prefix[nprob];
    for (unsigned long long t = blockIdx.x; t < total; t += gridDim.x) {
        const int p = find_problem(prefix, nprob, t);
        const BatchProb& B = probs[p];
        const int X = B.G.X, Y = B.G.Y;
        const unsigned tx = (unsigned)(X + 31) / 32, ty = (unsigned)(Y + 31) / 32;
        const unsigned long long local = t - prefix[p];
        const int x0 = (int)(local % tx) * 32, y0 = (int)((local / tx) % ty) * 32;
        const size_t slab = (size_t)X * Y * (size_t)(local / ((unsigned long long)tx * ty));
        for (int r = threadIdx.y; r < 32; r += 8) {
            const int x = x0 + threadIdx.x, y = y0 + r;
            if (x < X && y < Y) tile[r][threadIdx.x] = B.f[slab + (size_t)y * X + x];
        }
        __syncthreads();
        for (int r = threadIdx.y; r < 32; r += 8) {
            const int y = y0 + threadIdx.x, x = x0 + r;
            if (x < X && y < Y) B.f_t[slab + (size_t)x * Y + y] = tile[threadIdx.x][r];
        }
        __syncthreads();
    }
}

template <int ZC>
__global__ void __launch_bounds__(128) bp_kernel(const BatchProb* __restrict__ probs,
                                                  const unsigned long long* __restrict__ prefix,
                                                  const int* __restrict__ perm, int nprob,
                                                  unsigned long long* __restrict__ counter)
{
    extern __shared__ float smem[];
    float* acc = smem;
    float4* szb = reinterpret_cast<float4*>(smem + ZC * 128);
    __shared__ unsigned long long s_tile;
    const int tid = threadIdx.x + threadIdx.y * 32;
    const unsigned long long total = prefix[nprob];
    for (;;) {
        if (tid == 0) s_tile = atomicAdd(counter, 1ull);
        __syncthreads();
        const unsigned long long t = s_tile;
        if (t >= total) return;
        const int q = find_problem(prefix, nprob, t);
        const BatchProb& B = probs[perm[q]];
        const ExactGeom G = B.G;
        const unsigned long long local = t - prefix[q];
        const unsigned bx = (unsigned)(local % B.bp_bx);
        const unsigned by = (unsigned)((local / B.bp_bx) % B.bp_by);
        const unsigned bz = (unsigned)(local / ((unsigned long long)B.bp_bx * B.bp_by));
        for (int z = tid; z < G.Nv; z += 128) {
            const ZParam zz = B.zp[z];
            const bool pos = zz.S > 0.0f;
            szb[z] = make_float4(fabsf(zz.S), pos ? zz.O : -zz.O, (float)zz.kc, pos ? 1.0f : -1.0f);
        }
#pragma unroll
        for (int k = 0; k < ZC; ++k) acc[k * 128 + tid] = 0.0f;
        __syncthreads();
        const int i = (int)bx * 32 + threadIdx.x;
        const int j = (int)by * 4 + threadIdx.y;
        const int k0 = (int)bz * ZC;
        const int k1 = min(k0 + ZC, G.Z);
        if (i < G.X && j < G.Y) {
            exact::bp_gather_column<ZC, 2, false, float>(G, B.txy, B.kxy, B.cs, B.w, 0u, B.nviews, B.ratio, szb,
                                                         acc, tid, i, j, k0, k1);
            for (int k = k0; k < k1; ++k) {
                const size_t vox = (size_t)i + (size_t)j * G.X + (size_t)k * G.X * G.Y;
                const float ht = acc[(k - k0) * 128 + tid];
                const float s = B.sens[vox];
                const float f = B.f[vox];
                B.f[vox] = (s != 0.0f) ? __fdiv_rn(__fmul_rn(f, ht), s) : 0.0f;
            }
        }
        __syncthreads();
    }
}

}  // namespace batch

struct BatchChoice {
    int zc = 32;
    int fp_ctas = 0;
    int bp_ctas = 0;
};

}  // namespace rb

using namespace rb;

struct recon_batch {
    std::vector<recon_plan_t> plans;
    int device = 0;
    bool kahan = true;
    std::vector<BatchProb> host;
    BatchProb* d_probs = nullptr;
    unsigned long long* d_fp_prefix = nullptr;
    unsigned long long* d_tr_prefix = nullptr;  // transpose tiles
    int sm_count = 148;
    unsigned long long* d_bp_prefix[2] = {nullptr, nullptr};  // per zc candidate
    int* d_perm[2] = {nullptr, nullptr};
    unsigned long long* d_counters = nullptr;
    size_t max_nv = 0;
    std::string key;
    BatchChoice choice;
    bool tuned = false;
    cudaStream_t cap_stream = nullptr;
    cudaGraphExec_t exec = nullptr;
    const float* const* graph_g = nullptr;

    ~recon_batch()
    {
        if (exec) cudaGraphExecDestroy(exec);
        if (cap_stream) cudaStreamDestroy(cap_stream);
        cudaFree(d_probs);
        cudaFree(d_fp_prefix);
        cudaFree(d_tr_prefix);
        for (int k = 0; k < 2; ++k) {
            cudaFree(d_bp_prefix[k]);
            cudaFree(d_perm[k]);
        }
        cudaFree(d_counters);
        for (auto p : plans) recon_plan_destroy(p);
    }
};

namespace {

const int kZC[2] = {16, 32};

std::map<std::string, BatchChoice>& tune_cache()
{
    static std::map<std::string, BatchChoice> c;
    return c;
}

recon_status_t build_order(recon_batch& b, int zci)
{
    const int ZC = kZC[zci];
    const int n = (int)b.host.size();
    std::vector<double> cost(n);
    std::vector<unsigned long long> tiles(n);
    for (int p = 0; p < n; ++p) {
        const ExactGeom& G = b.host[p].G;
        const unsigned bx = (G.X + 31) / 32, by = (G.Y + 3) / 4, bz = (G.Z + ZC - 1) / ZC;
        tiles[p] = (unsigned long long)bx * by * bz;
        // per tile: views x detector rows a chunk of ZC voxels spans
        cost[p] = (double)b.host[p].nviews * std::min(ZC, G.Z) * (double)G.Nv / G.Z;
    }
    std::vector<int> perm(n);
    std::iota(perm.begin(), perm.end(), 0);
    std::stable_sort(perm.begin(), perm.end(), [&](int a, int c) { return cost[a] > cost[c]; });
    std::vector<unsigned long long> prefix(n + 1, 0);
    for (int q = 0; q < n; ++q) prefix[q + 1] = prefix[q] + tiles[perm[q]];
    RB_CUDA(cudaMalloc(&b.d_bp_prefix[zci], (n + 1) * sizeof(unsigned long long)));
    RB_CUDA(cudaMalloc(&b.d_perm[zci], n * sizeof(int)));
    RB_CUDA(cudaMemcpy(b.d_bp_prefix[zci], prefix.data(), (n + 1) * sizeof(unsigned long long),
                       cudaMemcpyHostToDevice));
    RB_CUDA(cudaMemcpy(b.d_perm[zci], perm.data(), n * sizeof(int), cudaMemcpyHostToDevice));
    return RECON_OK;
}

template <int ZC>
size_t bp_smem(const recon_batch& b)
{
    return (size_t)ZC * 128 * sizeof(float) + b.max_nv * sizeof(float4);
}

recon_status_t launch_iteration(recon_batch& b, const BatchChoice& c, cudaStream_t s)
{
    const int n = (int)b.host.size();
    const int zci = (c.zc == 16) ? 0 : 1;
    RB_CUDA(cudaMemsetAsync(b.d_counters, 0, 2 * sizeof(unsigned long long), s));
    batch::transpose_kernel<<<b.sm_count * 8, dim3(32, 8), 0, s>>>(b.d_probs, b.d_tr_prefix, n);
    RB_CUDA(cudaGetLastError());
    if (b.kahan)
        batch::fp_kernel<true><<<c.fp_ctas, dim3(32, 4), 0, s>>>(b.d_probs, b.d_fp_prefix, n, b.d_counters);
    else
        batch::fp_kernel<false><<<c.fp_ctas, dim3(32, 4), 0, s>>>(b.d_probs, b.d_fp_prefix, n, b.d_counters);
    RB_CUDA(cudaGetLastError());
    if (c.zc == 16)
        batch::bp_kernel<16><<<c.bp_ctas, dim3(32, 4), bp_smem<16>(b), s>>>(b.d_probs, b.d_bp_prefix[zci],
                                                                            b.d_perm[zci], n, b.d_counters + 1);
    else
        batch::bp_kernel<32><<<c.bp_ctas, dim3(32, 4), bp_smem<32>(b), s>>>(b.d_probs, b.d_bp_prefix[zci],
                                                                            b.d_perm[zci], n, b.d_counters + 1);
    RB_CUDA(cudaGetLastError());
    return RECON_OK;
}

recon_status_t capture(recon_batch& b, const BatchChoice& c)
{
    // the dynamic shared memory limit is per kernel, process-wide: set it for
    // this batch's largest detector before every capture
    if (c.zc == 16)
        RB_CUDA(cudaFuncSetAttribute(batch::bp_kernel<16>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)bp_smem<16>(b)));
    else
        RB_CUDA(cudaFuncSetAttribute(batch::bp_kernel<32>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)bp_smem<32>(b)));
    if (b.exec) {
        cudaGraphExecDestroy(b.exec);
        b.exec = nullptr;
    }
    cudaGraph_t graph = nullptr;
    RB_CUDA(cudaStreamBeginCapture(b.cap_stream, cudaStreamCaptureModeThreadLocal));
    recon_status_t st = launch_iteration(b, c, b.cap_stream);
    cudaError_t e = cudaStreamEndCapture(b.cap_stream, &graph);
    if (st != RECON_OK) {
        if (graph) cudaGraphDestroy(graph);
        return st;
    }
    if (e != cudaSuccess) return cuda_fail(e, "graph capture");
    e = cudaGraphInstantiate(&b.exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) return cuda_fail(e, "graph instantiate");
    return RECON_OK;
}

recon_status_t occupancy(recon_batch& b, int zc, int& fp_ctas, int& bp_ctas)
{
    int sms = 148, nfp = 1, nbp = 1;
    RB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b.device));
    if (b.kahan) RB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nfp, batch::fp_kernel<true>, 128, 0));
    else RB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nfp, batch::fp_kernel<false>, 128, 0));
    if (zc == 16) {
        RB_CUDA(cudaFuncSetAttribute(batch::bp_kernel<16>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)bp_smem<16>(b)));
        RB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nbp, batch::bp_kernel<16>, 128, bp_smem<16>(b)));
    } else {
        RB_CUDA(cudaFuncSetAttribute(batch::bp_kernel<32>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)bp_smem<32>(b)));
        RB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nbp, batch::bp_kernel<32>, 128, bp_smem<32>(b)));
    }
    fp_ctas = sms * std::max(1, nfp);
    bp_ctas = sms * std::max(1, nbp);
    return RECON_OK;
}

// Time graph replays of each candidate on the caller's data, restoring the
// images afterwards.
recon_status_t autotune(recon_batch& b, float* const* d_f)
{
    auto it = tune_cache().find(b.key);
    if (it != tune_cache().end()) {
        b.choice = it->second;
        return capture(b, b.choice);
    }
    size_t total = 0;
    for (auto& h : b.host) total += (size_t)h.G.X * h.G.Y * h.G.Z;
    float* save = nullptr;
    RB_CUDA(cudaMalloc(&save, total * sizeof(float)));
    size_t off = 0;
    for (size_t p = 0; p < b.host.size(); ++p) {
        const size_t n = (size_t)b.host[p].G.X * b.host[p].G.Y * b.host[p].G.Z;
        cudaMemcpyAsync(save + off, d_f[p], n * sizeof(float), cudaMemcpyDeviceToDevice, b.cap_stream);
        off += n;
    }
    std::vector<BatchChoice> cands;
    for (int zc : {16, 32}) {
        int fpc, bpc;
        recon_status_t st = occupancy(b, zc, fpc, bpc);
        if (st != RECON_OK) {
            cudaFree(save);
            return st;
        }
        cands.push_back({zc, fpc, bpc});
        if (bpc > 148) cands.push_back({zc, fpc, bpc / 2});
    }
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    float best = 1e30f;
    BatchChoice pick = cands.front();
    for (const auto& c : cands) {
        if (capture(b, c) != RECON_OK) continue;
        cudaGraphLaunch(b.exec, b.cap_stream);
        cudaEventRecord(e0, b.cap_stream);
        cudaGraphLaunch(b.exec, b.cap_stream);
        cudaGraphLaunch(b.exec, b.cap_stream);
        cudaEventRecord(e1, b.cap_stream);
        cudaEventSynchronize(e1);
        float ms = 0.f;
        cudaEventElapsedTime(&ms, e0, e1);
        if (ms < best) {
            best = ms;
            pick = c;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    off = 0;
    for (size_t p = 0; p < b.host.size(); ++p) {
        const size_t n = (size_t)b.host[p].G.X * b.host[p].G.Y * b.host[p].G.Z;
        cudaMemcpyAsync(d_f[p], save + off, n * sizeof(float), cudaMemcpyDeviceToDevice, b.cap_stream);
        off += n;
    }
    cudaStreamSynchronize(b.cap_stream);
    cudaFree(save);
    RB_CUDA(cudaGetLastError());
    b.choice = pick;
    tune_cache()[b.key] = pick;
    return capture(b, pick);
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
    b->kahan = (opt.sum == RECON_SUM_KAHAN);
    std::string key = std::to_string(n) + (b->kahan ? "k" : "p");
    for (int p = 0; p < n; ++p) {
        recon_plan_t plan = nullptr;
        RB_CHECK(recon_plan_create(&geoms[p], &opt, &plan));
        b->plans.push_back(plan);
        if (geoms[p].scan.NumProj == 0) return fail(RECON_ERR_INVALID_ARGUMENT, "every problem needs views");
        RB_CHECK(recon_mlem_prepare(plan, nullptr));
        Plan& P = *plan;
        BatchProb h{};
        h.G = P.eg;
        h.txy = P.d_txy;
        h.kxy = P.d_kxy;
        h.cs = P.d_cs;
        h.zp = P.d_zp;
        h.w = P.d_w;
        h.sens = P.d_sens;
        h.ratio = static_cast<float*>(P.d_ratio);
        h.f_t = P.d_vol_t;
        h.nviews = P.nviews;
        h.fp_tx = (P.eg.Nu + 31) / 32;
        h.fp_ty = (P.eg.Nv + 3) / 4;
        h.bp_bx = (P.eg.X + 31) / 32;
        h.bp_by = (P.eg.Y + 3) / 4;
        b->max_nv = std::max(b->max_nv, (size_t)P.eg.Nv);
        b->host.push_back(h);
        const recon_geometry_t& g = geoms[p];
        key += "|" + std::to_string(g.vox.Xdim) + "x" + std::to_string(g.vox.Ydim) + "x" + std::to_string(g.vox.Zdim) +
               "/" + std::to_string(g.scan.NumProj) + "/" + std::to_string(g.det.NumAxPixels) + "x" +
               std::to_string(g.det.NumTAxPixels);
    }
    b->key = key;
    RB_CUDA(cudaSetDevice(b->device));
    std::vector<unsigned long long> fp_prefix(n + 1, 0);
    for (int p = 0; p < n; ++p)
        fp_prefix[p + 1] = fp_prefix[p] + (unsigned long long)b->host[p].nviews * b->host[p].fp_tx * b->host[p].fp_ty;
    RB_CUDA(cudaMalloc(&b->d_fp_prefix, (n + 1) * sizeof(unsigned long long)));
    RB_CUDA(cudaMemcpy(b->d_fp_prefix, fp_prefix.data(), (n + 1) * sizeof(unsigned long long), cudaMemcpyHostToDevice));
    std::vector<unsigned long long> tr_prefix(n + 1, 0);
    for (int p = 0; p < n; ++p) {
        const ExactGeom& G = b->host[p].G;
        tr_prefix[p + 1] = tr_prefix[p] + (unsigned long long)((G.X + 31) / 32) * ((G.Y + 31) / 32) * G.Z;
    }
    RB_CUDA(cudaMalloc(&b->d_tr_prefix, (n + 1) * sizeof(unsigned long long)));
    RB_CUDA(cudaMemcpy(b->d_tr_prefix, tr_prefix.data(), (n + 1) * sizeof(unsigned long long), cudaMemcpyHostToDevice));
    RB_CUDA(cudaDeviceGetAttribute(&b->sm_count, cudaDevAttrMultiProcessorCount, b->device));
    for (int zci = 0; zci < 2; ++zci) RB_CHECK(build_order(*b, zci));
    RB_CUDA(cudaMalloc(&b->d_probs, n * sizeof(BatchProb)));
    RB_CUDA(cudaMalloc(&b->d_counters, 2 * sizeof(unsigned long long)));
    RB_CUDA(cudaStreamCreateWithFlags(&b->cap_stream, cudaStreamNonBlocking));
    RB_CUDA(cudaDeviceSynchronize());
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
    const size_t n = b->host.size();
    for (size_t p = 0; p < n; ++p)
        if (!d_g[p] || !d_f[p]) return fail(RECON_ERR_INVALID_ARGUMENT, "NULL problem buffer");
    RB_CUDA(cudaSetDevice(b->device));
    cudaStream_t s = as_stream(stream);
    // the work runs on the graph's stream, ordered after the caller's stream
    cudaEvent_t ev;
    RB_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    RB_CUDA(cudaEventRecord(ev, s));
    RB_CUDA(cudaStreamWaitEvent(b->cap_stream, ev, 0));
    for (size_t p = 0; p < n; ++p) {
        b->host[p].g = d_g[p];
        b->host[p].f = d_f[p];
        if (init_ones) {
            const size_t nv = (size_t)b->host[p].G.X * b->host[p].G.Y * b->host[p].G.Z;
            RB_CHECK(launch_fill(d_f[p], 1.0f, nv, b->cap_stream));
        }
    }
    RB_CUDA(cudaMemcpyAsync(b->d_probs, b->host.data(), n * sizeof(BatchProb), cudaMemcpyHostToDevice,
                            b->cap_stream));
    RB_CUDA(cudaStreamSynchronize(b->cap_stream));  // host descriptors must outlive the copy
    if (!b->tuned) {
        RB_CHECK(autotune(*b, d_f));
        b->tuned = true;
    }
    for (unsigned it = 0; it < iters; ++it) RB_CUDA(cudaGraphLaunch(b->exec, b->cap_stream));
    RB_CUDA(cudaEventRecord(ev, b->cap_stream));
    RB_CUDA(cudaStreamWaitEvent(s, ev, 0));
    cudaEventDestroy(ev);
    return RECON_OK;
}

}  // extern "C"
