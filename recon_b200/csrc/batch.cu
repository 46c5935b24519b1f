// batch.cu -- many independent MLEM reconstructions per launch.
//
// One iteration of all problems is four kernels, captured once in a CUDA
// graph and replayed:
//  1. a transpose of every image (the forward walk reads the xy-transposed
//     copy for views whose detector rows run along y), which also clears
//     every problem's max-|ratio| slot;
//  2. the forward projection with the ratio fused in, a persistent kernel
//     over the 32x4-ray blocks of every problem that can cross its volume
//     (the plans' culled tile lists), recording each problem's max |ratio|;
//  3. the back projection of the ratios, a persistent kernel over the same
//     ray tiles, adding to each problem's fixed-point accumulators;
//  4. the update f <- f * Ht / sens of every problem, which also clears the
//     accumulators.
// CTAs of 2 and 3 pull tile indices from atomic counters; problems are queued
// largest first, so the last tiles are small.  The per-ray work is the same
// device code as the single-problem kernels (exact_device.cuh) and the back
// projection sums exactly, so each problem's image is bit-identical to
// recon_mlem on its own plan whatever the tile order.  The number of resident
// CTAs of kernels 2 and 3 is picked by timing graph replays on the first call
// (cached per set of shapes for the process).
#include <algorithm>
#include <climits>
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
    float* f_t;                    // xy-transposed copy of f, made before each forward projection
    unsigned long long* acc;       // back projection accumulators, image layout [nvox]
    unsigned long long* acc_t;     // and xy-transposed [nvox]
    unsigned* bpmax;               // max |ratio| of the current iteration (float bits)
    float max_len;                 // longest segment (fixed-point scale)
    int count_bits;                // contributions per voxel, as bits (fixed-point scale)
    const uint2* tiles;            // ray blocks that can cross the volume ({view, tu | tv << 16})
    unsigned ntiles;
    unsigned nviews;
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

// f -> f_t of every problem, 32x32 tiles (one z slice each) spread over a
// grid-stride loop; prefix[p] counts the tiles of problems before p.  Block 0
// also clears every problem's max-|ratio| slot for the forward kernel.
__global__ void __launch_bounds__(256) transpose_kernel(const BatchProb* __restrict__ probs,
                                                         const unsigned long long* __restrict__ prefix, int nprob)
{
    __shared__ float tile[32][33];
    if (blockIdx.x == 0)
        for (int p = threadIdx.x + threadIdx.y * 32; p < nprob; p += 256) *probs[p].bpmax = 0u;
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

// Ray tile t of the queue: problem perm[q], view and the 32x4 block of rays.
struct RayTile {
    int p, u, v;
    unsigned view;
};

__device__ __forceinline__ RayTile ray_tile(const BatchProb* probs, const unsigned long long* prefix,
                                            const int* perm, int nprob, unsigned long long t)
{
    const int q = find_problem(prefix, nprob, t);
    const int p = perm[q];
    const uint2 tile = probs[p].tiles[t - prefix[q]];
    return RayTile{p, (int)(tile.y & 0xffffu) * 32 + (int)threadIdx.x, (int)(tile.y >> 16) * 4 + (int)threadIdx.y,
                   tile.x};
}

// Next tile index for the whole CTA (one atomic per tile).
__device__ __forceinline__ unsigned long long next_tile(unsigned long long* counter, unsigned long long* s_tile,
                                                        int tid)
{
    if (tid == 0) *s_tile = atomicAdd(counter, 1ull);
    __syncthreads();
    const unsigned long long t = *s_tile;
    __syncthreads();
    return t;
}

template <bool KAHAN>
__global__ void __launch_bounds__(128) fp_kernel(const BatchProb* __restrict__ probs,
                                                  const unsigned long long* __restrict__ prefix,
                                                  const int* __restrict__ perm, int nprob,
                                                  unsigned long long* __restrict__ counter)
{
    __shared__ unsigned long long s_tile;
    const int tid = threadIdx.x + threadIdx.y * 32;
    const unsigned long long total = prefix[nprob];
    for (;;) {
        const unsigned long long t = next_tile(counter, &s_tile, tid);
        if (t >= total) return;
        const RayTile R = ray_tile(probs, prefix, perm, nprob, t);
        const BatchProb& B = probs[R.p];
        const ExactGeom G = B.G;
        unsigned m = 0;
        if (R.u < G.Nu && R.v < G.Nv) {
            const size_t pix = (size_t)R.u + (size_t)R.v * G.Nu;
            const float4 T = __ldg(B.txy + (size_t)R.view * G.Nu + R.u);
            const int2 K = __ldg(B.kxy + (size_t)R.view * G.Nu + R.u);
            const ZParam Z = B.zp[R.v];
            const float w = __ldg(B.w + pix);
            const exact::VolView V = exact::vol_view_for(__ldg(B.cs + R.view), B.f, B.f_t, G.X, G.Y);
            const float hf = w * exact::fp_ray_sum<KAHAN>(G, T, K, Z, V);
            const size_t n = (size_t)R.view * G.Nu * G.Nv + pix;
            const float gv = __ldg(B.g + n);
            const float ratio = (hf != 0.0f) ? __fdiv_rn(gv, hf) : 0.0f;
            const float out = ratio * w;
            B.ratio[n] = out;
            m = __float_as_uint(fabsf(out));
        }
        for (int o = 16; o > 0; o >>= 1) m = max(m, __shfl_xor_sync(0xffffffffu, m, o));
        if (threadIdx.x == 0 && m) atomicMax(B.bpmax, m);
    }
}

__global__ void __launch_bounds__(128) bp_kernel(const BatchProb* __restrict__ probs,
                                                  const unsigned long long* __restrict__ prefix,
                                                  const int* __restrict__ perm, int nprob,
                                                  unsigned long long* __restrict__ counter)
{
    __shared__ unsigned long long s_tile;
    const int tid = threadIdx.x + threadIdx.y * 32;
    const unsigned long long total = prefix[nprob];
    for (;;) {
        const unsigned long long t = next_tile(counter, &s_tile, tid);
        if (t >= total) return;
        const RayTile R = ray_tile(probs, prefix, perm, nprob, t);
        const BatchProb& B = probs[R.p];
        const ExactGeom G = B.G;
        if (R.u >= G.Nu || R.v >= G.Nv) continue;
        const int F = exact::fix_exponent(*B.bpmax, B.max_len, B.count_bits);
        if (F == INT_MIN) continue;
        const float val = B.ratio[(size_t)R.view * G.Nu * G.Nv + (size_t)R.u + (size_t)R.v * G.Nu];
        if (val == 0.0f) continue;
        const float2 C = __ldg(B.cs + R.view);
        exact::bp_ray_slab(G, __ldg(B.txy + (size_t)R.view * G.Nu + R.u), __ldg(B.kxy + (size_t)R.view * G.Nu + R.u),
                           B.zp[R.v], 0, G.Z, val * ldexpf(1.0f, F), fabsf(C.y) > fabsf(C.x), B.acc, B.acc_t);
    }
}

// f <- (sens != 0) ? f * Ht / sens : 0 for every voxel of every problem;
// prefix[p] counts the voxels of problems before p.
__global__ void __launch_bounds__(256) update_kernel(const BatchProb* __restrict__ probs,
                                                      const unsigned long long* __restrict__ prefix, int nprob)
{
    const unsigned long long total = prefix[nprob];
    for (unsigned long long t = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x; t < total;
         t += (unsigned long long)gridDim.x * blockDim.x) {
        const int p = find_problem(prefix, nprob, t);
        const BatchProb& B = probs[p];
        const ExactGeom G = B.G;
        const size_t i = (size_t)(t - prefix[p]);
        const int x = (int)(i % G.X), y = (int)((i / G.X) % G.Y), z = (int)(i / ((size_t)G.X * G.Y));
        const int F = exact::fix_exponent(*B.bpmax, B.max_len, B.count_bits);
        const float ht = exact::bp_slab_value(G, x, y, z, F, B.acc, B.acc_t);
        const float sv = B.sens[i];
        B.f[i] = (sv != 0.0f) ? __fdiv_rn(__fmul_rn(B.f[i], ht), sv) : 0.0f;
    }
}

}  // namespace batch

struct BatchChoice {
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
    unsigned long long* d_ray_prefix = nullptr;  // ray tiles, problems in queue order
    int* d_perm = nullptr;                       // queue order -> problem
    unsigned long long* d_tr_prefix = nullptr;   // transpose tiles
    unsigned long long* d_vox_prefix = nullptr;  // voxels
    unsigned long long* d_acc = nullptr;         // all problems' accumulators
    unsigned long long* d_counters = nullptr;
    int sm_count = 148;
    std::string key;
    BatchChoice choice;
    bool tuned = false;
    cudaStream_t cap_stream = nullptr;
    cudaGraphExec_t exec = nullptr;

    ~recon_batch()
    {
        if (exec) cudaGraphExecDestroy(exec);
        if (cap_stream) cudaStreamDestroy(cap_stream);
        cudaFree(d_probs);
        cudaFree(d_ray_prefix);
        cudaFree(d_perm);
        cudaFree(d_tr_prefix);
        cudaFree(d_vox_prefix);
        cudaFree(d_acc);
        cudaFree(d_counters);
        for (auto p : plans) recon_plan_destroy(p);
    }
};

namespace {

std::map<std::string, BatchChoice>& tune_cache()
{
    static std::map<std::string, BatchChoice> c;
    return c;
}

recon_status_t upload(unsigned long long** d, const std::vector<unsigned long long>& h)
{
    RB_CUDA(cudaMalloc(d, h.size() * sizeof(unsigned long long)));
    RB_CUDA(cudaMemcpy(*d, h.data(), h.size() * sizeof(unsigned long long), cudaMemcpyHostToDevice));
    return RECON_OK;
}

recon_status_t launch_iteration(recon_batch& b, const BatchChoice& c, cudaStream_t s)
{
    const int n = (int)b.host.size();
    RB_CUDA(cudaMemsetAsync(b.d_counters, 0, 2 * sizeof(unsigned long long), s));
    batch::transpose_kernel<<<b.sm_count * 8, dim3(32, 8), 0, s>>>(b.d_probs, b.d_tr_prefix, n);
    RB_CUDA(cudaGetLastError());
    if (b.kahan)
        batch::fp_kernel<true><<<c.fp_ctas, dim3(32, 4), 0, s>>>(b.d_probs, b.d_ray_prefix, b.d_perm, n,
                                                                 b.d_counters);
    else
        batch::fp_kernel<false><<<c.fp_ctas, dim3(32, 4), 0, s>>>(b.d_probs, b.d_ray_prefix, b.d_perm, n,
                                                                  b.d_counters);
    RB_CUDA(cudaGetLastError());
    batch::bp_kernel<<<c.bp_ctas, dim3(32, 4), 0, s>>>(b.d_probs, b.d_ray_prefix, b.d_perm, n, b.d_counters + 1);
    RB_CUDA(cudaGetLastError());
    batch::update_kernel<<<b.sm_count * 8, 256, 0, s>>>(b.d_probs, b.d_vox_prefix, n);
    RB_CUDA(cudaGetLastError());
    return RECON_OK;
}

recon_status_t capture(recon_batch& b, const BatchChoice& c)
{
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

// Time graph replays of each candidate on the caller's data, restoring the
// images afterwards.
recon_status_t autotune(recon_batch& b, float* const* d_f)
{
    auto it = tune_cache().find(b.key);
    if (it != tune_cache().end()) {
        b.choice = it->second;
        return capture(b, b.choice);
    }
    int nfp = 1, nbp = 1;
    if (b.kahan) RB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nfp, batch::fp_kernel<true>, 128, 0));
    else RB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nfp, batch::fp_kernel<false>, 128, 0));
    RB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nbp, batch::bp_kernel, 128, 0));
    nfp = std::max(1, nfp);
    nbp = std::max(1, nbp);
    std::vector<BatchChoice> cands;
    for (int fdiv : {1, 2})
        for (int bdiv : {1, 2}) cands.push_back({b.sm_count * std::max(1, nfp / fdiv), b.sm_count * std::max(1, nbp / bdiv)});
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
    size_t nvox_total = 0;
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
        h.bpmax = P.d_bpmax;
        h.max_len = bp_max_len(P);
        h.count_bits = bp_count_bits(P, P.nviews);
        h.nviews = P.nviews;
        h.tiles = P.fp_tiles.d;
        h.ntiles = P.fp_tiles.prefix.empty() ? 0u : P.fp_tiles.prefix.back();
        b->host.push_back(h);
        nvox_total += P.nvox;
        const recon_geometry_t& g = geoms[p];
        key += "|" + std::to_string(g.vox.Xdim) + "x" + std::to_string(g.vox.Ydim) + "x" + std::to_string(g.vox.Zdim) +
               "/" + std::to_string(g.scan.NumProj) + "/" + std::to_string(g.det.NumAxPixels) + "x" +
               std::to_string(g.det.NumTAxPixels);
    }
    b->key = key;
    RB_CUDA(cudaSetDevice(b->device));
    RB_CUDA(cudaDeviceGetAttribute(&b->sm_count, cudaDevAttrMultiProcessorCount, b->device));
    // accumulators: two per problem, cleared once here and by every update
    RB_CUDA(cudaMalloc(&b->d_acc, 2 * nvox_total * sizeof(unsigned long long)));
    RB_CUDA(cudaMemset(b->d_acc, 0, 2 * nvox_total * sizeof(unsigned long long)));
    size_t off = 0;
    for (auto& h : b->host) {
        const size_t nv = (size_t)h.G.X * h.G.Y * h.G.Z;
        h.acc = b->d_acc + off;
        h.acc_t = b->d_acc + off + nv;
        off += 2 * nv;
    }
    // ray tiles, largest problems (most ray-voxel work) first
    std::vector<double> work(n);
    for (int p = 0; p < n; ++p) {
        const BatchProb& h = b->host[p];
        work[p] = (double)h.nviews * h.G.Nu * h.G.Nv * (double)(h.G.X + h.G.Y + h.G.Z);
    }
    std::vector<int> perm(n);
    std::iota(perm.begin(), perm.end(), 0);
    std::stable_sort(perm.begin(), perm.end(), [&](int a, int c) { return work[a] > work[c]; });
    std::vector<unsigned long long> ray_prefix(n + 1, 0), tr_prefix(n + 1, 0), vox_prefix(n + 1, 0);
    for (int q = 0; q < n; ++q) {
        const BatchProb& h = b->host[perm[q]];
        ray_prefix[q + 1] = ray_prefix[q] + h.ntiles;
    }
    for (int p = 0; p < n; ++p) {
        const BatchProb& h = b->host[p];
        tr_prefix[p + 1] = tr_prefix[p] + (unsigned long long)((h.G.X + 31) / 32) * ((h.G.Y + 31) / 32) * h.G.Z;
        vox_prefix[p + 1] = vox_prefix[p] + (unsigned long long)h.G.X * h.G.Y * h.G.Z;
    }
    RB_CHECK(upload(&b->d_ray_prefix, ray_prefix));
    RB_CHECK(upload(&b->d_tr_prefix, tr_prefix));
    RB_CHECK(upload(&b->d_vox_prefix, vox_prefix));
    RB_CUDA(cudaMalloc(&b->d_perm, n * sizeof(int)));
    RB_CUDA(cudaMemcpy(b->d_perm, perm.data(), n * sizeof(int), cudaMemcpyHostToDevice));
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
