// noalloc.cu -- COMPAT back projection of one view with no device allocation.
//
// recon_compat_bp_view_noalloc takes a geometry instead of a plan.  The
// per-call device state the COMPAT back projector needs (the view angle, the
// view's step count, the image's max |value| and the 64-bit fixed-point
// accumulator) lives in one file-scope __device__ array, so the call never
// allocates or frees device memory.  Its address is looked up once per
// device, on the first call on that device.  The work is the same
// compat_bp_view path a COMPAT plan runs: a host-only Plan describes the
// geometry and its device fields point into the scratch array.
//
// Limits:
//  * at most RECON_NOALLOC_MAX_VOXELS voxels (larger volumes are rejected
//    before any device work);
//  * one scratch array per device, shared by every caller in the process:
//    calls that may overlap in time on one device (different streams,
//    different host threads) race on it and corrupt each other's result.
//    Calls in one stream are ordered and safe;
//  * the first call on a device looks up the scratch address (and may load
//    the library's device code), so make it before any stream capture; the
//    address is kept for the process's life, so the entry point must not be
//    called after a cudaDeviceReset of that device.
#include <cmath>
#include <mutex>

#include "internal.h"

namespace rb {
namespace {

constexpr size_t kHeaderWords = 32;  // 256 bytes: angle, loopN, maxabs slots
constexpr size_t kMaxDevices = 64;

// [0] view angle (float), [1] loopN (unsigned), [2] max |img| bits (unsigned),
// [kHeaderWords ...] fixed-point accumulator, one word per voxel
static __device__ __align__(256) unsigned long long g_noalloc_scratch[kHeaderWords + RECON_NOALLOC_MAX_VOXELS];

std::mutex g_setup_mutex;
unsigned long long* g_scratch_addr[kMaxDevices] = {};

recon_status_t scratch_for_device(int device, unsigned long long** out)
{
    std::lock_guard<std::mutex> lock(g_setup_mutex);
    if (!g_scratch_addr[device]) {
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(no-alloc scratch)");
        if (!p) return fail(RECON_ERR_CUDA, "no-alloc scratch has no device address");
        g_scratch_addr[device] = static_cast<unsigned long long*>(p);
    }
    *out = g_scratch_addr[device];
    return RECON_OK;
}

}  // namespace
}  // namespace rb

using namespace rb;

extern "C" recon_status_t recon_compat_bp_view_noalloc(const recon_geometry_t* geom, const float* d_img,
                                                       float angle_deg, float* d_vol, void* stream)
{
    if (!geom || !d_img || !d_vol) return fail(RECON_ERR_INVALID_ARGUMENT, "NULL argument");
    if (!std::isfinite(angle_deg)) return fail(RECON_ERR_INVALID_ARGUMENT, "angle must be finite");
    const size_t nvox = (size_t)geom->vox.Xdim * geom->vox.Ydim * geom->vox.Zdim;
    if (geom->vox.Xdim > 0 && geom->vox.Ydim > 0 && geom->vox.Zdim > 0 && nvox > RECON_NOALLOC_MAX_VOXELS)
        return fail(RECON_ERR_UNSUPPORTED, "volume exceeds the no-alloc scratch (RECON_NOALLOC_MAX_VOXELS voxels); "
                                           "use a plan");
    int device = -1;
    RB_CUDA(cudaGetDevice(&device));
    if (device < 0 || (size_t)device >= kMaxDevices) return fail(RECON_ERR_UNSUPPORTED, "device ordinal too large");
    Plan P;  // host description only: owns no device memory, frees nothing
    P.device = device;
    RB_CHECK(describe_compat_geometry(*geom, P));
    unsigned long long* scratch = nullptr;
    RB_CHECK(scratch_for_device(device, &scratch));
    P.d_angles = reinterpret_cast<float*>(scratch + 0);
    P.d_loopN = reinterpret_cast<unsigned*>(scratch + 1);
    P.d_maxabs = reinterpret_cast<unsigned*>(scratch + 2);
    P.d_fix = scratch + kHeaderWords;
    cudaStream_t s = as_stream(stream);
    // the accumulator must start at zero (the angle, loopN and maxabs slots
    // are written or cleared by the projector itself)
    RB_CUDA(cudaMemsetAsync(P.d_fix, 0, P.nvox * sizeof(unsigned long long), s));
    // view slot 0 (= P.nviews): angle and step count set up for this call
    return compat_bp_view(P, d_img, 0, true, angle_deg, d_vol, false, s);
}
