// stt_noalloc.cu -- the ray-driven backprojector for callers that cannot
// allocate device memory.
//
// stt_bp_ray keeps its per-voxel (contribution, weight) accumulators in memory
// the context allocates on first use.  Some callers cannot let a library call
// cudaMalloc: a plugin inside a host application that has reserved the GPU's
// memory up front through its own allocator, or a real-time pipeline that
// cannot afford the device-wide synchronisation cudaMalloc and cudaFree can
// imply.  stt_bp_ray_noalloc does the same work with the accumulators in a
// fixed-size array compiled into this library instead: it allocates nothing.
//
// The array holds STT_BP_RAY_NOALLOC_MAX_VOXELS (2^21 = 128^3) float2 entries,
// 16 MiB that every GPU which loads libstt.so keeps until the process exits.
// All calls on a device share it, so calls that overlap on the GPU (on
// different streams, contexts or host threads) race on it; serialise them.
// Each call clears the part it uses before scattering, so nothing is carried
// over from an earlier call.  The first call on a device looks the array's
// device address up (cudaGetSymbolAddress, with that device current); make
// that first call before any stream capture.
#include <mutex>
#include <string>

#include "stt.h"
#include "stt_internal.cuh"
#include "stt_kernels.h"

// Context internals (stt_capi.cu).
extern "C" stt_status stt_internal_geom(stt_ctx *ctx, const void **geom, const void **views);
extern "C" stt_status stt_internal_set_error(stt_ctx *ctx, stt_status st, const char *msg);

static __device__ __align__(256) float2 g_bp_ray_scratch[STT_BP_RAY_NOALLOC_MAX_VOXELS];

namespace {

constexpr int kMaxDevices = 64;
std::mutex g_scratch_mu;
float2 *g_scratch_ptr[kMaxDevices] = {};

// Device address of g_bp_ray_scratch on the current device, looked up once per
// device.  In host code the symbol itself is only a host-side stand-in.
stt_status scratch_on_current_device(stt_ctx *ctx, float2 **out) {
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess)
        return stt_internal_set_error(ctx, STT_ERR_CUDA, (std::string("cudaGetDevice: ") + cudaGetErrorString(e)).c_str());
    if (dev < 0 || dev >= kMaxDevices)
        return stt_internal_set_error(ctx, STT_ERR_UNSUPPORTED, "stt_bp_ray_noalloc: device ordinal above 63");
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    if (!g_scratch_ptr[dev]) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_bp_ray_scratch);
        if (e != cudaSuccess || !p)
            return stt_internal_set_error(
                ctx, STT_ERR_CUDA, (std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e)).c_str());
        g_scratch_ptr[dev] = static_cast<float2 *>(p);
    }
    *out = g_scratch_ptr[dev];
    return STT_OK;
}

}  // namespace

extern "C" stt_status stt_bp_ray_noalloc(stt_ctx *ctx, const float *corr, float *vol, float gmax, int view,
                                         void *stream) {
    const void *gp = nullptr, *vp = nullptr;
    stt_status st = stt_internal_geom(ctx, &gp, &vp);  // also makes the context's device current
    if (st) return st;
    const stt::GeomDev &g = *static_cast<const stt::GeomDev *>(gp);
    if (!corr || !vol) return stt_internal_set_error(ctx, STT_ERR_INVALID, "null corr or vol");
    if (view < 0 || view >= g.n_views)
        return stt_internal_set_error(ctx, STT_ERR_INVALID, "view outside the geometry's view list");
    const long long n = (long long)g.nx * g.ny * g.nz;
    if (n > (long long)STT_BP_RAY_NOALLOC_MAX_VOXELS) {
        const std::string msg = "stt_bp_ray_noalloc: the volume has " + std::to_string(n) +
                                " voxels, more than the fixed scratch of " +
                                std::to_string((long long)STT_BP_RAY_NOALLOC_MAX_VOXELS) +
                                " voxels (128^3); use stt_bp_ray";
        return stt_internal_set_error(ctx, STT_ERR_INVALID, msg.c_str());
    }
    float2 *acc = nullptr;
    if ((st = scratch_on_current_device(ctx, &acc))) return st;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    cudaError_t e = cudaMemsetAsync(acc, 0, (size_t)n * sizeof(float2), s);
    if (e == cudaSuccess) {
        const stt::ViewSel sel{view, nullptr, 0, view};
        e = stt::launch_bp_ray(g, static_cast<const stt::ViewRec *>(vp), sel, corr, acc, vol, gmax, s);
    }
    if (e != cudaSuccess)
        return stt_internal_set_error(ctx, STT_ERR_CUDA, (std::string("stt_bp_ray_noalloc: ") + cudaGetErrorString(e)).c_str());
    return STT_OK;
}
