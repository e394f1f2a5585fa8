// host_api.cpp -- host-pointer entry points (include/stt_host.h): stage the
// arrays to the device, call the C ABI of libstt.so, copy the results back.
#include <cuda_runtime_api.h>

#include <cstring>
#include <string>
#include <vector>

#include "stt_host.h"

namespace stt_facade {

thread_local std::string g_err;
thread_local int g_device = 0;

void set_error(const std::string &m) { g_err = m; }

// Owns device buffers for one call.
class DeviceArena {
public:
    ~DeviceArena() {
        for (void *p : ptrs_) cudaFree(p);
    }
    float *alloc(size_t n) {
        void *p = nullptr;
        if (cudaMalloc(&p, n * sizeof(float) + 16) != cudaSuccess) {
            cudaGetLastError();
            return nullptr;
        }
        ptrs_.push_back(p);
        return static_cast<float *>(p);
    }
    float *upload(const float *src, size_t n) {
        float *p = alloc(n);
        if (p && src && cudaMemcpy(p, src, n * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess) return nullptr;
        return p;
    }

private:
    std::vector<void *> ptrs_;
};

int cuda_status(cudaError_t e, const char *where) {
    if (e == cudaSuccess) return STT_OK;
    set_error(std::string(where) + ": " + cudaGetErrorString(e));
    return STT_ERR_CUDA;
}

int lib_status(int st) {
    if (st != STT_OK) set_error(stt_last_error(nullptr));
    return st;
}

bool zero_min_box(const float *aabb, float box[3]) {
    if (aabb[0] != 0.0f || aabb[2] != 0.0f || aabb[4] != 0.0f) return false;
    box[0] = aabb[1];
    box[1] = aabb[3];
    box[2] = aabb[5];
    return true;
}

}  // namespace stt_facade

using namespace stt_facade;

extern "C" {

const char *stt_host_last_error(void) { return g_err.c_str(); }

int stt_host_set_device(int device) {
    g_device = device;
    return cuda_status(cudaSetDevice(device), "cudaSetDevice");
}

int stt_host_warp(const int *dim, const float *aabb, const float *vel, const float *src, int nc, float dt,
                  float *out) {
    if (!dim || !aabb || !vel || !src || !out || nc < 1) return set_error("null argument"), STT_ERR_INVALID;
    float box[3];
    if (!zero_min_box(aabb, box)) return set_error("aabb must start at the origin"), STT_ERR_UNSUPPORTED;
    if (int st = cuda_status(cudaSetDevice(g_device), "cudaSetDevice")) return st;
    const size_t n = (size_t)dim[0] * dim[1] * dim[2];
    DeviceArena a;
    float *dv = a.upload(vel, 3 * n), *ds = a.upload(src, nc * n), *dout = a.alloc(nc * n);
    if (!dv || !ds || !dout) return set_error("device allocation or upload failed"), STT_ERR_NOMEM;
    if (int st = lib_status(stt_warp_box(dim, box, dv, ds, nc, dt, dout, nullptr))) return st;
    return cuda_status(cudaMemcpy(out, dout, nc * n * sizeof(float), cudaMemcpyDeviceToHost), "download");
}

int stt_host_flow_level(const int *dim, const float *aabb, const int *roi, const float *I1, const float *I2,
                        float *V, float *Y, float tol, float lambda, int max_iter, int norm, int n_warps,
                        float huber, int *iters) {
    if (!dim || !aabb || !roi || !I1 || !I2 || !V || !Y) return set_error("null argument"), STT_ERR_INVALID;
    float box[3];
    if (!zero_min_box(aabb, box)) return set_error("aabb must start at the origin"), STT_ERR_UNSUPPORTED;
    if (int st = cuda_status(cudaSetDevice(g_device), "cudaSetDevice")) return st;
    const size_t n = (size_t)dim[0] * dim[1] * dim[2];
    stt_flow_params p{};
    p.tol = tol;
    p.lambda = lambda;
    p.huber = huber;
    p.eta = 1.0f;
    p.sigma = 0.0f;
    p.max_iter = max_iter;
    p.norm = norm;
    p.n_warps = n_warps;
    p.scales = 1;
    stt_flow *f = nullptr;
    if (int st = lib_status(stt_flow_create(g_device, dim, &p, &f))) return st;
    DeviceArena a;
    float *d1 = a.upload(I1, n), *d2 = a.upload(I2, n), *dv = a.upload(V, 3 * n), *dy = a.upload(Y, 10 * n);
    int st = (!d1 || !d2 || !dv || !dy) ? (set_error("device allocation or upload failed"), STT_ERR_NOMEM) : STT_OK;
    if (!st && (st = stt_flow_level(f, dim, box, roi, d1, d2, dv, dy, nullptr)) != STT_OK)
        set_error(stt_flow_last_error(f));
    if (!st && iters) {
        int ne = 0;
        std::vector<int> its(n_warps > 0 ? n_warps : 1);
        if ((st = stt_flow_stats(f, &ne, its.data(), nullptr)) == STT_OK)
            std::memcpy(iters, its.data(), sizeof(int) * (size_t)n_warps);
        else
            set_error(stt_flow_last_error(f));
    }
    if (!st) st = cuda_status(cudaMemcpy(V, dv, 3 * n * sizeof(float), cudaMemcpyDeviceToHost), "download V");
    if (!st) st = cuda_status(cudaMemcpy(Y, dy, 10 * n * sizeof(float), cudaMemcpyDeviceToHost), "download Y");
    stt_flow_destroy(f);
    return st;
}

int stt_host_flow_multiscale(const int *dim, const float *I1, const float *I2, const float *Vin,
                             const float *Y0, float *Vout, float tol, float lambda, int max_iter, int norm,
                             int n_warps, float eta, float sigma, int scales, float huber, const int *cut) {
    if (!dim || !I1 || !I2 || !Vin || !Vout || !cut) return set_error("null argument"), STT_ERR_INVALID;
    if (int st = cuda_status(cudaSetDevice(g_device), "cudaSetDevice")) return st;
    const size_t n = (size_t)dim[0] * dim[1] * dim[2];
    stt_flow_params p{};
    p.tol = tol;
    p.lambda = lambda;
    p.huber = huber;
    p.eta = eta;
    p.sigma = sigma;
    p.max_iter = max_iter;
    p.norm = norm;
    p.n_warps = n_warps;
    p.scales = scales;
    std::memcpy(p.cut, cut, sizeof(p.cut));
    stt_flow *f = nullptr;
    if (int st = lib_status(stt_flow_create(g_device, dim, &p, &f))) return st;
    DeviceArena a;
    float *d1 = a.upload(I1, n), *d2 = a.upload(I2, n), *dv = a.upload(Vin, 3 * n);
    float *dy = Y0 ? a.upload(Y0, 10 * n) : nullptr;
    int st = (!d1 || !d2 || !dv || (Y0 && !dy)) ? (set_error("device allocation or upload failed"), STT_ERR_NOMEM)
                                                : STT_OK;
    if (!st && (st = stt_flow_multiscale(f, d1, d2, dv, dy, nullptr)) != STT_OK) set_error(stt_flow_last_error(f));
    if (!st) st = cuda_status(cudaMemcpy(Vout, dv, 3 * n * sizeof(float), cudaMemcpyDeviceToHost), "download V");
    stt_flow_destroy(f);
    return st;
}

}  // extern "C"
