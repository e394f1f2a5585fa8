// host_solver.cpp -- the space-time primal-dual solve on host buffers
// (stt_host_solver_* of include/stt_host.h): the call a host application
// makes in place of ST_Tomography::Render's image phase
// (S/ST_Tomo/ST_Tomography.cpp:475-607), with its volumes, flows and
// projection stack in host memory.
//
// A handle keeps `slots` complete copies of the device state, each with its
// own stt_solver (the captured CUDA graph of one iteration), and three
// streams shared by the slots: uploads, compute, read-backs.  submit() puts a
// step on the next slot: the inputs go up on the upload stream, the compute
// stream resets the duals and runs the iterations once they have landed, and
// the read-back stream copies the volumes out once they are done.  With two
// slots, step i+1's upload and step i-1's read-back run while step i
// computes; wait() completes the oldest step.  With page-locked host buffers
// the copies are asynchronous; pageable ones work but serialise the copies.
#include <cuda_runtime_api.h>

#include <cstring>
#include <deque>
#include <string>
#include <vector>

#include "stt_host.h"

namespace stt_facade {
void set_error(const std::string &m);
extern thread_local int g_device;
}  // namespace stt_facade

using stt_facade::set_error;

struct stt_host_solver {
    struct Slot {
        float *vol = nullptr, *xbar = nullptr, *xprev = nullptr, *ytv = nullptr, *ytp = nullptr, *ybc = nullptr,
              *flow = nullptr, *proj = nullptr;
        stt_solver *solver = nullptr;
        cudaEvent_t uploaded = nullptr, computed = nullptr, freed = nullptr;
        bool busy = false;
    };
    int device = 0;
    stt_ctx *ctx = nullptr;
    stt_solve_cfg cfg{};
    size_t n = 0, npix = 0;
    int F = 0, V = 0;
    std::vector<Slot> slots;
    std::deque<int> pending;  // slots submitted and not yet waited for, oldest first
    int next = 0;
    cudaStream_t up = nullptr, compute = nullptr, down = nullptr;
    cudaStream_t poll = nullptr;  // reads a completed step's status word; holds nothing else
};

namespace {

int cuda_err(cudaError_t e, const char *where) {
    if (e == cudaSuccess) return STT_OK;
    set_error(std::string(where) + ": " + cudaGetErrorString(e));
    return STT_ERR_CUDA;
}

#define HCUDA(call, where)                                  \
    do {                                                    \
        int st_ = cuda_err((call), where);                  \
        if (st_) return st_;                                \
    } while (0)

int alloc(float *&p, size_t count) {
    if (cudaMalloc((void **)&p, count * sizeof(float)) != cudaSuccess) {
        cudaGetLastError();
        p = nullptr;
        set_error("cudaMalloc of the host solver's device state failed");
        return STT_ERR_NOMEM;
    }
    return STT_OK;
}

// Completes the oldest pending step: its read-back has landed in vol_out.
int wait_oldest(stt_host_solver *h) {
    if (h->pending.empty()) return STT_OK;
    const int k = h->pending.front();
    h->pending.pop_front();
    stt_host_solver::Slot &s = h->slots[k];
    s.busy = false;
    HCUDA(cudaEventSynchronize(s.freed), "cudaEventSynchronize");
    // on a stream of its own: the compute stream may already hold the next
    // step, and waiting for it here would stall the pipeline
    const stt_status st = stt_solver_poll_status(s.solver, h->poll);
    if (st != STT_OK) {
        set_error(stt_solver_last_error(s.solver));
        return st;
    }
    return STT_OK;
}

}  // namespace

extern "C" {

int stt_host_solver_create(const stt_geometry *g, const stt_solve_cfg *cfg, int slots, stt_host_solver **out) {
    if (!g || !cfg || !out || slots < 1 || slots > 8) return set_error("null argument or slots outside 1..8"), STT_ERR_INVALID;
    if (cfg->halo) return set_error("the host solver runs whole sequences (no halo)"), STT_ERR_UNSUPPORTED;
    if (cfg->storage != STT_DTYPE_F32)
        return set_error("the host solver takes FP32 host arrays (storage must be STT_DTYPE_F32)"), STT_ERR_UNSUPPORTED;
    *out = nullptr;
    stt_host_solver *h = new stt_host_solver();
    h->device = stt_facade::g_device;
    h->cfg = *cfg;
    h->F = cfg->n_frames;
    h->V = cfg->views_per_frame;
    h->n = (size_t)g->nx * g->ny * g->nz;
    h->npix = (size_t)g->W * g->H;
    auto bail = [&](int st) {
        std::string keep = stt_host_last_error();
        stt_host_solver_destroy(h);
        set_error(keep);
        return st;
    };
    if (int st = cuda_err(cudaSetDevice(h->device), "cudaSetDevice")) return bail(st);
    if (int st = stt_create(&h->ctx, h->device)) return set_error(stt_last_error(nullptr)), bail(st);
    if (int st = stt_set_geometry(h->ctx, g)) return set_error(stt_last_error(h->ctx)), bail(st);
    const size_t n = h->n, F = (size_t)h->F;
    h->slots.resize(slots);
    for (stt_host_solver::Slot &s : h->slots) {
        int st = STT_OK;
        if (!st) st = alloc(s.vol, (F + 1) * n);
        if (!st) st = alloc(s.xbar, (F + 1) * n);
        if (!st) st = alloc(s.xprev, F * n);
        if (!st) st = alloc(s.ytv, 3 * F * n);
        if (!st) st = alloc(s.ytp, F * n);
        if (!st) st = alloc(s.ybc, F * n);
        if (!st) st = alloc(s.flow, 3 * F * n);
        if (!st) st = alloc(s.proj, F * (size_t)h->V * h->npix);
        if (st) return bail(st);
        stt_pd_state state{};
        state.vol = s.vol;
        state.xbar = s.xbar;
        state.xprev = s.xprev;
        state.ytv = s.ytv;
        state.ytp = s.ytp;
        state.ybc = s.ybc;
        state.flow = s.flow;
        state.proj = s.proj;
        if ((st = stt_solver_create(h->ctx, cfg, &state, &s.solver))) return set_error(stt_last_error(h->ctx)), bail(st);
        if ((st = cuda_err(cudaEventCreateWithFlags(&s.uploaded, cudaEventDisableTiming), "event"))) return bail(st);
        if ((st = cuda_err(cudaEventCreateWithFlags(&s.computed, cudaEventDisableTiming), "event"))) return bail(st);
        if ((st = cuda_err(cudaEventCreateWithFlags(&s.freed, cudaEventDisableTiming), "event"))) return bail(st);
    }
    for (cudaStream_t *sp : {&h->up, &h->compute, &h->down, &h->poll})
        if (int st = cuda_err(cudaStreamCreateWithFlags(sp, cudaStreamNonBlocking), "stream")) return bail(st);
    *out = h;
    return STT_OK;
}

int stt_host_solver_submit(stt_host_solver *h, const float *vol, const float *flow, const float *proj, int n_iters,
                           float *vol_out) {
    if (!h || !vol || !flow || !proj || n_iters < 0) return set_error("null argument or n_iters < 0"), STT_ERR_INVALID;
    HCUDA(cudaSetDevice(h->device), "cudaSetDevice");
    const int k = h->next;
    h->next = (h->next + 1) % (int)h->slots.size();
    stt_host_solver::Slot &s = h->slots[k];
    while (s.busy)  // every slot in use: complete the oldest steps until this one is free
        if (int st = wait_oldest(h)) return st;
    const size_t n = h->n, F = (size_t)h->F, vb = n * sizeof(float);
    // inputs: after the slot's previous read-back
    HCUDA(cudaStreamWaitEvent(h->up, s.freed, 0), "stream wait");
    HCUDA(cudaMemcpyAsync(s.vol, vol, F * vb, cudaMemcpyHostToDevice, h->up), "upload volumes");
    HCUDA(cudaMemcpyAsync(s.flow, flow, 3 * F * vb, cudaMemcpyHostToDevice, h->up), "upload flows");
    HCUDA(cudaMemcpyAsync(s.proj, proj, F * h->V * h->npix * sizeof(float), cudaMemcpyHostToDevice, h->up),
          "upload projections");
    HCUDA(cudaEventRecord(s.uploaded, h->up), "event record");
    // compute: the duplicated last frame (VolumeData.cpp:124-126), X_bar = V,
    // zero duals, then the iterations from the first view order on
    HCUDA(cudaStreamWaitEvent(h->compute, s.uploaded, 0), "stream wait");
    HCUDA(cudaMemcpyAsync(s.vol + F * n, s.vol + (F - 1) * n, vb, cudaMemcpyDeviceToDevice, h->compute), "copy");
    HCUDA(cudaMemcpyAsync(s.xbar, s.vol, (F + 1) * vb, cudaMemcpyDeviceToDevice, h->compute), "copy");
    HCUDA(cudaMemsetAsync(s.xprev, 0, F * vb, h->compute), "clear");
    HCUDA(cudaMemsetAsync(s.ytv, 0, 3 * F * vb, h->compute), "clear");
    HCUDA(cudaMemsetAsync(s.ytp, 0, F * vb, h->compute), "clear");
    HCUDA(cudaMemsetAsync(s.ybc, 0, F * vb, h->compute), "clear");
    if (int st = stt_solver_set_iteration(s.solver, 0, h->compute)) return set_error(stt_solver_last_error(s.solver)), st;
    if (n_iters > 0)
        if (int st = stt_solver_iterate(s.solver, n_iters, h->compute))
            return set_error(stt_solver_last_error(s.solver)), st;
    HCUDA(cudaEventRecord(s.computed, h->compute), "event record");
    // read-back
    HCUDA(cudaStreamWaitEvent(h->down, s.computed, 0), "stream wait");
    if (vol_out) HCUDA(cudaMemcpyAsync(vol_out, s.vol, F * vb, cudaMemcpyDeviceToHost, h->down), "read back");
    HCUDA(cudaEventRecord(s.freed, h->down), "event record");
    s.busy = true;
    h->pending.push_back(k);
    return STT_OK;
}

int stt_host_solver_wait(stt_host_solver *h) {
    if (!h) return set_error("null handle"), STT_ERR_INVALID;
    HCUDA(cudaSetDevice(h->device), "cudaSetDevice");
    return wait_oldest(h);
}

int stt_host_solver_pending(const stt_host_solver *h) { return h ? (int)h->pending.size() : 0; }

int stt_host_solver_destroy(stt_host_solver *h) {
    if (!h) return STT_OK;
    cudaSetDevice(h->device);
    if (h->up) cudaStreamSynchronize(h->up);
    if (h->compute) cudaStreamSynchronize(h->compute);
    if (h->down) cudaStreamSynchronize(h->down);
    for (stt_host_solver::Slot &s : h->slots) {
        if (s.solver) stt_solver_destroy(s.solver);
        for (cudaEvent_t e : {s.uploaded, s.computed, s.freed})
            if (e) cudaEventDestroy(e);
        for (float *p : {s.vol, s.xbar, s.xprev, s.ytv, s.ytp, s.ybc, s.flow, s.proj}) cudaFree(p);
    }
    for (cudaStream_t st : {h->up, h->compute, h->down, h->poll})
        if (st) cudaStreamDestroy(st);
    if (h->ctx) stt_destroy(h->ctx);
    delete h;
    return STT_OK;
}

}  // extern "C"
