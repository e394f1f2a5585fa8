// stt_solver.cu -- one space-time primal-dual iteration of ST_Tomography::Render
// (S/ST_Tomo/ST_Tomography.cpp:492-607) over all frames, enqueued three ways:
//
//   STT_SOLVE_PLAIN    the per-view GPU form: frames in order, every view's
//                      forward projection, correction and backprojection as
//                      separate launches from a host loop, host sync per view;
//   STT_SOLVE_STREAMS  the batched form enqueued directly: all duals first,
//                      then the per-frame primal + SART + over-relaxation
//                      chains on one stream per frame, FP fused with the
//                      correction;
//   STT_SOLVE_GRAPH    the batched form captured once into a CUDA graph and
//                      replayed (the view order is drawn on the device from a
//                      counter, so every replay gets a fresh seeded order);
//   STT_SOLVE_PERSISTENT the whole iteration of every frame (view order,
//                      warps, dual and primal steps, SART, ROI mask,
//                      over-relaxation) in one persistent cooperative launch
//                      (k_iter_persistent, k_persist.cu), captured and
//                      replayed as a graph.
//
// Reordering "all duals, then every frame's primal chain" is exact: frame f's
// dual reads X_bar[f], X_bar[f+1] and flow[f] only, and X_bar[f] is rewritten
// only by frame f's own over-relaxation (ST_Tomography.cpp:503-534 vs :598),
// which the graph orders after the duals of frames f-1 and f.
#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "stt.h"
#include "stt_ctx.h"
#include "stt_internal.cuh"
#include "stt_kernels.h"

namespace stt {
namespace {

// One thread per local frame: Fisher-Yates with SplitMix64 (the same stream
// as stt_permutation), then thread 0 advances the iteration counter.  Local
// frame f is frame frame0 + f of a sequence of `total` frames.
__global__ void k_make_perm(unsigned long long seed, unsigned long long *counter, int frames, int total, int frame0,
                            int views, int *perm) {
    const int f = threadIdx.x + blockIdx.x * blockDim.x;
    const unsigned long long iter = *counter;
    if (f < frames) view_order(seed, iter, total, frame0 + f, views, perm + (size_t)f * views);
    __syncthreads();
    if (f == 0) *counter = iter + 1;
}

}  // namespace

cudaError_t launch_make_perm(unsigned long long seed, unsigned long long *counter, int frames, int total,
                             int frame0, int views, int *perm, cudaStream_t s) {
    if (frames > 1024) return cudaErrorInvalidValue;  // one block, one thread per frame
    k_make_perm<<<1, ((frames + 31) / 32) * 32, 0, s>>>(seed, counter, frames, total, frame0, views, perm);
    return cudaGetLastError();
}

__global__ void k_set_counter(unsigned long long *counter, unsigned long long v) { *counter = v; }

cudaError_t launch_set_counter(unsigned long long *counter, unsigned long long v, cudaStream_t s) {
    k_set_counter<<<1, 1, 0, s>>>(counter, v);
    return cudaGetLastError();
}

void host_perm(unsigned long long seed, unsigned long long iter, int frames, int f, int views, int *p) {
    view_order(seed, iter, frames, f, views, p);
}

}  // namespace stt

// The context internals the solver needs (defined in stt_capi.cu).
extern "C" stt_status stt_internal_geom(stt_ctx *ctx, const void **geom, const void **views);

struct stt_solver {
    stt_ctx *ctx = nullptr;
    stt_solve_cfg cfg{};
    stt_pd_state st{};
    const stt::GeomDev *g = nullptr;
    const stt::ViewRec *views = nullptr;
    int F = 0, V = 0;
    int total_frames = 0;  // frames of the whole (possibly sharded) sequence
    size_t n = 0, npix = 0;
    float *warpbuf = nullptr;  // F volumes: backward-warped X_bar[f+1], then forward-warped Y_bc[f-1]
    float *corr = nullptr;     // F correction images
    float *ax = nullptr;       // plain form: forward projection image
    void *volt = nullptr;      // F z-fastest volume copies (views gathering along x), in the state's storage
    float *raylen = nullptr;   // F sticky ray-length images
    float2 *acc = nullptr;     // ray-based BP accumulators, F volumes
    int *perm = nullptr;       // F x V device view order
    unsigned long long *counter = nullptr;
    int *status = nullptr;     // raised by a bounded device-side wait that gave up
    unsigned long long host_iter = 0;
    std::vector<cudaStream_t> streams;
    std::vector<cudaEvent_t> ev_dual, ev_done;
    cudaEvent_t ev_fork = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaGraph_t pgraph[2] = {nullptr, nullptr};
    cudaGraphExec_t pexec[2] = {nullptr, nullptr};
    long long launches_per_iter = 0;
    long long phase_launches[2] = {0, 0};
    std::vector<stt::CorrTex> corr_tex;  // batched modes: per frame, the correction as a texture
    std::vector<stt::FpSlabMaps> fpmaps;  // batched modes: per frame, TMA maps of the volume and its copy
    std::vector<stt::FpTex> fptex;  // batched modes, a tld4 gather form: per frame, the volume's textures
    stt::SweepJob *jobs_d = nullptr;  // STT_SOLVE_PERSISTENT: one job per frame
    unsigned *sweep_bar = nullptr;    // the jobs' barrier and ticket words (4 per frame), then the grid's
    int sweep_blocks = 0;
    bool sweep_wide = false;
    bool sweep_direct = false;        // the cooperative launch could not be captured
    std::string err;
};

namespace {

stt_status sfail(stt_solver *s, stt_status st, const std::string &m) {
    if (s) s->err = m;
    return st;
}

// A failed CUDA call: its error is read and cleared (cudaGetLastError), so a
// non-sticky error does not resurface in a later, unrelated launch check.
#define SCUDA(s, call, where)                                                                         \
    do {                                                                                              \
        cudaError_t e_ = (call);                                                                      \
        if (e_ != cudaSuccess) {                                                                      \
            cudaGetLastError();                                                                       \
            return sfail(s, STT_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(e_));      \
        }                                                                                             \
    } while (0)

stt::PdParams pdp(const stt_pd_params &p) {
    stt::PdParams q;
    q.sigma = p.sigma;
    q.tau = p.tau;
    q.tv_w = p.tv_w;
    q.tp_w = p.tp_w;
    q.bc_w = p.bc_w;
    q.hf = p.huber_factor;
    q.gmax = p.gmax;
    for (int i = 0; i < 8; ++i) q.cut[i] = p.cut[i];
    return q;
}

// The primal volumes (vol, xbar, xprev) and the sinogram stack in the state's
// storage T: float, or BF16 bits (unsigned short) with stt_solve_cfg.storage.
template <typename T>
T *vol_of(stt_solver *s, float *base, int f) {
    return reinterpret_cast<T *>(base) + (size_t)f * s->n;
}

// Frame f's dual step: backward warp of X_bar[f+1] along flow[f]
// (ST_Tomography.cpp:502-503) then the fused dual kernel (:504-534).
template <typename T>
stt_status enqueue_dual(stt_solver *s, int f, cudaStream_t cs, long long &nl) {
    const int d[3] = {s->g->nx, s->g->ny, s->g->nz};
    const size_t n = s->n;
    float *bw = s->warpbuf + f * n;
    const T *xf = vol_of<T>(s, s->st.xbar, f), *xf1 = vol_of<T>(s, s->st.xbar, f + 1);
    SCUDA(s, stt::launch_warp(d, s->st.flow + (size_t)f * 3 * n, xf1, 1, -1.0f, bw, cs, s->status), "warp (dual)");
    SCUDA(s, stt::launch_pd_dual(d, pdp(s->cfg.pd), xf, xf1, bw, s->st.ytv + (size_t)f * 3 * n, s->st.ytp + f * n,
                                 s->st.ybc + f * n, cs),
          "pd_dual");
    nl += 2;
    return STT_OK;
}

// Frame f's primal step (ST_Tomography.cpp:536-578): forward warp of
// Y_bc[f-1] along flow[f-1] for f > 0, then the fused primal kernel.
// With a halo, local frame 0 continues the previous shard: its "f-1" terms
// come from ytp_halo / ybc_halo / flow_halo.
template <typename T>
stt_status enqueue_primal(stt_solver *s, int f, cudaStream_t cs, long long &nl) {
    const int d[3] = {s->g->nx, s->g->ny, s->g->nz};
    const size_t n = s->n;
    float *fw = s->warpbuf + f * n;
    const bool first = (f == 0) && !s->cfg.halo;
    const float *ytp_prev = nullptr, *ybc_prev = nullptr, *flow_prev = nullptr;
    if (f > 0) {
        ytp_prev = s->st.ytp + (f - 1) * n;
        ybc_prev = s->st.ybc + (f - 1) * n;
        flow_prev = s->st.flow + (size_t)(f - 1) * 3 * n;
    } else if (s->cfg.halo) {
        ytp_prev = s->st.ytp_halo;
        ybc_prev = s->st.ybc_halo;
        flow_prev = s->st.flow_halo;
    }
    if (!first) {
        SCUDA(s, stt::launch_warp(d, flow_prev, ybc_prev, 1, 1.0f, fw, cs, s->status), "warp (primal)");
        ++nl;
    }
    SCUDA(s, stt::launch_pd_primal(d, pdp(s->cfg.pd), first, ytp_prev, s->st.ytp + f * n, first ? nullptr : fw,
                                   s->st.ybc + f * n, s->st.ytv + (size_t)f * 3 * n, vol_of<T>(s, s->st.vol, f),
                                   vol_of<T>(s, s->st.xprev, f), cs),
          "pd_primal");
    ++nl;
    return STT_OK;
}

// SART(f) (ST_Tomography.cpp:616-808) as fused launches, views read from the
// device-side order, then the ROI mask (:793-804) fused with the
// over-relaxation X_bar[f] = 2V - X_prev (:586-604).
// The fused forward projection of one view: FP32 storage through the tuned
// gather variant and, where the maps apply, the slab-staged kernel; BF16
// storage through the gather kernel.  Returns the kernels launched.
int fp_corr(stt_solver *s, int f, const float *vol, const float *volt, const stt::ViewSel &sel, const float *stack,
            float *rl, float *corr, cudaStream_t cs, unsigned long long surf, cudaError_t &e) {
    const stt::FpSlabMaps *maps = s->fpmaps.empty() ? nullptr : &s->fpmaps[f];
    e = stt::launch_fp_corr(*s->g, s->views, vol, volt, sel, stack, rl, corr, cs, surf, maps, s->status,
                            s->ctx->tuning.fp, s->fptex.empty() ? nullptr : &s->fptex[f]);
    return (maps && maps->ok) ? 2 : 1;  // slab-staged + gather kernels, or gather only
}

int fp_corr(stt_solver *s, int f, const unsigned short *vol, const unsigned short *volt, const stt::ViewSel &sel,
            const unsigned short *stack, float *rl, float *corr, cudaStream_t cs, unsigned long long surf,
            cudaError_t &e) {
    const stt::FpSlabMaps *maps = s->fpmaps.empty() ? nullptr : &s->fpmaps[f];
    e = stt::launch_fp_corr(*s->g, s->views, vol, volt, sel, stack, rl, corr, cs, surf, maps, s->status,
                            s->ctx->tuning.fp16, s->fptex.empty() ? nullptr : &s->fptex[f]);
    return (maps && maps->ok) ? 2 : 1;
}

template <typename T>
stt_status enqueue_sart_batched(stt_solver *s, int f, cudaStream_t cs, long long &nl) {
    const stt::GeomDev &g = *s->g;
    const int V = s->V;
    T *vol = vol_of<T>(s, s->st.vol, f);
    float *corr = s->corr + f * s->npix;
    const T *stack = reinterpret_cast<const T *>(s->st.proj) + (size_t)f * V * s->npix;
    const int voxel = s->cfg.bp_mode == 0;
    T *volt = reinterpret_cast<T *>(s->volt) + f * s->n;
    for (int i = 0; i < V; ++i) {
        const stt::ViewSel sel{0, s->perm + (size_t)f * V, i, f * V};
        SCUDA(s, stt::launch_transpose_for_view(g, s->views, sel, vol, volt, cs), "transpose");
        const bool tex = voxel && !s->corr_tex.empty();
        cudaError_t e = cudaSuccess;
        nl += fp_corr(s, f, vol, volt, sel, stack, voxel ? s->raylen + f * s->npix : nullptr, corr, cs,
                      tex ? s->corr_tex[f].surf : 0, e);
        SCUDA(s, e, "fp_corr");
        if (voxel)
            SCUDA(s, stt::launch_bp_voxel(g, s->views, sel, corr, vol, (float)s->cfg.alpha, s->cfg.pd.gmax, cs,
                                          tex ? s->corr_tex[f].tex : 0, s->ctx->tuning.bp),
                  "bp_voxel");
        else
            SCUDA(s, stt::launch_bp_ray(g, s->views, sel, corr, s->acc + f * s->n, vol, s->cfg.pd.gmax, cs,
                                        s->ctx->tuning.ray),
                  "bp_ray");
        nl += voxel ? 2 : 3;
    }
    const int d[3] = {g.nx, g.ny, g.nz};
    SCUDA(s, stt::launch_roi_apply(d, s->cfg.roi_cut, s->cfg.pd.cut, vol, vol_of<T>(s, s->st.xprev, f),
                                   vol_of<T>(s, s->st.xbar, f), cs),
          "roi_apply");
    ++nl;
    return STT_OK;
}

bool bf16(const stt_solver *s) { return s->cfg.storage == STT_DTYPE_BF16; }

// Phase 0: the view order, then every frame's dual on its own stream.  With
// `join` the frame streams rejoin `main` (phases run separately).
stt_status enqueue_phase0(stt_solver *s, cudaStream_t main, long long &nl, bool join) {
    const int F = s->F;
    SCUDA(s, stt::launch_make_perm(s->cfg.seed, s->counter, F, s->total_frames, s->cfg.frame_offset, s->V, s->perm,
                                   main),
          "make_perm");
    ++nl;
    SCUDA(s, cudaEventRecord(s->ev_fork, main), "event record");
    for (int f = 0; f < F; ++f) SCUDA(s, cudaStreamWaitEvent(s->streams[f], s->ev_fork, 0), "stream wait");
    for (int f = 0; f < F; ++f) {
        stt_status st = bf16(s) ? enqueue_dual<unsigned short>(s, f, s->streams[f], nl)
                                : enqueue_dual<float>(s, f, s->streams[f], nl);
        if (st) return st;
        SCUDA(s, cudaEventRecord(s->ev_dual[f], s->streams[f]), "event record");
        if (join) SCUDA(s, cudaStreamWaitEvent(main, s->ev_dual[f], 0), "stream wait");
    }
    return STT_OK;
}

// Phase 1: per frame, after the previous frame's dual, the primal step, SART
// and the ROI/over-relaxation; the frame chains rejoin `main`.  With `fork`
// (the phases enqueued separately) they first wait for `main`, which phase 0
// has joined already (every dual is done; work the caller queued between the
// phases is ordered too), so no frame waits on a phase-0 event: in the
// captured form those events belong to the other phase's graph.
stt_status enqueue_phase1(stt_solver *s, cudaStream_t main, long long &nl, bool fork) {
    const int F = s->F;
    if (fork) {
        SCUDA(s, cudaEventRecord(s->ev_fork, main), "event record");
        for (int f = 0; f < F; ++f) SCUDA(s, cudaStreamWaitEvent(s->streams[f], s->ev_fork, 0), "stream wait");
    }
    for (int f = 0; f < F; ++f) {
        cudaStream_t cs = s->streams[f];
        if (f > 0 && !fork) SCUDA(s, cudaStreamWaitEvent(cs, s->ev_dual[f - 1], 0), "stream wait");
        stt_status st = bf16(s) ? enqueue_primal<unsigned short>(s, f, cs, nl) : enqueue_primal<float>(s, f, cs, nl);
        if (st) return st;
        if ((st = bf16(s) ? enqueue_sart_batched<unsigned short>(s, f, cs, nl)
                          : enqueue_sart_batched<float>(s, f, cs, nl)))
            return st;
        SCUDA(s, cudaEventRecord(s->ev_done[f], cs), "event record");
        SCUDA(s, cudaStreamWaitEvent(main, s->ev_done[f], 0), "stream wait");
    }
    return STT_OK;
}

stt_status enqueue_batched(stt_solver *s, cudaStream_t main, long long &nl) {
    stt_status st = enqueue_phase0(s, main, nl, false);
    if (st) return st;
    return enqueue_phase1(s, main, nl, false);
}

// STT_SOLVE_PERSISTENT, before the sweep: per frame, after the previous
// frame's dual, the primal step; the frame chains rejoin `main` (`fork`: as in
// enqueue_phase1).
stt_status enqueue_primals(stt_solver *s, cudaStream_t main, long long &nl, bool fork) {
    const int F = s->F;
    if (fork) {
        SCUDA(s, cudaEventRecord(s->ev_fork, main), "event record");
        for (int f = 0; f < F; ++f) SCUDA(s, cudaStreamWaitEvent(s->streams[f], s->ev_fork, 0), "stream wait");
    }
    for (int f = 0; f < F; ++f) {
        cudaStream_t cs = s->streams[f];
        if (f > 0 && !fork) SCUDA(s, cudaStreamWaitEvent(cs, s->ev_dual[f - 1], 0), "stream wait");
        stt_status st = bf16(s) ? enqueue_primal<unsigned short>(s, f, cs, nl) : enqueue_primal<float>(s, f, cs, nl);
        if (st) return st;
        SCUDA(s, cudaEventRecord(s->ev_done[f], cs), "event record");
        SCUDA(s, cudaStreamWaitEvent(main, s->ev_done[f], 0), "stream wait");
    }
    return STT_OK;
}

// Every frame's SART call, ROI mask and over-relaxation: one persistent launch.
stt_status enqueue_sweep(stt_solver *s, cudaStream_t main, long long &nl) {
    SCUDA(s, cudaMemsetAsync(s->sweep_bar, 0, 4 * (size_t)s->F * sizeof(unsigned), main), "barrier reset");
    SCUDA(s, stt::launch_sweep_persistent(s->jobs_d, s->F, s->sweep_blocks, bf16(s), s->sweep_wide, s->status, main),
          "persistent sweep");
    ++nl;
    return STT_OK;
}

// The whole iteration: one cooperative launch (view orders, warps, duals,
// primals, SART calls, ROI masks, over-relaxations of every frame), or, with
// more frames than resident blocks, the duals and primals as launches and
// then the sweep.
stt_status enqueue_persistent(stt_solver *s, cudaStream_t main, long long &nl) {
    if (s->F <= s->sweep_blocks) {
        SCUDA(s, cudaMemsetAsync(s->sweep_bar, 0, (4 * (size_t)s->F + 2) * sizeof(unsigned), main), "barrier reset");
        SCUDA(s, stt::launch_iter_persistent(s->jobs_d, s->F, s->sweep_blocks, bf16(s), s->sweep_wide,
                                             s->sweep_bar + 4 * s->F, s->status, main),
              "persistent iteration");
        ++nl;
        return STT_OK;
    }
    stt_status st = enqueue_phase0(s, main, nl, false);
    if (!st) st = enqueue_primals(s, main, nl, false);
    if (!st) st = enqueue_sweep(s, main, nl);
    return st;
}

// The solver's frames as persistent-sweep jobs; the caller sets block0,
// nblocks and bar.
void fill_jobs(const stt_solver *s, stt::SweepJob *jobs) {
    const size_t es = s->cfg.storage == STT_DTYPE_BF16 ? 2 : 4, n = s->n, npix = s->npix;
    const int V = s->V;
    for (int f = 0; f < s->F; ++f) {
        stt::SweepJob &J = jobs[f];
        J = stt::SweepJob{};
        J.g = *s->g;
        J.views = s->views;
        J.perm = s->perm + (size_t)f * V;
        J.view_base = f * V;
        J.V = V;
        J.vol = reinterpret_cast<unsigned char *>(s->st.vol) + (size_t)f * n * es;
        J.volt = static_cast<unsigned char *>(s->volt) + (size_t)f * n * es;
        J.stack = reinterpret_cast<const unsigned char *>(s->st.proj) + (size_t)f * V * npix * es;
        J.raylen = s->raylen + (size_t)f * npix;
        J.corr = s->corr + (size_t)f * npix;
        J.xprev = reinterpret_cast<unsigned char *>(s->st.xprev) + (size_t)f * n * es;
        J.xbar = reinterpret_cast<unsigned char *>(s->st.xbar) + (size_t)f * n * es;
        J.alpha = (float)s->cfg.alpha;
        J.gmax = s->cfg.pd.gmax;
        for (int q = 0; q < 8; ++q) J.roi[q] = s->cfg.roi_cut[q], J.pdcut[q] = s->cfg.pd.cut[q];
        const int nmax = std::max(s->g->nx, std::max(s->g->ny, s->g->nz));
        J.work = (double)V * ((double)n + (double)npix * nmax / 2.0);
        // the whole-iteration launch: view order, warps, dual and primal steps
        const stt_pd_params &pd = s->cfg.pd;
        J.sigma = pd.sigma, J.tau = pd.tau, J.tv_w = pd.tv_w, J.tp_w = pd.tp_w, J.bc_w = pd.bc_w;
        J.hf = pd.huber_factor;
        J.first = f == 0 && !s->cfg.halo;
        J.xbar1 = reinterpret_cast<const unsigned char *>(s->st.xbar) + (size_t)(f + 1) * n * es;
        J.flow = s->st.flow + (size_t)f * 3 * n;
        J.flow_prev = f > 0 ? s->st.flow + (size_t)(f - 1) * 3 * n : nullptr;
        J.ytv = s->st.ytv + (size_t)f * 3 * n;
        J.ytp = s->st.ytp + (size_t)f * n;
        J.ybc = s->st.ybc + (size_t)f * n;
        J.ytp_prev = f > 0 ? s->st.ytp + (size_t)(f - 1) * n : nullptr;
        J.ybc_prev = f > 0 ? s->st.ybc + (size_t)(f - 1) * n : nullptr;
        J.seed = s->cfg.seed;
        J.counter = s->counter;
        J.frame_seq = s->cfg.frame_offset + f;
        J.frames_total = s->total_frames;
        J.counter_owner = f == 0;
    }
}

// Captures `enqueue` into a graph: the instantiated graph, or null with the
// failure cleared (the caller then enqueues directly).
cudaGraphExec_t try_capture(stt_solver *s, cudaGraph_t &graph, long long &nl,
                            stt_status (*enqueue)(stt_solver *, cudaStream_t, long long &), stt_status &st) {
    graph = nullptr;
    cudaStream_t cap;
    if (cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking) != cudaSuccess) {
        cudaGetLastError();
        return nullptr;
    }
    cudaGraphExec_t exec = nullptr;
    if (cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
        st = enqueue(s, cap, nl);
        cudaGraph_t g = nullptr;
        const cudaError_t ce = cudaStreamEndCapture(cap, &g);
        if (!st && ce == cudaSuccess && g && cudaGraphInstantiate(&exec, g, 0) == cudaSuccess) {
            graph = g;
        } else {
            if (g) cudaGraphDestroy(g);
            exec = nullptr;
        }
    }
    cudaGetLastError();
    cudaStreamDestroy(cap);
    return exec;
}

// The per-view form: frame by frame as the reference loops, each view's
// forward projection, correction and backprojection as separate launches,
// and a host synchronisation after every view.
template <typename T>
stt_status plain_frame_tail(stt_solver *s, int f, cudaStream_t cs, long long &nl);

// phase -1: the reference's interleaved frame loop; phase 0: every dual;
// phase 1: every frame's primal, SART and over-relaxation.
template <typename T>
stt_status run_plain_t(stt_solver *s, cudaStream_t cs, long long &nl, int phase) {
    const int F = s->F;
    for (int f = 0; f < F; ++f) {
        stt_status st = STT_OK;
        if (phase <= 0 && (st = enqueue_dual<T>(s, f, cs, nl))) return st;
        if (phase == 0) continue;
        if ((st = enqueue_primal<T>(s, f, cs, nl))) return st;
        if ((st = plain_frame_tail<T>(s, f, cs, nl))) return st;
    }
    if (phase == 0) {
        SCUDA(s, cudaStreamSynchronize(cs), "synchronize");
        return STT_OK;
    }
    ++s->host_iter;
    // keep the device counter in step so that the modes can be mixed
    SCUDA(s, cudaMemcpyAsync(s->counter, &s->host_iter, sizeof(unsigned long long), cudaMemcpyHostToDevice, cs),
          "counter update");
    SCUDA(s, cudaStreamSynchronize(cs), "synchronize");
    return STT_OK;
}

stt_status run_plain(stt_solver *s, cudaStream_t cs, long long &nl, int phase) {
    return bf16(s) ? run_plain_t<unsigned short>(s, cs, nl, phase) : run_plain_t<float>(s, cs, nl, phase);
}

cudaError_t fp_view(const stt::GeomDev &g, const stt::ViewRec *views, const float *vol, const float *volt, int view,
                    float *ax, float *rl, cudaStream_t cs) {
    return stt::launch_fp(g, views, vol, volt, view, 1, ax, rl, nullptr, cs);
}

cudaError_t fp_view(const stt::GeomDev &g, const stt::ViewRec *views, const unsigned short *vol,
                    const unsigned short *volt, int view, float *ax, float *rl, cudaStream_t cs) {
    return stt::launch_fp_bf16(g, views, vol, volt, view, 1, ax, rl, nullptr, cs);
}

template <typename T>
stt_status plain_frame_tail(stt_solver *s, int f, cudaStream_t cs, long long &nl) {
    const stt::GeomDev &g = *s->g;
    const int V = s->V;
    const int d[3] = {g.nx, g.ny, g.nz};
    std::vector<int> perm(V);
    const int voxel = s->cfg.bp_mode == 0;
    {
        stt::host_perm(s->cfg.seed, s->host_iter, s->total_frames, s->cfg.frame_offset + f, V, perm.data());
        T *vol = vol_of<T>(s, s->st.vol, f);
        float *corr = s->corr + f * s->npix;
        float *rl = s->raylen + f * s->npix;
        for (int i = 0; i < V; ++i) {
            const int view = f * V + perm[i];
            const T *b = reinterpret_cast<const T *>(s->st.proj) + ((size_t)f * V + perm[i]) * s->npix;
            const stt::ViewSel sel{view, nullptr, 0, view};
            T *volt = reinterpret_cast<T *>(s->volt) + f * s->n;
            SCUDA(s, stt::launch_transpose_for_view(g, s->views, sel, vol, volt, cs), "transpose");
            ++nl;
            if (voxel) {
                SCUDA(s, fp_view(g, s->views, vol, volt, view, s->ax, rl, cs), "fp");
                SCUDA(s, stt::launch_correction((long long)s->npix, b, s->ax, rl, corr, cs), "correction");
                SCUDA(s, stt::launch_bp_voxel(g, s->views, sel, corr, vol, (float)s->cfg.alpha, s->cfg.pd.gmax, cs),
                      "bp_voxel");
                nl += 3;
            } else {
                // ray-based: the producer is reset after every view (L = 0 on a miss)
                SCUDA(s, stt::launch_fill_zero(rl, (long long)s->npix, cs), "fill");
                SCUDA(s, fp_view(g, s->views, vol, volt, view, s->ax, rl, cs), "fp");
                SCUDA(s, stt::launch_correction((long long)s->npix, b, s->ax, rl, corr, cs), "correction");
                SCUDA(s, stt::launch_bp_ray(g, s->views, sel, corr, s->acc + f * s->n, vol, s->cfg.pd.gmax, cs,
                                            s->ctx->tuning.ray),
                      "bp_ray");
                nl += 5;
            }
            SCUDA(s, cudaStreamSynchronize(cs), "per-view synchronize");
        }
        SCUDA(s, stt::launch_roi_apply(d, s->cfg.roi_cut, s->cfg.pd.cut, vol, vol_of<T>(s, s->st.xprev, f),
                                       vol_of<T>(s, s->st.xbar, f), cs),
              "roi_apply");
        ++nl;
    }
    return STT_OK;
}

template <typename T>
stt_status alloc(stt_solver *s, T *&p, size_t count, const char *what) {
    cudaError_t e = cudaMalloc((void **)&p, count * sizeof(T));
    if (e != cudaSuccess) {
        p = nullptr;
        return sfail(s, STT_ERR_NOMEM, std::string("cudaMalloc(") + what + "): " + cudaGetErrorString(e));
    }
    return STT_OK;
}

}  // namespace

extern "C" {

stt_status stt_solver_iterate_phase(stt_solver *s, int phase, void *stream);

stt_status stt_solver_create(stt_ctx *ctx, const stt_solve_cfg *cfg, const stt_pd_state *state,
                             stt_solver **out) {
    if (!ctx || !cfg || !state || !out) return STT_ERR_INVALID;
    *out = nullptr;
    const void *gp = nullptr, *vp = nullptr;
    stt_status st = stt_internal_geom(ctx, &gp, &vp);
    if (st) return st;
    const stt::GeomDev *g = (const stt::GeomDev *)gp;
    if (cfg->n_frames < 1 || cfg->views_per_frame < 1 || (long long)cfg->n_frames * cfg->views_per_frame > g->n_views)
        return STT_ERR_INVALID;
    if (cfg->bp_mode != 0 && cfg->bp_mode != 1) return STT_ERR_INVALID;
    if (cfg->mode < STT_SOLVE_PLAIN || cfg->mode > STT_SOLVE_PERSISTENT) return STT_ERR_INVALID;
    if (cfg->mode == STT_SOLVE_PERSISTENT && cfg->bp_mode != 0) return STT_ERR_INVALID;  // voxel-based only
    if (cfg->storage != STT_DTYPE_F32 && cfg->storage != STT_DTYPE_BF16) return STT_ERR_INVALID;
    if (!state->vol || !state->xbar || !state->xprev || !state->ytv || !state->ytp || !state->ybc ||
        !state->flow || !state->proj)
        return STT_ERR_INVALID;
    if (cfg->halo && (!state->ytp_halo || !state->ybc_halo || !state->flow_halo)) return STT_ERR_INVALID;
    if (cfg->autotune && !ctx->tuned && (st = stt_autotune(ctx, nullptr, nullptr))) return st;
    if (cfg->n_frames > 1024) return STT_ERR_INVALID;
    const int total = cfg->total_frames > 0 ? cfg->total_frames : cfg->n_frames;
    if (cfg->frame_offset < 0 || (long long)cfg->frame_offset + cfg->n_frames > total) return STT_ERR_INVALID;
    stt_solver *s = new stt_solver();
    s->ctx = ctx;
    s->cfg = *cfg;
    s->st = *state;
    s->g = g;
    s->views = (const stt::ViewRec *)vp;
    s->F = cfg->n_frames;
    s->V = cfg->views_per_frame;
    s->total_frames = total;
    s->n = (size_t)g->nx * g->ny * g->nz;
    s->npix = (size_t)g->W * g->H;
    const int F = s->F;
    stt_status e = STT_OK;
    if (!e) e = alloc(s, s->warpbuf, (size_t)F * s->n, "warp buffers");
    if (!e) e = alloc(s, s->corr, (size_t)F * s->npix, "corrections");
    if (!e) e = alloc(s, s->ax, s->npix, "projection");
    if (!e) {
        unsigned char *vt = nullptr;
        e = alloc(s, vt, (size_t)F * s->n * (cfg->storage == STT_DTYPE_BF16 ? 2 : 4), "transposed volumes");
        s->volt = vt;
    }
    if (!e) e = alloc(s, s->raylen, (size_t)F * s->npix, "ray lengths");
    if (!e) e = alloc(s, s->perm, (size_t)F * s->V, "view order");
    if (!e) e = alloc(s, s->counter, 1, "iteration counter");
    if (!e) e = alloc(s, s->status, 1, "status word");
    if (!e && cfg->bp_mode == 1) e = alloc(s, s->acc, (size_t)F * s->n, "ray-BP accumulators");
    if (e) {
        stt_solver_destroy(s);
        return e;
    }
    // no views staged for this storage (the tuner found one gather launch per
    // view faster than the two kernels): no maps, one launch per view
    const bool any_staged = (cfg->storage == STT_DTYPE_F32 ? ctx->staged_bins : ctx->staged_bins16) != 0;
    // (the persistent sweep gathers with loads: no maps, textures or texture copy of the correction)
    const bool per_view_kernels = cfg->mode == STT_SOLVE_STREAMS || cfg->mode == STT_SOLVE_GRAPH;
    if (per_view_kernels && any_staged) {
        s->fpmaps.resize(F);
        for (int f = 0; f < F; ++f) {  // where the maps do not apply, ok stays 0 and every view gathers
            if (cfg->storage == STT_DTYPE_F32)
                stt::make_fp_slab_maps(*g, s->st.vol + f * s->n, static_cast<float *>(s->volt) + f * s->n,
                                       s->fpmaps[f], ctx->tuning.slab);
            else
                stt::make_fp_slab_maps(*g, reinterpret_cast<const unsigned short *>(s->st.vol) + f * s->n,
                                       static_cast<unsigned short *>(s->volt) + f * s->n, s->fpmaps[f],
                                       ctx->tuning.slab);
        }
    }
    if (per_view_kernels && cfg->storage == STT_DTYPE_F32 && stt::is_tex_fp_variant(ctx->tuning.fp)) {
        s->fptex.resize(F);  // where they cannot be made, ok stays 0 and the loads run
        for (int f = 0; f < F; ++f)
            stt::make_fp_tex(*g, s->st.vol + f * s->n, static_cast<float *>(s->volt) + f * s->n, s->fptex[f]);
    }
    if (per_view_kernels && cfg->storage == STT_DTYPE_BF16 && ctx->tuning.fp16 == 1) {
        s->fptex.resize(F);
        for (int f = 0; f < F; ++f)
            stt::make_fp_tex(*g, reinterpret_cast<const unsigned short *>(s->st.vol) + f * s->n,
                             static_cast<unsigned short *>(s->volt) + f * s->n, s->fptex[f]);
    }
    if (per_view_kernels && cfg->bp_mode == 0) {
        s->corr_tex.resize(F);
        for (int f = 0; f < F; ++f)
            if (stt::make_corr_tex(g->W, g->H, s->corr_tex[f]) != cudaSuccess) {
                cudaGetLastError();
                stt_solver_destroy(s);
                return STT_ERR_NOMEM;
            }
    }
    if (cfg->mode == STT_SOLVE_PERSISTENT) {
        s->sweep_wide = (long long)g->nx * g->ny * g->nz >= (1LL << 31);  // 64-bit gather offsets
        s->sweep_blocks = stt::sweep_max_blocks(cfg->storage == STT_DTYPE_BF16, s->sweep_wide);
        std::vector<stt::SweepJob> jobs(F);
        fill_jobs(s, jobs.data());
        if (s->sweep_blocks < 1) {
            stt_solver_destroy(s);
            return STT_ERR_CUDA;  // the occupancy query failed
        }
        stt::sweep_plan(jobs.data(), F, s->sweep_blocks);
        e = alloc(s, s->sweep_bar, 4 * (size_t)F + 2, "sweep barriers");  // 4 per frame, then the grid's
        unsigned char *jd = nullptr;
        if (!e) e = alloc(s, jd, F * sizeof(stt::SweepJob), "sweep jobs");
        s->jobs_d = reinterpret_cast<stt::SweepJob *>(jd);
        if (e) {
            stt_solver_destroy(s);
            return e;
        }
        for (int f = 0; f < F; ++f) jobs[f].bar = s->sweep_bar + 4 * f;
        if (cudaMemcpy(s->jobs_d, jobs.data(), F * sizeof(stt::SweepJob), cudaMemcpyHostToDevice) != cudaSuccess) {
            cudaGetLastError();
            stt_solver_destroy(s);
            return STT_ERR_CUDA;
        }
    }
    cudaError_t ce = cudaMemset(s->raylen, 0, (size_t)F * s->npix * sizeof(float));
    if (ce == cudaSuccess) ce = cudaMemset(s->counter, 0, sizeof(unsigned long long));
    if (ce == cudaSuccess) ce = cudaMemset(s->status, 0, sizeof(int));
    if (ce == cudaSuccess && s->acc) ce = cudaMemset(s->acc, 0, (size_t)F * s->n * sizeof(float2));
    s->streams.resize(F);
    s->ev_dual.resize(F);
    s->ev_done.resize(F);
    for (int f = 0; f < F && ce == cudaSuccess; ++f) {
        ce = cudaStreamCreateWithFlags(&s->streams[f], cudaStreamNonBlocking);
        if (ce == cudaSuccess) ce = cudaEventCreateWithFlags(&s->ev_dual[f], cudaEventDisableTiming);
        if (ce == cudaSuccess) ce = cudaEventCreateWithFlags(&s->ev_done[f], cudaEventDisableTiming);
    }
    if (ce == cudaSuccess) ce = cudaEventCreateWithFlags(&s->ev_fork, cudaEventDisableTiming);
    if (ce == cudaSuccess) ce = cudaDeviceSynchronize();
    if (ce != cudaSuccess) {
        stt_solver_destroy(s);
        return STT_ERR_CUDA;
    }
    *out = s;
    return STT_OK;
}

stt_status stt_solver_iterate(stt_solver *s, int n_iters, void *stream) {
    if (!s || n_iters < 0) return STT_ERR_INVALID;
    cudaStream_t cs = reinterpret_cast<cudaStream_t>(stream);
    for (int it = 0; it < n_iters; ++it) {
        long long nl = 0;
        stt_status st = STT_OK;
        if (s->cfg.halo) {  // a sharded solve runs its two phases (the caller exchanges halos in between)
            if ((st = stt_solver_iterate_phase(s, 0, stream))) return st;
            if ((st = stt_solver_iterate_phase(s, 1, stream))) return st;
            continue;
        }
        if (s->cfg.mode == STT_SOLVE_PLAIN) {
            st = run_plain(s, cs, nl, -1);
        } else if (s->cfg.mode == STT_SOLVE_STREAMS) {
            st = enqueue_batched(s, cs, nl);
            ++s->host_iter;
        } else if (s->cfg.mode == STT_SOLVE_PERSISTENT) {
            if (!s->exec && !s->sweep_direct) {
                stt_status cst = STT_OK;
                s->exec = try_capture(s, s->graph, nl, enqueue_persistent, cst);
                if (s->exec) s->launches_per_iter = nl;
                else s->sweep_direct = true, s->err.clear();
            }
            if (s->exec) {
                SCUDA(s, cudaGraphLaunch(s->exec, cs), "graph launch");
                nl = s->launches_per_iter;
            } else {
                nl = 0;
                st = enqueue_persistent(s, cs, nl);
            }
            ++s->host_iter;
        } else {
            if (!s->exec) {
                cudaStream_t cap;
                SCUDA(s, cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking), "capture stream");
                SCUDA(s, cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal), "begin capture");
                st = enqueue_batched(s, cap, nl);
                cudaGraph_t graph = nullptr;
                cudaError_t ce = cudaStreamEndCapture(cap, &graph);
                cudaStreamDestroy(cap);
                if (st) {
                    if (graph) cudaGraphDestroy(graph);
                    return st;
                }
                if (ce != cudaSuccess) return sfail(s, STT_ERR_CUDA, std::string("end capture: ") + cudaGetErrorString(ce));
                s->graph = graph;
                SCUDA(s, cudaGraphInstantiate(&s->exec, graph, 0), "graph instantiate");
                s->launches_per_iter = nl;
            }
            SCUDA(s, cudaGraphLaunch(s->exec, cs), "graph launch");
            nl = s->launches_per_iter;
            ++s->host_iter;
        }
        if (st) return st;
        s->launches_per_iter = nl;
    }
    return STT_OK;
}

stt_status stt_solver_iterate_phase(stt_solver *s, int phase, void *stream) {
    if (!s || (phase != 0 && phase != 1)) return STT_ERR_INVALID;
    cudaStream_t cs = reinterpret_cast<cudaStream_t>(stream);
    long long nl = 0;
    stt_status st = STT_OK;
    if (s->cfg.mode == STT_SOLVE_PLAIN) {
        st = run_plain(s, cs, nl, phase);
    } else if (s->cfg.mode == STT_SOLVE_STREAMS) {
        st = phase == 0 ? enqueue_phase0(s, cs, nl, true) : enqueue_phase1(s, cs, nl, true);
        if (phase == 1) ++s->host_iter;
    } else if (s->cfg.mode == STT_SOLVE_PERSISTENT) {
        // (enqueued directly: a handful of launches per phase)
        if (phase == 0) {
            st = enqueue_phase0(s, cs, nl, true);
        } else {
            st = enqueue_primals(s, cs, nl, true);
            if (!st) st = enqueue_sweep(s, cs, nl);
            ++s->host_iter;
        }
    } else {
        if (!s->pexec[phase]) {
            cudaStream_t cap;
            SCUDA(s, cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking), "capture stream");
            SCUDA(s, cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal), "begin capture");
            st = phase == 0 ? enqueue_phase0(s, cap, nl, true) : enqueue_phase1(s, cap, nl, true);
            cudaGraph_t graph = nullptr;
            cudaError_t ce = cudaStreamEndCapture(cap, &graph);
            cudaStreamDestroy(cap);
            if (st) {
                if (graph) cudaGraphDestroy(graph);
                return st;
            }
            if (ce != cudaSuccess) return sfail(s, STT_ERR_CUDA, std::string("end capture: ") + cudaGetErrorString(ce));
            s->pgraph[phase] = graph;
            SCUDA(s, cudaGraphInstantiate(&s->pexec[phase], graph, 0), "graph instantiate");
            s->phase_launches[phase] = nl;
        }
        SCUDA(s, cudaGraphLaunch(s->pexec[phase], cs), "graph launch");
        nl = s->phase_launches[phase];
        if (phase == 1) ++s->host_iter;
    }
    if (st) return st;
    s->phase_launches[phase] = nl;
    s->launches_per_iter = s->phase_launches[0] + s->phase_launches[1];
    return STT_OK;
}

stt_status stt_solver_set_iteration(stt_solver *s, unsigned long long iter, void *stream) {
    if (!s) return STT_ERR_INVALID;
    s->host_iter = iter;
    SCUDA(s, stt::launch_set_counter(s->counter, iter, reinterpret_cast<cudaStream_t>(stream)), "counter update");
    return STT_OK;
}

stt_status stt_solver_stats(const stt_solver *s, long long *launches_per_iter, unsigned long long *iterations) {
    if (!s) return STT_ERR_INVALID;
    if (launches_per_iter) *launches_per_iter = s->launches_per_iter;
    if (iterations) *iterations = s->host_iter;
    return STT_OK;
}

stt_status stt_solver_persistent_info(const stt_solver *s, int *blocks, int *graph) {
    if (!s) return STT_ERR_INVALID;
    const bool p = s->cfg.mode == STT_SOLVE_PERSISTENT;
    if (blocks) *blocks = p ? s->sweep_blocks : 0;
    if (graph) *graph = p && s->exec ? 1 : 0;
    return STT_OK;
}

stt_status stt_solver_poll_status(stt_solver *s, void *stream) {
    if (!s) return STT_ERR_INVALID;
    cudaStream_t cs = reinterpret_cast<cudaStream_t>(stream);
    int flag = 0;
    SCUDA(s, cudaMemcpyAsync(&flag, s->status, sizeof(int), cudaMemcpyDeviceToHost, cs), "read status word");
    SCUDA(s, cudaStreamSynchronize(cs), "cudaStreamSynchronize");
    if (!flag) return STT_OK;
    SCUDA(s, cudaMemsetAsync(s->status, 0, sizeof(int), cs), "clear status word");
    SCUDA(s, cudaStreamSynchronize(cs), "cudaStreamSynchronize");
    return sfail(s, STT_ERR_TIMEOUT,
                 "a bounded device-side wait gave up: a TMA copy into shared memory did not land within about 0.1 s "
                 "(the results were computed from global memory instead), or a barrier of the persistent sweep "
                 "waited about 5 s (it was abandoned: the iteration's results are not valid)");
}

const char *stt_solver_last_error(const stt_solver *s) { return s ? s->err.c_str() : ""; }

stt_status stt_solver_destroy(stt_solver *s) {
    if (!s) return STT_OK;
    if (s->exec) cudaGraphExecDestroy(s->exec);
    if (s->graph) cudaGraphDestroy(s->graph);
    for (int p = 0; p < 2; ++p) {
        if (s->pexec[p]) cudaGraphExecDestroy(s->pexec[p]);
        if (s->pgraph[p]) cudaGraphDestroy(s->pgraph[p]);
    }
    for (auto st : s->streams)
        if (st) cudaStreamDestroy(st);
    for (auto e : s->ev_dual)
        if (e) cudaEventDestroy(e);
    for (auto e : s->ev_done)
        if (e) cudaEventDestroy(e);
    if (s->ev_fork) cudaEventDestroy(s->ev_fork);
    for (auto &t : s->corr_tex) stt::free_corr_tex(t);
    for (auto &t : s->fptex) stt::destroy_fp_tex(t);
    cudaFree(s->jobs_d);
    cudaFree(s->sweep_bar);
    cudaFree(s->warpbuf);
    cudaFree(s->corr);
    cudaFree(s->ax);
    cudaFree(s->volt);
    cudaFree(s->raylen);
    cudaFree(s->acc);
    cudaFree(s->perm);
    cudaFree(s->counter);
    cudaFree(s->status);
    delete s;
    return STT_OK;
}

// Hooks of the batch's persistent form (stt_batch.cu), for a solver created
// with STT_SOLVE_PERSISTENT: one iteration's steps before the sweep, joined
// into `stream`; the solver's frames as sweep jobs (block ranges and barrier
// words are the caller's); the end of an iteration whose sweep the caller
// launched; the status word its sweep should raise.
stt_status stt_internal_solver_presweep(stt_solver *s, void *stream) {
    if (!s || s->cfg.mode != STT_SOLVE_PERSISTENT) return STT_ERR_INVALID;
    long long nl = 0;
    cudaStream_t cs = reinterpret_cast<cudaStream_t>(stream);
    stt_status st = enqueue_phase0(s, cs, nl, false);
    if (!st) st = enqueue_primals(s, cs, nl, false);
    return st;
}

int stt_internal_solver_jobs(const stt_solver *s, void *jobs) {
    if (!s || !jobs) return 0;
    fill_jobs(s, static_cast<stt::SweepJob *>(jobs));
    return s->F;
}

void stt_internal_solver_end_iteration(stt_solver *s) {
    if (s) ++s->host_iter;
}

int *stt_internal_solver_status(stt_solver *s) { return s ? s->status : nullptr; }

stt_status stt_solver_frame_order(unsigned long long seed, unsigned long long iter, int n_frames, int frame,
                                  int views, int *perm_out) {
    if (n_frames < 1 || frame < 0 || frame >= n_frames || views < 1 || !perm_out) return STT_ERR_INVALID;
    stt::host_perm(seed, iter, n_frames, frame, views, perm_out);
    return STT_OK;
}

}  // extern "C"
