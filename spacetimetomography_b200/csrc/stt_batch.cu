// stt_batch.cu -- many independent single-frame reconstructions of uneven
// size solved together: each instance is a one-frame primal-dual TV + SART
// solve (ST_Tomography::Render's iteration with one frame, whose temporal and
// brightness-constancy weights are zero) on its own context and stream, and
// one iteration of all of them is enqueued together -- or captured once into
// one CUDA graph and replayed.  The instances share nothing, so their views
// run concurrently and small instances fill the GPU that one alone leaves idle.
// In the persistent form (STT_SOLVE_PERSISTENT) ONE cooperative launch runs
// the whole iteration of every instance side by side -- view order, warps,
// dual and primal steps, SART call, ROI mask and over-relaxation -- the
// resident blocks split between the instances in proportion to their work
// (k_iter_persistent, k_persist.cu); the iteration is captured into a graph
// and replayed.  (More instances than resident blocks: the duals and primals
// run as launches on the instances' streams and the SART calls in rounds.)
#include <string>
#include <vector>

#include "stt.h"
#include "stt_internal.cuh"
#include "stt_kernels.h"

struct stt_batch {
    struct Inst {
        stt_ctx *ctx = nullptr;
        stt_solver *solver = nullptr;
        float *user_vol = nullptr;  // (BF16 values when the instance's storage is BF16)
        unsigned char *state = nullptr;  // vol 2n | xbar 2n | xprev n (storage), then FP32 ytv 3n | ytp n | ybc n | flow 3n
        size_t n = 0;
        size_t es = 4;       // bytes per stored primal value
        size_t primal = 0;   // bytes of the primal block (the FP32 duals follow it)
        stt_instance cfg{};  // the caller's description (its vol and proj stay the caller's)
        cudaStream_t stream = nullptr;
        cudaEvent_t done = nullptr;
    };
    std::vector<Inst> inst;
    int mode = STT_SOLVE_GRAPH;
    cudaEvent_t fork = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    bool skip_copy = false;  // timing runs do not copy results into the callers' volumes
    // STT_SOLVE_PERSISTENT: one sweep job per instance, their barrier words,
    // the launch's blocks, storage and index width, the sweep's status word
    stt::SweepJob *jobs_d = nullptr;
    unsigned *bar = nullptr;
    int *status = nullptr;
    int sweep_blocks = 0, rounds = 0;
    bool bf16 = false, wide = false, direct = false;
    int staging_timed = 0, all_gather = 0;
    float ms_split = 0.0f, ms_gather = 0.0f;
    std::string err;
};

extern "C" stt_status stt_internal_set_error(stt_ctx *ctx, stt_status st, const char *msg);
extern "C" stt_status stt_internal_solver_presweep(stt_solver *s, void *stream);
extern "C" int stt_internal_solver_jobs(const stt_solver *s, void *jobs);
extern "C" void stt_internal_solver_end_iteration(stt_solver *s);

namespace {

stt_status bfail(stt_batch *b, stt_status st, const std::string &m) {
    b->err = m;
    return st;
}

#define BCUDA(b, call, where)                                                                               \
    do {                                                                                                    \
        cudaError_t e_ = (call);                                                                            \
        if (e_ != cudaSuccess) return bfail(b, STT_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(e_)); \
    } while (0)

// One iteration of every instance, enqueued on the instances' streams,
// forked from and joined back to `main`.
stt_status enqueue_all(stt_batch *b, cudaStream_t main) {
    BCUDA(b, cudaEventRecord(b->fork, main), "event record");
    for (size_t i = 0; i < b->inst.size(); ++i) {
        stt_batch::Inst &in = b->inst[i];
        BCUDA(b, cudaStreamWaitEvent(in.stream, b->fork, 0), "stream wait");
        stt_status st = stt_solver_iterate(in.solver, 1, in.stream);
        if (st) return bfail(b, st, "instance " + std::to_string(i) + ": " + stt_solver_last_error(in.solver));
        if (!b->skip_copy)
            BCUDA(b, cudaMemcpyAsync(in.user_vol, in.state, in.n * in.es, cudaMemcpyDeviceToDevice, in.stream),
                  "copy result");
        BCUDA(b, cudaEventRecord(in.done, in.stream), "event record");
        BCUDA(b, cudaStreamWaitEvent(main, in.done, 0), "stream wait");
    }
    return STT_OK;
}

// The persistent form: every instance's steps before its SART call on its own
// stream, then one launch for all SART calls, then the results.
stt_status enqueue_all_persistent(stt_batch *b, cudaStream_t main) {
    const int ni = (int)b->inst.size();
    if (ni <= b->sweep_blocks) {  // the whole iteration of every instance: one launch
        BCUDA(b, cudaMemsetAsync(b->bar, 0, (4 * (size_t)ni + 2) * sizeof(unsigned), main), "barrier reset");
        BCUDA(b, stt::launch_iter_persistent(b->jobs_d, ni, b->sweep_blocks, b->bf16, b->wide, b->bar + 4 * ni,
                                             b->status, main),
              "persistent iteration");
        for (stt_batch::Inst &in : b->inst) {
            stt_internal_solver_end_iteration(in.solver);
            if (!b->skip_copy)
                BCUDA(b, cudaMemcpyAsync(in.user_vol, in.state, in.n * in.es, cudaMemcpyDeviceToDevice, main),
                      "copy result");
        }
        return STT_OK;
    }
    BCUDA(b, cudaEventRecord(b->fork, main), "event record");
    for (size_t i = 0; i < b->inst.size(); ++i) {
        stt_batch::Inst &in = b->inst[i];
        BCUDA(b, cudaStreamWaitEvent(in.stream, b->fork, 0), "stream wait");
        stt_status st = stt_internal_solver_presweep(in.solver, in.stream);
        if (st) return bfail(b, st, "instance " + std::to_string(i) + ": " + stt_solver_last_error(in.solver));
        BCUDA(b, cudaEventRecord(in.done, in.stream), "event record");
        BCUDA(b, cudaStreamWaitEvent(main, in.done, 0), "stream wait");
    }
    const int n = (int)b->inst.size();
    BCUDA(b, cudaMemsetAsync(b->bar, 0, 4 * (size_t)n * sizeof(unsigned), main), "barrier reset");
    BCUDA(b, stt::launch_sweep_persistent(b->jobs_d, n, b->sweep_blocks, b->bf16, b->wide, b->status, main),
          "persistent sweep");
    for (stt_batch::Inst &in : b->inst) {
        stt_internal_solver_end_iteration(in.solver);
        if (!b->skip_copy)
            BCUDA(b, cudaMemcpyAsync(in.user_vol, in.state, in.n * in.es, cudaMemcpyDeviceToDevice, main),
                  "copy result");
    }
    return STT_OK;
}

// The instances' sweep jobs, the launch's blocks split between them.
stt_status build_sweep(stt_batch *b) {
    const int n = (int)b->inst.size();
    std::vector<stt::SweepJob> jobs(n);
    b->bf16 = b->inst[0].cfg.storage == STT_DTYPE_BF16;
    b->wide = false;
    for (int i = 0; i < n; ++i) {
        if (stt_internal_solver_jobs(b->inst[i].solver, &jobs[i]) != 1)
            return bfail(b, STT_ERR_INVALID, "instance " + std::to_string(i) + ": sweep job");
        const stt::GeomDev &g = jobs[i].g;
        b->wide |= (long long)g.nx * g.ny * g.nz >= (1LL << 31);
    }
    b->sweep_blocks = stt::sweep_max_blocks(b->bf16, b->wide);
    if (b->sweep_blocks < 1) return bfail(b, STT_ERR_CUDA, "occupancy of the persistent sweep");
    b->rounds = stt::sweep_plan(jobs.data(), n, b->sweep_blocks);
    if (cudaMalloc(&b->bar, (4 * (size_t)n + 2) * sizeof(unsigned)) != cudaSuccess ||  // 4 per instance, the grid's
        cudaMalloc(&b->jobs_d, n * sizeof(stt::SweepJob)) != cudaSuccess ||
        cudaMalloc(&b->status, sizeof(int)) != cudaSuccess) {
        cudaGetLastError();
        return bfail(b, STT_ERR_NOMEM, "persistent sweep buffers");
    }
    for (int i = 0; i < n; ++i) jobs[i].bar = b->bar + 4 * i;
    if (cudaMemcpy(b->jobs_d, jobs.data(), n * sizeof(stt::SweepJob), cudaMemcpyHostToDevice) != cudaSuccess ||
        cudaMemset(b->status, 0, sizeof(int)) != cudaSuccess) {
        cudaGetLastError();
        return bfail(b, STT_ERR_CUDA, "persistent sweep set-up");
    }
    return STT_OK;
}

// The instance's solver state from its start volume: vol (and the duplicated
// last frame) and X_bar = the caller's volume; X_prev, the duals and the flow
// zero.
cudaError_t init_state(stt_batch::Inst &in) {
    const size_t n1 = in.n, es = in.es;
    unsigned char *vol = in.state, *xbar = vol + 2 * n1 * es, *xprev = xbar + 2 * n1 * es;
    float *ytv = reinterpret_cast<float *>(in.state + in.primal);
    cudaError_t e = cudaMemset(xprev, 0, n1 * es);
    if (e == cudaSuccess) e = cudaMemset(ytv, 0, 8 * n1 * sizeof(float));  // ytv, ytp, ybc, flow
    if (e == cudaSuccess) e = cudaMemcpy(vol, in.user_vol, n1 * es, cudaMemcpyDeviceToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(vol + n1 * es, in.user_vol, n1 * es, cudaMemcpyDeviceToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(xbar, vol, 2 * n1 * es, cudaMemcpyDeviceToDevice);
    return e;
}

// (Re)creates the instance's one-frame solver with its context's current
// launch choices.
stt_status make_solver(stt_batch::Inst &in, bool persistent = false) {
    if (in.solver) {
        stt_solver_destroy(in.solver);
        in.solver = nullptr;
    }
    const stt_instance &I = in.cfg;
    const size_t n1 = in.n, es = in.es;
    unsigned char *vol = in.state, *xbar = vol + 2 * n1 * es, *xprev = xbar + 2 * n1 * es;
    float *ytv = reinterpret_cast<float *>(in.state + in.primal), *ytp = ytv + 3 * n1, *ybc = ytp + n1,
          *flow = ybc + n1;
    stt_solve_cfg cfg{};
    cfg.n_frames = 1;
    cfg.views_per_frame = I.n_views;
    cfg.bp_mode = I.bp_mode;
    cfg.alpha = I.alpha;
    cfg.pd = I.pd;
    cfg.pd.tp_w = 0.0f;  // one frame: no temporal or brightness-constancy term
    cfg.pd.bc_w = 0.0f;
    for (int q = 0; q < 8; ++q) cfg.roi_cut[q] = I.roi_cut[q];
    cfg.seed = I.seed;
    cfg.autotune = I.autotune;
    cfg.storage = I.storage;
    cfg.mode = persistent ? STT_SOLVE_PERSISTENT : STT_SOLVE_STREAMS;
    stt_pd_state state{};  // (BF16 storage: the primal pointers address BF16 arrays)
    state.vol = reinterpret_cast<float *>(vol);
    state.xbar = reinterpret_cast<float *>(xbar);
    state.xprev = reinterpret_cast<float *>(xprev);
    state.ytv = ytv;
    state.ytp = ytp;
    state.ybc = ybc;
    state.flow = flow;
    state.proj = I.proj;
    return stt_solver_create(I.ctx, &cfg, &state, &in.solver);
}

void drop_graph(stt_batch *b) {
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    b->exec = nullptr;
    b->graph = nullptr;
}

}  // namespace

extern "C" stt_status stt_batch_iterate(stt_batch *b, int n_iters, void *stream);

namespace {

// Milliseconds of one batched iteration (after one warm-up iteration, which
// also captures the graph), results not copied out; the caller re-initialises
// the states afterwards.
stt_status time_iteration(stt_batch *b, float &ms) {
    drop_graph(b);
    b->skip_copy = true;
    cudaStream_t s = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaError_t e = cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreate(&e0);
    if (e == cudaSuccess) e = cudaEventCreate(&e1);
    stt_status st = e == cudaSuccess ? STT_OK : bfail(b, STT_ERR_CUDA, "timing set-up");
    if (!st) st = stt_batch_iterate(b, 1, s);
    if (!st && (e = cudaEventRecord(e0, s)) != cudaSuccess) st = bfail(b, STT_ERR_CUDA, "event record");
    if (!st) st = stt_batch_iterate(b, 1, s);
    if (!st && ((e = cudaEventRecord(e1, s)) != cudaSuccess || (e = cudaEventSynchronize(e1)) != cudaSuccess))
        st = bfail(b, STT_ERR_CUDA, std::string("timing: ") + cudaGetErrorString(e));
    if (!st && (e = cudaEventElapsedTime(&ms, e0, e1)) != cudaSuccess) st = bfail(b, STT_ERR_CUDA, "elapsed time");
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (s) {
        cudaStreamSynchronize(s);
        cudaStreamDestroy(s);
    }
    if (st) cudaGetLastError();
    b->skip_copy = false;
    drop_graph(b);
    return st;
}

// Which views the slab-staged projector takes is tuned per instance on an
// otherwise idle GPU.  In a batch, the instances' views run side by side, and
// there every view gathering (one launch per view, no 37 KB of shared memory
// per block) can be faster: measured on the 64 uneven instances of the batch
// workload, 409 against 466 ms per iteration (BF16 storage 400 against 444).
// So a batch whose instances ask for tuning times one batched iteration both
// ways and keeps the faster; the states are re-initialised and the solvers
// re-created afterwards, so the solve starts as if untimed.
stt_status choose_staging(stt_batch *b) {
    const size_t n = b->inst.size();
    std::vector<stt_tuning> saved(n);
    bool any = false;
    for (size_t i = 0; i < n; ++i) {
        stt_status st = stt_get_tuning(b->inst[i].ctx, &saved[i]);
        if (st) return bfail(b, st, "instance " + std::to_string(i) + ": stt_get_tuning");
        any |= (b->inst[i].cfg.storage == STT_DTYPE_BF16 ? saved[i].staged_bins_bf16 : saved[i].staged_bins) != 0;
    }
    if (!any) return STT_OK;  // every view gathers already
    stt_status st = time_iteration(b, b->ms_split);
    for (size_t i = 0; i < n && !st; ++i) {  // the mask of the instance's own storage
        stt_tuning t = saved[i];
        if (b->inst[i].cfg.storage == STT_DTYPE_BF16) t.staged_bins_bf16 = 0;
        else t.staged_bins = 0;
        st = stt_set_tuning(b->inst[i].ctx, &t);
    }
    for (size_t i = 0; i < n && !st; ++i)
        if ((st = make_solver(b->inst[i]))) bfail(b, st, "instance " + std::to_string(i) + ": solver");
    for (size_t i = 0; i < n && !st; ++i)
        if (init_state(b->inst[i]) != cudaSuccess) st = bfail(b, STT_ERR_CUDA, "state reset");
    if (!st) st = time_iteration(b, b->ms_gather);
    if (st) return st;
    b->staging_timed = 1;
    b->all_gather = b->ms_gather < b->ms_split;
    if (!b->all_gather)
        for (size_t i = 0; i < n && !st; ++i) st = stt_set_tuning(b->inst[i].ctx, &saved[i]);
    // fresh solvers (iteration counters at 0, no sticky ray lengths) and states
    for (size_t i = 0; i < n && !st; ++i)
        if ((st = make_solver(b->inst[i]))) bfail(b, st, "instance " + std::to_string(i) + ": solver");
    for (size_t i = 0; i < n && !st; ++i)
        if (init_state(b->inst[i]) != cudaSuccess) st = bfail(b, STT_ERR_CUDA, "state reset");
    return st;
}

}  // namespace

extern "C" {

stt_status stt_batch_create(const stt_instance *instances, int n, int mode, stt_batch **out) {
    if (!instances || n < 1 || !out) return stt_internal_set_error(nullptr, STT_ERR_INVALID, "null argument or n < 1");
    if (mode != STT_SOLVE_STREAMS && mode != STT_SOLVE_GRAPH && mode != STT_SOLVE_PERSISTENT)
        return stt_internal_set_error(nullptr, STT_ERR_INVALID,
                                      "mode must be STT_SOLVE_STREAMS, STT_SOLVE_GRAPH or STT_SOLVE_PERSISTENT");
    const bool persistent = mode == STT_SOLVE_PERSISTENT;
    for (int i = 0; persistent && i < n; ++i)
        if (instances[i].bp_mode != 0 || instances[i].storage != instances[0].storage)
            return stt_internal_set_error(nullptr, STT_ERR_INVALID,
                                          "STT_SOLVE_PERSISTENT: every instance voxel-based (bp_mode 0), one storage");
    *out = nullptr;
    stt_batch *b = new stt_batch;
    b->mode = mode;
    b->inst.resize(n);
    auto bail = [&](stt_status st, const std::string &m) {
        stt_internal_set_error(nullptr, st, m.c_str());
        stt_batch_destroy(b);
        return st;
    };
    for (int i = 0; i < n; ++i) {
        const stt_instance &I = instances[i];
        stt_batch::Inst &in = b->inst[i];
        if (!I.ctx || !I.vol || !I.proj || I.n_views < 1)
            return bail(STT_ERR_INVALID, "instance " + std::to_string(i) + ": null ctx/vol/proj or no views");
        int dims[3];
        if (stt_ctx_dims(I.ctx, dims) != STT_OK)
            return bail(STT_ERR_STATE, "instance " + std::to_string(i) + ": no geometry set on its context");
        in.ctx = I.ctx;
        in.user_vol = I.vol;
        in.cfg = I;
        if (I.storage != STT_DTYPE_F32 && I.storage != STT_DTYPE_BF16)
            return bail(STT_ERR_INVALID, "instance " + std::to_string(i) + ": storage must be F32 or BF16");
        in.n = (size_t)dims[0] * dims[1] * dims[2];
        in.es = I.storage == STT_DTYPE_BF16 ? 2 : 4;
        in.primal = ((5 * in.n * in.es + 255) / 256) * 256;  // the FP32 duals start 256-byte aligned
        if (cudaMalloc(&in.state, in.primal + 8 * in.n * sizeof(float)) != cudaSuccess) {
            cudaGetLastError();
            return bail(STT_ERR_NOMEM, "instance " + std::to_string(i) + ": cudaMalloc of its solver state failed");
        }
        cudaError_t e = init_state(in);
        if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&in.stream, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&in.done, cudaEventDisableTiming);
        if (e != cudaSuccess) return bail(STT_ERR_CUDA, std::string("instance set-up: ") + cudaGetErrorString(e));
        stt_status st = make_solver(in, persistent);
        if (st) return bail(st, "instance " + std::to_string(i) + ": " + stt_last_error(I.ctx));
    }
    if (cudaEventCreateWithFlags(&b->fork, cudaEventDisableTiming) != cudaSuccess)
        return bail(STT_ERR_CUDA, "event create");
    bool tune = false;
    for (int i = 0; i < n; ++i) tune |= instances[i].autotune != 0;
    if (tune && !persistent) {  // (the persistent sweep has one projector: nothing to choose)
        const stt_status st = choose_staging(b);
        if (st) return bail(st, "batch staging choice: " + b->err);
    }
    if (persistent) {
        const stt_status st = build_sweep(b);
        if (st) return bail(st, b->err);
    }
    *out = b;
    return STT_OK;
}

stt_status stt_batch_iterate(stt_batch *b, int n_iters, void *stream) {
    if (!b || n_iters < 0) return STT_ERR_INVALID;
    cudaStream_t cs = reinterpret_cast<cudaStream_t>(stream);
    for (int it = 0; it < n_iters; ++it) {
        if (b->mode == STT_SOLVE_STREAMS) {
            stt_status st = enqueue_all(b, cs);
            if (st) return st;
            continue;
        }
        if (b->mode == STT_SOLVE_PERSISTENT && !b->exec && !b->direct) {
            // capture once; where the runtime refuses to capture the
            // cooperative launch, enqueue every iteration directly
            cudaStream_t cap;
            BCUDA(b, cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking), "capture stream");
            stt_status st = STT_OK;
            cudaGraph_t graph = nullptr;
            if (cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal) == cudaSuccess) {
                st = enqueue_all_persistent(b, cap);
                if (cudaStreamEndCapture(cap, &graph) != cudaSuccess) graph = nullptr;
            }
            cudaGetLastError();
            cudaStreamDestroy(cap);
            if (!st && graph && cudaGraphInstantiate(&b->exec, graph, 0) == cudaSuccess) {
                b->graph = graph;
            } else {
                if (graph) cudaGraphDestroy(graph);
                cudaGetLastError();
                b->exec = nullptr;
                b->direct = true;
            }
        }
        if (b->mode == STT_SOLVE_PERSISTENT && b->direct) {
            stt_status st = enqueue_all_persistent(b, cs);
            if (st) return st;
            continue;
        }
        if (!b->exec) {
            cudaStream_t cap;
            BCUDA(b, cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking), "capture stream");
            BCUDA(b, cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal), "begin capture");
            stt_status st = enqueue_all(b, cap);
            cudaGraph_t graph = nullptr;
            cudaError_t ce = cudaStreamEndCapture(cap, &graph);
            cudaStreamDestroy(cap);
            if (st) {
                if (graph) cudaGraphDestroy(graph);
                return st;
            }
            if (ce != cudaSuccess) return bfail(b, STT_ERR_CUDA, std::string("end capture: ") + cudaGetErrorString(ce));
            b->graph = graph;
            BCUDA(b, cudaGraphInstantiate(&b->exec, graph, 0), "graph instantiate");
        }
        BCUDA(b, cudaGraphLaunch(b->exec, cs), "graph launch");
    }
    return STT_OK;
}

stt_status stt_batch_poll_status(stt_batch *b, void *stream) {
    if (!b) return STT_ERR_INVALID;
    stt_status worst = STT_OK;
    if (b->status) {  // the persistent sweep's word
        cudaStream_t cs = reinterpret_cast<cudaStream_t>(stream);
        int flag = 0;
        BCUDA(b, cudaMemcpyAsync(&flag, b->status, sizeof(int), cudaMemcpyDeviceToHost, cs), "read status word");
        BCUDA(b, cudaStreamSynchronize(cs), "cudaStreamSynchronize");
        if (flag) {
            BCUDA(b, cudaMemsetAsync(b->status, 0, sizeof(int), cs), "clear status word");
            BCUDA(b, cudaStreamSynchronize(cs), "cudaStreamSynchronize");
            worst = bfail(b, STT_ERR_TIMEOUT,
                          "a barrier of the persistent iteration waited about 5 s: it was abandoned and the "
                          "iteration's results are not valid");
        }
    }
    for (size_t i = 0; i < b->inst.size(); ++i) {
        const stt_status st = stt_solver_poll_status(b->inst[i].solver, stream);
        if (st != STT_OK && worst == STT_OK) {
            worst = st;
            bfail(b, st, "instance " + std::to_string(i) + ": " + stt_solver_last_error(b->inst[i].solver));
        }
    }
    return worst;
}

stt_status stt_batch_staging(const stt_batch *b, int *timed, int *all_gather, float *ms_split, float *ms_gather) {
    if (!b) return STT_ERR_INVALID;
    if (timed) *timed = b->staging_timed;
    if (all_gather) *all_gather = b->all_gather;
    if (ms_split) *ms_split = b->ms_split;
    if (ms_gather) *ms_gather = b->ms_gather;
    return STT_OK;
}

const char *stt_batch_last_error(const stt_batch *b) { return b ? b->err.c_str() : "null batch"; }

stt_status stt_batch_destroy(stt_batch *b) {
    if (!b) return STT_OK;
    drop_graph(b);
    for (stt_batch::Inst &in : b->inst) {
        if (in.solver) stt_solver_destroy(in.solver);
        if (in.done) cudaEventDestroy(in.done);
        if (in.stream) cudaStreamDestroy(in.stream);
        cudaFree(in.state);
    }
    if (b->fork) cudaEventDestroy(b->fork);
    cudaFree(b->jobs_d);
    cudaFree(b->bar);
    cudaFree(b->status);
    delete b;
    return STT_OK;
}

}  // extern "C"
