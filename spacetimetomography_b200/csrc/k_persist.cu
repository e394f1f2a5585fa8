// k_persist.cu -- the persistent forms of the primal-dual iteration.
// k_iter_persistent: the whole iteration (S/ST_Tomo/ST_Tomography.cpp:492-607)
// of every frame -- or of every batch instance -- in ONE cooperative launch:
// view order, warps, dual and primal steps (see the kernel), then the SART
// call.  k_sweep_persistent: only the SART calls (every view of every
// frame's SART call, :616-808) and the ROI mask with the over-relaxation
// that follows them (:586-604, :793-804), for a sharded solve whose halos are
// exchanged between the phases.  Both run the SART calls as below.
//
// The jobs (SweepJob: one frame or one instance each) share the launch's
// blocks in proportion to their work and run side by side; only when there
// are more jobs than resident blocks do they run in rounds (a block moves on
// to its job of the next round as soon as its own is done: jobs are
// independent, so there is no barrier between rounds).  Measured on the 10
// frames of 256^3 with 36 views each: side by side 160 ms per iteration, one
// frame after another on every block 179 ms -- a block then has two detector
// tiles per view, the slowest block sets each phase's time, and every barrier
// spans all 1036 blocks.  A job's blocks walk its views in the frame's order;
// per view, three phases separated by the job's own barrier:
//   transpose  (views that gather along x) the z-fastest copy of the volume,
//              32 x 32 tiles through shared memory;
//   project    the forward projection with the SART correction, one thread
//              per detector pixel, 32 x 4 pixel tiles (k_fp_corr's arithmetic:
//              the same samples, Kahan order and epilogue);
//   backproject the voxel-based backprojection, one thread per (x, z) column
//              walking 16 voxels up y (bp_column, the column walk of the
//              per-view kernel);
// and after the last view the ROI mask and the over-relaxation.  Each phase's
// tiles go round-robin over the job's blocks, so the block that owns a
// pixel's sticky ray length or a voxel column is the same for every view.
//
// What one launch changes: no launch gaps between the ~3 V dependent steps of
// a sweep, and all frames' (instances') sweeps side by side.  What it costs:
// data that the launch itself writes (the volume, its copy, the correction)
// cannot be read through the texture or read-only paths, whose caches are not
// kept coherent within a launch, so the gathers are plain L1-cached loads
// (after each barrier's acquire) instead of the per-view kernels' tld4
// gathers, and every phase runs at the launch's one occupancy.
//
// The barrier: a block's thread 0 makes the block's writes visible
// (__threadfence), adds one arrival to the job's counter, and polls it with
// acquire loads until all of the job's blocks have arrived.  The launch is
// cooperative, so every block is resident and every wait ends (a block that
// reaches a job early waits for the job's other blocks to finish their
// previous round's jobs); the poll is still bounded (about 5 s by the global
// timer): a wait that runs out raises the job's abort word and the status
// word (STT_WAIT_TIMEOUT_FLAG), and every block of the job leaves at its next
// barrier.
#include "stt_internal.cuh"
#include "stt_kernels.h"
#include "stt_voxel.cuh"
#include "warp_dev.cuh"

#include <algorithm>

namespace stt {

namespace {

constexpr int SWEEP_THREADS = 128;
constexpr int SWEEP_COL = 16;                              // voxels per column of the backprojection
constexpr unsigned long long SWEEP_WAIT_NS = 5000000000ull;  // bound of one barrier wait

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ unsigned ld_acquire(const unsigned *p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p) : "memory");
    return v;
}

// The job's barrier: true when all `target` arrivals are in (the job's blocks
// have passed it as many times), false when the job aborted.
__device__ __forceinline__ bool sweep_barrier(unsigned *bar, unsigned target, int *status) {
    __shared__ int ok;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        atomicAdd(bar, 1u);
        const unsigned long long t0 = global_ns();
        int good = 1;
        while (ld_acquire(bar) < target) {
            if (ld_acquire(bar + 1)) {
                good = 0;
                break;
            }
            if (global_ns() - t0 > SWEEP_WAIT_NS) {
                atomicExch(bar + 1, 1u);
                atomicOr(status, STT_WAIT_TIMEOUT_FLAG);
                good = 0;
                break;
            }
            __nanosleep(64);
        }
        __threadfence();
        ok = good;
    }
    __syncthreads();
    return ok != 0;
}

// Tiles [0, ntiles) of one phase handed out by the job's ticket counter:
// thread 0 takes the next ticket while the block works on the current tile
// (the atomic's latency hides behind the tile), so blocks that drew cheap
// tiles take more and no block waits at the phase's barrier for a slow
// static share.  `base` is the counter's value at the phase's start: every
// block's last draw overshoots by one, so a phase uses ntiles + nblocks
// tickets and the next phase starts there.  Which block computes a tile does
// not change its values.
template <typename Work>
__device__ __forceinline__ void dynamic_tiles(unsigned *ticket, unsigned base, int ntiles, Work &&work) {
    __shared__ int next;
    if (threadIdx.x == 0) next = (int)(atomicAdd(ticket, 1u) - base);
    __syncthreads();
    int t = next;
    while (t < ntiles) {
        __syncthreads();  // every thread has read `next`
        unsigned drawn = 0;
        if (threadIdx.x == 0) drawn = atomicAdd(ticket, 1u);
        work(t);
        if (threadIdx.x == 0) next = (int)(drawn - base);
        __syncthreads();
        t = next;
    }
}

// The forward projection with the correction of pixel (i, j)
// (k_fp_corr's body, corners by plain loads).
template <typename I, typename T>
__device__ __forceinline__ void sweep_fp_pixel(const GeomDev &g, const ViewRec &vr, const T *vol, const T *volt,
                                               const T *b, float *raylen, float *corr, int i, int j) {
    Ray r;
    make_ray(g, vr, i, j, r);
    const size_t pix = i + (size_t)j * g.W;
    float L, sum = 0.0f;
    if (r.tnear < r.tfar) {
        if (volt && vr.layout == 1) {
            const Strides st = zyx_strides(g);
            sum = fp_ray_sum_with<FP_GROUP, false>(
                g, [=](int, const FpCell &c, float v[8]) { fp_corners<2, I, T, true>(volt, st, c, v); }, r, nullptr);
        } else {
            const Strides st = xyz_strides(g);
            sum = fp_ray_sum_with<FP_GROUP, false>(
                g, [=](int, const FpCell &c, float v[8]) { fp_corners<0, I, T, true>(vol, st, c, v); }, r, nullptr);
        }
        L = r.tfar - r.tnear;
        raylen[pix] = L;
    } else {
        L = raylen[pix];
    }
    corr[pix] = __fdiv_rn(__fsub_rn(ld_voxel(b + pix), sum), __fadd_rn(L, 1.0f));
}

// One job on this block (rank `rank` of the job's nblocks): false when the
// job aborted.
// passed: the job barriers this block has passed before the call.
template <typename T, typename I>
__device__ __forceinline__ bool run_job(const SweepJob &J, int rank, T (*tile)[33], int *status,
                                       unsigned passed = 0) {
    const GeomDev g = J.g;
    const int nb = J.nblocks;
    T *vol = static_cast<T *>(J.vol);
    T *volt = static_cast<T *>(J.volt);
    const T *stack = static_cast<const T *>(J.stack);
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const size_t nxy = (size_t)g.nx * g.ny, nzy = (size_t)g.nz * g.ny, npix = (size_t)g.W * g.H;
    unsigned tickets = 0;  // the job's ticket counter at the next dynamic phase's start
    for (int v = 0; v < J.V; ++v) {
        const int local = J.perm[v];  // (a plain load: the whole-iteration launch draws perm itself)
        const ViewRec &vr = J.views[J.view_base + local];
        if (volt && vr.layout == 1) {  // the z-fastest copy this view gathers from
            const int tx = (g.nx + 31) / 32, tz = (g.nz + 31) / 32;
            for (int t = rank; t < tx * tz * g.ny; t += nb) {
                const int x0 = (t % tx) * 32, z0 = ((t / tx) % tz) * 32, y = t / (tx * tz);
                for (int r = warp; r < 32; r += SWEEP_THREADS / 32)
                    if (x0 + lane < g.nx && z0 + r < g.nz)
                        tile[r][lane] = vol[(x0 + lane) + (size_t)y * g.nx + (size_t)(z0 + r) * nxy];
                __syncthreads();
                for (int r = warp; r < 32; r += SWEEP_THREADS / 32)
                    if (x0 + r < g.nx && z0 + lane < g.nz)
                        volt[(z0 + lane) + (size_t)y * g.nz + (size_t)(x0 + r) * nzy] = tile[lane][r];
                __syncthreads();
            }
            if (!sweep_barrier(J.bar, ++passed * nb, status)) return false;
        }
        {  // forward projection + correction (tiles of uneven cost: handed out dynamically)
            const T *b = stack + (size_t)local * npix;
            const int tw = (g.W + 31) / 32, th = (g.H + 3) / 4;
            dynamic_tiles(J.bar + 2, tickets, tw * th, [&](int t) {
                const int i = (t % tw) * 32 + lane, j = (t / tw) * 4 + warp;
                if (i < g.W && j < g.H) sweep_fp_pixel<I>(g, vr, vol, volt, b, J.raylen, J.corr, i, j);
            });
            tickets += (unsigned)(tw * th + nb);
        }
        if (!sweep_barrier(J.bar, ++passed * nb, status)) return false;
        {  // voxel-based backprojection (columns outside the view's shadow are cheap: dynamic too)
            const int cx = (g.nx + SWEEP_THREADS - 1) / SWEEP_THREADS, cy = (g.ny + SWEEP_COL - 1) / SWEEP_COL;
            const BpRowsLoad rows{J.corr, g.W};
            dynamic_tiles(J.bar + 2, tickets, cx * cy * g.nz, [&](int t) {
                const int x = (t % cx) * SWEEP_THREADS + threadIdx.x, y0 = ((t / cx) % cy) * SWEEP_COL;
                const int z = t / (cx * cy);
                if (x < g.nx) bp_column<SWEEP_COL, false>(g, vr, rows, vol, x, y0, z, J.alpha, J.gmax);
            });
            tickets += (unsigned)(cx * cy * g.nz + nb);
        }
        if (!sweep_barrier(J.bar, ++passed * nb, status)) return false;
    }
    // the ROI mask and the over-relaxation (the job's last step: nothing of
    // this job reads it before the launch ends)
    const int rx = (g.nx + SWEEP_THREADS - 1) / SWEEP_THREADS;
    const T *xprev = static_cast<const T *>(J.xprev);
    T *xbar = static_cast<T *>(J.xbar);
    for (int t = rank; t < rx * g.ny * g.nz; t += nb) {
        const int i = (t % rx) * SWEEP_THREADS + threadIdx.x, j = (t / rx) % g.ny, k = t / (rx * g.ny);
        if (i < g.nx) roi_apply_at(i, j, k, g.nx, g.ny, g.nz, J.roi, J.pdcut, vol, xprev, xbar);
    }
    return true;
}

// Seven blocks per SM: 72 registers, no spills (eight would spill); 1036
// resident blocks on 148 SMs.  jobs: sorted by round; a block runs, round
// after round, the job whose block range holds it.
template <typename T, typename I>
__global__ void __launch_bounds__(SWEEP_THREADS, 7) k_sweep_persistent(const SweepJob *__restrict__ jobs, int njobs,
                                                                       int *status) {
    __shared__ T tile[32][33];
    const int b = (int)blockIdx.x;
    for (int q = 0; q < njobs; ++q) {
        const SweepJob &J = jobs[q];
        if (b < J.block0 || b >= J.block0 + J.nblocks) continue;  // another block's job of this round
        if (!run_job<T, I>(J, b - J.block0, tile, status)) return;
    }
}

// The whole primal-dual iteration of every job in one cooperative launch
// (ST_Tomography.cpp:492-607; one round: a block per job at least).  Per job
// (frame): its view order (from the iteration counter, which its owner job
// advances once every job has read it); over its voxels the backward warp
// of X_bar[f+1] along flow[f] and the dual step; a barrier of the whole grid
// (frame f's primal step reads frame f-1's duals); over its voxels the
// forward warp of Y_bc[f-1] along flow[f-1] and the primal step; the job's
// barrier; then the SART call, ROI mask and over-relaxation of run_job.  The
// warp is the gather form's trace and sample (trace_cell, sample_cell), the
// dual and primal steps the per-voxel functions of the separate kernels
// (pd_dual_at, pd_primal_at), the warped value passed in a register; the
// duals the primal step reads were written in this launch, so it loads them
// (and the warp's taps of Y_bc[f-1]) with plain loads.
template <typename T, typename I>
__global__ void __launch_bounds__(SWEEP_THREADS, 7) k_iter_persistent(const SweepJob *__restrict__ jobs, int njobs,
                                                                      unsigned *gbar, int *status) {
    __shared__ T tile[32][33];
    const int b = (int)blockIdx.x;
    int q = 0;
    while (q + 1 < njobs && b >= jobs[q + 1].block0) ++q;
    const SweepJob &J = jobs[q];
    const int rank = b - J.block0, nb = J.nblocks;
    const warpdev::Dim3i d{J.g.nx, J.g.ny, J.g.nz};
    const int gx = (d.x + SWEEP_THREADS - 1) / SWEEP_THREADS;
    const long long rows = (long long)gx * d.y * d.z;
    const T *xbar = static_cast<const T *>(J.xbar), *xbar1 = static_cast<const T *>(J.xbar1);
    if (rank == 0 && threadIdx.x == 0) view_order(J.seed, *J.counter, J.frames_total, J.frame_seq, J.V, J.perm);
    for (long long t = rank; t < rows; t += nb) {  // backward warp + dual step
        const int i = (int)(t % gx) * SWEEP_THREADS + threadIdx.x, j = (int)((t / gx) % d.y);
        const int k = (int)(t / ((long long)gx * d.y));
        if (i < d.x) {
            warpdev::Cell s;
            warpdev::trace_cell(d, J.flow, -1.0f, i, j, k, s);
            float bw[1];
            warpdev::sample_cell<1, false, T>(xbar1, 0, s, bw);
            pd_dual_at(i, j, k, d.x, d.y, d.z, J.sigma, J.tv_w, J.tp_w, J.bc_w, J.hf, J.pdcut, xbar, xbar1, bw[0],
                       J.ytv, J.ytp, J.ybc);
        }
    }
    if (!sweep_barrier(gbar, gridDim.x, status)) return;
    if (J.counter_owner && rank == 0 && threadIdx.x == 0) *J.counter += 1;
    T *vol = static_cast<T *>(J.vol), *xprev = static_cast<T *>(J.xprev);
    for (long long t = rank; t < rows; t += nb) {  // forward warp + primal step
        const int i = (int)(t % gx) * SWEEP_THREADS + threadIdx.x, j = (int)((t / gx) % d.y);
        const int k = (int)(t / ((long long)gx * d.y));
        if (i < d.x) {
            float fw = 0.0f;
            if (!J.first) {
                warpdev::Cell s;
                warpdev::trace_cell(d, J.flow_prev, 1.0f, i, j, k, s);
                float v[1];
                warpdev::sample_cell<1, false, float, true>(J.ybc_prev, 0, s, v);
                fw = v[0];
            }
            pd_primal_at<true>(i, j, k, d.x, d.y, d.z, J.tau, J.gmax, J.pdcut, J.first, J.ytp_prev, J.ytp, fw, J.ybc,
                               J.ytv, vol, xprev);
        }
    }
    if (!sweep_barrier(J.bar, nb, status)) return;  // (the SART call reads every voxel of the volume)
    run_job<T, I>(J, rank, tile, status, 1);
}

template <typename T, typename I>
const void *sweep_kernel() {
    return reinterpret_cast<const void *>(&k_sweep_persistent<T, I>);
}

template <typename T, typename I>
const void *iter_kernel() {
    return reinterpret_cast<const void *>(&k_iter_persistent<T, I>);
}

const void *pick(bool bf16, bool wide, bool whole = false) {
    if (whole) {
        if (bf16) return wide ? iter_kernel<unsigned short, long long>() : iter_kernel<unsigned short, int>();
        return wide ? iter_kernel<float, long long>() : iter_kernel<float, int>();
    }
    if (bf16) return wide ? sweep_kernel<unsigned short, long long>() : sweep_kernel<unsigned short, int>();
    return wide ? sweep_kernel<float, long long>() : sweep_kernel<float, int>();
}

}  // namespace

int sweep_max_blocks(bool bf16, bool wide) {
    // (the smaller of the two kernels' resident blocks: one plan serves both)
    int per_sm = 0, per_sm2 = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm2, pick(bf16, wide, true), SWEEP_THREADS, 0) !=
        cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, pick(bf16, wide), SWEEP_THREADS, 0) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return (per_sm2 < per_sm ? per_sm2 : per_sm) * sm_count();
}

namespace {
// One round's jobs [q0, q1) share all nblocks: every job one block, the rest
// in proportion to the work.
void split_round(SweepJob *jobs, int q0, int q1, int nblocks) {
    double total = 0.0;
    for (int q = q0; q < q1; ++q) total += jobs[q].work > 0.0 ? jobs[q].work : 1.0;
    const int spare = nblocks - (q1 - q0);
    int given = 0;
    for (int q = q0; q < q1; ++q) {
        const double w = jobs[q].work > 0.0 ? jobs[q].work : 1.0;
        jobs[q].nblocks = 1 + (int)((double)spare * w / total);
        given += jobs[q].nblocks;
    }
    for (int q = q0; given < nblocks; q = q + 1 < q1 ? q + 1 : q0, ++given) ++jobs[q].nblocks;
    int b0 = 0;
    for (int q = q0; q < q1; ++q) {
        jobs[q].block0 = b0;
        b0 += jobs[q].nblocks;
    }
}
}  // namespace

int sweep_plan(SweepJob *jobs, int njobs, int nblocks) {
    if (njobs < 1 || nblocks < 1) return 0;
    // largest first, at most nblocks jobs a round
    std::stable_sort(jobs, jobs + njobs, [](const SweepJob &a, const SweepJob &b) { return a.work > b.work; });
    int rounds = 0;
    for (int q0 = 0; q0 < njobs; q0 += nblocks, ++rounds) {
        const int q1 = q0 + nblocks < njobs ? q0 + nblocks : njobs;
        split_round(jobs, q0, q1, nblocks);
        for (int k = q0; k < q1; ++k) jobs[k].round = rounds;
    }
    return rounds;
}

cudaError_t launch_iter_persistent(const SweepJob *jobs_d, int njobs, int nblocks, bool bf16, bool wide,
                                   unsigned *gbar, int *status, cudaStream_t s) {
    if (njobs < 1 || nblocks < njobs) return cudaErrorInvalidValue;  // one round
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(nblocks);
    cfg.blockDim = dim3(SWEEP_THREADS);
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    void *args[] = {(void *)&jobs_d, (void *)&njobs, (void *)&gbar, (void *)&status};
    return cudaLaunchKernelExC(&cfg, pick(bf16, wide, true), args);
}

cudaError_t launch_sweep_persistent(const SweepJob *jobs_d, int njobs, int nblocks, bool bf16, bool wide,
                                    int *status, cudaStream_t s) {
    if (njobs < 1 || nblocks < 1) return cudaErrorInvalidValue;
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(nblocks);
    cfg.blockDim = dim3(SWEEP_THREADS);
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    void *args[] = {(void *)&jobs_d, (void *)&njobs, (void *)&status};
    return cudaLaunchKernelExC(&cfg, pick(bf16, wide), args);
}

}  // namespace stt
