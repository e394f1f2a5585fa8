// stt_flow.cu -- host side of the optical flow in include/stt.h: the
// multiscale driver of optical_flow::L1Huber_OF_MultiScale3D
// (S/ST_Tomo/optical_flow.h:630-734), the per-level loop of L1Huber_OF
// (:83-623), and the CImg blur/resize sequencing.  Kernels are in k_flow.cu.
//
// Reference paths are relative to gmzang/SpaceTimeTomography (S/ = SpaceTimeTomography/).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "stt.h"
#include "stt_kernels.h"

extern "C" stt_status stt_internal_set_error(stt_ctx *ctx, stt_status st, const char *msg);

namespace {

constexpr int kTableCap = 8192;  // longest resized axis
constexpr int kFlowMaxDim = 4096;  // flow extents (10 channel planes * nz must fit a grid's z extent)

struct Level {
    int d[3];
    long long n;
};

long long vol(const int *d) { return (long long)d[0] * d[1] * d[2]; }

// CImg::deriche order-0 coefficients (CImg.h:32941-32961), float arithmetic
// with std::exp on floats as CImg evaluates them.
stt::DericheCoef deriche_coefs(float sigma) {
    const float nnsigma = sigma < 0.1f ? 0.1f : sigma, alpha = 1.695f / nnsigma,
                ema = (float)std::exp(-alpha), ema2 = (float)std::exp(-2 * alpha), b1 = -2 * ema, b2 = ema2;
    const float k = (1 - ema) * (1 - ema) / (1 + 2 * alpha * ema - ema2);
    stt::DericheCoef c;
    c.a0 = k;
    c.a1 = k * (alpha - 1) * ema;
    c.a2 = k * (alpha + 1) * ema;
    c.a3 = -k * ema2;
    c.b1 = b1;
    c.b2 = b2;
    c.coefp = (c.a0 + c.a1) / (1 + b1 + b2);
    c.coefn = (c.a2 + c.a3) / (1 + b1 + b2);
    return c;
}

cudaStream_t S(void *s) { return reinterpret_cast<cudaStream_t>(s); }

}  // namespace

struct stt_flow {
    int device = 0;
    std::string err;
    int dims[3] = {0, 0, 0};
    long long nmax = 0;
    stt_flow_params p{};
    std::vector<Level> lev;  // coarse first; the last one is the full size
    // device memory
    std::vector<void *> allocs;
    float *blur1 = nullptr, *blur2 = nullptr;  // blurred full-size images
    std::vector<float *> pyr1, pyr2;           // the coarser levels of the pyramid
    float *vbuf[2] = {nullptr, nullptr};       // flow of the coarser levels
    float *ybuf[2] = {nullptr, nullptr};       // dual of every level
    float *yw = nullptr, *vpp = nullptr, *kty = nullptr, *u = nullptr, *tau = nullptr, *sig2 = nullptr,
          *i2w = nullptr, *k4prev = nullptr;
    int *tsrc = nullptr;
    double *tfrac = nullptr;
    double *resid = nullptr;
    int *done = nullptr;
    int *iters = nullptr;
    float *errs = nullptr;
    int n_stat = 0, stat_cap = 0;
    // The stop flag as the host last saw it: at every residual check the flag
    // is copied into a slot of this pinned ring behind an event, so the host
    // can stop enqueuing a warp whose iterations stopped (enqueue_level).
    static constexpr int kRing = 8, kLookahead = 4;
    int *done_host = nullptr;
    cudaEvent_t ring_ev[kRing] = {};

    stt_status fail(stt_status st, const std::string &m) {
        err = m;
        return st;
    }
    stt_status cuda(cudaError_t e, const char *where) {
        if (e == cudaSuccess) return STT_OK;
        return fail(STT_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
    }
    template <typename T>
    stt_status alloc(T **ptr, long long count) {
        void *q = nullptr;
        if (cudaMalloc(&q, (size_t)std::max<long long>(count, 1) * sizeof(T)) != cudaSuccess) {
            cudaGetLastError();
            return fail(STT_ERR_NOMEM, "cudaMalloc of " + std::to_string(count * sizeof(T)) + " bytes failed");
        }
        allocs.push_back(q);
        *ptr = static_cast<T *>(q);
        return STT_OK;
    }
    ~stt_flow() {
        for (void *q : allocs) cudaFree(q);
        for (cudaEvent_t e : ring_ev)
            if (e) cudaEventDestroy(e);
        if (done_host) cudaFreeHost(done_host);
    }
};

#define FLOW_TRY(expr)                    \
    do {                                  \
        stt_status st_ = (expr);          \
        if (st_ != STT_OK) return st_;    \
    } while (0)
#define FLOW_CUDA(f, call, where) FLOW_TRY((f)->cuda((call), (where)))

namespace {

// Deriche blur along x, y, z of every axis longer than 1 (CImg::blur,
// CImg.h:33249-33262), in place, one channel at a time; scratch = f->i2w.
stt_status enqueue_blur(stt_flow *f, const int *d, int nc, float sigma, float *img, cudaStream_t s) {
    if (sigma < 0.1f) return STT_OK;  // deriche() leaves the image unchanged
    const stt::DericheCoef c = deriche_coefs(sigma);
    for (int ch = 0; ch < nc; ++ch)
        for (int axis = 0; axis < 3; ++axis)
            if (d[axis] > 1)
                FLOW_CUDA(f, stt::launch_deriche(d, 1, axis, c, img + ch * vol(d), f->i2w, s), "k_deriche_line");
    return STT_OK;
}

// get_resize(odim, nc, 5): one pass per axis whose extent changes, x then y
// then z, one channel at a time, ping-ponging through f->i2w and f->sig2
// (both free between levels).
stt_status enqueue_resize(stt_flow *f, const int *di, int nc, const float *in, const int *dout, float *out,
                          cudaStream_t s) {
    int axes[3], na = 0;
    for (int a = 0; a < 3; ++a)
        if (di[a] != dout[a]) axes[na++] = a;
    if (na == 0) {
        if (in != out)
            FLOW_CUDA(f, cudaMemcpyAsync(out, in, sizeof(float) * vol(di) * nc, cudaMemcpyDeviceToDevice, s),
                      "resize copy");
        return STT_OK;
    }
    for (int ch = 0; ch < nc; ++ch) {
        int cur[3] = {di[0], di[1], di[2]};
        const float *src = in + ch * vol(di);
        for (int q = 0; q < na; ++q) {
            const int a = axes[q];
            stt::ResizeAxis ra{};
            ra.axis = a;
            ra.nc = 1;
            ra.ix = cur[0];
            ra.iy = cur[1];
            ra.iz = cur[2];
            ra.old_n = cur[a];
            ra.new_n = dout[a];
            cur[a] = dout[a];
            ra.ox = cur[0];
            ra.oy = cur[1];
            ra.oz = cur[2];
            ra.mode = ra.new_n < ra.old_n ? 0 : 1;
            if (ra.mode == 1) {
                FLOW_CUDA(f, stt::launch_resize_table(ra.old_n, ra.new_n, f->tsrc, f->tfrac, s), "k_resize_table");
                ra.src = f->tsrc;
                ra.frac = f->tfrac;
            }
            float *dst = q == na - 1 ? out + ch * vol(dout) : (q % 2 == 0 ? f->i2w : f->sig2);
            FLOW_CUDA(f, stt::launch_resize_axis(ra, src, dst, s), "k_resize_axis");
            src = dst;
        }
    }
    return STT_OK;
}

// One L1Huber_OF call (optical_flow.h:83-623) on a level of size d.  The
// flow alternates between V and f->vpp: iteration `it` reads buffer
// (it-1)&1 and writes buffer it&1; k_flow_settle brings the last one back
// into V at the end of every warp.
stt_status enqueue_level(stt_flow *f, const int *d, const float *box, const int *roi6, const float *i1,
                         const float *i2, float *V, float *Y, int stat0, cudaStream_t s) {
    const stt_flow_params &p = f->p;
    const long long n = vol(d);
    const stt::FlowRoi roi{roi6[0], roi6[1], roi6[2], roi6[3], roi6[4], roi6[5]};
    const float sigma1 = std::min(1.0f / 3.0f, std::min(1.0f / 3.0f, 1.0f / 3.0f));
    const float hf = 1.0f / (1.0f + sigma1 * p.huber / p.lambda);
    float *vb[2] = {V, f->vpp};
    FLOW_CUDA(f, cudaMemcpyAsync(f->yw, Y, sizeof(float) * 10 * n, cudaMemcpyDeviceToDevice, s), "copy Y");
    FLOW_CUDA(f, cudaMemcpyAsync(f->vpp, V, sizeof(float) * 3 * n, cudaMemcpyDeviceToDevice, s), "copy V");
    FLOW_CUDA(f, cudaMemsetAsync(f->kty, 0, sizeof(float) * 3 * n, s), "clear Kty");
    const bool runs = 1.0f > p.tol;  // err starts at 1 (optical_flow.h:305-306)
    const int last = p.max_iter + 1;
    bool any_dual = false;
    // Once a warp's check has stopped it, the launches of its remaining
    // iterations return at once, but each still costs its full grid (about
    // 75 us per iteration at 256^3; with the reference's parameters the warps
    // of a 256^3 multiscale solve stop after 400-1000 of their 3001
    // iterations).  So after every check the stop flag is copied to pinned
    // host memory behind an event; the host stays at most kLookahead checks
    // ahead of the device, and when a copy that has landed shows the warp
    // stopped, the rest of its iterations are not enqueued (they would have
    // done nothing: the same results, and the same iteration counts, which
    // the check recorded when it stopped).  Not while the stream is being
    // captured: then every iteration is enqueued.
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    if (cudaStreamIsCapturing(s, &cap) != cudaSuccess) {
        cudaGetLastError();
        cap = cudaStreamCaptureStatusActive;
    }
    const bool poll = cap == cudaStreamCaptureStatusNone;
    for (int w = 0; w < p.n_warps; ++w) {
        int *it_slot = f->iters + stat0 + w;
        float *err_slot = f->errs + stat0 + w;
        FLOW_CUDA(f, stt::launch_flow_reset(f->done, f->resid, it_slot, err_slot, s), "k_flow_reset");
        FLOW_CUDA(f, stt::launch_warp_box(d, box, V, i2, 1, -1.0f, f->i2w, s), "k_warp_box");
        FLOW_CUDA(f, stt::launch_flow_setup(d, roi, f->i2w, i1, V, f->u, f->tau, f->sig2, f->k4prev, s),
                  "k_flow_setup");
        if (!runs) continue;
        int pushed = 0, seen = 0;  // checks whose flag copy was enqueued / looked at
        for (int it = 1; it <= last; ++it) {
            int flags = (it % 50 == 0 ? 1 : 0) | ((it + 1) % 50 == 0 ? 2 : 0);
            if (it == 1) flags |= any_dual ? 8 : 4;
            const float *vin = vb[(it - 1) & 1];
            float *vout = vb[it & 1];
            FLOW_CUDA(f, stt::launch_flow_primal(d, roi, f->yw, f->u, f->tau, vin, vout, f->kty, flags, f->resid,
                                                 f->done, s),
                      "k_flow_primal");
            FLOW_CUDA(f, stt::launch_flow_dual(d, vout, vin, f->u, f->sig2, f->k4prev, f->yw, sigma1, hf, p.lambda,
                                               p.norm == 4 ? 1 : 0, flags, f->resid, f->done, s),
                      "k_flow_dual");
            if ((flags & 1) || it == last)
                FLOW_CUDA(f, stt::launch_flow_check(f->resid, n, p.tol, it, flags & 1, it == last, f->done, it_slot,
                                                    err_slot, s),
                          "k_flow_check");
            if (poll && (flags & 1) && it < last) {
                // at most kLookahead checks (kLookahead * 50 iterations) ahead of the
                // device: past that, wait for the oldest copy, so that no more than
                // those iterations are enqueued after the warp stopped
                if (pushed - seen >= stt_flow::kLookahead) {
                    FLOW_CUDA(f, cudaEventSynchronize(f->ring_ev[seen % stt_flow::kRing]), "cudaEventSynchronize");
                    if (f->done_host[seen % stt_flow::kRing]) break;
                    ++seen;
                }
                const int q = pushed++ % stt_flow::kRing;
                FLOW_CUDA(f, cudaMemcpyAsync(f->done_host + q, f->done, sizeof(int), cudaMemcpyDeviceToHost, s),
                          "copy stop flag");
                FLOW_CUDA(f, cudaEventRecord(f->ring_ev[q], s), "event record");
                bool stopped = false;
                while (seen < pushed) {
                    const cudaError_t qe = cudaEventQuery(f->ring_ev[seen % stt_flow::kRing]);
                    if (qe == cudaErrorNotReady) {
                        cudaGetLastError();  // (not an error: the copy has not landed yet)
                        break;
                    }
                    FLOW_CUDA(f, qe, "cudaEventQuery");
                    if (f->done_host[seen % stt_flow::kRing]) {
                        stopped = true;
                        break;
                    }
                    ++seen;
                }
                if (stopped) break;
            }
        }
        any_dual = true;
        FLOW_CUDA(f, stt::launch_flow_settle(3 * n, it_slot, f->vpp, V, s), "k_flow_settle");
    }
    FLOW_CUDA(f, stt::launch_copy_roi(d, 10, roi, f->yw, Y, s), "k_copy_roi");
    return STT_OK;
}

stt_status check_params(const stt_flow_params *p, std::string &why) {
    if (!p) return why = "null params", STT_ERR_INVALID;
    if (p->scales < 1) return why = "scales must be >= 1", STT_ERR_INVALID;
    if (p->n_warps < 0 || p->max_iter < 0 || p->max_iter > 100000000)
        return why = "n_warps must be >= 0 and max_iter in [0, 1e8]", STT_ERR_INVALID;
    if (!(p->lambda > 0.0f)) return why = "lambda must be > 0", STT_ERR_INVALID;
    if (!(p->eta > 0.0f) || p->eta > 1.0f) return why = "eta must be in (0, 1]", STT_ERR_INVALID;
    for (int q = 0; q < 6; ++q)
        if (p->cut[q] < 0) return why = "cut entries must be >= 0", STT_ERR_INVALID;
    return STT_OK;
}

}  // namespace

extern "C" {

stt_status stt_flow_create(int device, const int *dims, const stt_flow_params *p, stt_flow **out) {
    if (!out || !dims) return stt_internal_set_error(nullptr, STT_ERR_INVALID, "null argument");
    *out = nullptr;
    std::string why;
    if (check_params(p, why) != STT_OK) return stt_internal_set_error(nullptr, STT_ERR_INVALID, why.c_str());
    for (int a = 0; a < 3; ++a)
        if (dims[a] < 3 || dims[a] > kFlowMaxDim)
            return stt_internal_set_error(nullptr, STT_ERR_INVALID, "flow dims must be in [3, 4096]");
    if (vol(dims) * 10 >= (1LL << 31))  // the kernels address the 10 dual planes with 32-bit offsets
        return stt_internal_set_error(nullptr, STT_ERR_INVALID, "flow volume too large (10 * voxels must be < 2^31)");
    // Pyramid sizes (optical_flow.h:659-677): dims * eta^s, eta^s accumulated in float.
    std::vector<Level> lev;
    float t_eta = 1.0f;
    for (int sc = 0; sc < p->scales; ++sc) {
        Level L;
        for (int a = 0; a < 3; ++a) L.d[a] = (int)((float)dims[a] * t_eta);
        L.n = vol(L.d);
        if (L.d[0] < 3 || L.d[1] < 3 || L.d[2] < 3)
            return stt_internal_set_error(nullptr, STT_ERR_INVALID,
                                          "a pyramid level is smaller than 3 voxels along an axis: "
                                          "use fewer scales or a larger eta");
        lev.insert(lev.begin(), L);
        t_eta = t_eta * p->eta;
    }
    if (cudaSetDevice(device) != cudaSuccess) {
        cudaGetLastError();
        return stt_internal_set_error(nullptr, STT_ERR_CUDA, "cudaSetDevice failed");
    }
    auto *f = new stt_flow;
    f->device = device;
    f->p = *p;
    std::memcpy(f->dims, dims, sizeof(f->dims));
    f->nmax = vol(dims);
    f->lev = lev;
    const long long n = f->nmax;
    long long coarse_max = 1;
    for (size_t l = 0; l + 1 < f->lev.size(); ++l) coarse_max = std::max(coarse_max, f->lev[l].n);
    stt_status st = STT_OK;
    auto A = [&](auto **ptr, long long count) {
        if (st == STT_OK) st = f->alloc(ptr, count);
    };
    A(&f->blur1, n);
    A(&f->blur2, n);
    f->pyr1.assign(f->lev.size(), nullptr);
    f->pyr2.assign(f->lev.size(), nullptr);
    for (size_t l = 0; l + 1 < f->lev.size(); ++l) {
        A(&f->pyr1[l], f->lev[l].n);
        A(&f->pyr2[l], f->lev[l].n);
    }
    for (int b = 0; b < 2; ++b) {
        A(&f->vbuf[b], 3 * coarse_max);
        A(&f->ybuf[b], 10 * n);
    }
    A(&f->yw, 10 * n);
    A(&f->vpp, 3 * n);
    A(&f->k4prev, n);
    A(&f->kty, 3 * n);
    A(&f->u, 4 * n);
    A(&f->tau, 3 * n);
    A(&f->sig2, n);
    A(&f->i2w, n);
    A(&f->tsrc, kTableCap);
    A(&f->tfrac, kTableCap);
    A(&f->resid, 2);
    A(&f->done, 1);
    f->stat_cap = std::max(1, (int)f->lev.size() * std::max(1, p->n_warps));
    A(&f->iters, f->stat_cap);
    A(&f->errs, f->stat_cap);
    if (st == STT_OK && cudaHostAlloc((void **)&f->done_host, stt_flow::kRing * sizeof(int), cudaHostAllocDefault) !=
                            cudaSuccess) {
        cudaGetLastError();
        f->done_host = nullptr;
        st = f->fail(STT_ERR_NOMEM, "cudaHostAlloc of the stop-flag ring failed");
    }
    for (int q = 0; q < stt_flow::kRing && st == STT_OK; ++q)
        if (cudaEventCreateWithFlags(&f->ring_ev[q], cudaEventDisableTiming) != cudaSuccess) {
            cudaGetLastError();
            st = f->fail(STT_ERR_CUDA, "event create");
        }
    if (st != STT_OK) {
        std::string m = f->err;
        delete f;
        return stt_internal_set_error(nullptr, st, m.c_str());
    }
    *out = f;
    return STT_OK;
}

const char *stt_flow_last_error(const stt_flow *f) { return f ? f->err.c_str() : "null flow"; }

stt_status stt_flow_destroy(stt_flow *f) {
    if (f) {
        cudaSetDevice(f->device);
        delete f;
    }
    return STT_OK;
}

stt_status stt_flow_multiscale(stt_flow *f, const float *I1, const float *I2, float *V, const float *Y0,
                               void *stream) {
    if (!f) return stt_internal_set_error(nullptr, STT_ERR_INVALID, "null flow");
    if (!I1 || !I2 || !V) return f->fail(STT_ERR_INVALID, "null I1, I2 or V");
    FLOW_CUDA(f, cudaSetDevice(f->device), "cudaSetDevice");
    cudaStream_t s = S(stream);
    const long long n = f->nmax;
    const int L = (int)f->lev.size();
    const int *full = f->dims;
    // blurred images (optical_flow.h:636-637)
    FLOW_CUDA(f, cudaMemcpyAsync(f->blur1, I1, sizeof(float) * n, cudaMemcpyDeviceToDevice, s), "copy I1");
    FLOW_CUDA(f, cudaMemcpyAsync(f->blur2, I2, sizeof(float) * n, cudaMemcpyDeviceToDevice, s), "copy I2");
    FLOW_TRY(enqueue_blur(f, full, 1, f->p.sigma, f->blur1, s));
    FLOW_TRY(enqueue_blur(f, full, 1, f->p.sigma, f->blur2, s));
    // pyramid (optical_flow.h:663-677): every level resized from the full size
    for (int l = 0; l + 1 < L; ++l) {
        FLOW_TRY(enqueue_resize(f, full, 1, f->blur1, f->lev[l].d, f->pyr1[l], s));
        FLOW_TRY(enqueue_resize(f, full, 1, f->blur2, f->lev[l].d, f->pyr2[l], s));
    }
    // Starting point of the coarsest level; the finer levels start from the
    // upsampled result of the level below (optical_flow.h:718-729).
    float *v_cur = L == 1 ? V : f->vbuf[0];
    float *y_cur = f->ybuf[0];
    if (L > 1) FLOW_TRY(enqueue_resize(f, full, 3, V, f->lev[0].d, v_cur, s));
    if (Y0) FLOW_TRY(enqueue_resize(f, full, 10, Y0, f->lev[0].d, y_cur, s));
    else FLOW_CUDA(f, cudaMemsetAsync(y_cur, 0, sizeof(float) * 10 * f->lev[0].n, s), "clear Y");
    const float box[3] = {(float)full[0], (float)full[1], (float)full[2]};
    f->n_stat = L * f->p.n_warps;
    for (int l = 0; l < L; ++l) {
        const Level &lv = f->lev[l];
        int roi[6];
        for (int q = 0; q < 6; ++q)
            roi[q] = (int)((float)f->p.cut[q] * ((float)lv.d[q / 2] / (float)full[q / 2]));
        const float *i1 = l + 1 < L ? f->pyr1[l] : f->blur1;
        const float *i2 = l + 1 < L ? f->pyr2[l] : f->blur2;
        FLOW_TRY(enqueue_level(f, lv.d, box, roi, i1, i2, v_cur, y_cur, l * f->p.n_warps, s));
        if (l + 1 < L) {
            const Level &nx = f->lev[l + 1];
            float *v_next = l + 2 == L ? V : f->vbuf[(l + 1) % 2];
            float *y_next = f->ybuf[(l + 1) % 2];
            FLOW_TRY(enqueue_resize(f, lv.d, 3, v_cur, nx.d, v_next, s));
            FLOW_TRY(enqueue_resize(f, lv.d, 10, y_cur, nx.d, y_next, s));
            v_cur = v_next;
            y_cur = y_next;
        }
    }
    return STT_OK;
}

stt_status stt_flow_level(stt_flow *f, const int *dim, const float *box, const int *roi, const float *I1,
                          const float *I2, float *V, float *Y, void *stream) {
    if (!f) return stt_internal_set_error(nullptr, STT_ERR_INVALID, "null flow");
    if (!dim || !box || !roi || !I1 || !I2 || !V || !Y) return f->fail(STT_ERR_INVALID, "null argument");
    for (int a = 0; a < 3; ++a)
        if (dim[a] < 3) return f->fail(STT_ERR_INVALID, "level extents must be >= 3");
    if (vol(dim) > f->nmax) return f->fail(STT_ERR_INVALID, "level larger than the created volume");
    for (int q = 0; q < 6; ++q)
        if (roi[q] < 0) return f->fail(STT_ERR_INVALID, "roi entries must be >= 0");
    FLOW_CUDA(f, cudaSetDevice(f->device), "cudaSetDevice");
    f->n_stat = f->p.n_warps;
    return enqueue_level(f, dim, box, roi, I1, I2, V, Y, 0, S(stream));
}

stt_status stt_flow_stats(stt_flow *f, int *n_entries, int *iters, float *err) {
    if (!f) return stt_internal_set_error(nullptr, STT_ERR_INVALID, "null flow");
    FLOW_CUDA(f, cudaSetDevice(f->device), "cudaSetDevice");
    FLOW_CUDA(f, cudaDeviceSynchronize(), "cudaDeviceSynchronize");
    if (n_entries) *n_entries = f->n_stat;
    if (iters && f->n_stat)
        FLOW_CUDA(f, cudaMemcpy(iters, f->iters, sizeof(int) * f->n_stat, cudaMemcpyDeviceToHost), "read iterations");
    if (err && f->n_stat)
        FLOW_CUDA(f, cudaMemcpy(err, f->errs, sizeof(float) * f->n_stat, cudaMemcpyDeviceToHost), "read residuals");
    return STT_OK;
}

stt_status stt_flow_blur(stt_flow *f, const int *dim, int nc, float sigma, float *img, void *stream) {
    if (!f) return stt_internal_set_error(nullptr, STT_ERR_INVALID, "null flow");
    if (!dim || !img || nc < 1) return f->fail(STT_ERR_INVALID, "null argument or nc < 1");
    if (dim[0] < 1 || dim[1] < 1 || dim[2] < 1 || dim[0] > kFlowMaxDim || dim[1] > kFlowMaxDim ||
        dim[2] > kFlowMaxDim || vol(dim) > f->nmax)
        return f->fail(STT_ERR_INVALID, "blur size out of range (each channel at most the created volume)");
    FLOW_CUDA(f, cudaSetDevice(f->device), "cudaSetDevice");
    return enqueue_blur(f, dim, nc, sigma, img, S(stream));
}

stt_status stt_flow_resize(stt_flow *f, const int *dim, int nc, const float *in, const int *odim, float *out,
                           void *stream) {
    if (!f) return stt_internal_set_error(nullptr, STT_ERR_INVALID, "null flow");
    if (!dim || !odim || !in || !out || nc < 1) return f->fail(STT_ERR_INVALID, "null argument or nc < 1");
    int cur[3] = {dim[0], dim[1], dim[2]};
    for (int a = 0; a < 3; ++a) {
        if (dim[a] < 2 || odim[a] < 1 || odim[a] > kTableCap)
            return f->fail(STT_ERR_INVALID, "resize extents out of range (input >= 2, output in [1, 8192])");
        cur[a] = odim[a];
        if (vol(cur) > f->nmax)
            return f->fail(STT_ERR_INVALID, "resize intermediate larger than the created volume");
    }
    if (in == out) return f->fail(STT_ERR_INVALID, "resize cannot run in place");
    FLOW_CUDA(f, cudaSetDevice(f->device), "cudaSetDevice");
    return enqueue_resize(f, dim, nc, in, odim, out, S(stream));
}

stt_status stt_warp_box(const int *dim, const float *box, const float *vel, const float *src, int nc, float dt,
                        float *out, void *stream) {
    if (!dim || !box || !vel || !src || !out)
        return stt_internal_set_error(nullptr, STT_ERR_INVALID, "null argument");
    if (dim[0] < 3 || dim[1] < 3 || dim[2] < 3)
        return stt_internal_set_error(nullptr, STT_ERR_INVALID, "warp needs every dimension >= 3");
    if (nc < 1) return stt_internal_set_error(nullptr, STT_ERR_INVALID, "nc must be >= 1");
    for (int a = 0; a < 3; ++a)
        if (!(box[a] > 0.0f)) return stt_internal_set_error(nullptr, STT_ERR_INVALID, "box extents must be > 0");
    cudaError_t e = stt::launch_warp_box(dim, box, vel, src, nc, dt, out, S(stream));
    if (e != cudaSuccess)
        return stt_internal_set_error(nullptr, STT_ERR_CUDA, (std::string("k_warp_box: ") + cudaGetErrorString(e)).c_str());
    return STT_OK;
}

stt_status stt_image_gradient(const int *dim, const float *img, float *grad, void *stream) {
    if (!dim || !img || !grad) return stt_internal_set_error(nullptr, STT_ERR_INVALID, "null argument");
    if (dim[0] < 1 || dim[1] < 1 || dim[2] < 1)
        return stt_internal_set_error(nullptr, STT_ERR_INVALID, "extents must be >= 1");
    cudaError_t e = stt::launch_gradient(dim, img, grad, S(stream));
    if (e != cudaSuccess)
        return stt_internal_set_error(nullptr, STT_ERR_CUDA, (std::string("k_gradient: ") + cudaGetErrorString(e)).c_str());
    return STT_OK;
}

}  // extern "C"
