// k_warp.cu -- semi-Lagrangian tricubic warp (S/ST_Tomo/warping.h:49-145) and
// its vector-Jacobian product.
//
// One thread per output voxel, x fastest.  Per voxel: the velocity at the
// cell centre (an exact grid read: the Catmull-Rom sampler interpolates, and
// the centre lands on a node), one clamped tricubic velocity sample at the
// half-traced point (3 channels sharing one 64-tap stencil) and one clamped
// tricubic sample of every source channel at the traced point.  Taps come from
// L1/L2 through the read-only path; the cell corners of the clamp are taps of
// the stencil, so a sample is at most 64 loads per channel.  The kernel is
// bound by L1 load wavefronts, not by HBM.
#include <climits>

#include "stt_internal.cuh"
#include "stt_kernels.h"
#include "stt_tma.cuh"
#include "warp_dev.cuh"

namespace stt {

namespace {

using namespace warpdev;

// Blocks of 32 x 4 voxels: a warp is one x-run of 32, so every tap load of a
// warp reads ~32 consecutive floats, and the block's four rows share most of
// their stencil rows in L1.  All offsets are 32-bit (the host bounds
// n * max(nc, 3) below 2^31).
constexpr int WARP_BX = 32, WARP_BY = 4;

// T: the source's storage (float, or BF16 bits widened exactly to FP32).
template <typename T>
__global__ void __launch_bounds__(WARP_BX *WARP_BY) k_warp(const Dim3i d, const float *__restrict__ vel,
                                                           const T *__restrict__ src, int nc, float dt,
                                                           float *__restrict__ out) {
    const int i = blockIdx.x * WARP_BX + threadIdx.x;
    const int j = blockIdx.y * WARP_BY + threadIdx.y, k = blockIdx.z;
    if (i >= d.x || j >= d.y) return;
    const int n = d.x * d.y * d.z;
    Cell s;
    trace_cell(d, vel, dt, i, j, k, s);
    const int o = i + j * d.x + k * d.x * d.y;
    for (int ch = 0; ch < nc; ++ch) {
        float v[1];
        sample_cell<1>(src + (size_t)ch * n, 0, s, v);
        out[o + (size_t)ch * n] = v[0];
    }
}

// Staged form: the three velocity planes around the block's half-traced
// points come into shared memory with one 4D TMA box, and the velocity sample
// (three quarters of the warp's taps) reads them there.  Each thread finds the
// first tap of its velocity stencil after the exact centre read; the block's
// minimum places the box (x rounded down to 16 bytes); a stencil that does not
// fit in the box (a rough flow, a copy that did not land within the bounded
// wait) reads global memory.  The taps and the arithmetic are those of k_warp,
// so the outputs are the same bits.  The source sample stays on the L1 path.
constexpr int VX = 40, VY = 10, VZ = 6;  // velocity box (x, y, z) per plane; VX*4 is a multiple of 16
constexpr int VBOX = VX * VY * VZ;
constexpr long long WARP_WAIT_CYCLES = 200000000LL;  // about 0.1 s

// Status word of the warps launched without one (stt_warp, stt_warp_box on
// their own): one per device, read and cleared by stt_warp_poll_status.
__device__ int g_warp_wait_status;

template <typename T>
__global__ void __launch_bounds__(WARP_BX *WARP_BY) k_warp_staged(const Dim3i d,
                                                                  const __grid_constant__ CUtensorMap vmap,
                                                                  const float *__restrict__ vel,
                                                                  const T *__restrict__ src, int nc, float dt,
                                                                  float *__restrict__ out, int *status) {
    __shared__ alignas(128) float vbox[3 * VBOX];
    __shared__ uint64_t bar;
    __shared__ int red[3 * WARP_BY];
    const int i = blockIdx.x * WARP_BX + threadIdx.x;
    const int j = blockIdx.y * WARP_BY + threadIdx.y, k = blockIdx.z;
    const bool live = i < d.x && j < d.y;
    const int n = d.x * d.y * d.z;
    const float h = -dt;
    const float p[3] = {(float)i + 0.5f, (float)j + 0.5f, (float)k + 0.5f};
    float p2[3] = {0.0f, 0.0f, 0.0f}, g2[3] = {1.0f, 1.0f, 1.0f};
    int b0[3] = {INT_MAX, INT_MAX, INT_MAX};  // first tap of the velocity stencil
    if (live) {
        // cell centre (warping.h:25-29); the velocity there is an exact node read
        const int ci = min(max(i, 1), d.x - 2), cj = min(max(j, 1), d.y - 2), ck = min(max(k, 1), d.z - 2);
        const int c = ci + cj * d.x + ck * d.x * d.y;
        const float v1[3] = {__ldg(vel + c), __ldg(vel + n + c), __ldg(vel + 2 * n + c)};
        // trace (warping.h:100-114): p2 = p + h v(p); p0 = p2 - h v(p2); q = p2 + (p - p0)/2
#pragma unroll
        for (int a = 0; a < 3; ++a) p2[a] = __fadd_rn(p[a], __fmul_rn(h, v1[a]));
        g2[0] = to_grid(p2[0], d.x, nullptr);
        g2[1] = to_grid(p2[1], d.y, nullptr);
        g2[2] = to_grid(p2[2], d.z, nullptr);
#pragma unroll
        for (int a = 0; a < 3; ++a) b0[a] = (int)g2[a] - 1;
    }
    int m[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) m[a] = __reduce_min_sync(0xffffffffu, b0[a]);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int a = 0; a < 3; ++a) red[3 * threadIdx.y + a] = m[a];
    }
    const bool lead = threadIdx.x == 0 && threadIdx.y == 0;
    if (lead) {
        tma::mbar_init(&bar, 1);
        tma::fence_barrier_init();
    }
    __syncthreads();
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        m[a] = red[a];
#pragma unroll
        for (int w = 1; w < WARP_BY; ++w) m[a] = min(m[a], red[3 * w + a]);
    }
    const bool any = m[0] != INT_MAX;  // uniform: some voxel of the block is inside the volume
    const int ox = (m[0] >> 2) << 2, oy = m[1], oz = m[2];
    if (any && lead) {
        tma::mbar_arrive_expect_tx(&bar, 3u * VBOX * sizeof(float));
        tma::load_box_4d(vbox, &vmap, ox, oy, oz, 0, &bar);
    }
    bool staged = false;
    if (any) {
        staged = tma::mbar_wait(&bar, 0, WARP_WAIT_CYCLES);
        if (!staged) {
            // An error, reported through the status word.  The velocity sample
            // reads global memory instead (same bits); the box is not read, but
            // the block waits (bounded) once more so that it does not exit with
            // the copy still writing into its shared memory.
            atomicExch(status ? status : &g_warp_wait_status, STT_WAIT_TIMEOUT_FLAG);
            tma::mbar_wait(&bar, 0, WARP_WAIT_CYCLES);
        }
    }
    if (!live) return;
    Cell s2;
    cell_setup(d, g2, s2);
    float v2[3];
    const unsigned lx = (unsigned)(b0[0] - ox), ly = (unsigned)(b0[1] - oy), lz = (unsigned)(b0[2] - oz);
    if (staged && lx <= VX - 4 && ly <= VY - 4 && lz <= VZ - 4) {
        Cell sl = s2;  // the same weights and edge flags, box-local offsets
        sl.sy = VX;
        sl.sz = VX * VY;
        sl.x.lo = (int)lx;
        sl.y.lo = (int)ly * VX;
        sl.z.lo = (int)lz * VX * VY;
        sample_cell<3, true>(vbox, VBOX, sl, v2);
    } else {
        sample_cell<3>(vel, n, s2, v2);
    }
    float q[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const float p0 = __fsub_rn(p2[a], __fmul_rn(h, v2[a]));
        q[a] = __fadd_rn(p2[a], __fmul_rn(0.5f, __fsub_rn(p[a], p0)));
    }
    const float gq[3] = {to_grid(q[0], d.x, nullptr), to_grid(q[1], d.y, nullptr), to_grid(q[2], d.z, nullptr)};
    Cell s;
    cell_setup(d, gq, s);
    const int o = i + j * d.x + k * d.x * d.y;
    for (int ch = 0; ch < nc; ++ch) {
        float v[1];
        sample_cell<1>(src + (size_t)ch * n, 0, s, v);
        out[o + (size_t)ch * n] = v[0];
    }
}

// ---- VJP ---------------------------------------------------------------
// For one clamped sample: which branch the clamp took and, when unclamped,
// the spatial gradient of the Catmull-Rom value (zero along an axis whose
// grid coordinate was clamped to [1, dim-2]).
struct SampleD {
    float value;
    int branch;        // 0 interior, 1 clamped to max corner, 2 clamped to min corner
    long long corner;  // arg-max / arg-min corner index when branch != 0
    float grad[3];
};

__device__ __forceinline__ void cr_dweights(float d, float w[4]) {
    float d2 = d * d;
    w[0] = 0.5f * (-1.0f + 4.0f * d - 3.0f * d2);
    w[1] = 0.5f * (-10.0f * d + 9.0f * d2);
    w[2] = 0.5f * (1.0f + 8.0f * d - 9.0f * d2);
    w[3] = 0.5f * (-2.0f * d + 3.0f * d2);
}

__device__ __forceinline__ void sample_d(const float *__restrict__ img, const Stencil &s,
                                         const bool clamped[3], SampleD &r) {
    float dwx[4], dwy[4], dwz[4];
    cr_dweights(s.dx, dwx);
    cr_dweights(s.dy, dwy);
    cr_dweights(s.dz, dwz);
    // Separable sums in the forward sampler's order (x taps, then rows, then
    // planes): per row its value and x-slope, per plane its value and x- and
    // y-slopes, then the sample's value and gradient.
    float val = 0.0f, gx = 0.0f, gy = 0.0f, gz = 0.0f;
#pragma unroll 1
    for (int c = 0; c < 4; ++c) {
        float pv = 0.0f, px = 0.0f, py = 0.0f;
#pragma unroll
        for (int b = 0; b < 4; ++b) {
            const float *row = img + s.yo[b] + s.zo[c];
            const float t0 = __ldg(row + s.xo[0]), t1 = __ldg(row + s.xo[1]), t2 = __ldg(row + s.xo[2]),
                        t3 = __ldg(row + s.xo[3]);
            const float xv = s.wx[0] * t0 + s.wx[1] * t1 + s.wx[2] * t2 + s.wx[3] * t3;
            const float xd = dwx[0] * t0 + dwx[1] * t1 + dwx[2] * t2 + dwx[3] * t3;
            pv += s.wy[b] * xv;
            px += s.wy[b] * xd;
            py += dwy[b] * xv;
        }
        val += s.wz[c] * pv;
        gx += s.wz[c] * px;
        gy += s.wz[c] * py;
        gz += dwz[c] * pv;
    }
    long long imn = s.c0, imx = s.c0;
    float mn = __ldg(img + s.c0), mx = mn;
    const int off[7] = {s.sx1, s.sx1 + s.sy1, s.sy1, s.sz1, s.sx1 + s.sz1, s.sx1 + s.sy1 + s.sz1,
                        s.sy1 + s.sz1};
#pragma unroll
    for (int k = 0; k < 7; ++k) {
        float v = __ldg(img + s.c0 + off[k]);
        if (v < mn) { mn = v; imn = s.c0 + off[k]; }
        if (mx < v) { mx = v; imx = s.c0 + off[k]; }
    }
    r.grad[0] = r.grad[1] = r.grad[2] = 0.0f;
    if (val > mx) {
        r.value = mx; r.branch = 1; r.corner = imx;
    } else if (val < mn) {
        r.value = mn; r.branch = 2; r.corner = imn;
    } else {
        r.value = val; r.branch = 0; r.corner = -1;
        r.grad[0] = clamped[0] ? 0.0f : gx;
        r.grad[1] = clamped[1] ? 0.0f : gy;
        r.grad[2] = clamped[2] ? 0.0f : gz;
    }
}

__device__ __forceinline__ void scatter_sample(float *__restrict__ bar, const Stencil &s,
                                               const SampleD &r, float g) {
    if (g == 0.0f) return;
    if (r.branch != 0) {
        atomicAdd(bar + r.corner, g);
        return;
    }
#pragma unroll 1
    for (int c = 0; c < 4; ++c)
#pragma unroll
        for (int b = 0; b < 4; ++b) {
            float wbc = g * s.wy[b] * s.wz[c];
            float *row = bar + s.yo[b] + s.zo[c];
#pragma unroll
            for (int a = 0; a < 4; ++a) {
                float w = s.wx[a] * wbc;
                if (w != 0.0f) atomicAdd(row + s.xo[a], w);
            }
        }
}

// q = p + (h/2) v(p) + (h/2) v(p2), p2 = p + h v(p).  Reverse mode:
//   out_c = S(src_c, q)        -> src_bar, q_bar
//   q_bar -> v2_bar = (h/2) q_bar;  p2_bar = q_bar/2 + J_v(p2)^T v2_bar
//   v1_bar = (h/2) q_bar' ... folded: v1_bar = h * p2_bar (p2 = p + h v1)
// The centre read v(p) is an exact node value, so its adjoint is a single add.
__global__ void __launch_bounds__(128) k_warp_vjp(const Dim3i d, const float *__restrict__ vel,
                                                  const float *__restrict__ src, int nc, float dt,
                                                  const float *__restrict__ out_bar,
                                                  float *__restrict__ src_bar,
                                                  float *__restrict__ vel_bar) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y, k = blockIdx.z;
    if (i >= d.x) return;
    const size_t n = (size_t)d.x * d.y * d.z;
    const float h = -dt;
    float q[3], p2[3], v1[3], v2[3];
    trace(d, vel, n, i, j, k, h, q, p2, v1, v2);
    bool cq[3];
    float gq[3] = {to_grid(q[0], d.x, &cq[0]), to_grid(q[1], d.y, &cq[1]), to_grid(q[2], d.z, &cq[2])};
    Stencil sq;
    make_stencil(d, gq, sq);
    const size_t o = i + (size_t)j * d.x + (size_t)k * d.x * d.y;
    float qbar[3] = {0.0f, 0.0f, 0.0f};
    for (int c = 0; c < nc; ++c) {
        const float ob = __ldg(out_bar + o + c * n);
        if (ob == 0.0f) continue;
        SampleD r;
        sample_d(src + c * n, sq, cq, r);
        if (src_bar) scatter_sample(src_bar + c * n, sq, r, ob);
        qbar[0] += ob * r.grad[0];
        qbar[1] += ob * r.grad[1];
        qbar[2] += ob * r.grad[2];
    }
    if (!vel_bar) return;
    if (qbar[0] == 0.0f && qbar[1] == 0.0f && qbar[2] == 0.0f) return;
    bool c2[3];
    float g2[3] = {to_grid(p2[0], d.x, &c2[0]), to_grid(p2[1], d.y, &c2[1]), to_grid(p2[2], d.z, &c2[2])};
    Stencil s2;
    make_stencil(d, g2, s2);
    float v2bar[3], p2bar[3] = {0.5f * qbar[0], 0.5f * qbar[1], 0.5f * qbar[2]};
#pragma unroll
    for (int a = 0; a < 3; ++a) v2bar[a] = 0.5f * h * qbar[a];
#pragma unroll 1
    for (int a = 0; a < 3; ++a) {
        SampleD r;
        sample_d(vel + a * n, s2, c2, r);
        scatter_sample(vel_bar + a * n, s2, r, v2bar[a]);
        p2bar[0] += v2bar[a] * r.grad[0];
        p2bar[1] += v2bar[a] * r.grad[1];
        p2bar[2] += v2bar[a] * r.grad[2];
    }
    const int ci = min(max(i, 1), d.x - 2), cj = min(max(j, 1), d.y - 2), ck = min(max(k, 1), d.z - 2);
    const size_t cc = ci + (size_t)cj * d.x + (size_t)ck * d.x * d.y;
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        float g = h * p2bar[a];
        if (g != 0.0f) atomicAdd(vel_bar + a * n + cc, g);
    }
}

}  // namespace

cudaError_t warp_poll_status(int *flag, cudaStream_t s) {
    *flag = 0;
    cudaError_t e = cudaMemcpyFromSymbolAsync(flag, g_warp_wait_status, sizeof(int), 0, cudaMemcpyDeviceToHost, s);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    if (e == cudaSuccess && *flag) {
        const int zero = 0;
        e = cudaMemcpyToSymbolAsync(g_warp_wait_status, &zero, sizeof(int), 0, cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
    }
    return e;
}

namespace {
template <typename T>
cudaError_t warp_any(const int *dim, const float *vel, const T *src, int nc, float dt, float *out, cudaStream_t s,
                     int *status) {
    Dim3i d{dim[0], dim[1], dim[2]};
    const dim3 grid((d.x + WARP_BX - 1) / WARP_BX, (d.y + WARP_BY - 1) / WARP_BY, d.z), block(WARP_BX, WARP_BY);
    CUtensorMap vmap;
    const unsigned box[4] = {VX, VY, VZ, 3};
    if (encode_planes_map(&vmap, vel, d.x, d.y, d.z, 3, box))
        k_warp_staged<T><<<grid, block, 0, s>>>(d, vmap, vel, src, nc, dt, out, status);
    else
        k_warp<T><<<grid, block, 0, s>>>(d, vel, src, nc, dt, out);
    return cudaGetLastError();
}
}  // namespace

cudaError_t launch_warp(const int *dim, const float *vel, const float *src, int nc, float dt,
                        float *out, cudaStream_t s, int *status) {
    return warp_any(dim, vel, src, nc, dt, out, s, status);
}

cudaError_t launch_warp(const int *dim, const float *vel, const unsigned short *src, int nc, float dt,
                        float *out, cudaStream_t s, int *status) {
    return warp_any(dim, vel, src, nc, dt, out, s, status);
}

cudaError_t launch_warp_vjp(const int *dim, const float *vel, const float *src, int nc, float dt,
                            const float *out_bar, float *src_bar, float *vel_bar, cudaStream_t s) {
    Dim3i d{dim[0], dim[1], dim[2]};
    k_warp_vjp<<<dim3((d.x + 127) / 128, d.y, d.z), 128, 0, s>>>(d, vel, src, nc, dt, out_bar,
                                                                  src_bar, vel_bar);
    return cudaGetLastError();
}

}  // namespace stt
