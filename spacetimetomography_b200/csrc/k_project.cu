// k_project.cu -- ray-driven kernels: forward projection, forward projection
// fused with the SART correction, the ray-driven backprojection scatter and
// the exact adjoint A^T.
//
// One thread per detector pixel.  A 128-thread block covers a 16x8 pixel
// tile; each warp covers an 8x4 sub-tile so that the 32 rays of a warp stay
// close together in the volume and their trilinear gathers share L1 lines.
// The volume is read through the read-only path (ld.global.nc); at the sizes
// of the headline workloads (256^3 fp32 = 64 MiB) it stays resident in the
// 126 MB L2.
#include "stt_internal.cuh"
#include "stt_kernels.h"

namespace stt {

namespace {

__device__ __forceinline__ bool tile_pixel(const GeomDev &g, int &i, int &j) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    i = blockIdx.x * 16 + (w & 1) * 8 + (lane & 7);
    j = blockIdx.y * 8 + (w >> 1) * 4 + (lane >> 3);
    return i < g.W && j < g.H;
}

// GenerateImage_MT (S/ImageFormationModel/TypicalRayProducer.core.h:168-224)
// for views [view0, view0 + gridDim.z).
__global__ void __launch_bounds__(128) k_fp(const GeomDev g, const ViewRec *__restrict__ views,
                                            const float *__restrict__ vol, int view0,
                                            float *__restrict__ proj, float *__restrict__ raylen,
                                            float *__restrict__ weight) {
    int i, j;
    if (!tile_pixel(g, i, j)) return;
    const int v = blockIdx.z;
    Ray r;
    make_ray(g, views[view0 + v], i, j, r);
    Kahan acc{0.0f, 0.0f};
    int count = 0;
    const bool hit = r.tnear < r.tfar;
    if (hit) {
        march(g, r, [&](const float p[3]) {
            Taps t;
            make_taps(g, p, t);
            acc.add(tri_value(vol, t) * g.sd);
            ++count;
        });
    }
    const size_t o = (size_t)v * g.W * g.H + i + (size_t)j * g.W;
    proj[o] = acc.s;
    if (raylen && hit) raylen[o] = r.tfar - r.tnear;
    if (weight) weight[o] = (float)count;
}

// Forward projection of one view with the SART correction as epilogue
// (ST_Tomography.cpp:667-676; Factor = 1 and pY == 0 in the reference, so
// c = (b - Ax) / (L + 1)).  L is the sticky ray length of the producer:
// updated where the ray hits, kept where it misses; with no state buffer
// (ray-based SART, whose producer is reset after every view) a miss gives L = 0.
__global__ void __launch_bounds__(128) k_fp_corr(const GeomDev g, const ViewRec *__restrict__ views,
                                                 const float *__restrict__ vol, const ViewSel sel,
                                                 const float *__restrict__ b_stack,
                                                 float *__restrict__ raylen_state,
                                                 float *__restrict__ corr) {
    int i, j;
    if (!tile_pixel(g, i, j)) return;
    int local;
    const int view = sel_view(sel, local);
    const float *b = b_stack + (size_t)local * g.W * g.H;
    Ray r;
    make_ray(g, views[view], i, j, r);
    Kahan acc{0.0f, 0.0f};
    const size_t pix = i + (size_t)j * g.W;
    float L;
    if (r.tnear < r.tfar) {
        march(g, r, [&](const float p[3]) {
            Taps t;
            make_taps(g, p, t);
            acc.add(tri_value(vol, t) * g.sd);
        });
        L = r.tfar - r.tnear;
        if (raylen_state) raylen_state[pix] = L;
    } else {
        L = raylen_state ? raylen_state[pix] : 0.0f;
    }
    corr[pix] = __fdiv_rn(__fsub_rn(__ldg(b + pix), acc.s), __fadd_rn(L, 1.0f));
}

// BP-mode march (SingleScalarVolume.core.h:128-143, UpdateContributionSum
// :73-84): every sample scatters (c*w_k, w_k) into the interleaved
// accumulator of its 8 clamped corners with one vector atomic each.
__global__ void __launch_bounds__(128) k_bp_ray_scatter(const GeomDev g,
                                                        const ViewRec *__restrict__ views,
                                                        const ViewSel sel,
                                                        const float *__restrict__ corr,
                                                        float2 *__restrict__ acc) {
    int i, j;
    if (!tile_pixel(g, i, j)) return;
    int local;
    const int view = sel_view(sel, local);
    Ray r;
    make_ray(g, views[view], i, j, r);
    if (!(r.tnear < r.tfar)) return;
    const float c = __ldg(corr + i + (size_t)j * g.W);
    march(g, r, [&](const float p[3]) {
        Taps t;
        make_taps(g, p, t);
        float w[8];
        tri_weights(t, w);
#pragma unroll
        for (int k = 0; k < 8; ++k) atomicAdd(acc + tap_index(t, k), make_float2(c * w[k], w[k]));
    });
}

// Exact adjoint of k_fp: vol_bar[corner] += sd * w_k * y for every sample,
// the entry sample twice, clamped corners collapsing as in the forward pass.
__global__ void __launch_bounds__(128) k_fp_adjoint(const GeomDev g, const ViewRec *__restrict__ views,
                                                    int view0, const float *__restrict__ proj_bar,
                                                    float *__restrict__ vol_bar) {
    int i, j;
    if (!tile_pixel(g, i, j)) return;
    const int v = blockIdx.z;
    const float y = __ldg(proj_bar + (size_t)v * g.W * g.H + i + (size_t)j * g.W);
    if (y == 0.0f) return;
    Ray r;
    make_ray(g, views[view0 + v], i, j, r);
    if (!(r.tnear < r.tfar)) return;
    const float ys = y * g.sd;
    march(g, r, [&](const float p[3]) {
        Taps t;
        make_taps(g, p, t);
        float w[8];
        tri_weights(t, w);
#pragma unroll
        for (int k = 0; k < 8; ++k) atomicAdd(vol_bar + tap_index(t, k), ys * w[k]);
    });
}

// Ray-BP normalisation (ST_Tomography.cpp:746-762): vol += contrib/weight,
// clamped with the reference macros so 0/0 = NaN becomes 0; the accumulator
// is reset for the next view (TypicalRayProducer::Initial, TypicalRayProducer.cpp:91-95).
__global__ void k_bp_ray_update(long long n, float2 *__restrict__ acc, float *__restrict__ vol,
                                float gmax) {
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n;
         k += (long long)gridDim.x * blockDim.x) {
        float2 a = acc[k];
        float v = vol[k] + __fdiv_rn(a.x, a.y);
        vol[k] = rmax(rmin(gmax, v), 0.0f);
        acc[k] = make_float2(0.0f, 0.0f);
    }
}

// Stand-alone SART correction (ST_Tomography.cpp:667-676) for the unfused
// per-view form: the ray lengths are the sticky state k_fp updated on hits.
__global__ void k_correction(long long n, const float *__restrict__ b, const float *__restrict__ ax,
                             const float *__restrict__ raylen, float *__restrict__ corr) {
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n;
         k += (long long)gridDim.x * blockDim.x)
        corr[k] = __fdiv_rn(__fsub_rn(b[k], ax[k]), __fadd_rn(raylen ? raylen[k] : 0.0f, 1.0f));
}

__global__ void k_fill_zero(long long n, float *__restrict__ p) {
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n;
         k += (long long)gridDim.x * blockDim.x)
        p[k] = 0.0f;
}

dim3 ray_grid(const GeomDev &g, int nviews) {
    return dim3((g.W + 15) / 16, (g.H + 7) / 8, nviews);
}

}  // namespace

int grid_stride_blocks(long long n, int threads) {
    long long b = (n + threads - 1) / threads;
    const long long cap = 148LL * 16;  // 16 resident 256-thread blocks per SM on 148 SMs
    return (int)(b < cap ? (b < 1 ? 1 : b) : cap);
}

cudaError_t launch_fp(const GeomDev &g, const ViewRec *views, const float *vol, int view0,
                      int nviews, float *proj, float *raylen, float *weight, cudaStream_t s) {
    k_fp<<<ray_grid(g, nviews), 128, 0, s>>>(g, views, vol, view0, proj, raylen, weight);
    return cudaGetLastError();
}

cudaError_t launch_fp_corr(const GeomDev &g, const ViewRec *views, const float *vol, const ViewSel &sel,
                           const float *b_stack, float *raylen_state, float *corr, cudaStream_t s) {
    k_fp_corr<<<ray_grid(g, 1), 128, 0, s>>>(g, views, vol, sel, b_stack, raylen_state, corr);
    return cudaGetLastError();
}

cudaError_t launch_correction(long long n, const float *b, const float *ax, const float *raylen,
                              float *corr, cudaStream_t s) {
    k_correction<<<grid_stride_blocks(n, 256), 256, 0, s>>>(n, b, ax, raylen, corr);
    return cudaGetLastError();
}

cudaError_t launch_bp_ray(const GeomDev &g, const ViewRec *views, const ViewSel &sel, const float *corr,
                          float2 *acc, float *vol, float gmax, cudaStream_t s) {
    k_bp_ray_scatter<<<ray_grid(g, 1), 128, 0, s>>>(g, views, sel, corr, acc);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    const long long n = (long long)g.nx * g.ny * g.nz;
    k_bp_ray_update<<<grid_stride_blocks(n, 256), 256, 0, s>>>(n, acc, vol, gmax);
    return cudaGetLastError();
}

cudaError_t launch_fp_adjoint(const GeomDev &g, const ViewRec *views, int view0, int nviews,
                              const float *proj_bar, float *vol_bar, cudaStream_t s) {
    k_fp_adjoint<<<ray_grid(g, nviews), 128, 0, s>>>(g, views, view0, proj_bar, vol_bar);
    return cudaGetLastError();
}

cudaError_t launch_fill_zero(float *p, long long n, cudaStream_t s) {
    k_fill_zero<<<grid_stride_blocks(n, 256), 256, 0, s>>>(n, p);
    return cudaGetLastError();
}

}  // namespace stt
