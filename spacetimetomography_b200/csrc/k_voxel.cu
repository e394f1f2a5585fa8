// k_voxel.cu -- voxel-driven kernels: the voxel-based (gather) backprojector,
// the primal-dual dual/primal/over-relaxation steps and the ROI mask.
//
// All of these stream the volume once in x-fastest order: one thread per
// voxel along x, blocks of 128 threads, grid (ceil(nx/128), ny, nz), so every
// warp reads and writes 128 contiguous bytes per array.  The stencil
// neighbours (x+-1, y+-1, z+-1) come from L1/L2.
#include "stt_internal.cuh"
#include "stt_kernels.h"

namespace stt {

namespace {

// ROI box of the primal-dual loops (ST_Tomography.cpp:514, 565, 593).
__device__ __forceinline__ bool roi_out(int i, int j, int k, int nx, int ny, int nz, const int *cut) {
    return i < cut[0] || i > nx - cut[1] || j < cut[2] || j > ny - cut[3] || k < cut[4] ||
           k > nz - cut[5];
}

// ROI mask (ST_Tomography.cpp:303-329); note the literal 7 in the y test of :324.
__device__ __forceinline__ float roi_value(int i, int j, int k, int nx, int ny, int nz, const int *cut) {
    float r = 1.0f;
    if (((i < cut[6]) && (k < cut[7])) || ((i < cut[6]) && (k > (nz - cut[7])))) r = 0.0f;
    if (((i > (nx - cut[6])) && (k < cut[7])) || ((i > (nx - cut[6])) && (k > (nz - cut[7])))) r = 0.0f;
    if (((k < cut[6]) && (i < cut[7])) || ((k < cut[6]) && (i > (nx - cut[7])))) r = 0.0f;
    if (((k > (nz - cut[6])) && (i < cut[7])) || ((k > (nz - cut[6])) && (i > (nx - cut[7])))) r = 0.0f;
    if (i < cut[0] || i > nx - cut[1] || j < cut[2] || j > ny - 7 || k < cut[4] || k > nz - cut[5]) r = 0.0f;
    return r;
}

struct Cut8 {
    int c[8];
};

// Voxel-based backprojection (ST_Tomography.cpp:690-730): project the voxel
// centre, Catmull-Rom 4x4 gather of the correction image (y first, then x),
// vol += alpha*val, clamp to [0, gmax]; voxels whose footprint leaves
// [2, W-2) x [2, H-2) are untouched.  With TEX the 16 taps come from four
// tld4 gathers of the correction's one-layer texture copy (one request per
// 2x2 texels instead of one per texel); the values and the arithmetic are
// the same.
template <bool TEX>
__global__ void __launch_bounds__(128) k_bp_voxel(const GeomDev g, const ViewRec *__restrict__ views,
                                                  const ViewSel sel, const float *__restrict__ corr,
                                                  float *__restrict__ vol, float alpha, float gmax,
                                                  unsigned long long corr_tex) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y, z = blockIdx.z;
    if (x >= g.nx) return;
    int local;
    const ViewRec &v = views[sel_view(sel, local)];
    const float fx = (float)x, fy = (float)y, fz = (float)z;
    const float cxm = v.A[0] * fx + v.A[1] * fy + v.A[2] * fz + v.b[0];
    const float cym = v.A[3] * fx + v.A[4] * fy + v.A[5] * fz + v.b[1];
    const float czm = v.A[6] * fx + v.A[7] * fy + v.A[8] * fz + v.b[2];
    const float upx = g.cx + __fdiv_rn(cxm, -czm) * g.sdd_ds;
    const float upy = g.cy + __fdiv_rn(cym, -czm) * g.sdd_ds;
    if (!(upx >= 2.0f && upx < (float)(g.W - 2) && upy >= 2.0f && upy < (float)(g.H - 2))) return;
    const int px = (int)upx, py = (int)upy;
    float wx[4], wy[4];
    cr_weights(upx - (float)px, wx);
    cr_weights(upy - (float)py, wy);
    float tap[4][4];  // tap[a][b]: column px-1+a, row py-1+b
    if (TEX) {
        const float4 g00 = gather_layer(corr_tex, px - 1, py - 1, 0), g10 = gather_layer(corr_tex, px + 1, py - 1, 0);
        const float4 g01 = gather_layer(corr_tex, px - 1, py + 1, 0), g11 = gather_layer(corr_tex, px + 1, py + 1, 0);
        tap[0][0] = g00.w, tap[0][1] = g00.x, tap[0][2] = g01.w, tap[0][3] = g01.x;
        tap[1][0] = g00.z, tap[1][1] = g00.y, tap[1][2] = g01.z, tap[1][3] = g01.y;
        tap[2][0] = g10.w, tap[2][1] = g10.x, tap[2][2] = g11.w, tap[2][3] = g11.x;
        tap[3][0] = g10.z, tap[3][1] = g10.y, tap[3][2] = g11.z, tap[3][3] = g11.y;
    } else {
        const float *c0 = corr + (size_t)(py - 1) * g.W + (px - 1);
#pragma unroll
        for (int a = 0; a < 4; ++a)
#pragma unroll
            for (int b = 0; b < 4; ++b) tap[a][b] = __ldg(c0 + a + b * g.W);
    }
    float val = 0.0f;
#pragma unroll
    for (int a = 0; a < 4; ++a) {
        float s = wy[0] * tap[a][0] + wy[1] * tap[a][1] + wy[2] * tap[a][2] + wy[3] * tap[a][3];
        val += wx[a] * s;
    }
    const size_t o = x + (size_t)y * g.nx + (size_t)z * g.nx * g.ny;
    float nv = vol[o] + alpha * val;
    vol[o] = rmax(rmin(gmax, nv), 0.0f);
}

// Dual step of one frame (ST_Tomography.cpp:504-534), fused:
//   whole volume:     ytp += sigma*(xf1 - xf);  ybc += sigma*(bw - xf)
//   interior & ROI:   ytv_c += sigma*(xf(p+e_c) - xf(p))*hf, clamp +-tv_w;
//                     ytp = ytp*tp_w/(tp_w + 2 sigma);  ybc clamp +-bc_w
__global__ void __launch_bounds__(128) k_pd_dual(int nx, int ny, int nz, float sigma, float tv_w,
                                                 float tp_w, float bc_w, float hf, Cut8 cut,
                                                 const float *__restrict__ xf,
                                                 const float *__restrict__ xf1,
                                                 const float *__restrict__ bw, float *__restrict__ ytv,
                                                 float *__restrict__ ytp, float *__restrict__ ybc) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y, k = blockIdx.z;
    if (i >= nx) return;
    const size_t sy = nx, sz = (size_t)nx * ny, n = sz * nz;
    const size_t p = i + j * sy + k * sz;
    const float x0 = __ldg(xf + p);
    float tp = ytp[p] + sigma * (__ldg(xf1 + p) - x0);
    float bc = ybc[p] + sigma * (__ldg(bw + p) - x0);
    const bool inner = i >= 1 && i < nx - 1 && j >= 1 && j < ny - 1 && k >= 1 && k < nz - 1 &&
                       !roi_out(i, j, k, nx, ny, nz, cut.c);
    if (inner) {
        float y0 = ytv[p] + sigma * (__ldg(xf + p + 1) - x0) * hf;
        float y1 = ytv[p + n] + sigma * (__ldg(xf + p + sy) - x0) * hf;
        float y2 = ytv[p + 2 * n] + sigma * (__ldg(xf + p + sz) - x0) * hf;
        ytv[p] = rmax(-tv_w, rmin(tv_w, y0));
        ytv[p + n] = rmax(-tv_w, rmin(tv_w, y1));
        ytv[p + 2 * n] = rmax(-tv_w, rmin(tv_w, y2));
        tp = __fdiv_rn(tp * tp_w, tp_w + 2.0f * sigma);
        bc = rmax(-bc_w, rmin(bc_w, bc));
    }
    ytp[p] = tp;
    ybc[p] = bc;
}

// Primal step of one frame (ST_Tomography.cpp:536-578), fused: xprev = vol;
// vol -= tau*(-ytp); vol -= tau*(-ybc) for the first frame, otherwise
// vol -= tau*(ytp_prev - ytp); vol -= tau*(fw - ybc); then on the interior
// ROI vol -= tau*(-div ytv) and clamp to [0, gmax].
__global__ void __launch_bounds__(128) k_pd_primal(int nx, int ny, int nz, float tau, float gmax,
                                                   Cut8 cut, int first,
                                                   const float *__restrict__ ytp_prev,
                                                   const float *__restrict__ ytp,
                                                   const float *__restrict__ fw,
                                                   const float *__restrict__ ybc,
                                                   const float *__restrict__ ytv,
                                                   float *__restrict__ vol, float *__restrict__ xprev) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y, k = blockIdx.z;
    if (i >= nx) return;
    const size_t sy = nx, sz = (size_t)nx * ny, n = sz * nz;
    const size_t p = i + j * sy + k * sz;
    float v = vol[p];
    xprev[p] = v;
    if (first) {
        v = v - tau * (-__ldg(ytp + p));
        v = v - tau * (-__ldg(ybc + p));
    } else {
        v = v - tau * (__ldg(ytp_prev + p) - __ldg(ytp + p));
        v = v - tau * (__ldg(fw + p) - __ldg(ybc + p));
    }
    const bool inner = i >= 1 && i < nx - 1 && j >= 1 && j < ny - 1 && k >= 1 && k < nz - 1 &&
                       !roi_out(i, j, k, nx, ny, nz, cut.c);
    if (inner) {
        const float *y0 = ytv, *y1 = ytv + n, *y2 = ytv + 2 * n;
        float y = -(__ldg(y0 + p) - __ldg(y0 + p - 1) + __ldg(y1 + p) - __ldg(y1 + p - sy) +
                    __ldg(y2 + p) - __ldg(y2 + p - sz));
        v = v - tau * y;
        v = rmax(rmin(gmax, v), 0.0f);
    }
    vol[p] = v;
}

// Over-relaxation (ST_Tomography.cpp:586-604): xbar = 2*vol - xprev in the ROI box.
__global__ void __launch_bounds__(128) k_pd_extrapolate(int nx, int ny, int nz, Cut8 cut,
                                                        const float *__restrict__ vol,
                                                        const float *__restrict__ xprev,
                                                        float *__restrict__ xbar) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y, k = blockIdx.z;
    if (i >= nx || roi_out(i, j, k, nx, ny, nz, cut.c)) return;
    const size_t p = i + (size_t)j * nx + (size_t)k * nx * ny;
    xbar[p] = 2.0f * __ldg(vol + p) - __ldg(xprev + p);
}

// End of a SART call (ST_Tomography.cpp:793-804) optionally fused with the
// over-relaxation that follows it in the primal-dual loop (:586-604):
// vol *= roi; if xbar: xbar = 2*vol - xprev in the ROI box.
__global__ void __launch_bounds__(128) k_roi_apply(int nx, int ny, int nz, Cut8 cut, Cut8 pdcut,
                                                   float *__restrict__ vol,
                                                   const float *__restrict__ xprev,
                                                   float *__restrict__ xbar) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y, k = blockIdx.z;
    if (i >= nx) return;
    const size_t p = i + (size_t)j * nx + (size_t)k * nx * ny;
    float v = vol[p] * roi_value(i, j, k, nx, ny, nz, cut.c);
    vol[p] = v;
    if (xbar && !roi_out(i, j, k, nx, ny, nz, pdcut.c)) xbar[p] = 2.0f * v - __ldg(xprev + p);
}

__global__ void __launch_bounds__(128) k_roi_mask(int nx, int ny, int nz, Cut8 cut, float *__restrict__ roi) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y, k = blockIdx.z;
    if (i >= nx) return;
    roi[i + (size_t)j * nx + (size_t)k * nx * ny] = roi_value(i, j, k, nx, ny, nz, cut.c);
}

// ---- FP64 helpers of the power iteration --------------------------------------
// out[0] += sum a*b (FP64 products and sums; one double atomic per block).
__global__ void __launch_bounds__(256) k_dot_f64(long long n, const float *__restrict__ a,
                                                 const float *__restrict__ b, double *__restrict__ out) {
    double s = 0.0;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x)
        s += (double)__ldg(a + k) * (double)__ldg(b + k);
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    __shared__ double part[8];
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) t += part[w];
        atomicAdd(out, t);
    }
}

// x *= 1/sqrt(*norm2) (the factor formed in FP64); x = 0 when the norm is 0.
__global__ void __launch_bounds__(256) k_scale_inv_sqrt(long long n, float *__restrict__ x,
                                                        const double *__restrict__ norm2) {
    const double q = *norm2;
    const float f = q > 0.0 ? (float)(1.0 / sqrt(q)) : 0.0f;
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n; k += (long long)gridDim.x * blockDim.x)
        x[k] *= f;
}

// Seeded start vector: uniform in [0.5, 1.5) from SplitMix64 of (seed, index).
__global__ void __launch_bounds__(256) k_fill_seeded(long long n, unsigned long long seed, float *__restrict__ x) {
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n;
         k += (long long)gridDim.x * blockDim.x) {
        unsigned long long z = seed + 0x9E3779B97F4A7C15ULL * (unsigned long long)(k + 1);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
        z ^= z >> 31;
        x[k] = 0.5f + (float)(z >> 40) * (1.0f / 16777216.0f);
    }
}

dim3 vox_grid(int nx, int ny, int nz) { return dim3((nx + 127) / 128, ny, nz); }

Cut8 to_cut(const int *c) {
    Cut8 r;
    for (int q = 0; q < 8; ++q) r.c[q] = c ? c[q] : 0;
    return r;
}

}  // namespace

cudaError_t launch_dot_f64(long long n, const float *a, const float *b, double *out, cudaStream_t s) {
    k_dot_f64<<<grid_stride_blocks(n, 256), 256, 0, s>>>(n, a, b, out);
    return cudaGetLastError();
}

cudaError_t launch_scale_inv_sqrt(long long n, float *x, const double *norm2, cudaStream_t s) {
    k_scale_inv_sqrt<<<grid_stride_blocks(n, 256), 256, 0, s>>>(n, x, norm2);
    return cudaGetLastError();
}

cudaError_t launch_fill_seeded(long long n, unsigned long long seed, float *x, cudaStream_t s) {
    k_fill_seeded<<<grid_stride_blocks(n, 256), 256, 0, s>>>(n, seed, x);
    return cudaGetLastError();
}

cudaError_t launch_bp_voxel(const GeomDev &g, const ViewRec *views, const ViewSel &sel, const float *corr,
                            float *vol, float alpha, float gmax, cudaStream_t s, unsigned long long corr_tex) {
    if (corr_tex)
        k_bp_voxel<true><<<vox_grid(g.nx, g.ny, g.nz), 128, 0, s>>>(g, views, sel, corr, vol, alpha, gmax, corr_tex);
    else
        k_bp_voxel<false><<<vox_grid(g.nx, g.ny, g.nz), 128, 0, s>>>(g, views, sel, corr, vol, alpha, gmax, 0);
    return cudaGetLastError();
}

cudaError_t launch_pd_dual(const int *d, const PdParams &p, const float *xf, const float *xf1,
                           const float *bw, float *ytv, float *ytp, float *ybc, cudaStream_t s) {
    k_pd_dual<<<vox_grid(d[0], d[1], d[2]), 128, 0, s>>>(d[0], d[1], d[2], p.sigma, p.tv_w, p.tp_w,
                                                         p.bc_w, p.hf, to_cut(p.cut), xf, xf1, bw,
                                                         ytv, ytp, ybc);
    return cudaGetLastError();
}

cudaError_t launch_pd_primal(const int *d, const PdParams &p, int first, const float *ytp_prev,
                             const float *ytp, const float *fw, const float *ybc, const float *ytv,
                             float *vol, float *xprev, cudaStream_t s) {
    k_pd_primal<<<vox_grid(d[0], d[1], d[2]), 128, 0, s>>>(d[0], d[1], d[2], p.tau, p.gmax,
                                                           to_cut(p.cut), first, ytp_prev, ytp, fw,
                                                           ybc, ytv, vol, xprev);
    return cudaGetLastError();
}

cudaError_t launch_pd_extrapolate(const int *d, const int *cut, const float *vol, const float *xprev,
                                  float *xbar, cudaStream_t s) {
    k_pd_extrapolate<<<vox_grid(d[0], d[1], d[2]), 128, 0, s>>>(d[0], d[1], d[2], to_cut(cut), vol,
                                                                xprev, xbar);
    return cudaGetLastError();
}

cudaError_t launch_roi_apply(const int *d, const int *roi_cut, const int *pd_cut, float *vol,
                             const float *xprev, float *xbar, cudaStream_t s) {
    k_roi_apply<<<vox_grid(d[0], d[1], d[2]), 128, 0, s>>>(d[0], d[1], d[2], to_cut(roi_cut),
                                                           to_cut(pd_cut), vol, xprev, xbar);
    return cudaGetLastError();
}

cudaError_t launch_roi_mask(const int *d, const int *cut, float *roi, cudaStream_t s) {
    k_roi_mask<<<vox_grid(d[0], d[1], d[2]), 128, 0, s>>>(d[0], d[1], d[2], to_cut(cut), roi);
    return cudaGetLastError();
}

}  // namespace stt
