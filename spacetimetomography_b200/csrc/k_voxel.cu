// k_voxel.cu -- voxel-driven kernels: the voxel-based (gather) backprojector,
// the primal-dual dual/primal/over-relaxation steps and the ROI mask.
//
// All of these stream the volume once in x-fastest order: one thread per
// voxel along x, blocks of 128 threads, grid (ceil(nx/128), ny, nz), so every
// warp reads and writes 128 contiguous bytes per array.  The stencil
// neighbours (x+-1, y+-1, z+-1) come from L1/L2.
#include "stt_internal.cuh"
#include "stt_kernels.h"
#include "stt_voxel.cuh"

namespace stt {

namespace {

template <bool TEX, typename T>
__global__ void __launch_bounds__(128) k_bp_voxel(const GeomDev g, const ViewRec *__restrict__ views,
                                                  const ViewSel sel, const float *__restrict__ corr,
                                                  T *__restrict__ vol, float alpha, float gmax,
                                                  unsigned long long corr_tex) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    if (x >= g.nx) return;
    int local;
    const ViewRec &v = views[sel_view(sel, local)];
    if (TEX)
        bp_voxel_at(g, v, BpRowsTex{corr_tex}, vol, x, blockIdx.y, blockIdx.z, alpha, gmax);
    else
        bp_voxel_at(g, v, BpRowsLdg{corr, g.W}, vol, x, blockIdx.y, blockIdx.z, alpha, gmax);
}

// Column form, texture taps (bp_column in stt_voxel.cuh): one thread per
// (x, z) walks K voxels up y.  Column length K: 16 by default; the autotuner
// may pick 8 or 32 (the voxels' values do not depend on which thread walks
// them).
constexpr int BP_COL = 16;

// Ten 128-thread blocks per SM (48 registers, no spills): the walk is bound
// by texture latency, so the extra warps pay (10 blocks: 104.1 ms per
// iteration of the 10 x 256^3 solve against 106.6 ms with the compiler's
// 52 registers and 9 blocks).
//
// PF: before the walk, every thread asks L2 for its column's K voxels
// (prefetch.global.L2: no register, no scoreboard).  Where the volume does not
// fit in L2 (512^3 FP32 is 512 MiB against 126 MB), the walk's one load per
// voxel otherwise waits for HBM with a single load in flight per thread, and
// ten blocks of them keep too few bytes in flight to cover HBM latency.  The
// values read, and so the bits written, are the same.
template <int K = BP_COL, typename T = float, bool PF = false>
__global__ void __launch_bounds__(128, 10) k_bp_voxel_cols(const GeomDev g, const ViewRec *__restrict__ views,
                                                       const ViewSel sel, T *__restrict__ vol, float alpha,
                                                       float gmax, unsigned long long tex) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    if (x >= g.nx) return;
    int local;
    const ViewRec &v = views[sel_view(sel, local)];
    bp_column<K, PF>(g, v, BpRowsTex{tex}, vol, x, blockIdx.y * K, blockIdx.z, alpha, gmax);
}

// The dual and primal steps of one frame (pd_dual_at, pd_primal_at in
// stt_voxel.cuh), one thread per voxel.
template <typename T>
__global__ void __launch_bounds__(128) k_pd_dual(int nx, int ny, int nz, float sigma, float tv_w,
                                                 float tp_w, float bc_w, float hf, Cut8 cut,
                                                 const T *__restrict__ xf,
                                                 const T *__restrict__ xf1,
                                                 const float *__restrict__ bw, float *__restrict__ ytv,
                                                 float *__restrict__ ytp, float *__restrict__ ybc) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y, k = blockIdx.z;
    if (i >= nx) return;
    const size_t p = i + (size_t)j * nx + (size_t)k * nx * ny;
    pd_dual_at(i, j, k, nx, ny, nz, sigma, tv_w, tp_w, bc_w, hf, cut.c, xf, xf1, __ldg(bw + p), ytv, ytp, ybc);
}

template <typename T>
__global__ void __launch_bounds__(128) k_pd_primal(int nx, int ny, int nz, float tau, float gmax,
                                                   Cut8 cut, int first,
                                                   const float *__restrict__ ytp_prev,
                                                   const float *__restrict__ ytp,
                                                   const float *__restrict__ fw,
                                                   const float *__restrict__ ybc,
                                                   const float *__restrict__ ytv,
                                                   T *__restrict__ vol, T *__restrict__ xprev) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y, k = blockIdx.z;
    if (i >= nx) return;
    const size_t p = i + (size_t)j * nx + (size_t)k * nx * ny;
    pd_primal_at<false>(i, j, k, nx, ny, nz, tau, gmax, cut.c, first, ytp_prev, ytp, first ? 0.0f : __ldg(fw + p),
                        ybc, ytv, vol, xprev);
}

// Over-relaxation (ST_Tomography.cpp:586-604): xbar = 2*vol - xprev in the ROI box.
template <typename T>
__global__ void __launch_bounds__(128) k_pd_extrapolate(int nx, int ny, int nz, Cut8 cut,
                                                        const T *__restrict__ vol,
                                                        const T *__restrict__ xprev,
                                                        T *__restrict__ xbar) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y, k = blockIdx.z;
    if (i >= nx || roi_out(i, j, k, nx, ny, nz, cut.c)) return;
    const size_t p = i + (size_t)j * nx + (size_t)k * nx * ny;
    st_stored(xbar + p, 2.0f * ld_voxel(vol + p) - ld_voxel(xprev + p));
}

// End of a SART call (ST_Tomography.cpp:793-804) optionally fused with the
// over-relaxation that follows it in the primal-dual loop (:586-604)
// (roi_apply_at).
template <typename T>
__global__ void __launch_bounds__(128) k_roi_apply(int nx, int ny, int nz, Cut8 cut, Cut8 pdcut,
                                                   T *__restrict__ vol,
                                                   const T *__restrict__ xprev,
                                                   T *__restrict__ xbar) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nx) return;
    roi_apply_at(i, (int)blockIdx.y, (int)blockIdx.z, nx, ny, nz, cut.c, pdcut.c, vol, xprev, xbar);
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

namespace {
template <int K, typename T, bool PF = false>
void bp_cols(const GeomDev &g, const ViewRec *views, const ViewSel &sel, T *vol, float alpha, float gmax,
             cudaStream_t s, unsigned long long tex) {
    k_bp_voxel_cols<K, T, PF><<<dim3((g.nx + 127) / 128, (g.ny + K - 1) / K, g.nz), 128, 0, s>>>(
        g, views, sel, vol, alpha, gmax, tex);
}

template <typename T>
cudaError_t bp_voxel_any(const GeomDev &g, const ViewRec *views, const ViewSel &sel, const float *corr, T *vol,
                         float alpha, float gmax, cudaStream_t s, unsigned long long corr_tex, int bp_variant) {
    if (corr_tex) {
        switch (bp_variant) {
        case 1: bp_cols<8>(g, views, sel, vol, alpha, gmax, s, corr_tex); break;
        case 2: bp_cols<32>(g, views, sel, vol, alpha, gmax, s, corr_tex); break;
        case 3: bp_cols<16, T, true>(g, views, sel, vol, alpha, gmax, s, corr_tex); break;
        case 4: bp_cols<32, T, true>(g, views, sel, vol, alpha, gmax, s, corr_tex); break;
        default: bp_cols<BP_COL>(g, views, sel, vol, alpha, gmax, s, corr_tex); break;
        }
    } else {
        k_bp_voxel<false, T><<<vox_grid(g.nx, g.ny, g.nz), 128, 0, s>>>(g, views, sel, corr, vol, alpha, gmax, 0);
    }
    return cudaGetLastError();
}

template <typename T>
cudaError_t pd_dual_any(const int *d, const PdParams &p, const T *xf, const T *xf1, const float *bw, float *ytv,
                        float *ytp, float *ybc, cudaStream_t s) {
    k_pd_dual<T><<<vox_grid(d[0], d[1], d[2]), 128, 0, s>>>(d[0], d[1], d[2], p.sigma, p.tv_w, p.tp_w, p.bc_w, p.hf,
                                                            to_cut(p.cut), xf, xf1, bw, ytv, ytp, ybc);
    return cudaGetLastError();
}

template <typename T>
cudaError_t pd_primal_any(const int *d, const PdParams &p, int first, const float *ytp_prev, const float *ytp,
                          const float *fw, const float *ybc, const float *ytv, T *vol, T *xprev, cudaStream_t s) {
    k_pd_primal<T><<<vox_grid(d[0], d[1], d[2]), 128, 0, s>>>(d[0], d[1], d[2], p.tau, p.gmax, to_cut(p.cut), first,
                                                              ytp_prev, ytp, fw, ybc, ytv, vol, xprev);
    return cudaGetLastError();
}

template <typename T>
cudaError_t roi_apply_any(const int *d, const int *roi_cut, const int *pd_cut, T *vol, const T *xprev, T *xbar,
                          cudaStream_t s) {
    k_roi_apply<T><<<vox_grid(d[0], d[1], d[2]), 128, 0, s>>>(d[0], d[1], d[2], to_cut(roi_cut), to_cut(pd_cut), vol,
                                                              xprev, xbar);
    return cudaGetLastError();
}

template <typename T>
cudaError_t pd_extrapolate_any(const int *d, const int *cut, const T *vol, const T *xprev, T *xbar, cudaStream_t s) {
    k_pd_extrapolate<T><<<vox_grid(d[0], d[1], d[2]), 128, 0, s>>>(d[0], d[1], d[2], to_cut(cut), vol, xprev, xbar);
    return cudaGetLastError();
}
}  // namespace

cudaError_t make_corr_tex(int W, int H, CorrTex &o) {
    o = CorrTex{};
    cudaChannelFormatDesc cd = cudaCreateChannelDesc<float>();
    cudaError_t e = cudaMalloc3DArray(&o.arr, &cd, make_cudaExtent(W, H, 1), cudaArrayLayered | cudaArraySurfaceLoadStore);
    if (e != cudaSuccess) return e;
    cudaResourceDesc rd{};
    rd.resType = cudaResourceTypeArray;
    rd.res.array.array = o.arr;
    cudaTextureDesc td{};
    td.addressMode[0] = td.addressMode[1] = td.addressMode[2] = cudaAddressModeClamp;
    td.filterMode = cudaFilterModePoint;
    td.readMode = cudaReadModeElementType;
    td.normalizedCoords = 0;
    cudaTextureObject_t t = 0;
    cudaSurfaceObject_t sf = 0;
    if ((e = cudaCreateTextureObject(&t, &rd, &td, nullptr)) == cudaSuccess) e = cudaCreateSurfaceObject(&sf, &rd);
    o.tex = t;
    o.surf = sf;
    o.W = W;
    o.H = H;
    if (e != cudaSuccess) free_corr_tex(o);
    return e;
}

void free_corr_tex(CorrTex &o) {
    if (o.surf) cudaDestroySurfaceObject((cudaSurfaceObject_t)o.surf);
    if (o.tex) cudaDestroyTextureObject((cudaTextureObject_t)o.tex);
    if (o.arr) cudaFreeArray(o.arr);
    o = CorrTex{};
}

const char *bp_variant_name(int v) {
    static const char *names[kBpVariants] = {"columns of 16 voxels", "columns of 8 voxels", "columns of 32 voxels",
                                             "columns of 16 voxels, L2 prefetch", "columns of 32 voxels, L2 prefetch"};
    return v >= 0 && v < kBpVariants ? names[v] : "?";
}

cudaError_t launch_bp_voxel(const GeomDev &g, const ViewRec *views, const ViewSel &sel, const float *corr,
                            float *vol, float alpha, float gmax, cudaStream_t s, unsigned long long corr_tex,
                            int bp_variant) {
    return bp_voxel_any(g, views, sel, corr, vol, alpha, gmax, s, corr_tex, bp_variant);
}

cudaError_t launch_bp_voxel(const GeomDev &g, const ViewRec *views, const ViewSel &sel, const float *corr,
                            unsigned short *vol, float alpha, float gmax, cudaStream_t s, unsigned long long corr_tex,
                            int bp_variant) {
    return bp_voxel_any(g, views, sel, corr, vol, alpha, gmax, s, corr_tex, bp_variant);
}

cudaError_t launch_pd_dual(const int *d, const PdParams &p, const float *xf, const float *xf1,
                           const float *bw, float *ytv, float *ytp, float *ybc, cudaStream_t s) {
    return pd_dual_any(d, p, xf, xf1, bw, ytv, ytp, ybc, s);
}

cudaError_t launch_pd_dual(const int *d, const PdParams &p, const unsigned short *xf, const unsigned short *xf1,
                           const float *bw, float *ytv, float *ytp, float *ybc, cudaStream_t s) {
    return pd_dual_any(d, p, xf, xf1, bw, ytv, ytp, ybc, s);
}

cudaError_t launch_pd_primal(const int *d, const PdParams &p, int first, const float *ytp_prev,
                             const float *ytp, const float *fw, const float *ybc, const float *ytv,
                             float *vol, float *xprev, cudaStream_t s) {
    return pd_primal_any(d, p, first, ytp_prev, ytp, fw, ybc, ytv, vol, xprev, s);
}

cudaError_t launch_pd_primal(const int *d, const PdParams &p, int first, const float *ytp_prev,
                             const float *ytp, const float *fw, const float *ybc, const float *ytv,
                             unsigned short *vol, unsigned short *xprev, cudaStream_t s) {
    return pd_primal_any(d, p, first, ytp_prev, ytp, fw, ybc, ytv, vol, xprev, s);
}

cudaError_t launch_pd_extrapolate(const int *d, const int *cut, const float *vol, const float *xprev,
                                  float *xbar, cudaStream_t s) {
    return pd_extrapolate_any(d, cut, vol, xprev, xbar, s);
}

cudaError_t launch_pd_extrapolate(const int *d, const int *cut, const unsigned short *vol,
                                  const unsigned short *xprev, unsigned short *xbar, cudaStream_t s) {
    return pd_extrapolate_any(d, cut, vol, xprev, xbar, s);
}

cudaError_t launch_roi_apply(const int *d, const int *roi_cut, const int *pd_cut, float *vol,
                             const float *xprev, float *xbar, cudaStream_t s) {
    return roi_apply_any(d, roi_cut, pd_cut, vol, xprev, xbar, s);
}

cudaError_t launch_roi_apply(const int *d, const int *roi_cut, const int *pd_cut, unsigned short *vol,
                             const unsigned short *xprev, unsigned short *xbar, cudaStream_t s) {
    return roi_apply_any(d, roi_cut, pd_cut, vol, xprev, xbar, s);
}

cudaError_t launch_roi_mask(const int *d, const int *cut, float *roi, cudaStream_t s) {
    k_roi_mask<<<vox_grid(d[0], d[1], d[2]), 128, 0, s>>>(d[0], d[1], d[2], to_cut(cut), roi);
    return cudaGetLastError();
}

}  // namespace stt
