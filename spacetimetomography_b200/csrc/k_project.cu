// k_project.cu -- ray-driven kernels: forward projection, forward projection
// fused with the SART correction, the ray-driven backprojection scatter and
// the exact adjoint A^T.
//
// One thread per detector pixel.  A 128-thread block covers 32x4 pixels: each
// warp is 32 consecutive detector columns of one row, so at every step its 32
// samples lie along the detector's u axis in the volume.  For views whose rays
// run mostly along z, u maps to the volume's x axis, which is contiguous in
// memory; for views whose rays run mostly along x, u maps to z and the forward
// projector gathers from a z-fastest transposed copy (ViewRec::layout), so
// either way a warp's gathers touch few cache lines.  The volume is read
// through the read-only path (ld.global.nc); at the headline sizes (256^3 fp32
// = 64 MiB) it stays resident in the 126 MB L2.
#include "stt_internal.cuh"
#include "stt_kernels.h"

namespace stt {

namespace {

__device__ __forceinline__ bool tile_pixel(const GeomDev &g, int &i, int &j) {
    i = blockIdx.x * 32 + (threadIdx.x & 31);
    j = blockIdx.y * 4 + (threadIdx.x >> 5);
    return i < g.W && j < g.H;
}

// The ray sum gathered from the z-fastest transposed copy for layout-1 views
// when one is given, else from the volume (fp_ray_sum_with).
template <int FAST, typename I, int G = FP_GROUP, bool PK = false, typename T>
__device__ __forceinline__ float fp_ray_sum_from(const GeomDev &g, const T *__restrict__ src, const Strides &st,
                                                 const Ray &r, int *count) {
    return fp_ray_sum_with<G, PK>(
        g, [=](int, const FpCell &c, float v[8]) { fp_corners<FAST, I>(src, st, c, v); }, r, count);
}

// The ray sum through the textures of FpTex: the transposed copy's for
// layout-1 views when there is one, as fp_ray_sum reads the arrays.
template <int G = FP_GROUP, bool PK = false, typename T = float>
__device__ __forceinline__ float fp_ray_sum_tex(const GeomDev &g, const ViewRec &v, const FpTex &tex, const Ray &r) {
    if (tex.z && v.layout == 1) {
        const unsigned long long t = tex.z;
        const int row = g.nz;
        return fp_ray_sum_with<G, PK>(
            g, [=](int, const FpCell &c, float w[8]) { fp_corners_tex<2, T>(t, row, c, w); }, r, nullptr);
    }
    const unsigned long long t = tex.x;
    const int row = g.nx;
    return fp_ray_sum_with<G, PK>(
        g, [=](int, const FpCell &c, float w[8]) { fp_corners_tex<0, T>(t, row, c, w); }, r, nullptr);
}

template <typename I, int G = FP_GROUP, bool PK = false, typename T>
__device__ __forceinline__ float fp_ray_sum(const GeomDev &g, const ViewRec &v, const T *__restrict__ vol,
                                            const T *__restrict__ vol_t, const Ray &r, int *count) {
    if (vol_t && v.layout == 1) return fp_ray_sum_from<2, I, G, PK>(g, vol_t, zyx_strides(g), r, count);
    return fp_ray_sum_from<0, I, G, PK>(g, vol, xyz_strides(g), r, count);
}

// Detector tile of a block of NW warps for the tunable projector variants:
// a warp covers WX x (32/WX) pixels (WX consecutive columns of 32/WX rows),
// the NW warps are stacked along the rows.  WX = 32, NW = 4 is tile_pixel.
template <int WX, int NW>
__device__ __forceinline__ bool tile_pixel_t(const GeomDev &g, int &i, int &j) {
    constexpr int WY = 32 / WX;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    i = blockIdx.x * WX + (lane % WX);
    j = (blockIdx.y * NW + w) * WY + lane / WX;
    return i < g.W && j < g.H;
}

// GenerateImage_MT (S/ImageFormationModel/TypicalRayProducer.core.h:168-224)
// for views [view0, view0 + gridDim.z).  T = float, or unsigned short for a
// BF16-stored volume (taps widened to FP32; the march and the sums are FP32).
template <typename I, typename T>
__global__ void __launch_bounds__(128) k_fp(const GeomDev g, const ViewRec *__restrict__ views,
                                            const T *__restrict__ vol, const T *__restrict__ vol_t,
                                            int view0, float *__restrict__ proj, float *__restrict__ raylen,
                                            float *__restrict__ weight) {
    int i, j;
    if (!tile_pixel(g, i, j)) return;
    const int v = blockIdx.z;
    const ViewRec &vr = views[view0 + v];
    Ray r;
    make_ray(g, vr, i, j, r);
    int count = 0;
    const bool hit = r.tnear < r.tfar;
    const float sum = hit ? fp_ray_sum<I>(g, vr, vol, vol_t, r, &count) : 0.0f;
    const size_t o = (size_t)v * g.W * g.H + i + (size_t)j * g.W;
    proj[o] = sum;
    if (raylen && hit) raylen[o] = r.tfar - r.tnear;
    if (weight) weight[o] = (float)count;
}

// Forward projection of one view with the SART correction as epilogue
// (ST_Tomography.cpp:667-676; Factor = 1 and pY == 0 in the reference, so
// c = (b - Ax) / (L + 1)).  L is the sticky ray length of the producer:
// updated where the ray hits, kept where it misses; with no state buffer
// (ray-based SART, whose producer is reset after every view) a miss gives L = 0.
// Tunable variants (fp_variant_name): the block's detector tile (WX, NW), the
// samples in flight per step (G) and whether pairs of samples share packed
// FP32x2 instructions (PK) change only which thread projects which ray, how
// far ahead its loads run and how many instructions carry the same roundings,
// never a ray's arithmetic.
// T, B: the storage of the volume and of the sinogram stack (float, or BF16
// bits widened exactly to FP32).
// TX: the corners come from the textures of `tex` (FP32 volumes below 2^31
// voxels), not from vol and vol_t.
template <typename I, int WX = 32, int NW = 4, int G = FP_GROUP, bool PK = false, typename T = float,
          typename B = float, bool TX = false>
__global__ void __launch_bounds__(32 * NW) k_fp_corr(const GeomDev g, const ViewRec *__restrict__ views,
                                                     const T *__restrict__ vol, const T *__restrict__ vol_t,
                                                     const ViewSel sel, const B *__restrict__ b_stack,
                                                     float *__restrict__ raylen_state,
                                                     float *__restrict__ corr, unsigned long long corr_surf,
                                                     int skip_staged, const FpTex tex) {
    int i, j;
    if (!tile_pixel_t<WX, NW>(g, i, j)) return;
    int local;
    const int view = sel_view(sel, local);
    const B *b = b_stack + (size_t)local * g.W * g.H;
    const ViewRec &vr = views[view];
    if (skip_staged && view_staged<T>(vr)) return;  // the slab-staged kernel projects this view
    Ray r;
    make_ray(g, vr, i, j, r);
    const size_t pix = i + (size_t)j * g.W;
    float L, sum = 0.0f;
    if (r.tnear < r.tfar) {
        if constexpr (TX)
            sum = fp_ray_sum_tex<G, PK, T>(g, vr, tex, r);
        else
            sum = fp_ray_sum<I, G, PK>(g, vr, vol, vol_t, r, nullptr);
        L = r.tfar - r.tnear;
        if (raylen_state) raylen_state[pix] = L;
    } else {
        L = raylen_state ? raylen_state[pix] : 0.0f;
    }
    const float c = __fdiv_rn(__fsub_rn(ld_voxel(b + pix), sum), __fadd_rn(L, 1.0f));
    corr[pix] = c;
    // the copy the voxel-driven backprojector gathers from with tld4
    if (corr_surf) surf2DLayeredwrite(c, corr_surf, i * (int)sizeof(float), j, 0, cudaBoundaryModeZero);
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
        scatter_corners(acc, t, c, w);
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
        // x-neighbour corners inside the volume whose first address is 8-byte
        // aligned (the caller's vol_bar may start anywhere on 4 bytes): one
        // vector atomic (the same terms)
#pragma unroll
        for (int m = 0; m < 8; m += 2) {
            const long long idx = tap_index(t, m);
            if (t.dx == 1 && !(reinterpret_cast<uintptr_t>(vol_bar + idx) & 7)) {
                atomicAdd(reinterpret_cast<float2 *>(vol_bar + idx), make_float2(ys * w[m], ys * w[m + 1]));
            } else {
                atomicAdd(vol_bar + idx, ys * w[m]);
                atomicAdd(vol_bar + idx + t.dx, ys * w[m + 1]);
            }
        }
    });
}

// Ray-BP normalisation (ST_Tomography.cpp:746-762): vol += contrib/weight,
// clamped with the reference macros so 0/0 = NaN becomes 0; the accumulator
// is reset for the next view (TypicalRayProducer::Initial, TypicalRayProducer.cpp:91-95).
template <typename T>
__global__ void k_bp_ray_update(long long n, float2 *__restrict__ acc, T *__restrict__ vol, float gmax) {
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n;
         k += (long long)gridDim.x * blockDim.x) {
        float2 a = acc[k];
        float v = ld_stored(vol + k) + __fdiv_rn(a.x, a.y);
        st_stored(vol + k, rmax(rmin(gmax, v), 0.0f));
        acc[k] = make_float2(0.0f, 0.0f);
    }
}

// Adds the scatter accumulators to caller arrays and clears them: the raw
// contributions and weights of the reference's backprojection mode
// (SingleScalarVolume.core.h:128-143, read back through
// TypicalRayProducer::GetContributions / GetTotalWeight).
__global__ void k_acc_split(long long n, float2 *__restrict__ acc, float *__restrict__ contrib,
                            float *__restrict__ wsum) {
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n;
         k += (long long)gridDim.x * blockDim.x) {
        const float2 a = acc[k];
        contrib[k] += a.x;
        wsum[k] += a.y;
        acc[k] = make_float2(0.0f, 0.0f);
    }
}

// Stand-alone SART correction (ST_Tomography.cpp:667-676) for the unfused
// per-view form: the ray lengths are the sticky state k_fp updated on hits.
template <typename B>
__global__ void k_correction(long long n, const B *__restrict__ b, const float *__restrict__ ax,
                             const float *__restrict__ raylen, float *__restrict__ corr) {
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n;
         k += (long long)gridDim.x * blockDim.x)
        corr[k] = __fdiv_rn(__fsub_rn(ld_voxel(b + k), ax[k]), __fadd_rn(raylen ? raylen[k] : 0.0f, 1.0f));
}

// z-fastest copy of an x-fastest volume: out[z + y*nz + x*nz*ny] = in[x + y*nx + z*nx*ny].
// One 64x64 (x, z) tile of one y plane per block of 32x8 threads, through
// shared memory.  Interior tiles move two elements per access (8-byte float2
// or 4-byte ushort2 rows) when nx and nz are even and both arrays aligned to
// a pair; edge tiles move one.
template <typename T>
struct Pair2;
template <>
struct Pair2<float> {
    typedef float2 type;
};
template <>
struct Pair2<unsigned short> {
    typedef ushort2 type;
};

template <typename T>
__device__ __forceinline__ void transpose_tile(int nx, int ny, int nz, const T *__restrict__ in,
                                               T *__restrict__ out) {
    typedef typename Pair2<T>::type P;
    __shared__ T tile[64][65];  // tile[z - z0][x - x0]
    const int x0 = blockIdx.x * 64, z0 = blockIdx.y * 64, y = blockIdx.z;
    const size_t nxy = (size_t)nx * ny, nzy = (size_t)nz * ny;
    const T *src = in + (size_t)y * nx + x0 + (size_t)z0 * nxy;
    T *dst = out + (size_t)y * nz + z0 + (size_t)x0 * nzy;
    const int tx = threadIdx.x;
    const bool pairs = x0 + 64 <= nx && z0 + 64 <= nz && !(nx & 1) && !(nz & 1) &&
                       !(((uintptr_t)in | (uintptr_t)out) % sizeof(P));
    if (pairs) {
#pragma unroll
        for (int r = threadIdx.y; r < 64; r += 8) {
            const P v = reinterpret_cast<const P *>(src + r * nxy)[tx];
            tile[r][2 * tx] = v.x;
            tile[r][2 * tx + 1] = v.y;
        }
        __syncthreads();
#pragma unroll
        for (int r = threadIdx.y; r < 64; r += 8) {
            P v;
            v.x = tile[2 * tx][r];
            v.y = tile[2 * tx + 1][r];
            reinterpret_cast<P *>(dst + r * nzy)[tx] = v;
        }
    } else {
        for (int r = threadIdx.y; r < 64; r += 8)
            for (int c = tx; c < 64; c += 32)
                if (x0 + c < nx && z0 + r < nz) tile[r][c] = src[c + r * nxy];
        __syncthreads();
        for (int r = threadIdx.y; r < 64; r += 8)
            for (int c = tx; c < 64; c += 32)
                if (x0 + r < nx && z0 + c < nz) dst[c + r * nzy] = tile[c][r];
    }
}

template <typename T>
__global__ void __launch_bounds__(256) k_transpose_xz(int nx, int ny, int nz, const T *__restrict__ in,
                                                      T *__restrict__ out) {
    transpose_tile(nx, ny, nz, in, out);
}

// The transpose, only if the selected view gathers from the z-fastest copy
// (the choice is read on the device, so a captured graph can hold it).
template <typename T>
__global__ void __launch_bounds__(256) k_transpose_for_view(int nx, int ny, int nz,
                                                            const ViewRec *__restrict__ views, const ViewSel sel,
                                                            const T *__restrict__ in, T *__restrict__ out) {
    int local;
    if (views[sel_view(sel, local)].layout != 1) return;
    transpose_tile(nx, ny, nz, in, out);
}

__global__ void k_fill_zero(long long n, float *__restrict__ p) {
    for (long long k = blockIdx.x * (long long)blockDim.x + threadIdx.x; k < n;
         k += (long long)gridDim.x * blockDim.x)
        p[k] = 0.0f;
}

// 32-bit gather offsets when every voxel index fits.
bool small_volume(const GeomDev &g) { return (long long)g.nx * g.ny * g.nz < (1LL << 31); }

dim3 ray_grid(const GeomDev &g, int nviews) {
    return dim3((g.W + 31) / 32, (g.H + 3) / 4, nviews);
}

dim3 transpose_grid(const GeomDev &g) { return dim3((g.nx + 63) / 64, (g.nz + 63) / 64, g.ny); }

// The gather ceiling of the forward projector: each ray of one view takes as
// many samples as its clip length holds, at the projector's step from its
// entry point, with the projector's cell, 8-corner gather and trilinear
// interpolation (G = 4 samples' loads in flight, packed pairs when PK; the
// corners as tld4 gathers of texture `tex` when TX), and none of its march
// control (no segment splits, no per-sample bound, a plain sum).  No
// counterpart in the reference: a measurement of the rate the gathers alone
// reach on a volume, the on-chip roofline of the projectors.
template <int FAST, bool PK, bool TX = false>
__global__ void __launch_bounds__(128) k_gather_ceiling(const GeomDev g, const ViewRec *__restrict__ views, int view,
                                                        const float *__restrict__ src, unsigned long long tex,
                                                        float *__restrict__ out, int *__restrict__ count) {
    int i, j;
    if (!tile_pixel(g, i, j)) return;
    Ray r;
    make_ray(g, views[view], i, j, r);
    const size_t pix = i + (size_t)j * g.W;
    float sum = 0.0f;
    int n = 0;
    if (r.tnear < r.tfar) {
        const Strides st = FAST ? zyx_strides(g) : xyz_strides(g);
        n = min((int)((r.tfar - r.tnear) / g.sd) + 1, 1 << 22);
        float p[3], step[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            p[k] = __fmaf_rn(r.vu[k], r.tnear, r.vz[k]);  // explicit roundings: every instantiation alike
            step[k] = __fmul_rn(r.vu[k], g.sd);
        }
        constexpr int G = 4;
        int k = 0;
        for (; k + G <= n; k += G) {
            float q[G][3];
            FpCell c[G];
            float v[G][8];
#pragma unroll
            for (int s = 0; s < G; ++s)
#pragma unroll
                for (int a = 0; a < 3; ++a) q[s][a] = __fmaf_rn((float)s, step[a], p[a]);
#pragma unroll
            for (int a = 0; a < 3; ++a) p[a] = __fmaf_rn((float)G, step[a], p[a]);
            if constexpr (PK) {
#pragma unroll
                for (int s = 0; s < G; s += 2) fp_cell2(g, q[s], q[s + 1], c[s], c[s + 1]);
            } else {
#pragma unroll
                for (int s = 0; s < G; ++s) fp_cell(g, q[s], c[s]);
            }
#pragma unroll
            for (int s = 0; s < G; ++s) {
                if constexpr (TX)
                    fp_corners_tex<FAST>(tex, FAST ? g.nz : g.nx, c[s], v[s]);
                else
                    fp_corners<FAST, int>(src, st, c[s], v[s]);
            }
            if constexpr (PK) {
#pragma unroll
                for (int s = 0; s < G; s += 2) {
                    const float2 t = trilerp2(v[s], v[s + 1], c[s], c[s + 1]);
                    sum = __fadd_rn(sum, __fadd_rn(t.x, t.y));
                }
            } else {  // the same additions as the packed form
#pragma unroll
                for (int s = 0; s < G; s += 2)
                    sum = __fadd_rn(sum, __fadd_rn(trilerp(v[s], c[s]), trilerp(v[s + 1], c[s + 1])));
            }
        }
        for (; k < n; ++k) {
            FpCell c;
            fp_cell(g, p, c);
            float v[8];
            if constexpr (TX)
                fp_corners_tex<FAST>(tex, FAST ? g.nz : g.nx, c, v);
            else
                fp_corners<FAST, int>(src, st, c, v);
            sum = __fadd_rn(sum, trilerp(v, c));
#pragma unroll
            for (int a = 0; a < 3; ++a) p[a] = __fadd_rn(p[a], step[a]);
        }
    }
    out[pix] = __fmul_rn(sum, g.sd);
    if (count) count[pix] = n;
}

}  // namespace

int sm_count() {
    // multiProcessorCount of each device, read once per device (148 on B200)
    static int cached[64] = {0};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) {
        cudaGetLastError();
        return 148;
    }
    if (!cached[dev]) {
        int n = 0;
        if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || n < 1) {
            cudaGetLastError();
            n = 148;
        }
        cached[dev] = n;
    }
    return cached[dev];
}

int grid_stride_blocks(long long n, int threads) {
    long long b = (n + threads - 1) / threads;
    // grid-stride loops: at most 8 resident 256-thread blocks per SM (2048 threads)
    const long long cap = (long long)sm_count() * (2048 / (threads > 0 ? threads : 256));
    return (int)(b < cap ? (b < 1 ? 1 : b) : cap);
}

cudaError_t launch_fp(const GeomDev &g, const ViewRec *views, const float *vol, const float *vol_t, int view0,
                      int nviews, float *proj, float *raylen, float *weight, cudaStream_t s) {
    if (small_volume(g))
        k_fp<int, float><<<ray_grid(g, nviews), 128, 0, s>>>(g, views, vol, vol_t, view0, proj, raylen, weight);
    else
        k_fp<long long, float><<<ray_grid(g, nviews), 128, 0, s>>>(g, views, vol, vol_t, view0, proj, raylen, weight);
    return cudaGetLastError();
}

namespace {

// One launch of gather variant <WX, NW, G, PK, TX>: a block is NW warps of WX x (32/WX) pixels.
template <int WX, int NW, int G, bool PK = false, bool TX = false>
void fp_corr_variant(const GeomDev &g, const ViewRec *views, const float *vol, const float *vol_t, const ViewSel &sel,
                     const float *b_stack, float *raylen_state, float *corr, cudaStream_t s,
                     unsigned long long corr_surf, int skip, const FpTex &tex = FpTex{}) {
    constexpr int TH = (32 / WX) * NW;  // detector rows per block
    k_fp_corr<int, WX, NW, G, PK, float, float, TX>
        <<<dim3((g.W + WX - 1) / WX, (g.H + TH - 1) / TH, 1), 32 * NW, 0, s>>>(
            g, views, vol, vol_t, sel, b_stack, raylen_state, corr, corr_surf, skip, tex);
}

// Device limits of pitch-linear 2D textures, read once per device.
struct TexLimits {
    int width = 0, height = 0, pitch = 0, pitch_align = 0, base_align = 0;
};

bool tex_limits(TexLimits &l) {
    static TexLimits cache[64];
    static bool have[64] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return false;
    if (!have[dev]) {
        TexLimits t;
        if (cudaDeviceGetAttribute(&t.width, cudaDevAttrMaxTexture2DLinearWidth, dev) != cudaSuccess ||
            cudaDeviceGetAttribute(&t.height, cudaDevAttrMaxTexture2DLinearHeight, dev) != cudaSuccess ||
            cudaDeviceGetAttribute(&t.pitch, cudaDevAttrMaxTexture2DLinearPitch, dev) != cudaSuccess ||
            cudaDeviceGetAttribute(&t.pitch_align, cudaDevAttrTexturePitchAlignment, dev) != cudaSuccess ||
            cudaDeviceGetAttribute(&t.base_align, cudaDevAttrTextureAlignment, dev) != cudaSuccess) {
            cudaGetLastError();
            return false;
        }
        cache[dev] = t;
        have[dev] = true;
    }
    l = cache[dev];
    return true;
}

bool slices_fit(const TexLimits &l, const void *p, long long width, long long rows, int esize) {
    const long long pitch = width * (long long)esize;
    return p && width >= 2 && rows >= 2 && width <= l.width && rows <= l.height && pitch <= l.pitch &&
           !(l.pitch_align > 0 && pitch % l.pitch_align) && !(l.base_align > 0 && (uintptr_t)p % l.base_align);
}

// A point-sampled, clamped texture of `rows` rows of `width` texels over
// linear memory (FP32 texels, or 16-bit unsigned ones holding BF16 bits); 0
// where the limits do not admit it.
template <typename T>
unsigned long long slices_texture(const TexLimits &l, const T *p, long long width, long long rows) {
    const long long pitch = width * (long long)sizeof(T);
    if (!slices_fit(l, p, width, rows, (int)sizeof(T))) return 0;
    cudaResourceDesc rd{};
    rd.resType = cudaResourceTypePitch2D;
    rd.res.pitch2D.devPtr = const_cast<T *>(p);
    rd.res.pitch2D.desc = cudaCreateChannelDesc<T>();
    rd.res.pitch2D.width = (size_t)width;
    rd.res.pitch2D.height = (size_t)rows;
    rd.res.pitch2D.pitchInBytes = (size_t)pitch;
    cudaTextureDesc td{};
    td.addressMode[0] = td.addressMode[1] = cudaAddressModeClamp;
    td.filterMode = cudaFilterModePoint;
    td.readMode = cudaReadModeElementType;
    cudaTextureObject_t t = 0;
    if (cudaCreateTextureObject(&t, &rd, &td, nullptr) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return (unsigned long long)t;
}

}  // namespace

const char *fp_variant_name(int v) {
    static const char *names[kFpVariants] = {"32x4 rays per block, 4 samples in flight",
                                             "32x2 rays per block, 4 in flight",
                                             "32x8 rays per block, 4 in flight",
                                             "warps of 16x2 rays, 16x8 per block, 4 in flight",
                                             "warps of 8x4 rays, 8x16 per block, 4 in flight",
                                             "32x4 rays per block, 2 in flight",
                                             "32x4 rays per block, 8 in flight",
                                             "32x4 rays per block, 4 in flight, packed pairs",
                                             "32x4 rays per block, 8 in flight, packed pairs",
                                             "32x8 rays per block, 4 in flight, packed pairs",
                                             "warps of 8x4 rays, 8x16 per block, 8 in flight, packed pairs, tld4 corners",
                                             "32x4 rays per block, 8 in flight, packed pairs, tld4 corners"};
    return v >= 0 && v < kFpVariants ? names[v] : "?";
}

bool is_tex_fp_variant(int fp_variant) { return fp_variant == 10 || fp_variant == 11; }

const char *fp16_variant_name(int v) {
    static const char *names[kFp16Variants] = {"32x4 rays per block, 4 samples in flight",
                                               "warps of 8x4 rays, 8 in flight, packed pairs, tld4 corners"};
    return v >= 0 && v < kFp16Variants ? names[v] : "?";
}

namespace {
template <typename T>
bool make_fp_tex_any(const GeomDev &g, const T *vol, const T *vol_t, FpTex &t) {
    t = FpTex{};
    TexLimits l;
    if (!small_volume(g) || !tex_limits(l)) return false;
    const unsigned long long x = slices_texture(l, vol, (long long)g.nx * g.ny, g.nz);
    if (!x) return false;
    unsigned long long z = 0;
    if (vol_t && !(z = slices_texture(l, vol_t, (long long)g.nz * g.ny, g.nx))) {
        cudaDestroyTextureObject((cudaTextureObject_t)x);
        return false;
    }
    t.x = x;
    t.z = z;
    t.ok = 1;
    t.esize = (int)sizeof(T);
    return true;
}
}  // namespace

bool make_fp_tex(const GeomDev &g, const float *vol, const float *vol_t, FpTex &t) {
    return make_fp_tex_any(g, vol, vol_t, t);
}

bool make_fp_tex(const GeomDev &g, const unsigned short *vol, const unsigned short *vol_t, FpTex &t) {
    return make_fp_tex_any(g, vol, vol_t, t);
}

bool fp_tex_fits(const GeomDev &g, const void *vol, int esize) {
    TexLimits l;
    if (!small_volume(g) || !tex_limits(l)) return false;
    const void *aligned = reinterpret_cast<const void *>((uintptr_t)(l.base_align > 0 ? l.base_align : 256));
    return slices_fit(l, vol, (long long)g.nx * g.ny, g.nz, esize) &&
           slices_fit(l, aligned, (long long)g.nz * g.ny, g.nx, esize);
}

void destroy_fp_tex(FpTex &t) {
    if (t.x) cudaDestroyTextureObject((cudaTextureObject_t)t.x);
    if (t.z) cudaDestroyTextureObject((cudaTextureObject_t)t.z);
    t = FpTex{};
}

cudaError_t launch_fp_corr(const GeomDev &g, const ViewRec *views, const float *vol, const float *vol_t,
                           const ViewSel &sel, const float *b_stack, float *raylen_state, float *corr,
                           cudaStream_t s, unsigned long long corr_surf, const FpSlabMaps *maps, int *status,
                           int fp_variant, const FpTex *tex) {
    const int skip = maps && maps->ok && maps->esize == 4 && (!vol_t || maps->has_z);
    // a texture variant whose textures are missing, or do not cover vol_t,
    // runs the load-based variant of the same shape
    if (is_tex_fp_variant(fp_variant) && !(tex && tex->ok && tex->esize == 4 && (!vol_t || tex->z)))
        fp_variant = fp_variant == 10 ? 4 : 8;
    FpTex tx = tex ? *tex : FpTex{};
    if (!vol_t) tx.z = 0;  // without the copy every view reads the volume, as the loads do
    if (skip) {
        cudaError_t e = launch_fp_corr_slab(g, views, *maps, vol, vol_t, sel, b_stack, raylen_state, corr, s,
                                            corr_surf, status);
        if (e != cudaSuccess) return e;
    }
    if (!small_volume(g)) {
        k_fp_corr<long long><<<ray_grid(g, 1), 128, 0, s>>>(g, views, vol, vol_t, sel, b_stack, raylen_state, corr,
                                                            corr_surf, skip, FpTex{});
        return cudaGetLastError();
    }
    switch (fp_variant) {
    case 1: fp_corr_variant<32, 2, 4>(g, views, vol, vol_t, sel, b_stack, raylen_state, corr, s, corr_surf, skip); break;
    case 2: fp_corr_variant<32, 8, 4>(g, views, vol, vol_t, sel, b_stack, raylen_state, corr, s, corr_surf, skip); break;
    case 3: fp_corr_variant<16, 4, 4>(g, views, vol, vol_t, sel, b_stack, raylen_state, corr, s, corr_surf, skip); break;
    case 4: fp_corr_variant<8, 4, 4>(g, views, vol, vol_t, sel, b_stack, raylen_state, corr, s, corr_surf, skip); break;
    case 5: fp_corr_variant<32, 4, 2>(g, views, vol, vol_t, sel, b_stack, raylen_state, corr, s, corr_surf, skip); break;
    case 6: fp_corr_variant<32, 4, 8>(g, views, vol, vol_t, sel, b_stack, raylen_state, corr, s, corr_surf, skip); break;
    case 7: fp_corr_variant<32, 4, 4, true>(g, views, vol, vol_t, sel, b_stack, raylen_state, corr, s, corr_surf, skip); break;
    case 8: fp_corr_variant<32, 4, 8, true>(g, views, vol, vol_t, sel, b_stack, raylen_state, corr, s, corr_surf, skip); break;
    case 9: fp_corr_variant<32, 8, 4, true>(g, views, vol, vol_t, sel, b_stack, raylen_state, corr, s, corr_surf, skip); break;
    case 10:
        fp_corr_variant<8, 4, 8, true, true>(g, views, vol, vol_t, sel, b_stack, raylen_state, corr, s, corr_surf,
                                             skip, tx);
        break;
    case 11:
        fp_corr_variant<32, 4, 8, true, true>(g, views, vol, vol_t, sel, b_stack, raylen_state, corr, s, corr_surf,
                                              skip, tx);
        break;
    default: fp_corr_variant<32, 4, 4>(g, views, vol, vol_t, sel, b_stack, raylen_state, corr, s, corr_surf, skip); break;
    }
    return cudaGetLastError();
}

cudaError_t launch_transpose(const GeomDev &g, const float *in, float *out, cudaStream_t s) {
    k_transpose_xz<float><<<transpose_grid(g), dim3(32, 8), 0, s>>>(g.nx, g.ny, g.nz, in, out);
    return cudaGetLastError();
}

cudaError_t launch_fp_bf16(const GeomDev &g, const ViewRec *views, const unsigned short *vol,
                           const unsigned short *vol_t, int view0, int nviews, float *proj, float *raylen,
                           float *weight, cudaStream_t s) {
    if (small_volume(g))
        k_fp<int, unsigned short><<<ray_grid(g, nviews), 128, 0, s>>>(g, views, vol, vol_t, view0, proj, raylen, weight);
    else
        k_fp<long long, unsigned short><<<ray_grid(g, nviews), 128, 0, s>>>(g, views, vol, vol_t, view0, proj, raylen,
                                                                            weight);
    return cudaGetLastError();
}

cudaError_t launch_transpose_bf16(const GeomDev &g, const unsigned short *in, unsigned short *out, cudaStream_t s) {
    k_transpose_xz<unsigned short><<<transpose_grid(g), dim3(32, 8), 0, s>>>(g.nx, g.ny, g.nz, in, out);
    return cudaGetLastError();
}

cudaError_t launch_transpose_for_view(const GeomDev &g, const ViewRec *views, const ViewSel &sel, const float *in,
                                      float *out, cudaStream_t s) {
    k_transpose_for_view<float><<<transpose_grid(g), dim3(32, 8), 0, s>>>(g.nx, g.ny, g.nz, views, sel, in, out);
    return cudaGetLastError();
}

cudaError_t launch_transpose_for_view(const GeomDev &g, const ViewRec *views, const ViewSel &sel,
                                      const unsigned short *in, unsigned short *out, cudaStream_t s) {
    k_transpose_for_view<unsigned short><<<transpose_grid(g), dim3(32, 8), 0, s>>>(g.nx, g.ny, g.nz, views, sel, in,
                                                                                  out);
    return cudaGetLastError();
}

cudaError_t launch_correction(long long n, const float *b, const float *ax, const float *raylen,
                              float *corr, cudaStream_t s) {
    k_correction<float><<<grid_stride_blocks(n, 256), 256, 0, s>>>(n, b, ax, raylen, corr);
    return cudaGetLastError();
}

cudaError_t launch_correction(long long n, const unsigned short *b, const float *ax, const float *raylen,
                              float *corr, cudaStream_t s) {
    k_correction<unsigned short><<<grid_stride_blocks(n, 256), 256, 0, s>>>(n, b, ax, raylen, corr);
    return cudaGetLastError();
}

cudaError_t launch_fp_corr(const GeomDev &g, const ViewRec *views, const unsigned short *vol,
                           const unsigned short *vol_t, const ViewSel &sel, const unsigned short *b_stack,
                           float *raylen_state, float *corr, cudaStream_t s, unsigned long long corr_surf,
                           const FpSlabMaps *maps, int *status, int fp_variant16, const FpTex *tex) {
    typedef unsigned short U;
    const int skip = maps && maps->ok && maps->esize == 2 && (!vol_t || maps->has_z);
    if (skip) {
        cudaError_t e = launch_fp_corr_slab(g, views, *maps, vol, vol_t, sel, b_stack, raylen_state, corr, s,
                                            corr_surf, status);
        if (e != cudaSuccess) return e;
    }
    if (fp_variant16 == 1 && tex && tex->ok && tex->esize == 2 && (!vol_t || tex->z) && small_volume(g)) {
        FpTex tx = *tex;
        if (!vol_t) tx.z = 0;
        constexpr int WX = 8, NW = 4, TH = (32 / WX) * NW;
        k_fp_corr<int, WX, NW, 8, true, U, U, true><<<dim3((g.W + WX - 1) / WX, (g.H + TH - 1) / TH, 1), 32 * NW, 0, s>>>(
            g, views, vol, vol_t, sel, b_stack, raylen_state, corr, corr_surf, skip, tx);
        return cudaGetLastError();
    }
    if (small_volume(g))
        k_fp_corr<int, 32, 4, FP_GROUP, false, U, U><<<ray_grid(g, 1), 128, 0, s>>>(
            g, views, vol, vol_t, sel, b_stack, raylen_state, corr, corr_surf, skip, FpTex{});
    else
        k_fp_corr<long long, 32, 4, FP_GROUP, false, U, U><<<ray_grid(g, 1), 128, 0, s>>>(
            g, views, vol, vol_t, sel, b_stack, raylen_state, corr, corr_surf, skip, FpTex{});
    return cudaGetLastError();
}

const char *ray_variant_name(int v) {
    static const char *names[kRayVariants] = {"global vector atomic per corner", "shared-memory box per slab"};
    return v >= 0 && v < kRayVariants ? names[v] : "?";
}

int default_ray_variant(const GeomDev &g) { return (long long)g.nx * g.ny * g.nz >= (1LL << 26) ? 1 : 0; }

// The scatter of the ray-driven backprojection: ray variant 1 (the slab box,
// below 2^31 voxels) or 0 (a global vector atomic per corner).
static cudaError_t bp_ray_scatter_any(const GeomDev &g, const ViewRec *views, const ViewSel &sel, const float *corr,
                                      float2 *acc, cudaStream_t s, int ray_variant) {
    if (ray_variant < 0) ray_variant = default_ray_variant(g);
    if (ray_variant == 1 && small_volume(g)) return launch_bp_ray_scatter_slab(g, views, sel, corr, acc, s);
    k_bp_ray_scatter<<<ray_grid(g, 1), 128, 0, s>>>(g, views, sel, corr, acc);
    return cudaGetLastError();
}

cudaError_t launch_bp_ray(const GeomDev &g, const ViewRec *views, const ViewSel &sel, const float *corr,
                          float2 *acc, float *vol, float gmax, cudaStream_t s, int ray_variant) {
    cudaError_t e = bp_ray_scatter_any(g, views, sel, corr, acc, s, ray_variant);
    if (e != cudaSuccess) return e;
    const long long n = (long long)g.nx * g.ny * g.nz;
    k_bp_ray_update<float><<<grid_stride_blocks(n, 256), 256, 0, s>>>(n, acc, vol, gmax);
    return cudaGetLastError();
}

cudaError_t launch_bp_ray(const GeomDev &g, const ViewRec *views, const ViewSel &sel, const float *corr,
                          float2 *acc, unsigned short *vol, float gmax, cudaStream_t s, int ray_variant) {
    cudaError_t e = bp_ray_scatter_any(g, views, sel, corr, acc, s, ray_variant);
    if (e != cudaSuccess) return e;
    const long long n = (long long)g.nx * g.ny * g.nz;
    k_bp_ray_update<unsigned short><<<grid_stride_blocks(n, 256), 256, 0, s>>>(n, acc, vol, gmax);
    return cudaGetLastError();
}

cudaError_t launch_bp_ray_scatter(const GeomDev &g, const ViewRec *views, const ViewSel &sel, const float *corr,
                                  float2 *acc, float *contrib, float *wsum, cudaStream_t s, int ray_variant) {
    cudaError_t e = bp_ray_scatter_any(g, views, sel, corr, acc, s, ray_variant);
    if (e != cudaSuccess) return e;
    const long long n = (long long)g.nx * g.ny * g.nz;
    k_acc_split<<<grid_stride_blocks(n, 256), 256, 0, s>>>(n, acc, contrib, wsum);
    return cudaGetLastError();
}

cudaError_t launch_fp_adjoint(const GeomDev &g, const ViewRec *views, int view0, int nviews,
                              const float *proj_bar, float *vol_bar, cudaStream_t s) {
    k_fp_adjoint<<<ray_grid(g, nviews), 128, 0, s>>>(g, views, view0, proj_bar, vol_bar);
    return cudaGetLastError();
}

cudaError_t launch_gather_ceiling(const GeomDev &g, const ViewRec *views, const ViewRec &host_view, int view,
                                  const float *vol, const float *vol_t, int packed, float *out, int *count,
                                  cudaStream_t s, const FpTex *tex) {
    if (!small_volume(g)) return cudaErrorInvalidValue;
    const bool zf = vol_t && host_view.layout == 1;
    const float *src = zf ? vol_t : vol;
    if (tex) {  // packed pairs, tld4 corners
        if (!tex->ok || (zf && !tex->z)) return cudaErrorInvalidValue;
        if (zf) k_gather_ceiling<2, true, true><<<ray_grid(g, 1), 128, 0, s>>>(g, views, view, src, tex->z, out, count);
        else k_gather_ceiling<0, true, true><<<ray_grid(g, 1), 128, 0, s>>>(g, views, view, src, tex->x, out, count);
        return cudaGetLastError();
    }
    if (zf && packed) k_gather_ceiling<2, true><<<ray_grid(g, 1), 128, 0, s>>>(g, views, view, src, 0, out, count);
    else if (zf) k_gather_ceiling<2, false><<<ray_grid(g, 1), 128, 0, s>>>(g, views, view, src, 0, out, count);
    else if (packed) k_gather_ceiling<0, true><<<ray_grid(g, 1), 128, 0, s>>>(g, views, view, src, 0, out, count);
    else k_gather_ceiling<0, false><<<ray_grid(g, 1), 128, 0, s>>>(g, views, view, src, 0, out, count);
    return cudaGetLastError();
}

cudaError_t launch_fill_zero(float *p, long long n, cudaStream_t s) {
    k_fill_zero<<<grid_stride_blocks(n, 256), 256, 0, s>>>(n, p);
    return cudaGetLastError();
}

}  // namespace stt
