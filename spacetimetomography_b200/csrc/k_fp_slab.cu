// k_fp_slab.cu -- forward projection + SART correction with the volume staged
// into shared memory by TMA, slab by slab.
//
// A block is the 32x4-pixel detector tile of k_fp_corr: 128 nearly parallel
// rays.  Along the volume copy's slowest axis (z for the x-fastest volume, x
// for the z-fastest copy: the axis the rays of the view mostly run along) the
// block walks slabs of SB-1 planes.  For each slab it loads, with one
// cp.async.bulk.tensor.3d, the FB x YB x SB box (fast, y, slow) that holds
// every trilinear tap of its rays' samples in those planes, double-buffered
// behind an mbarrier, and every ray takes the samples whose base plane lies
// in the slab from shared memory.  The 8 taps of a sample are then 8 shared
// loads at fixed offsets, in place of 8 global gathers whose warp-wide
// requests touch several cache lines each.
//
// Each ray keeps its own march (MarchGen: the samples of march(), in order)
// and its own Kahan sum; a slab only decides where a sample's taps are read.
// A sample whose taps are not in the box (a ray outside the box's extent, the
// pre-entry restart of the march walking back, a timed-out copy) reads them
// from global memory, and the samples left after the last slab are drained the
// same way, so the ray sums are those of k_fp_corr bit for bit.
#include <climits>
#include <cuda.h>
#include <cudaTypedefs.h>

#include "stt_internal.cuh"
#include "stt_kernels.h"
#include "stt_slab.cuh"
#include "stt_tma.cuh"

namespace stt {

namespace {

// A staged box (fast, y, slow) of voxels; its rows (FB voxels of FP32 or
// BF16) are multiples of 16 bytes.  The variants (slab_variant_name) hold
// different slices of the same taps: a sample whose taps are not in the box
// reads them from global memory, so every box gives the same bits.
template <int FB_, int YB_, int SB_>
struct SlabBox {
    static constexpr int FB = FB_, YB = YB_, SB = SB_;
    static constexpr int N = FB * YB * SB;
    static constexpr int SLAB = SB - 1;  // base planes per slab; the box also holds their +1 plane
    static_assert(FB % 8 == 0, "TMA box rows must be 16-byte multiples in FP32 and BF16");
};

// A staged voxel widened to FP32 (shared memory: plain loads).
__device__ __forceinline__ float sm_voxel(const float *p) { return *p; }
__device__ __forceinline__ float sm_voxel(const unsigned short *p) { return __uint_as_float((unsigned)*p << 16); }
using Box0 = SlabBox<48, 8, 12>;
using Box1 = SlabBox<48, 8, 8>;
using Box2 = SlabBox<64, 8, 10>;
using Box3 = SlabBox<40, 8, 16>;
constexpr long long WAIT_CYCLES = 200000000LL;  // about 0.1 s: a copy that never lands is an error
constexpr int WARPS = 4;                         // a block is 32 x WARPS detector pixels, one warp per row

// The march of one ray of the block, summed into `acc`, taps from the staged
// slabs where they are held.  PK: inside a segment, two samples at a time in
// the packed FP32x2 instructions (fp_cell2, trilerp2, the paired march step);
// the same samples are added in the same order with the same roundings, so
// the sum is the same bits.
// T: the volume's storage (float, or BF16 bits widened exactly to FP32).
template <bool ZF, class BX, bool PK, typename T>
__device__ __forceinline__ void slab_ray_sum(const GeomDev &g, const CUtensorMap *map, const T *__restrict__ src,
                                             bool hit, const Ray &r, T *buf, uint64_t *bar, int *red_s,
                                             int (*red)[2 * WARPS], volatile int *dead, int *status, Kahan &acc) {
    constexpr int FB = BX::FB, YB = BX::YB, SB = BX::SB, BOXN = BX::N, SLAB = BX::SLAB;
    constexpr unsigned BOX_BYTES = BX::N * sizeof(T);
    constexpr int ALIGN = 16 / sizeof(T);  // a TMA box starts on 16 bytes along its innermost axis
    const Strides st = ZF ? zyx_strides(g) : xyz_strides(g);
    MarchGen m;
    if (hit) m.init(g, r);
    else m.phase = 2;

    // The base planes the block's rays span and the direction they run in.
    int lo, hi;
    bool fwd;
    slab::block_span<ZF, WARPS>(g, r, hit, red_s, lo, hi, fwd, [&] {
        tma::mbar_init(&bar[0], 1);
        tma::mbar_init(&bar[1], 1);
        tma::fence_barrier_init();
        tma::prefetch_map(map);
        *dead = 0;
    });
    if (lo == INT_MAX) return;  // no ray of the block hits the volume
    const int nslab = (hi - lo) / SLAB + 1;
    auto slab_m0 = [&](int k) { return fwd ? lo + k * SLAB : hi - (SLAB - 1) - k * SLAB; };

    // slab 0
    int f0, y0;
    {
        slab::ray_box_low<ZF, SLAB>(g, r, hit, slab_m0(0), f0, y0);
        slab::block_min2<WARPS>(f0, y0, red[0]);
        if (f0 == INT_MAX) f0 = y0 = 0;
        f0 &= ~(ALIGN - 1);  // the box's innermost coordinate starts on 16 bytes (rounded down, also below 0)
        if (threadIdx.x == 0) {
            tma::mbar_arrive_expect_tx(&bar[0], BOX_BYTES);
            tma::load_box_3d(buf, map, f0, y0, slab_m0(0), &bar[0]);
        }
    }
    bool gave_up = false;  // a copy did not land: the remaining samples read global memory
    int drain0 = 0, drain1 = -1;  // after a give-up: the slabs whose copies may still be in flight
    for (int k = 0; k < nslab; ++k) {
        // issue slab k+1 into the other buffer (free since the barrier that ended slab k-1)
        int fn = 0, yn = 0;
        if (k + 1 < nslab && !gave_up) {
            slab::ray_box_low<ZF, SLAB>(g, r, hit, slab_m0(k + 1), fn, yn);
            slab::block_min2<WARPS>(fn, yn, red[(k + 1) & 1]);
            if (fn == INT_MAX) fn = yn = 0;
            fn &= ~(ALIGN - 1);
            if (threadIdx.x == 0) {
                const int nb = (k + 1) & 1;
                tma::mbar_arrive_expect_tx(&bar[nb], BOX_BYTES);
                tma::load_box_3d(buf + nb * BOXN, map, fn, yn, slab_m0(k + 1), &bar[nb]);
            }
        }
        bool staged = false;
        if (!gave_up) {
            staged = tma::mbar_wait(&bar[k & 1], (k >> 1) & 1, WAIT_CYCLES);
            if (!staged) {  // an error: reported through the status word, the block stops staging
                *dead = 1;
                if (status) atomicExch(status, STT_WAIT_TIMEOUT_FLAG);
            }
        }
        const T *bx = buf + (k & 1) * BOXN;
        const int m0 = slab_m0(k);
        // the base plane of a cell along the slab axis, and whether it belongs to a later slab
        auto plane = [&](const FpCell &c) { return ZF ? c.ix : c.iz; };
        auto is_later = [&](int bs) { return fwd ? bs > m0 + SLAB - 1 : bs < m0; };
        // a cell's 8 corners: from the staged box when they lie in it, else global memory
        auto corners = [&](const FpCell &c, int bs, float v[8]) {
            const unsigned of = (unsigned)((ZF ? c.iz : c.ix) - f0), oy = (unsigned)(c.iy - y0),
                           os = (unsigned)(bs - m0);
            if (staged && of <= FB - 2 && oy <= YB - 2 && os <= SB - 2) {
                const T *q = bx + (os * YB + oy) * FB + of;
                constexpr int P = FB * YB;  // plane stride
                if (!ZF) {  // fast = x, slow = z
                    v[0] = sm_voxel(q), v[1] = sm_voxel(q + 1), v[2] = sm_voxel(q + FB), v[3] = sm_voxel(q + FB + 1);
                    v[4] = sm_voxel(q + P), v[5] = sm_voxel(q + P + 1), v[6] = sm_voxel(q + P + FB),
                    v[7] = sm_voxel(q + P + FB + 1);
                } else {  // fast = z, slow = x
                    v[0] = sm_voxel(q), v[4] = sm_voxel(q + 1), v[2] = sm_voxel(q + FB), v[6] = sm_voxel(q + FB + 1);
                    v[1] = sm_voxel(q + P), v[5] = sm_voxel(q + P + 1), v[3] = sm_voxel(q + P + FB),
                    v[7] = sm_voxel(q + P + FB + 1);
                }
            } else {
                fp_corners<ZF ? 2 : 0, int>(src, st, c, v);
            }
        };
        // one sample: false (and nothing added) when it belongs to a later slab
        auto take = [&](const float p[3]) -> bool {
            FpCell c;
            fp_cell(g, p, c);
            const int bs = plane(c);
            if (is_later(bs)) return false;
            float v[8];
            corners(c, bs, v);
            acc.add(__fmul_rn(trilerp(v, c), g.sd));
            return true;
        };
        // two consecutive samples: how many were added before one belonged to a later slab
        auto take2 = [&](const float pa[3], const float pb[3]) -> int {
            FpCell ca, cb;
            fp_cell2(g, pa, pb, ca, cb);
            const int ba = plane(ca), bb = plane(cb);
            if (is_later(ba)) return 0;
            float va[8], vb[8];
            corners(ca, ba, va);
            if (is_later(bb)) {
                acc.add(__fmul_rn(trilerp(va, ca), g.sd));
                return 1;
            }
            corners(cb, bb, vb);
            const float2 s2 = __fmul2_rn(trilerp2(va, vb, ca, cb), make_float2(g.sd, g.sd));
            acc.add(s2.x);
            acc.add(s2.y);
            return 2;
        };
        bool later = false;
        while (!later && m.peek()) {
            if (m.phase == 0) {  // the entry sample
                later = !take(m.pos);
                if (!later) m.advance();
                continue;
            }
            // the rest of the current segment, from registers; (x, y) and
            // (t, z) advance as packed pairs (the same float additions)
            float t = m.t, p[3] = {m.pos[0], m.pos[1], m.pos[2]};
            int n = m.n;
            const float2 sxy = make_float2(m.d.step[0], m.d.step[1]), stz = make_float2(m.sd, m.d.step[2]);
            do {
                const float2 xy1 = __fadd2_rn(make_float2(p[0], p[1]), sxy);
                const float2 tz1 = __fadd2_rn(make_float2(t, p[2]), stz);
                if (PK && n + 1 < m.cap && tz1.x < m.tb) {  // the segment holds this sample and the next
                    const float q[3] = {xy1.x, xy1.y, tz1.y};
                    const int took = take2(p, q);
                    if (took < 2) {
                        if (took == 1) {
                            t = tz1.x;
                            p[0] = q[0], p[1] = q[1], p[2] = q[2];
                            ++n;
                        }
                        later = true;
                        break;
                    }
                    const float2 xy2 = __fadd2_rn(xy1, sxy), tz2 = __fadd2_rn(tz1, stz);
                    t = tz2.x;
                    p[0] = xy2.x, p[1] = xy2.y, p[2] = tz2.y;
                    n += 2;
                } else {
                    if (!take(p)) {
                        later = true;
                        break;
                    }
                    t = tz1.x;
                    p[0] = xy1.x, p[1] = xy1.y, p[2] = tz1.y;
                    ++n;
                }
            } while (n < m.cap && t < m.tb);
            m.t = t;
            m.n = n;
#pragma unroll
            for (int a = 0; a < 3; ++a) m.pos[a] = p[a];
        }
        __syncthreads();  // every ray is done with buffer k&1 before slab k+2 is loaded into it
        if (*dead != 0 && !gave_up) {
            // slab k's copy did not land in time, and slab k+1's was issued before that wait
            drain0 = k;
            drain1 = k + 1 < nslab ? k + 1 : k;
        }
        gave_up = *dead != 0;
        f0 = fn;
        y0 = yn;
    }
    if (gave_up) {
        // No block exits with a bulk copy still writing into its shared memory:
        // wait (again bounded) for every copy issued but not seen to land.  The
        // buffers are not read again; the samples above went to global memory.
        for (int k = drain0; k <= drain1; ++k) tma::mbar_wait(&bar[k & 1], (k >> 1) & 1, WAIT_CYCLES);
    }
    // samples outside the planes the slabs covered
    while (m.peek()) {
        FpCell c;
        fp_cell(g, m.pos, c);
        float v[8];
        fp_corners<ZF ? 2 : 0, int>(src, st, c, v);
        acc.add(__fmul_rn(trilerp(v, c), g.sd));
        m.advance();
    }
}

// k_fp_corr (GenerateImage_MT + the correction of ST_Tomography.cpp:667-676)
// with slab-staged gathers.  map_x covers `vol` (x-fastest), map_z `vol_t`
// (z-fastest), both with the box of BX; T and B are the storages of the
// volume and of the sinogram stack.
template <class BX, bool PK, typename T = float, typename B = float>
__global__ void __launch_bounds__(32 * WARPS) k_fp_corr_slab(const GeomDev g, const ViewRec *__restrict__ views,
                                                      const __grid_constant__ CUtensorMap map_x,
                                                      const __grid_constant__ CUtensorMap map_z,
                                                      const T *__restrict__ vol, const T *__restrict__ vol_t,
                                                      const ViewSel sel, const B *__restrict__ b_stack,
                                                      float *__restrict__ raylen_state, float *__restrict__ corr,
                                                      unsigned long long corr_surf, int *status) {
    __shared__ alignas(128) T buf[2 * BX::N];
    __shared__ uint64_t bar[2];
    __shared__ int red[2][2 * WARPS];
    __shared__ int red_s[3 * WARPS];
    __shared__ int dead;
    const int i = blockIdx.x * 32 + (threadIdx.x & 31);
    const int j = blockIdx.y * WARPS + (threadIdx.x >> 5);
    const bool valid = i < g.W && j < g.H;
    int local;
    const int view = sel_view(sel, local);
    const ViewRec &vr = views[view];
    if (!view_staged<T>(vr)) return;  // the gather kernel projects this view (uniform over the block)
    Ray r;
    bool hit = false;
    if (valid) {
        make_ray(g, vr, i, j, r);
        hit = r.tnear < r.tfar;
    }
    Kahan acc{0.0f, 0.0f};
    if (vol_t && vr.layout == 1)
        slab_ray_sum<true, BX, PK, T>(g, &map_z, vol_t, hit, r, buf, bar, red_s, red, &dead, status, acc);
    else
        slab_ray_sum<false, BX, PK, T>(g, &map_x, vol, hit, r, buf, bar, red_s, red, &dead, status, acc);
    if (!valid) return;
    const B *b = b_stack + (size_t)local * g.W * g.H;
    const size_t pix = i + (size_t)j * g.W;
    float L;
    if (hit) {
        L = r.tfar - r.tnear;
        if (raylen_state) raylen_state[pix] = L;
    } else {
        L = raylen_state ? raylen_state[pix] : 0.0f;
    }
    const float c = __fdiv_rn(__fsub_rn(ld_voxel(b + pix), acc.s), __fadd_rn(L, 1.0f));
    corr[pix] = c;
    if (corr_surf) surf2DLayeredwrite(c, corr_surf, i * (int)sizeof(float), j, 0, cudaBoundaryModeZero);
}

PFN_cuTensorMapEncodeTiled_v12000 encode_fn() {
    static const PFN_cuTensorMapEncodeTiled_v12000 fn = [] {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess) {
            cudaGetLastError();
            return (PFN_cuTensorMapEncodeTiled_v12000) nullptr;
        }
        return reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }();
    return fn;
}

// A 3D tensor map (fast, mid, slow) over `ptr` with the slab box `box`:
// FP32 elements, or 16-bit ones (BF16 bits, copied as they are).  The rows
// must be whole multiples of 16 bytes (fast a multiple of 4 or 8 elements).
bool encode_box_map(CUtensorMap *m, const void *ptr, size_t esize, int fast, int mid, int slow,
                    const cuuint32_t box[3]) {
    const PFN_cuTensorMapEncodeTiled_v12000 fn = encode_fn();
    if (!fn || !ptr || (reinterpret_cast<uintptr_t>(ptr) & 15) || ((size_t)fast * esize) % 16) return false;
    const cuuint64_t dims[3] = {(cuuint64_t)fast, (cuuint64_t)mid, (cuuint64_t)slow};
    const cuuint64_t strides[2] = {(cuuint64_t)fast * esize, (cuuint64_t)fast * mid * esize};
    const cuuint32_t estr[3] = {1, 1, 1};
    const CUtensorMapDataType dt = esize == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_UINT16;
    return fn(m, dt, 3, const_cast<void *>(ptr), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
              CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

}  // namespace

bool encode_planes_map(CUtensorMap *m, const float *ptr, int nx, int ny, int nz, int nc, const unsigned box[4]) {
    const PFN_cuTensorMapEncodeTiled_v12000 fn = encode_fn();
    if (!fn || !ptr || (reinterpret_cast<uintptr_t>(ptr) & 15) || (nx & 3) || ((box[0] * sizeof(float)) & 15))
        return false;
    const cuuint64_t dims[4] = {(cuuint64_t)nx, (cuuint64_t)ny, (cuuint64_t)nz, (cuuint64_t)nc};
    const cuuint64_t row = (cuuint64_t)nx * sizeof(float);
    const cuuint64_t strides[3] = {row, row * ny, row * ny * nz};
    const cuuint32_t bx[4] = {box[0], box[1], box[2], box[3]};
    const cuuint32_t estr[4] = {1, 1, 1, 1};
    return fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, const_cast<float *>(ptr), dims, strides, bx, estr,
              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

namespace {

template <class BX>
void box_dims(cuuint32_t box[3]) {
    box[0] = BX::FB;
    box[1] = BX::YB;
    box[2] = BX::SB;
}

template <class BX, bool PK, typename T, typename B>
cudaError_t launch_slab(const GeomDev &g, const ViewRec *views, const FpSlabMaps &m, const T *vol,
                        const T *vol_t, const ViewSel &sel, const B *b_stack, float *raylen_state, float *corr,
                        cudaStream_t s, unsigned long long corr_surf, int *status) {
    static const bool carve = [] {
        cudaFuncSetAttribute(k_fp_corr_slab<BX, PK, T, B>, cudaFuncAttributePreferredSharedMemoryCarveout,
                             cudaSharedmemCarveoutMaxShared);
        cudaGetLastError();
        return true;
    }();
    (void)carve;
    k_fp_corr_slab<BX, PK, T, B><<<dim3((g.W + 31) / 32, (g.H + WARPS - 1) / WARPS, 1), 32 * WARPS, 0, s>>>(
        g, views, m.x, m.z, vol, vol_t, sel, b_stack, raylen_state, corr, corr_surf, status);
    return cudaGetLastError();
}

}  // namespace

const char *slab_variant_name(int v) {
    static const char *names[kSlabVariants] = {"box 48x8x12", "box 48x8x8", "box 64x8x10", "box 40x8x16",
                                               "box 48x8x12, packed pairs", "box 48x8x8, packed pairs",
                                               "box 64x8x10, packed pairs", "box 40x8x16, packed pairs"};
    return v >= 0 && v < kSlabVariants ? names[v] : "?";
}

static bool make_maps(const GeomDev &g, const void *vol, const void *vol_t, size_t esize, FpSlabMaps &m,
                      int variant) {
    m = FpSlabMaps{};
    if ((long long)g.nx * g.ny * g.nz >= (1LL << 31)) return false;  // 32-bit fallback offsets
    if (variant < 0 || variant >= kSlabVariants) return false;
    cuuint32_t box[3];
    switch (variant & 3) {  // variants 4..7: the boxes of 0..3 with packed sample pairs
    case 1: box_dims<Box1>(box); break;
    case 2: box_dims<Box2>(box); break;
    case 3: box_dims<Box3>(box); break;
    default: box_dims<Box0>(box); break;
    }
    if (!encode_box_map(&m.x, vol, esize, g.nx, g.ny, g.nz, box)) return false;
    if (vol_t && !encode_box_map(&m.z, vol_t, esize, g.nz, g.ny, g.nx, box)) return false;
    m.ok = 1;
    m.has_z = vol_t != nullptr;
    m.variant = variant;
    m.esize = (int)esize;
    return true;
}

bool make_fp_slab_maps(const GeomDev &g, const float *vol, const float *vol_t, FpSlabMaps &m, int variant) {
    return make_maps(g, vol, vol_t, sizeof(float), m, variant);
}

bool make_fp_slab_maps(const GeomDev &g, const unsigned short *vol, const unsigned short *vol_t, FpSlabMaps &m,
                       int variant) {
    return make_maps(g, vol, vol_t, sizeof(unsigned short), m, variant & 3);  // scalar boxes in BF16
}

cudaError_t launch_fp_corr_slab(const GeomDev &g, const ViewRec *views, const FpSlabMaps &m, const unsigned short *vol,
                                const unsigned short *vol_t, const ViewSel &sel, const unsigned short *b_stack,
                                float *raylen_state, float *corr, cudaStream_t s, unsigned long long corr_surf,
                                int *status) {
    if (!m.ok || m.esize != 2 || (vol_t && !m.has_z)) return cudaErrorInvalidValue;
    typedef unsigned short U;
#define STT_SLAB16(BOX) \
    launch_slab<BOX, false, U, U>(g, views, m, vol, vol_t, sel, b_stack, raylen_state, corr, s, corr_surf, status)
    switch (m.variant & 3) {
    case 1: return STT_SLAB16(Box1);
    case 2: return STT_SLAB16(Box2);
    case 3: return STT_SLAB16(Box3);
    default: return STT_SLAB16(Box0);
    }
#undef STT_SLAB16
}

cudaError_t launch_fp_corr_slab(const GeomDev &g, const ViewRec *views, const FpSlabMaps &m, const float *vol,
                                const float *vol_t, const ViewSel &sel, const float *b_stack, float *raylen_state,
                                float *corr, cudaStream_t s, unsigned long long corr_surf, int *status) {
    if (!m.ok || m.esize != 4 || (vol_t && !m.has_z)) return cudaErrorInvalidValue;
#define STT_SLAB(B, P) launch_slab<B, P, float, float>(g, views, m, vol, vol_t, sel, b_stack, raylen_state, corr, s, \
                                                      corr_surf, status)
    switch (m.variant) {
    case 1: return STT_SLAB(Box1, false);
    case 2: return STT_SLAB(Box2, false);
    case 3: return STT_SLAB(Box3, false);
    case 4: return STT_SLAB(Box0, true);
    case 5: return STT_SLAB(Box1, true);
    case 6: return STT_SLAB(Box2, true);
    case 7: return STT_SLAB(Box3, true);
    default: return STT_SLAB(Box0, false);
    }
#undef STT_SLAB
}

}  // namespace stt
