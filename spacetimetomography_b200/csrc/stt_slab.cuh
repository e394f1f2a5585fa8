// stt_slab.cuh -- the slab walk shared by the kernels that stage a block's
// share of the volume in shared memory (k_fp_slab.cu: the forward projector
// reads its taps from a staged box; k_bp_slab.cu: the ray-driven
// backprojection accumulates into one).  A block is a 32 x NW tile of nearly
// parallel rays; it walks slabs of planes across the axis the rays mostly run
// along, and per slab a box (fast, y, slow) holds every trilinear corner of
// the samples whose base plane lies in the slab.
#pragma once

#include <climits>

#include "stt_internal.cuh"

namespace stt {
namespace slab {

__device__ __forceinline__ int warp_min(int v) { return __reduce_min_sync(0xffffffffu, v); }

// Block-wide minima of (a, b) over NW warps, through red[0..2*NW).  One barrier.
template <int NW>
__device__ __forceinline__ void block_min2(int &a, int &b, int *red) {
    a = warp_min(a);
    b = warp_min(b);
    const int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) {
        red[2 * w] = a;
        red[2 * w + 1] = b;
    }
    __syncthreads();
    a = red[0];
    b = red[1];
#pragma unroll
    for (int k = 1; k < NW; ++k) {
        a = min(a, red[2 * k]);
        b = min(b, red[2 * k + 1]);
    }
}

// Axes of a slab walk.  ZF = false: rays mostly along z; slabs across z
// (slow), the box's fast axis x.  ZF = true: rays mostly along x; slabs
// across x, the box's fast axis z.
template <bool ZF>
struct Axes {
    static constexpr int F = ZF ? 2 : 0;  // fast axis of the box
    static constexpr int S = ZF ? 0 : 2;  // slab axis
};

// Lowest (fast, y) base coordinates of the taps of this ray's samples whose
// slab coordinate lies in [m0, m0 + SLAB), with a voxel of margin; INT_MAX
// when the ray has none there.
template <bool ZF, int SLAB>
__device__ __forceinline__ void ray_box_low(const GeomDev &g, const Ray &r, bool hit, int m0, int &lf, int &ly) {
    constexpr int F = Axes<ZF>::F, S = Axes<ZF>::S;
    lf = INT_MAX;
    ly = INT_MAX;
    if (!hit) return;
    const float ta = __fdividef((float)m0 - 0.5f - r.vz[S], r.vu[S]);
    const float tb = __fdividef((float)(m0 + SLAB) + 0.5f - r.vz[S], r.vu[S]);
    const float tl = fmaxf(fminf(ta, tb), r.tnear - g.sd), th = fminf(fmaxf(ta, tb), r.tfar + g.sd);
    if (!(tl <= th)) return;
    const int dimF = ZF ? g.nz : g.nx;
    const float f = fminf(r.vz[F] + r.vu[F] * tl, r.vz[F] + r.vu[F] * th);
    const float y = fminf(r.vz[1] + r.vu[1] * tl, r.vz[1] + r.vu[1] * th);
    lf = (int)floorf(fminf(fmaxf(f, 0.0f), (float)(dimF - 1))) - 1;
    ly = (int)floorf(fminf(fmaxf(y, 0.0f), (float)(g.ny - 1))) - 1;
}

// Highest (fast, y) coordinates of the +1 corners of this ray's samples
// whose slab coordinate lies in [m0, m0 + SLAB), with a voxel of margin;
// INT_MIN when the ray has none there.
template <bool ZF, int SLAB>
__device__ __forceinline__ void ray_box_high(const GeomDev &g, const Ray &r, bool hit, int m0, int &hf, int &hy) {
    constexpr int F = Axes<ZF>::F, S = Axes<ZF>::S;
    hf = INT_MIN;
    hy = INT_MIN;
    if (!hit) return;
    const float ta = __fdividef((float)m0 - 0.5f - r.vz[S], r.vu[S]);
    const float tb = __fdividef((float)(m0 + SLAB) + 0.5f - r.vz[S], r.vu[S]);
    const float tl = fmaxf(fminf(ta, tb), r.tnear - g.sd), th = fminf(fmaxf(ta, tb), r.tfar + g.sd);
    if (!(tl <= th)) return;
    const int dimF = ZF ? g.nz : g.nx;
    const float f = fmaxf(r.vz[F] + r.vu[F] * tl, r.vz[F] + r.vu[F] * th);
    const float y = fmaxf(r.vz[1] + r.vu[1] * tl, r.vz[1] + r.vu[1] * th);
    hf = (int)floorf(fminf(fmaxf(f, 0.0f), (float)(dimF - 1))) + 2;
    hy = (int)floorf(fminf(fmaxf(y, 0.0f), (float)(g.ny - 1))) + 2;
}

// The base planes [lo, hi] (along the slab axis) the block's rays span and
// whether most of them run up that axis; lo = INT_MAX when no ray of the
// block hits the volume.  red_s: 3*NW ints; one barrier.  Thread 0 runs
// `init0` before the barrier (barrier set-up of the caller).
template <bool ZF, int NW, typename Init>
__device__ __forceinline__ void block_span(const GeomDev &g, const Ray &r, bool hit, int *red_s, int &lo, int &hi,
                                           bool &fwd, Init &&init0) {
    constexpr int S = Axes<ZF>::S;
    const int dimS = ZF ? g.nx : g.nz;
    int l = INT_MAX, nh = INT_MAX, up = 0;
    if (hit) {
        const float a = r.vz[S] + r.vu[S] * r.tnear, b = r.vz[S] + r.vu[S] * r.tfar;
        const float pl = fminf(fmaxf(fminf(a, b), 0.0f), (float)(dimS - 1));
        const float ph = fminf(fmaxf(fmaxf(a, b), 0.0f), (float)(dimS - 1));
        l = min((int)pl, dimS - 2);
        nh = -min((int)ph, dimS - 2);
        up = r.vu[S] > 0.0f ? 1 : -1;
    }
    l = warp_min(l);
    nh = warp_min(nh);
    up = __reduce_add_sync(0xffffffffu, up);
    const int w = threadIdx.x >> 5;
    if ((threadIdx.x & 31) == 0) {
        red_s[3 * w] = l;
        red_s[3 * w + 1] = nh;
        red_s[3 * w + 2] = up;
    }
    if (threadIdx.x == 0) init0();
    __syncthreads();
    l = red_s[0];
    nh = red_s[1];
    up = red_s[2];
#pragma unroll
    for (int k = 1; k < NW; ++k) {
        l = min(l, red_s[3 * k]);
        nh = min(nh, red_s[3 * k + 1]);
        up += red_s[3 * k + 2];
    }
    lo = l;
    hi = -nh;
    fwd = up >= 0;
}

}  // namespace slab
}  // namespace stt
