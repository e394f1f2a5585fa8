// warp_dev.cuh -- device helpers of the tricubic warp (S/ST_Tomo/warping.h:49-114):
// grid mapping, the CImg Catmull-Rom stencil, the 8-corner clamp and the trace.
#pragma once

#include "stt_internal.cuh"

namespace stt {
namespace warpdev {

struct Dim3i {
    int x, y, z;
};

// world (aabb = [0,dim]) -> cell grid, clamped to [1, dim-2] (warping.h:54-62).
__device__ __forceinline__ float to_grid(float p, int dim, bool *clamped) {
    float gw = __fdiv_rn(__fmul_rn((float)dim, p), (float)dim);
    float gq = gw - 0.5f;
    const float hi = (float)(dim - 2), lo = 1.0f;
    bool c = !(gq >= lo && gq <= hi);
    gq = (gq < hi) ? gq : hi;  // std::min(hi, g)
    gq = (lo < gq) ? gq : lo;  // std::max(lo, g)
    if (clamped) *clamped = c;
    return gq;
}

// Stencil of CImg::_cubic_atXYZ (CImg.h:13429-13438) for an already clamped
// coordinate: taps x-1, x, x+1 (only when the fraction is non-zero), x+2,
// clamped to the image.
struct Stencil {
    int xo[4], yo[4], zo[4];  // element offsets per axis
    float wx[4], wy[4], wz[4];
    float dx, dy, dz;
    long long c0;            // linear index of the integer corner (ix,iy,iz)
    int sx1, sy1, sz1;       // offsets to the +1 corner (for the 8-corner min/max)
};

__device__ __forceinline__ void axis_taps(float g, int dim, int stride, int o[4], float &d, int &ix) {
    int x = (int)g;
    d = g - (float)x;
    const int p = x - 1 < 0 ? 0 : x - 1;
    const int n = d > 0.0f ? x + 1 : x;
    const int a = x + 2 >= dim ? dim - 1 : x + 2;
    o[0] = p * stride;
    o[1] = x * stride;
    o[2] = n * stride;
    o[3] = a * stride;
    ix = x;
}

__device__ __forceinline__ void make_stencil(const Dim3i d, const float gq[3], Stencil &s) {
    int ix, iy, iz;
    axis_taps(gq[0], d.x, 1, s.xo, s.dx, ix);
    axis_taps(gq[1], d.y, d.x, s.yo, s.dy, iy);
    axis_taps(gq[2], d.z, d.x * d.y, s.zo, s.dz, iz);
    cr_weights(s.dx, s.wx);
    cr_weights(s.dy, s.wy);
    cr_weights(s.dz, s.wz);
    s.c0 = ix + (long long)iy * d.x + (long long)iz * d.x * d.y;
    s.sx1 = 1;
    s.sy1 = d.x;
    s.sz1 = d.x * d.y;
}

// sample_image (warping.h:49-88): Catmull-Rom value clamped to the min/max of
// the 8 corners of the cell.
__device__ __forceinline__ float sample_clamped(const float *__restrict__ img, const Stencil &s) {
    float val = 0.0f;
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        float yv = 0.0f;
#pragma unroll
        for (int b = 0; b < 4; ++b) {
            const float *row = img + s.yo[b] + s.zo[c];
            float xv = s.wx[0] * __ldg(row + s.xo[0]) + s.wx[1] * __ldg(row + s.xo[1]) +
                       s.wx[2] * __ldg(row + s.xo[2]) + s.wx[3] * __ldg(row + s.xo[3]);
            yv += s.wy[b] * xv;
        }
        val += s.wz[c] * yv;
    }
    const float *c0 = img + s.c0;
    float mn = __ldg(c0), mx = mn;
    const int off[7] = {s.sx1, s.sx1 + s.sy1, s.sy1, s.sz1, s.sx1 + s.sz1, s.sx1 + s.sy1 + s.sz1,
                        s.sy1 + s.sz1};
#pragma unroll
    for (int k = 0; k < 7; ++k) {
        float v = __ldg(c0 + off[k]);
        mn = (v < mn) ? v : mn;
        mx = (mx < v) ? v : mx;
    }
    float inner = (val < mx) ? val : mx;
    return (mn < inner) ? inner : mn;
}

// ---- forward sampler with 32-bit offsets and shared rows -------------------
// The grid coordinate g is already clamped to [1, dim-2], so with x = (int)g:
//  * taps x-1, x, x+1 are always inside the image.  CImg takes x instead of
//    x+1 when the fraction is 0, where the Catmull-Rom weight of that tap is
//    exactly 0: for finite data both give the same sum, and x+1 is then also
//    the cell's +1 corner, so the 8 corners are taps 1..2 on every axis and
//    need no loads of their own;
//  * tap x+2 leaves the image only when x = dim-2, i.e. g = dim-2 exactly and
//    the fraction is 0, where its weight is exactly 0: the tap is skipped
//    (a zero row or tap adds nothing), so no load ever leaves the image.
struct Axis {
    int lo;      // element offset of tap 0 (x-1) along this axis
    bool t3;     // tap 3 (x+2) inside the image
    float w[4];  // Catmull-Rom weights of the fraction
};

__device__ __forceinline__ void axis_setup(float g, int stride, int dim, Axis &a) {
    const int x = (int)g;
    cr_weights(g - (float)x, a.w);
    a.lo = (x - 1) * stride;
    a.t3 = x + 2 < dim;
}

struct Cell {
    Axis x, y, z;
    int sy, sz;  // row and plane strides
};

__device__ __forceinline__ void cell_setup(const Dim3i d, const float g[3], Cell &c) {
    c.sy = d.x;
    c.sz = d.x * d.y;
    axis_setup(g[0], 1, d.x, c.x);
    axis_setup(g[1], c.sy, d.y, c.y);
    axis_setup(g[2], c.sz, d.z, c.z);
}

// A tap: read-only global load (a BF16-stored image widened exactly), or a
// plain load when SHARED (img then points into shared memory, which the
// global read-only path cannot address).
// RW: a plain load of a global image that the running launch has written
// (the persistent iteration's Y_bc).
template <bool SHARED, typename T, bool RW = false>
__device__ __forceinline__ float ld_tap(const T *p) {
    if constexpr (SHARED) return *p;
    else if constexpr (RW) return ld_stored(p);
    else return ld_voxel(p);
}

// sample_image (warping.h:49-88) of NC planes that share one cell: the
// Catmull-Rom value of each, clamped to the min/max of its 8 cell corners.
// Plane p starts at img + p * pstride.  The sums run in the order of
// sample_clamped above (x taps, then rows, then planes), so both give the
// same bits.
template <int NC, bool SHARED = false, typename T = float, bool RW = false>
__device__ __forceinline__ void sample_cell(const T *__restrict__ img, int pstride, const Cell &s,
                                            float out[NC]) {
    float val[NC], mn[NC], mx[NC];
#pragma unroll
    for (int p = 0; p < NC; ++p) {
        val[p] = 0.0f;
        mn[p] = INFINITY;
        mx[p] = -INFINITY;
    }
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        if (c == 3 && !s.z.t3) break;
        float yv[NC];
#pragma unroll
        for (int p = 0; p < NC; ++p) yv[p] = 0.0f;
#pragma unroll
        for (int b = 0; b < 4; ++b) {
            if (b == 3 && !s.y.t3) break;
            const int row = s.x.lo + s.y.lo + b * s.sy + s.z.lo + c * s.sz;
#pragma unroll
            for (int p = 0; p < NC; ++p) {
                const T *r = img + p * pstride + row;
                const float t0 = ld_tap<SHARED, T, RW>(r), t1 = ld_tap<SHARED, T, RW>(r + 1),
                            t2 = ld_tap<SHARED, T, RW>(r + 2);
                const float t3 = s.x.t3 ? ld_tap<SHARED, T, RW>(r + 3) : 0.0f;
                const float xv = s.x.w[0] * t0 + s.x.w[1] * t1 + s.x.w[2] * t2 + s.x.w[3] * t3;
                yv[p] += s.y.w[b] * xv;
                if ((b == 1 || b == 2) && (c == 1 || c == 2)) {
                    mn[p] = fminf(mn[p], fminf(t1, t2));
                    mx[p] = fmaxf(mx[p], fmaxf(t1, t2));
                }
            }
        }
#pragma unroll
        for (int p = 0; p < NC; ++p) val[p] += s.z.w[c] * yv[p];
    }
#pragma unroll
    for (int p = 0; p < NC; ++p) out[p] = fmaxf(mn[p], fminf(val[p], mx[p]));
}

// The trace of voxel (i, j, k) through vel (warping.h:100-114) with step dt
// (the gather form's arithmetic: the exact centre read, the Catmull-Rom
// velocity sample at the half-traced point) and the cell of its end point.
__device__ __forceinline__ void trace_cell(const Dim3i d, const float *__restrict__ vel, float dt, int i, int j,
                                           int k, Cell &s) {
    const int n = d.x * d.y * d.z;
    const float h = -dt;
    // cell centre (warping.h:25-29); the velocity there is an exact node read
    const float p[3] = {(float)i + 0.5f, (float)j + 0.5f, (float)k + 0.5f};
    const int ci = min(max(i, 1), d.x - 2), cj = min(max(j, 1), d.y - 2), ck = min(max(k, 1), d.z - 2);
    const int c = ci + cj * d.x + ck * d.x * d.y;
    const float v1[3] = {__ldg(vel + c), __ldg(vel + n + c), __ldg(vel + 2 * n + c)};
    // trace (warping.h:100-114): p2 = p + h v(p); p0 = p2 - h v(p2); q = p2 + (p - p0)/2
    float p2[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) p2[a] = __fadd_rn(p[a], __fmul_rn(h, v1[a]));
    const float g2[3] = {to_grid(p2[0], d.x, nullptr), to_grid(p2[1], d.y, nullptr),
                         to_grid(p2[2], d.z, nullptr)};
    Cell s2;
    cell_setup(d, g2, s2);
    float v2[3];
    sample_cell<3>(vel, n, s2, v2);
    float q[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const float p0 = __fsub_rn(p2[a], __fmul_rn(h, v2[a]));
        q[a] = __fadd_rn(p2[a], __fmul_rn(0.5f, __fsub_rn(p[a], p0)));
    }
    const float gq[3] = {to_grid(q[0], d.x, nullptr), to_grid(q[1], d.y, nullptr), to_grid(q[2], d.z, nullptr)};
    cell_setup(d, gq, s);
}

__device__ __forceinline__ void trace(const Dim3i d, const float *__restrict__ vel, size_t n, int i,
                                      int j, int k, float h, float q[3], float p2[3], float v1[3],
                                      float v2[3]) {
    // cell centre (warping.h:25-29) and the velocity there (an exact node read)
    const float p[3] = {(float)i + 0.5f, (float)j + 0.5f, (float)k + 0.5f};
    const int ci = min(max(i, 1), d.x - 2), cj = min(max(j, 1), d.y - 2), ck = min(max(k, 1), d.z - 2);
    const size_t c = ci + (size_t)cj * d.x + (size_t)ck * d.x * d.y;
#pragma unroll
    for (int a = 0; a < 3; ++a) v1[a] = __ldg(vel + a * n + c);
    // trace (warping.h:100-114): p2 = p + h v(p); p0 = p2 - h v(p2); q = p2 + (p - p0)/2
#pragma unroll
    for (int a = 0; a < 3; ++a) p2[a] = __fadd_rn(p[a], __fmul_rn(h, v1[a]));
    float g2[3] = {to_grid(p2[0], d.x, nullptr), to_grid(p2[1], d.y, nullptr), to_grid(p2[2], d.z, nullptr)};
    Stencil s2;
    make_stencil(d, g2, s2);
#pragma unroll
    for (int a = 0; a < 3; ++a) v2[a] = sample_clamped(vel + a * n, s2);
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        float p0 = __fsub_rn(p2[a], __fmul_rn(h, v2[a]));
        q[a] = __fadd_rn(p2[a], __fmul_rn(0.5f, __fsub_rn(p[a], p0)));
    }
}

}  // namespace warpdev
}  // namespace stt
