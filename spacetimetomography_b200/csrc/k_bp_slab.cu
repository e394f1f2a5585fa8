// k_bp_slab.cu -- the scatter of the ray-driven backprojection with a
// shared-memory box per slab.
//
// The reference's backprojection mode (S/ImageFormationModel/
// SingleScalarVolume.core.h:73-84, 128-143, reached through the second march
// of ST_Tomography.cpp:735-739) adds c*w and w to the 8 trilinear corners of
// every sample of every ray.  Done with global atomics that is 8 vector
// atomics per sample, about 14 per voxel and view at 512^3 / 1024^2, and the
// scatter runs at the L2's atomic rate.  Here a block of 32 x 4 nearly
// parallel rays walks slabs of planes across the axis its rays run along (the
// slab walk of the staged projector, stt_slab.cuh); per slab its samples add
// into a shared-memory box that covers the block's footprint in the slab
// (shared atomics), and after a barrier every touched cell of the box goes to
// the global accumulator with one float2 atomic and is cleared.  A sample
// whose corners are not in the box (the march's pre-entry restart, a footprint
// the estimate missed) adds them to global memory directly, and so do the
// samples left after the last slab.  The terms are those of the global
// scatter; only the order of the float additions differs (which atomics make
// order-nondeterministic anyway).
#include <climits>

#include "stt_internal.cuh"
#include "stt_kernels.h"
#include "stt_slab.cuh"

namespace stt {

namespace {

constexpr int WARPS = 4;                     // a block is 32 x WARPS detector pixels, one warp per row
constexpr int FB = 48, YB = 8, SB = 12;      // the box (fast, y, slab axis); the footprint is usually smaller
constexpr int BOXN = FB * YB * SB;
constexpr int SLAB = SB - 1;                 // base planes per slab; the box also holds their +1 plane

// The 8 corners of one sample to global memory (k_bp_ray_scatter's update).
__device__ __forceinline__ void scatter_global(const GeomDev &g, const float p[3], float c, float2 *__restrict__ acc) {
    Taps t;
    make_taps(g, p, t);
    float w[8];
    tri_weights(t, w);
    scatter_corners(acc, t, c, w);
}

template <bool ZF>
__device__ __forceinline__ void scatter_slabs(const GeomDev &g, const Ray &r, bool hit, float c,
                                              float2 *__restrict__ acc, float *bc, float *bw, int *red_s,
                                              int (*red)[2 * WARPS]) {
    MarchGen m;
    if (hit) m.init(g, r);
    else m.phase = 2;
    int lo, hi;
    bool fwd;
    slab::block_span<ZF, WARPS>(g, r, hit, red_s, lo, hi, fwd, [] {});
    if (lo == INT_MAX) return;  // no ray of the block hits the volume (uniform)
    const int nslab = (hi - lo) / SLAB + 1;
    auto slab_m0 = [&](int k) { return fwd ? lo + k * SLAB : hi - (SLAB - 1) - k * SLAB; };
    for (int k = 0; k < nslab; ++k) {
        const int m0 = slab_m0(k);
        // the block's footprint in this slab: box origin (f0, y0) and extents
        int f0, y0, hf, hy;
        slab::ray_box_low<ZF, SLAB>(g, r, hit, m0, f0, y0);
        slab::ray_box_high<ZF, SLAB>(g, r, hit, m0, hf, hy);
        // block maxima as minima of the negated values (INT_MIN: no sample here)
        int nf1 = hf == INT_MIN ? INT_MAX : -hf, ny1 = hy == INT_MIN ? INT_MAX : -hy;
        slab::block_min2<WARPS>(f0, y0, red[0]);
        slab::block_min2<WARPS>(nf1, ny1, red[1]);
        if (f0 == INT_MAX || nf1 == INT_MAX) f0 = y0 = 0, nf1 = ny1 = 0;
        const int ef = min(FB, max(2, -nf1 - f0 + 1)), ey = min(YB, max(2, -ny1 - y0 + 1));
        // one sample: false (and nothing added) when it belongs to a later slab
        auto take = [&](const float p[3]) -> bool {
            const float px = rmax(rmin(p[0], (float)(g.nx - 1)), 0.0f);
            const float py = rmax(rmin(p[1], (float)(g.ny - 1)), 0.0f);
            const float pz = rmax(rmin(p[2], (float)(g.nz - 1)), 0.0f);
            const int ix = (int)px, iy = (int)py, iz = (int)pz;
            const int bs = ZF ? ix : iz;
            if (fwd ? bs > m0 + SLAB - 1 : bs < m0) return false;
            const unsigned of = (unsigned)((ZF ? iz : ix) - f0), oy = (unsigned)(iy - y0), os = (unsigned)(bs - m0);
            if (of <= (unsigned)(ef - 2) && oy <= (unsigned)(ey - 2) && os <= (unsigned)(SB - 2)) {
                Taps t;  // the same fractions and edge collapse as make_taps, box-local offsets
                t.fx = px - (float)ix;
                t.fy = py - (float)iy;
                t.fz = pz - (float)iz;
                const int sF = 1, sY = FB, sS = FB * YB;
                t.dx = (ix < g.nx - 1) ? (ZF ? sS : sF) : 0;
                t.dy = (iy < g.ny - 1) ? sY : 0;
                t.dz = (iz < g.nz - 1) ? (ZF ? sF : sS) : 0;
                t.base = (long long)((os * YB + oy) * FB + of);
                float w[8];
                tri_weights(t, w);
#pragma unroll
                for (int q = 0; q < 8; ++q) {
                    const int cell = (int)tap_index(t, q);
                    atomicAdd(bc + cell, c * w[q]);
                    atomicAdd(bw + cell, w[q]);
                }
            } else {
                scatter_global(g, p, c, acc);
            }
            return true;
        };
        bool later = false;
        while (!later && m.peek()) {
            if (m.phase == 0) {  // the entry sample
                later = !take(m.pos);
                if (!later) m.advance();
                continue;
            }
            // the rest of the current segment, from registers
            float t = m.t, p[3] = {m.pos[0], m.pos[1], m.pos[2]};
            int n = m.n;
            do {
                if (!take(p)) {
                    later = true;
                    break;
                }
                t = __fadd_rn(t, m.sd);
#pragma unroll
                for (int a = 0; a < 3; ++a) p[a] = __fadd_rn(p[a], m.d.step[a]);
                ++n;
            } while (n < m.cap && t < m.tb);
            m.t = t;
            m.n = n;
#pragma unroll
            for (int a = 0; a < 3; ++a) m.pos[a] = p[a];
        }
        __syncthreads();
        // every touched cell of the footprint to global memory once, cleared on the way
        const int cells = ef * ey * SB;
        for (int q = threadIdx.x; q < cells; q += 32 * WARPS) {
            const int of = q % ef, oy = (q / ef) % ey, os = q / (ef * ey);
            const int b = (os * YB + oy) * FB + of;
            const float wq = bw[b], cq = bc[b];
            if (wq != 0.0f || cq != 0.0f) {  // (a NaN contribution counts as touched and is cleared too)
                bc[b] = 0.0f;
                bw[b] = 0.0f;
                const int fi = f0 + of, yi = y0 + oy, si = m0 + os;
                const int x = ZF ? si : fi, z = ZF ? fi : si;
                // cells outside the volume are never touched (taps are clamped into it)
                atomicAdd(acc + (x + (size_t)yi * g.nx + (size_t)z * g.nx * g.ny), make_float2(cq, wq));
            }
        }
        __syncthreads();  // the box is clear before the next slab adds into it
    }
    // samples outside the planes the slabs covered
    while (m.peek()) {
        scatter_global(g, m.pos, c, acc);
        m.advance();
    }
}

__global__ void __launch_bounds__(32 * WARPS) k_bp_ray_scatter_slab(const GeomDev g, const ViewRec *__restrict__ views,
                                                                   const ViewSel sel, const float *__restrict__ corr,
                                                                   float2 *__restrict__ acc) {
    __shared__ float bc[BOXN], bw[BOXN];  // contributions and weights of the box
    __shared__ int red[2][2 * WARPS];
    __shared__ int red_s[3 * WARPS];
    for (int q = threadIdx.x; q < BOXN; q += 32 * WARPS) bc[q] = bw[q] = 0.0f;  // flushes keep it clear
    const int i = blockIdx.x * 32 + (threadIdx.x & 31);
    const int j = blockIdx.y * WARPS + (threadIdx.x >> 5);
    const bool valid = i < g.W && j < g.H;
    int local;
    const ViewRec &vr = views[sel_view(sel, local)];
    Ray r;
    bool hit = false;
    float c = 0.0f;
    if (valid) {
        make_ray(g, vr, i, j, r);
        hit = r.tnear < r.tfar;
        c = __ldg(corr + i + (size_t)j * g.W);
    }
    // (the barrier inside the span reduction also orders the clearing above)
    if (vr.layout == 1) scatter_slabs<true>(g, r, hit, c, acc, bc, bw, red_s, red);
    else scatter_slabs<false>(g, r, hit, c, acc, bc, bw, red_s, red);
}

}  // namespace

cudaError_t launch_bp_ray_scatter_slab(const GeomDev &g, const ViewRec *views, const ViewSel &sel, const float *corr,
                                       float2 *acc, cudaStream_t s) {
    if ((long long)g.nx * g.ny * g.nz >= (1LL << 31)) return cudaErrorInvalidValue;  // int box arithmetic
    k_bp_ray_scatter_slab<<<dim3((g.W + 31) / 32, (g.H + WARPS - 1) / WARPS, 1), 32 * WARPS, 0, s>>>(g, views, sel,
                                                                                                   corr, acc);
    return cudaGetLastError();
}

}  // namespace stt
