// stt_voxel.cuh -- device helpers of the voxel-driven steps, shared by the
// per-view kernels (k_voxel.cu) and the persistent sweep (k_persist.cu): the
// ROI tests, the voxel-based backprojection of one voxel and of one column,
// and the ROI mask with the over-relaxation.
//
// Paths cited are relative to the reference project root (gmzang/SpaceTimeTomography);
// S/ = SpaceTimeTomography/.
#pragma once

#include <climits>

#include "stt_internal.cuh"

namespace stt {

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

// End of a SART call (ST_Tomography.cpp:793-804) for voxel (i, j, k),
// optionally fused with the over-relaxation that follows it in the
// primal-dual loop (:586-604): vol *= roi; if xbar: xbar = 2*vol - xprev in
// the ROI box.  vol is read with a plain load (a launch may have written it).
template <typename T>
__device__ __forceinline__ void roi_apply_at(int i, int j, int k, int nx, int ny, int nz, const int *cut,
                                             const int *pdcut, T *vol, const T *xprev, T *xbar) {
    const size_t p = i + (size_t)j * nx + (size_t)k * nx * ny;
    const float v = ld_stored(vol + p) * roi_value(i, j, k, nx, ny, nz, cut);  // (a product by 0 or 1: exact)
    st_stored(vol + p, v);
    if (xbar && !roi_out(i, j, k, nx, ny, nz, pdcut)) st_stored(xbar + p, 2.0f * v - ld_voxel(xprev + p));
}

// A load of an FP32 array: through the read-only path, or (RW) a plain load
// for an array that the running launch has written (the persistent sweep).
template <bool RW>
__device__ __forceinline__ float ld_f(const float *p) {
    if constexpr (RW) return *p;
    else return __ldg(p);
}

// Dual step of one frame at voxel (i, j, k) (ST_Tomography.cpp:504-534), fused:
//   whole volume:     ytp += sigma*(xf1 - xf);  ybc += sigma*(bw - xf)
//   interior & ROI:   ytv_c += sigma*(xf(p+e_c) - xf(p))*hf, clamp +-tv_w;
//                     ytp = ytp*tp_w/(tp_w + 2 sigma);  ybc clamp +-bc_w
// bw: the backward-warped X_bar[f+1] at the voxel.  T: the storage of X_bar
// (the duals are FP32).
template <typename T>
__device__ __forceinline__ void pd_dual_at(int i, int j, int k, int nx, int ny, int nz, float sigma, float tv_w,
                                           float tp_w, float bc_w, float hf, const int *cut, const T *xf,
                                           const T *xf1, float bw, float *ytv, float *ytp, float *ybc) {
    const size_t sy = nx, sz = (size_t)nx * ny, n = sz * nz;
    const size_t p = i + j * sy + k * sz;
    const float x0 = ld_voxel(xf + p);
    float tp = ytp[p] + sigma * (ld_voxel(xf1 + p) - x0);
    float bc = ybc[p] + sigma * (bw - x0);
    const bool inner = i >= 1 && i < nx - 1 && j >= 1 && j < ny - 1 && k >= 1 && k < nz - 1 &&
                       !roi_out(i, j, k, nx, ny, nz, cut);
    if (inner) {
        float y0 = ytv[p] + sigma * (ld_voxel(xf + p + 1) - x0) * hf;
        float y1 = ytv[p + n] + sigma * (ld_voxel(xf + p + sy) - x0) * hf;
        float y2 = ytv[p + 2 * n] + sigma * (ld_voxel(xf + p + sz) - x0) * hf;
        ytv[p] = rmax(-tv_w, rmin(tv_w, y0));
        ytv[p + n] = rmax(-tv_w, rmin(tv_w, y1));
        ytv[p + 2 * n] = rmax(-tv_w, rmin(tv_w, y2));
        tp = __fdiv_rn(tp * tp_w, tp_w + 2.0f * sigma);
        bc = rmax(-bc_w, rmin(bc_w, bc));
    }
    ytp[p] = tp;
    ybc[p] = bc;
}

// Primal step of one frame at voxel (i, j, k) (ST_Tomography.cpp:536-578),
// fused: xprev = vol; vol -= tau*(-ytp); vol -= tau*(-ybc) for the first
// frame, otherwise vol -= tau*(ytp_prev - ytp); vol -= tau*(fw - ybc); then
// on the interior ROI vol -= tau*(-div ytv) and clamp to [0, gmax].  fw: the
// forward-warped Y_bc[f-1] at the voxel.  T: the storage of vol and xprev
// (the duals are FP32).  RW: the duals were written by the same launch.
template <bool RW, typename T>
__device__ __forceinline__ void pd_primal_at(int i, int j, int k, int nx, int ny, int nz, float tau, float gmax,
                                             const int *cut, int first, const float *ytp_prev, const float *ytp,
                                             float fw, const float *ybc, const float *ytv, T *vol, T *xprev) {
    const size_t sy = nx, sz = (size_t)nx * ny, n = sz * nz;
    const size_t p = i + j * sy + k * sz;
    float v = ld_stored(vol + p);
    st_stored(xprev + p, v);
    if (first) {
        v = v - tau * (-ld_f<RW>(ytp + p));
        v = v - tau * (-ld_f<RW>(ybc + p));
    } else {
        v = v - tau * (ld_f<RW>(ytp_prev + p) - ld_f<RW>(ytp + p));
        v = v - tau * (fw - ld_f<RW>(ybc + p));
    }
    const bool inner = i >= 1 && i < nx - 1 && j >= 1 && j < ny - 1 && k >= 1 && k < nz - 1 &&
                       !roi_out(i, j, k, nx, ny, nz, cut);
    if (inner) {
        const float *y0 = ytv, *y1 = ytv + n, *y2 = ytv + 2 * n;
        float y = -(ld_f<RW>(y0 + p) - ld_f<RW>(y0 + p - 1) + ld_f<RW>(y1 + p) - ld_f<RW>(y1 + p - sy) +
                    ld_f<RW>(y2 + p) - ld_f<RW>(y2 + p - sz));
        v = v - tau * y;
        v = rmax(rmin(gmax, v), 0.0f);
    }
    st_stored(vol + p, v);
}

// Voxel-based backprojection (ST_Tomography.cpp:690-730): project the voxel
// centre, Catmull-Rom 4x4 gather of the correction image (y first, then x),
// vol += alpha*val, clamp to [0, gmax]; voxels whose footprint leaves
// [2, W-2) x [2, H-2) are untouched.  Every product and sum is rounded on its
// own (explicit intrinsics), so the per-voxel and the column forms below give
// the same bits whichever way their taps are fetched.

// Camera coordinate r of voxel (fx, fy, fz): A[r]*(x, y, z) + b[r].
__device__ __forceinline__ float bp_cam(const ViewRec &v, int r, float fx, float fy, float fz) {
    return __fadd_rn(__fmaf_rn(v.A[3 * r + 2], fz, __fmaf_rn(v.A[3 * r + 1], fy, __fmul_rn(v.A[3 * r], fx))), v.b[r]);
}

// Detector coordinate c + cam/(-depth) * sdd/ds.
__device__ __forceinline__ float bp_pixel(float c, float cam, float ndepth, float sdd_ds) {
    return __fmaf_rn(__fdiv_rn(cam, ndepth), sdd_ds, c);
}

// Catmull-Rom weights of taps (-1, 0, +1, +2) at fraction d.
__device__ __forceinline__ void bp_weights(float d, float w[4]) {
    const float d2 = __fmul_rn(d, d), d3 = __fmul_rn(d2, d);
    w[0] = __fmul_rn(0.5f, __fsub_rn(__fmaf_rn(2.0f, d2, -d), d3));
    w[1] = __fadd_rn(1.0f, __fmul_rn(0.5f, __fmaf_rn(3.0f, d3, __fmul_rn(-5.0f, d2))));
    w[2] = __fmul_rn(0.5f, __fmaf_rn(-3.0f, d3, __fmaf_rn(4.0f, d2, d)));
    w[3] = __fmul_rn(0.5f, __fsub_rn(d3, d2));
}

// sum_a wx[a] * sum_b wy[b] * tap[a][b]; tap[a][b] is column px-1+a, row py-1+b.
__device__ __forceinline__ float bp_sum(const float tap[4][4], const float wx[4], const float wy[4]) {
    float val = 0.0f;
#pragma unroll
    for (int a = 0; a < 4; ++a) {
        const float s = __fmaf_rn(wy[3], tap[a][3],
                                  __fmaf_rn(wy[2], tap[a][2], __fmaf_rn(wy[1], tap[a][1], __fmul_rn(wy[0], tap[a][0]))));
        val = a == 0 ? __fmul_rn(wx[0], s) : __fmaf_rn(wx[a], s, val);
    }
    return val;
}

// T: the volume's storage (float, or BF16 bits widened to FP32 and rounded
// back to nearest even on store).
template <typename T>
__device__ __forceinline__ void bp_update(T *__restrict__ vol, size_t o, float alpha, float val, float gmax) {
    const float nv = __fmaf_rn(alpha, val, ld_stored(vol + o));
    st_stored(vol + o, rmax(rmin(gmax, nv), 0.0f));
}

// Fetchers of two correction rows, pyr and pyr + 1, at columns px-1 .. px+2
// (r0[a], r1[a]: column px-1+a).  All three return the stored values.
// From the correction's one-layer texture copy: two tld4 gathers.
struct BpRowsTex {
    unsigned long long tex;
    __device__ __forceinline__ void operator()(int px, int pyr, float r0[4], float r1[4]) const {
        const float4 gc = gather_layer(tex, px - 1, pyr, 0), gd = gather_layer(tex, px + 1, pyr, 0);
        r0[0] = gc.w, r0[1] = gc.z, r0[2] = gd.w, r0[3] = gd.z;
        r1[0] = gc.x, r1[1] = gc.y, r1[2] = gd.x, r1[3] = gd.y;
    }
};
// From the correction array through the read-only path (written by an
// earlier launch).
struct BpRowsLdg {
    const float *corr;
    int W;
    __device__ __forceinline__ void operator()(int px, int pyr, float r0[4], float r1[4]) const {
        const float *c0 = corr + (size_t)pyr * W + (px - 1);
#pragma unroll
        for (int a = 0; a < 4; ++a) r0[a] = __ldg(c0 + a), r1[a] = __ldg(c0 + W + a);
    }
};
// From the correction array with plain loads (written by the same launch).
struct BpRowsLoad {
    const float *corr;
    int W;
    __device__ __forceinline__ void operator()(int px, int pyr, float r0[4], float r1[4]) const {
        const float *c0 = corr + (size_t)pyr * W + (px - 1);
#pragma unroll
        for (int a = 0; a < 4; ++a) r0[a] = ld_stored(c0 + a), r1[a] = ld_stored(c0 + W + a);
    }
};

// One voxel, everything computed for it alone.
template <typename Rows, typename T>
__device__ __forceinline__ void bp_voxel_at(const GeomDev &g, const ViewRec &v, const Rows &rows, T *__restrict__ vol,
                                            int x, int y, int z, float alpha, float gmax) {
    const float fx = (float)x, fy = (float)y, fz = (float)z;
    const float ndepth = -bp_cam(v, 2, fx, fy, fz);
    const float upx = bp_pixel(g.cx, bp_cam(v, 0, fx, fy, fz), ndepth, g.sdd_ds);
    const float upy = bp_pixel(g.cy, bp_cam(v, 1, fx, fy, fz), ndepth, g.sdd_ds);
    if (!(upx >= 2.0f && upx < (float)(g.W - 2) && upy >= 2.0f && upy < (float)(g.H - 2))) return;
    const int px = (int)upx, py = (int)upy;
    float wx[4], wy[4], tap[4][4], r0[4], r1[4], r2[4], r3[4];
    bp_weights(upx - (float)px, wx);
    bp_weights(upy - (float)py, wy);
    rows(px, py - 1, r0, r1);
    rows(px, py + 1, r2, r3);
#pragma unroll
    for (int a = 0; a < 4; ++a) tap[a][0] = r0[a], tap[a][1] = r1[a], tap[a][2] = r2[a], tap[a][3] = r3[a];
    bp_update(vol, x + (size_t)y * g.nx + (size_t)z * g.nx * g.ny, alpha, bp_sum(tap, wx, wy), gmax);
}

// The column walk: voxels (x, y0 .. y0+K-1, z).  For a view whose matrix has
// A[1] == A[7] == 0 (every rotation about y) the voxel's detector column and
// depth do not depend on y: they are computed once (the y term of their sums
// is an exact zero, so the values are the per-voxel ones).  The detector row
// moves by about sdd/sid per voxel, and the 4x4 window's rows are kept in
// registers: a step of s = 0, 1 or 2 rows reuses two of them and fetches the
// two new ones.  Other views take the per-voxel form.
// PF: first ask L2 for the column's voxels (prefetch.global.L2).
template <int K, bool PF, typename Rows, typename T>
__device__ __forceinline__ void bp_column(const GeomDev &g, const ViewRec &v, const Rows &rows, T *__restrict__ vol,
                                          int x, int y0, int z, float alpha, float gmax) {
    const int y1 = min(y0 + K, g.ny);
    if (!(v.A[1] == 0.0f && v.A[7] == 0.0f)) {
        for (int y = y0; y < y1; ++y) bp_voxel_at(g, v, rows, vol, x, y, z, alpha, gmax);
        return;
    }
    const float fx = (float)x, fz = (float)z;
    const float ndepth = -bp_cam(v, 2, fx, (float)y0, fz);
    const float upx = bp_pixel(g.cx, bp_cam(v, 0, fx, (float)y0, fz), ndepth, g.sdd_ds);
    if (!(upx >= 2.0f && upx < (float)(g.W - 2))) return;
    const int px = (int)upx;
    if (PF) {
        const T *col = vol + x + (size_t)z * g.nx * g.ny;
        for (int y = y0; y < y1; ++y) asm volatile("prefetch.global.L2 [%0];" ::"l"(col + (size_t)y * g.nx));
    }
    float wx[4];
    bp_weights(upx - (float)px, wx);
    float R[4][4];  // R[a][b]: column px-1+a, row pyc-1+b
    int pyc = INT_MIN / 2;
    for (int y = y0; y < y1; ++y) {
        const float upy = bp_pixel(g.cy, bp_cam(v, 1, fx, (float)y, fz), ndepth, g.sdd_ds);
        if (!(upy >= 2.0f && upy < (float)(g.H - 2))) continue;
        const int py = (int)upy;
        float wy[4];
        bp_weights(upy - (float)py, wy);
        const int s = py - pyc;
        float r0[4], r1[4];  // rows py-1, py
        if (s >= 0 && s <= 2) {
#pragma unroll
            for (int a = 0; a < 4; ++a) {
                r0[a] = s == 0 ? R[a][0] : (s == 1 ? R[a][1] : R[a][2]);
                r1[a] = s == 0 ? R[a][1] : (s == 1 ? R[a][2] : R[a][3]);
            }
        } else {
            rows(px, py - 1, r0, r1);
        }
        float r2[4], r3[4];  // rows py+1, py+2
        rows(px, py + 1, r2, r3);
#pragma unroll
        for (int a = 0; a < 4; ++a) {
            R[a][0] = r0[a];
            R[a][1] = r1[a];
            R[a][2] = r2[a];
            R[a][3] = r3[a];
        }
        pyc = py;
        bp_update(vol, x + (size_t)y * g.nx + (size_t)z * g.nx * g.ny, alpha, bp_sum(R, wx, wy), gmax);
    }
}

}  // namespace stt
