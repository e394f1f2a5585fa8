// k_flow.cu -- kernels of the 3D TV-L1/Huber optical flow of
// S/ST_Tomo/optical_flow.h (L1Huber_OF :83-623, L1Huber_OF_MultiScale3D
// :630-734) and of the CImg operations it calls (S/ImageFormationModel/CImg.h):
// the order-0 Deriche blur (deriche :32917-33050), resizing by moving average
// (:28135-28195) and by Catmull-Rom interpolation (:28432-28560), central
// differences with Neumann boundaries (get_gradient :34570-34581) and the
// warp of S/ST_Tomo/warping.h:49-145 over a general bounding box.
//
// This file is compiled with -fmad=false: every float and double expression
// is rounded operation by operation in the reference's order, so a level of
// the flow reproduces the reference's CPU result bit for bit (the residual
// sums, which the reference accumulates in a racy loop, are the exception).
//
// Layout: planar x-fastest fields, idx = x + y*nx + z*nx*ny, channel planes of
// n = nx*ny*nz floats (CImg's layout).  Dual field y: 10 planes Y1|Y2|Y3|Y4.
// Per iteration the primal step reads y, u, tau and the flow and writes the
// next flow into a second buffer; the dual step reads both flows (K v and
// K v_old), u and sigma2 and updates y in place: 53 floats per voxel instead
// of the 70 of the reference's layout, which also stores K v (10 floats).
#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdint>

#include "stt_kernels.h"

namespace stt {
namespace {

// std::min / std::max exactly as the reference calls them.
__device__ __forceinline__ float smin(float a, float b) { return (b < a) ? b : a; }
__device__ __forceinline__ float smax(float a, float b) { return (a < b) ? b : a; }

struct Dims {
    int x, y, z;
};

__device__ __forceinline__ bool in_roi(const FlowRoi &r, const Dims &d, int i, int j, int k) {
    return k >= r.z0 && k < d.z - r.z1 && j >= r.y0 && j < d.y - r.y1 && i >= r.x0 && i < d.x - r.x1;
}

// ---- warp (warping.h:11-145) with aabb = [0, box] ---------------------------
// CImg::_cubic_atXYZ in its nested Catmull-Rom form (CImg.h:13429-13520): x
// rows first, then y, then z; taps clamped to the image, the "next" tap is
// x+1 only when the fraction is positive.
__device__ __forceinline__ float cimg_cr(float p, float c, float n, float a, float d) {
    return c + 0.5f * (d * (-p + n) + d * d * (2 * p - 5 * c + 4 * n - a) + d * d * d * (-p + 3 * c - 3 * n + a));
}

__device__ __forceinline__ void cimg_taps(float f, int dim, int t[4], float &d) {
    const float nf = f < 0.0f ? 0.0f : (f > (float)(dim - 1) ? (float)(dim - 1) : f);
    const int x = (int)nf;
    d = nf - (float)x;
    t[0] = x - 1 < 0 ? 0 : x - 1;
    t[1] = x;
    t[2] = d > 0.0f ? x + 1 : x;
    t[3] = x + 2 >= dim ? dim - 1 : x + 2;
}

// warping::sample_image: world point -> cell grid (aabb [0, box]), clamped to
// [1, dim-2], cubic value clamped to the min/max of the cell's 8 corners.
__device__ float sample_box(const float *__restrict__ img, const Dims &d, const float box[3], const float p[3]) {
    const int D[3] = {d.x, d.y, d.z};
    float g[3];
#pragma unroll
    for (int a = 0; a < 3; ++a) {
        const float gw = (float)D[a] * (p[a] - 0.0f) / (box[a] - 0.0f);
        float q = (float)((double)gw - 0.5);
        const float hi = (float)(D[a] - 2), lo = 1.0f;
        q = (q < hi) ? q : hi;
        q = (lo < q) ? q : lo;
        g[a] = q;
    }
    const long long sy = d.x, sz = (long long)d.x * d.y;
    const int ix = (int)g[0], iy = (int)g[1], iz = (int)g[2];
    const float *c0 = img + ix + iy * sy + iz * sz;
    float mn = __ldg(c0), mx = mn;
    const long long off[7] = {1, 1 + sy, sy, sz, 1 + sz, 1 + sy + sz, sy + sz};
#pragma unroll
    for (int k = 0; k < 7; ++k) {
        const float v = __ldg(c0 + off[k]);
        mn = (v < mn) ? v : mn;
        mx = (mx < v) ? v : mx;
    }
    int tx[4], ty[4], tz[4];
    float dx, dy, dz;
    cimg_taps(g[0], d.x, tx, dx);
    cimg_taps(g[1], d.y, ty, dy);
    cimg_taps(g[2], d.z, tz, dz);
    float zv[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) {
        float yv[4];
#pragma unroll
        for (int b = 0; b < 4; ++b) {
            const float *row = img + ty[b] * sy + tz[c] * sz;
            yv[b] = cimg_cr(__ldg(row + tx[0]), __ldg(row + tx[1]), __ldg(row + tx[2]), __ldg(row + tx[3]), dx);
        }
        zv[c] = cimg_cr(yv[0], yv[1], yv[2], yv[3], dy);
    }
    const float val = cimg_cr(zv[0], zv[1], zv[2], zv[3], dz);
    const float inner = (val < mx) ? val : mx;
    return (mn < inner) ? inner : mn;
}

// warping::warp: trace back from each cell centre with -dt (two-step
// semi-Lagrangian, warping.h:100-114), sample every source channel there.
__global__ void __launch_bounds__(128) k_warp_box(const Dims d, const float bx, const float by, const float bz,
                                                  const float *__restrict__ vel, const float *__restrict__ src, int nc,
                                                  float dt, float *__restrict__ out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y, k = blockIdx.z;
    if (i >= d.x) return;
    const long long n = (long long)d.x * d.y * d.z;
    const float box[3] = {bx, by, bz};
    const int ijk[3] = {i, j, k};
    const int D[3] = {d.x, d.y, d.z};
    float p[3], v[3], p2[3], q[3];
#pragma unroll
    for (int a = 0; a < 3; ++a)
        p[a] = (float)(0 + ((double)(float)ijk[a] + 0.5) * (double)(box[a] - 0) / (double)(float)D[a]);
    const float h = -dt;
#pragma unroll
    for (int c = 0; c < 3; ++c) v[c] = sample_box(vel + c * n, d, box, p);
#pragma unroll
    for (int c = 0; c < 3; ++c) p2[c] = p[c] + h * v[c];
#pragma unroll
    for (int c = 0; c < 3; ++c) v[c] = sample_box(vel + c * n, d, box, p2);
#pragma unroll
    for (int c = 0; c < 3; ++c) {
        const float p0 = p2[c] - h * v[c];
        q[c] = p2[c] + (float)(0.5 * (double)(p[c] - p0));
    }
    const long long o = i + (long long)j * d.x + (long long)k * d.x * d.y;
    for (int c = 0; c < nc; ++c) out[o + c * n] = sample_box(src + c * n, d, box, q);
}

// ---- per-warp setup (optical_flow.h:257-297) ---------------------------------
// Inside the ROI: the Neumann central gradient of the warped I2 and
// ut = I2w - I1 - grad.v.  Outside the ROI the reference leaves these arrays
// unset; here they are 0.  Everywhere: tau_c = 1/(4 + |u_c|) and
// sigma2 = 1/(|ux| + |uy| + |uz|) (infinite where the gradient vanishes).
// Before u is replaced, k4prev = u_prev . v keeps the data-term part of the
// previous warp's last K v, which the first dual step of this warp uses as
// its K v_old (the reference keeps Kx across warps, optical_flow.h:246, 394).
__global__ void __launch_bounds__(128) k_flow_setup(const Dims d, const FlowRoi roi, const float *__restrict__ i2w,
                                                    const float *__restrict__ i1, const float *__restrict__ v,
                                                    float *__restrict__ u, float *__restrict__ tau,
                                                    float *__restrict__ sig2, float *__restrict__ k4prev) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y, k = blockIdx.z;
    if (i >= d.x) return;
    const long long sy = d.x, sz = (long long)d.x * d.y, n = sz * d.z;
    const long long p = i + j * sy + k * sz;
    const float v1 = __ldg(v + p), v2 = __ldg(v + n + p), v3 = __ldg(v + 2 * n + p);
    k4prev[p] = u[p] * v1 + u[n + p] * v2 + u[2 * n + p] * v3;
    float ux = 0.0f, uy = 0.0f, uz = 0.0f, ut = 0.0f;
    if (in_roi(roi, d, i, j, k)) {
        const long long xm = i > 0 ? p - 1 : p, xp = i < d.x - 1 ? p + 1 : p;
        const long long ym = j > 0 ? p - sy : p, yp = j < d.y - 1 ? p + sy : p;
        const long long zm = k > 0 ? p - sz : p, zp = k < d.z - 1 ? p + sz : p;
        ux = (__ldg(i2w + xp) - __ldg(i2w + xm)) / 2;
        uy = (__ldg(i2w + yp) - __ldg(i2w + ym)) / 2;
        uz = (__ldg(i2w + zp) - __ldg(i2w + zm)) / 2;
        ut = __ldg(i2w + p) - __ldg(i1 + p) - ux * v1 - uy * v2 - uz * v3;
    }
    u[p] = ux;
    u[n + p] = uy;
    u[2 * n + p] = uz;
    u[3 * n + p] = ut;
    tau[p] = 1.0f / (4.0f / 1.0f + fabsf(ux));
    tau[n + p] = 1.0f / (4.0f / 1.0f + fabsf(uy));
    tau[2 * n + p] = 1.0f / (4.0f / 1.0f + fabsf(uz));
    sig2[p] = 1.0f / (fabsf(ux) + fabsf(uy) + fabsf(uz));
}

// Backward difference of S/ImageFormationModel/tools.cpp:146-192 (dxm3, dym3,
// dzm3) at coordinate c of n along a stride st, from the centre value a and
// the lower neighbour b (read only when c > 0): interior a - b, first a,
// last -b.
__device__ __forceinline__ float dm(float a, float b, int c, int n) {
    return (c > 0 && c < n - 1) ? a - b : (c == 0 ? a : -b);
}

// Forward difference of tools.cpp:126-138 (dxp3, dyp3, dzp3): upper
// neighbour b (read only when c < n-1) minus the centre a, 0 at the last.
__device__ __forceinline__ float dp(float a, float b, int c, int n) { return c < n - 1 ? b - a : 0.0f; }

// flags: bit 0 = residual iteration (iteration % 50 == 0); bit 1 = keep K^T y
// for the next iteration's residual; bit 2 = first iteration of the level
// (K v_old = 0, optical_flow.h:231-243); bit 3 = first iteration of a later
// warp (the data-term row of K v_old from k4prev).
constexpr int kResid = 1, kKeepKty = 2, kFirstOfLevel = 4, kFirstOfWarp = 8;

__device__ __forceinline__ void add_resid(double *resid, float r) {
    for (int o = 16; o > 0; o >>= 1) r += __shfl_down_sync(0xffffffffu, r, o);
    if ((threadIdx.x & 31) == 0 && r != 0.0f) atomicAdd(resid, (double)r);
}

// Offsets inside one level are 32-bit: the host keeps 10 * voxels < 2^31.
// Every load of a voxel's neighbourhood is issued before the arithmetic.

// Primal step over the ROI (optical_flow.h:314-370):
// Kty_c = -div_b(y_c) + u_c*y4; v_c -= tau_c*Kty_c, read from v_in and
// written to v_out (the dual step needs both).  Outside the ROI v_in and
// v_out hold the same, never-updated values.
__global__ void __launch_bounds__(128) k_flow_primal(const Dims d, const FlowRoi roi, const float *__restrict__ y,
                                                     const float *__restrict__ u, const float *__restrict__ tau,
                                                     const float *__restrict__ v_in, float *__restrict__ v_out,
                                                     float *__restrict__ kty, int flags, double *__restrict__ resid,
                                                     const int *__restrict__ done) {
    if (*done) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y, k = blockIdx.z;
    float pr = 0.0f;
    if (i < d.x && in_roi(roi, d, i, j, k)) {
        const int sy = d.x, sz = d.x * d.y, n = sz * d.z;
        const long long p = i + (long long)j * sy + (long long)k * sz;
        const float *yp = y + p;
        const int ox = i > 0 ? 1 : 0, oy = j > 0 ? sy : 0, oz = k > 0 ? sz : 0;
        float a[9], b[9];
#pragma unroll
        for (int q = 0; q < 9; ++q) {
            const int off = q * n, st = (q % 3 == 0) ? ox : (q % 3 == 1 ? oy : oz);
            a[q] = __ldg(yp + off);
            b[q] = __ldg(yp + off - st);
        }
        const float y4 = __ldg(yp + 9 * n);
        float uc[3], vo[3], t[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            uc[c] = __ldg(u + p + c * n);
            vo[c] = __ldg(v_in + p + c * n);
            t[c] = __ldg(tau + p + c * n);
        }
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            // -stepsizeD * dxm3 - ... with unit step sizes: (-1 * x) == -x and 1 * x == x exactly
            const float kt = -dm(a[3 * c], b[3 * c], i, d.x) - dm(a[3 * c + 1], b[3 * c + 1], j, d.y) -
                             dm(a[3 * c + 2], b[3 * c + 2], k, d.z) + uc[c] * y4;
            const float vn = vo[c] - t[c] * kt;
            v_out[p + c * n] = vn;
            if (flags & kResid) {
                const float r = fabsf((vo[c] - vn) / t[c] - kty[p + c * n] + kt);
                pr = c == 0 ? r : pr + r;
            }
            if (flags & kKeepKty) kty[p + c * n] = kt;
        }
    }
    if (flags & kResid) add_resid(resid, pr);
}

// Dual step over every voxel (optical_flow.h:374-497): K v by forward
// differences of v and u.v; over-relaxed ascent y + sigma1*(2 K v - K v_old),
// scaled by the Huber factor for norm 4; each y_c projected onto the
// lambda-ball; y4 clamped to [-1, 1].  K v_old, which the reference stores
// (10 floats per voxel), is recomputed here from v_old with the same float
// operations, so it is the same value.
__global__ void __launch_bounds__(128) k_flow_dual(const Dims d, const float *__restrict__ v,
                                                   const float *__restrict__ v_old, const float *__restrict__ u,
                                                   const float *__restrict__ sig2, const float *__restrict__ k4prev,
                                                   float *__restrict__ y, float sigma1, float hf, float lambda,
                                                   float lam2_lo, int huber, int flags, double *__restrict__ resid,
                                                   const int *__restrict__ done) {
    if (*done) return;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y, k = blockIdx.z;
    float dr = 0.0f;
    if (i < d.x) {
        const int sy = d.x, sz = d.x * d.y, n = sz * d.z;
        const long long p = i + (long long)j * sy + (long long)k * sz;
        const int ox = i < d.x - 1 ? 1 : 0, oy = j < d.y - 1 ? sy : 0, oz = k < d.z - 1 ? sz : 0;
        const bool zero_old = flags & kFirstOfLevel;
        const float *vp = v + p, *op = v_old + p;
        float vc[3], vx[3], vy[3], vz[3], oc[3], oxv[3], oyv[3], ozv[3];
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const int off = c * n;
            vc[c] = __ldg(vp + off);
            vx[c] = __ldg(vp + off + ox);
            vy[c] = __ldg(vp + off + oy);
            vz[c] = __ldg(vp + off + oz);
            if (!zero_old) {
                oc[c] = __ldg(op + off);
                oxv[c] = __ldg(op + off + ox);
                oyv[c] = __ldg(op + off + oy);
                ozv[c] = __ldg(op + off + oz);
            }
        }
        float *yp = y + p;
        float yo[10];
#pragma unroll
        for (int q = 0; q < 10; ++q) yo[q] = yp[q * n];
        const float u1 = __ldg(u + p), u2 = __ldg(u + p + n), u3 = __ldg(u + p + 2 * n), ut = __ldg(u + p + 3 * n);
        const float s2 = __ldg(sig2 + p);
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            // K v with unit step sizes (stepsizeD = 1: x * 1.0f == x, dropped)
            const float kn[3] = {dp(vc[c], vx[c], i, d.x), dp(vc[c], vy[c], j, d.y), dp(vc[c], vz[c], k, d.z)};
            float ko[3] = {0.0f, 0.0f, 0.0f};
            if (!zero_old) {
                ko[0] = dp(oc[c], oxv[c], i, d.x);
                ko[1] = dp(oc[c], oyv[c], j, d.y);
                ko[2] = dp(oc[c], ozv[c], k, d.z);
            }
            float yt[3];
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                const float t = yo[3 * c + a] + sigma1 * (kn[a] + kn[a] - ko[a]);
                yt[a] = huber ? t * hf : t;
            }
            // divisor = max(1, sqrt(s)/lambda) and y = yt/divisor.  Below
            // lam2_lo (< lambda^2 with margin) sqrt(s) rounds below lambda, so
            // the divisor is exactly 1 and y = yt exactly: skip the sqrt and
            // the divisions.
            const float ss = yt[0] * yt[0] + yt[1] * yt[1] + yt[2] * yt[2];
            float yn[3] = {yt[0], yt[1], yt[2]};
            if (!(ss < lam2_lo)) {
                const float div = smax(1.0f, sqrtf(ss) / lambda);
                if (div != 1.0f) {
                    yn[0] = yt[0] / div;
                    yn[1] = yt[1] / div;
                    yn[2] = yt[2] / div;
                }
            }
#pragma unroll
            for (int a = 0; a < 3; ++a) {
                yp[(3 * c + a) * n] = yn[a];
                if (flags & kResid) {
                    const float r = fabsf((yo[3 * c + a] - yn[a]) / sigma1 - ko[a] + kn[a]);
                    dr = (c == 0 && a == 0) ? r : dr + r;
                }
            }
        }
        const float k4 = u1 * vc[0] + u2 * vc[1] + u3 * vc[2];
        float k4o = 0.0f;
        if (flags & kFirstOfWarp) k4o = __ldg(k4prev + p);
        else if (!zero_old) k4o = u1 * oc[0] + u2 * oc[1] + u3 * oc[2];
        const float y4 = smax(-1.0f, smin(1.0f, yo[9] + s2 * (k4 + k4 - k4o + ut)));
        yp[9 * n] = y4;
        if (flags & kResid) dr = dr + fabsf((yo[9] - y4) / s2 - k4o + k4);
    }
    if (flags & kResid) add_resid(resid + 1, dr);
}

// End of a warp: the flow of the last iteration that ran lies in the second
// buffer when that count is odd; bring it back to the first.
__global__ void __launch_bounds__(256) k_flow_settle(long long n3, const int *__restrict__ iters,
                                                     const float *__restrict__ v_b, float *__restrict__ v_a) {
    if ((*iters & 1) == 0) return;
    for (long long q = blockIdx.x * (long long)blockDim.x + threadIdx.x; q < n3; q += (long long)gridDim.x * blockDim.x)
        v_a[q] = v_b[q];
}

// Stopping rule of optical_flow.h:306, 488-491: after a residual iteration
// err = (d^2 + p^2)/n, and the loop stops unless err > tol.  Records the
// iteration count of the warp (when it stops, or at the last iteration).
__global__ void k_flow_check(double *resid, long long n, float tol, int it, int is_resid, int is_last, int *done,
                             int *iters, float *err) {
    if (*done) return;
    if (is_resid) {
        const float pf = (float)resid[0], df = (float)resid[1];
        const float e = (df * df + pf * pf) / (float)n;
        *err = e;
        resid[0] = 0.0;
        resid[1] = 0.0;
        if (!(e > tol)) {
            *done = 1;
            *iters = it;
            return;
        }
    }
    if (is_last) *iters = it;
}

// Start of a warp: clear the stop flag and the residual sums, reset the
// iteration count and set the recorded residual to its initial value 1.
__global__ void k_flow_reset(int *done, double *resid, int *iters, float *err) {
    *done = 0;
    resid[0] = 0.0;
    resid[1] = 0.0;
    *iters = 0;
    *err = 1.0f;
}

// ---- CImg::deriche, order 0, Neumann (CImg.h:32917-33050) ---------------------
// One thread per line along `axis`, in place; the causal pass is buffered in
// `tmp` at the same positions.
__global__ void k_deriche_line(const Dims d, int nc, int axis, const DericheCoef c, float *__restrict__ img,
                               float *__restrict__ tmp) {
    const long long per_ch = axis == 0 ? (long long)d.y * d.z : axis == 1 ? (long long)d.x * d.z : (long long)d.x * d.y;
    const long long l = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (l >= per_ch * nc) return;
    const long long n3 = (long long)d.x * d.y * d.z;
    const int ch = (int)(l / per_ch);
    const long long r = l % per_ch;
    long long base, off;
    int N;
    if (axis == 0) {
        N = d.x;
        off = 1;
        base = r * d.x;
    } else if (axis == 1) {
        N = d.y;
        off = d.x;
        base = (r % d.x) + (r / d.x) * (long long)d.x * d.y;
    } else {
        N = d.z;
        off = (long long)d.x * d.y;
        base = r;
    }
    float *X = img + ch * n3 + base;
    float *Y = tmp + ch * n3 + base;
    float xp = X[0], yb = c.coefp * xp, yp = yb;
    for (int m = 0; m < N; ++m) {
        const float xc = X[m * off];
        const float yc = c.a0 * xc + c.a1 * xp - c.b1 * yp - c.b2 * yb;
        Y[m * off] = yc;
        xp = xc;
        yb = yp;
        yp = yc;
    }
    float xn = X[(N - 1) * off], xa = xn, yn = c.coefn * xn, ya = yn;
    for (int m = N - 1; m >= 0; --m) {
        const float xc = X[m * off];
        const float yc = c.a2 * xn + c.a3 * xa - c.b1 * yn - c.b2 * ya;
        xa = xn;
        xn = xc;
        ya = yn;
        yn = yc;
        X[m * off] = Y[m * off] + yc;
    }
}

// ---- CImg::get_resize(..., 5), one axis ---------------------------------------
// Source position of each output sample of a growing axis: CImg walks
// curr += (old-1)/(new-1) in double, clamped to old-1 (CImg.h:28445-28452);
// the walk is sequential, so one thread writes the table.
__global__ void k_resize_table(int old_n, int new_n, int *__restrict__ src, double *__restrict__ frac) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    const double fx = new_n > 1 ? ((double)old_n - 1.0) / (double)(new_n - 1) : 0.0;
    double curr = 0.0;
    for (int x = 0; x < new_n; ++x) {
        const unsigned s = (unsigned)curr;
        frac[x] = curr - (double)s;
        src[x] = (int)s;
        const double nxt = curr + fx, lim = (double)old_n - 1.0;
        curr = (nxt < lim) ? nxt : lim;
    }
}

// mode 0: moving average (resize type 2): output t covers [t*old, (t+1)*old)
// and source s covers [s*new, (s+1)*new) of a common grid; the overlaps are
// accumulated in source order and divided by the old extent.  mode 1:
// Catmull-Rom in double from the table, clamped to the float range.
__global__ void k_resize_axis(const ResizeAxis ra, const float *__restrict__ in, float *__restrict__ out) {
    const long long total = (long long)ra.ox * ra.oy * ra.oz * ra.nc;
    const long long id = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (id >= total) return;
    long long rem = id;
    int o[3];
    o[0] = (int)(rem % ra.ox);
    rem /= ra.ox;
    o[1] = (int)(rem % ra.oy);
    rem /= ra.oy;
    o[2] = (int)(rem % ra.oz);
    const int ch = (int)(rem / ra.oz);
    const long long st[3] = {1, ra.ix, (long long)ra.ix * ra.iy};
    const int t = o[ra.axis];
    o[ra.axis] = 0;
    const float *line = in + ch * (long long)ra.ix * ra.iy * ra.iz + o[0] * st[0] + o[1] * st[1] + o[2] * st[2];
    const long long ss = st[ra.axis];
    float res;
    if (ra.mode == 0) {
        const unsigned long long oldn = (unsigned)ra.old_n, nn = (unsigned)ra.new_n;
        const unsigned long long lo = (unsigned long long)t * oldn, hi = lo + oldn;
        float acc = 0.0f;
        for (unsigned long long s = lo / nn; s <= (hi - 1) / nn; ++s) {
            const unsigned long long a = s * nn > lo ? s * nn : lo;
            const unsigned long long b = (s + 1) * nn < hi ? (s + 1) * nn : hi;
            acc += __ldg(line + s * ss) * (float)(unsigned)(b - a);
        }
        res = acc / (float)(unsigned)oldn;
    } else {
        const int s = __ldg(ra.src + t);
        const double f = __ldg(ra.frac + t);
        const int m = ra.old_n;
        const double val1 = (double)__ldg(line + s * ss);
        const double val0 = s > 0 ? (double)__ldg(line + (s - 1) * ss) : val1;
        const double val2 = s <= m - 2 ? (double)__ldg(line + (s + 1) * ss) : val1;
        const double val3 = s < m - 2 ? (double)__ldg(line + (s + 2) * ss) : val2;
        const double val = val1 + 0.5f * (f * (-val0 + val2) + f * f * (2 * val0 - 5 * val1 + 4 * val2 - val3) +
                                          f * f * f * (-val0 + 3 * val1 - 3 * val2 + val3));
        res = (float)(val < -FLT_MAX ? -FLT_MAX : val > FLT_MAX ? FLT_MAX : val);
    }
    o[ra.axis] = t;
    out[ch * (long long)ra.ox * ra.oy * ra.oz + o[0] + (long long)o[1] * ra.ox + (long long)o[2] * ra.ox * ra.oy] = res;
}

// CImg::get_gradient("xyz", 0): 3 planes of central differences, Neumann.
__global__ void __launch_bounds__(128) k_gradient(const Dims d, const float *__restrict__ img, float *__restrict__ g) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y, k = blockIdx.z;
    if (i >= d.x) return;
    const long long sy = d.x, sz = (long long)d.x * d.y, n = sz * d.z;
    const long long p = i + j * sy + k * sz;
    const long long xm = i > 0 ? p - 1 : p, xp = i < d.x - 1 ? p + 1 : p;
    const long long ym = j > 0 ? p - sy : p, yp = j < d.y - 1 ? p + sy : p;
    const long long zm = k > 0 ? p - sz : p, zp = k < d.z - 1 ? p + sz : p;
    g[p] = (__ldg(img + xp) - __ldg(img + xm)) / 2;
    g[n + p] = (__ldg(img + yp) - __ldg(img + ym)) / 2;
    g[2 * n + p] = (__ldg(img + zp) - __ldg(img + zm)) / 2;
}

// dst = src inside the ROI, nc planes (the write-back of optical_flow.h:503-533).
__global__ void __launch_bounds__(128) k_copy_roi(const Dims d, int nc, const FlowRoi roi,
                                                  const float *__restrict__ src, float *__restrict__ dst) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const int j = blockIdx.y, k = blockIdx.z % d.z, c = blockIdx.z / d.z;
    if (i >= d.x || c >= nc || !in_roi(roi, d, i, j, k)) return;
    const long long p = c * (long long)d.x * d.y * d.z + i + (long long)j * d.x + (long long)k * d.x * d.y;
    dst[p] = src[p];
}

inline dim3 vox_grid(const int *d, int zmul = 1) {
    return dim3((unsigned)((d[0] + 127) / 128), (unsigned)d[1], (unsigned)(d[2] * zmul));
}

}  // namespace

cudaError_t launch_warp_box(const int *dim, const float *box, const float *vel, const float *src, int nc, float dt,
                            float *out, cudaStream_t s) {
    k_warp_box<<<vox_grid(dim), 128, 0, s>>>(Dims{dim[0], dim[1], dim[2]}, box[0], box[1], box[2], vel, src, nc, dt,
                                             out);
    return cudaGetLastError();
}

cudaError_t launch_flow_setup(const int *d, const FlowRoi &roi, const float *i2w, const float *i1, const float *v,
                              float *u, float *tau, float *sig2, float *k4prev, cudaStream_t s) {
    k_flow_setup<<<vox_grid(d), 128, 0, s>>>(Dims{d[0], d[1], d[2]}, roi, i2w, i1, v, u, tau, sig2, k4prev);
    return cudaGetLastError();
}

cudaError_t launch_flow_primal(const int *d, const FlowRoi &roi, const float *y, const float *u, const float *tau,
                               const float *v_in, float *v_out, float *kty, int flags, double *resid, const int *done,
                               cudaStream_t s) {
    k_flow_primal<<<vox_grid(d), 128, 0, s>>>(Dims{d[0], d[1], d[2]}, roi, y, u, tau, v_in, v_out, kty, flags, resid,
                                              done);
    return cudaGetLastError();
}

cudaError_t launch_flow_dual(const int *d, const float *v, const float *v_old, const float *u, const float *sig2,
                             const float *k4prev, float *y, float sigma1, float hf, float lambda, int huber, int flags,
                             double *resid, const int *done, cudaStream_t s) {
    // lam2_lo = lambda^2 (1 - 2^-20) rounded down: s < lam2_lo gives sqrt(s) < lambda (1 - 2^-21), whose float
    // rounding stays below lambda, so sqrt(s)/lambda rounds to at most 1.
    const double l2 = (double)lambda * (double)lambda * (1.0 - 1.0 / 1048576.0);
    float lam2_lo = (float)l2;
    if ((double)lam2_lo > l2) lam2_lo = std::nextafter(lam2_lo, 0.0f);
    k_flow_dual<<<vox_grid(d), 128, 0, s>>>(Dims{d[0], d[1], d[2]}, v, v_old, u, sig2, k4prev, y, sigma1, hf, lambda,
                                            lam2_lo, huber, flags, resid, done);
    return cudaGetLastError();
}

cudaError_t launch_flow_settle(long long n3, const int *iters, const float *v_b, float *v_a, cudaStream_t s) {
    k_flow_settle<<<grid_stride_blocks(n3, 256), 256, 0, s>>>(n3, iters, v_b, v_a);
    return cudaGetLastError();
}

cudaError_t launch_flow_check(double *resid, long long n, float tol, int it, int is_resid, int is_last, int *done,
                              int *iters, float *err, cudaStream_t s) {
    k_flow_check<<<1, 1, 0, s>>>(resid, n, tol, it, is_resid, is_last, done, iters, err);
    return cudaGetLastError();
}

cudaError_t launch_flow_reset(int *done, double *resid, int *iters, float *err, cudaStream_t s) {
    k_flow_reset<<<1, 1, 0, s>>>(done, resid, iters, err);
    return cudaGetLastError();
}

cudaError_t launch_deriche(const int *d, int nc, int axis, const DericheCoef &c, float *img, float *tmp,
                           cudaStream_t s) {
    const long long per_ch =
        axis == 0 ? (long long)d[1] * d[2] : axis == 1 ? (long long)d[0] * d[2] : (long long)d[0] * d[1];
    const long long lines = per_ch * nc;
    k_deriche_line<<<(unsigned)((lines + 127) / 128), 128, 0, s>>>(Dims{d[0], d[1], d[2]}, nc, axis, c, img, tmp);
    return cudaGetLastError();
}

cudaError_t launch_resize_table(int old_n, int new_n, int *src, double *frac, cudaStream_t s) {
    k_resize_table<<<1, 1, 0, s>>>(old_n, new_n, src, frac);
    return cudaGetLastError();
}

cudaError_t launch_resize_axis(const ResizeAxis &ra, const float *in, float *out, cudaStream_t s) {
    const long long total = (long long)ra.ox * ra.oy * ra.oz * ra.nc;
    k_resize_axis<<<(unsigned)((total + 255) / 256), 256, 0, s>>>(ra, in, out);
    return cudaGetLastError();
}

cudaError_t launch_gradient(const int *d, const float *img, float *g, cudaStream_t s) {
    k_gradient<<<vox_grid(d), 128, 0, s>>>(Dims{d[0], d[1], d[2]}, img, g);
    return cudaGetLastError();
}

cudaError_t launch_copy_roi(const int *d, int nc, const FlowRoi &roi, const float *src, float *dst, cudaStream_t s) {
    k_copy_roi<<<vox_grid(d, nc), 128, 0, s>>>(Dims{d[0], d[1], d[2]}, nc, roi, src, dst);
    return cudaGetLastError();
}

}  // namespace stt
