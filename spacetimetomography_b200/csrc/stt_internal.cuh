// stt_internal.cuh -- device-side records and helpers shared by the kernels of libstt.so.
//
// Paths cited are relative to the reference project root (gmzang/SpaceTimeTomography);
// S/ = SpaceTimeTomography/.
#pragma once

#ifndef cuda_runtime_h
#include <cuda_runtime.h>
#endif
#include <cuda_bf16.h>
#include <stdint.h>

namespace stt {

// Per-view projection record, built on the host in FP64 (stt_geometry.cpp).
//   Ray setup (ProduceRay, S/ImageFormationModel/TypicalRayProducer.core.h:32-69):
//     source `src` and the detector point of pixel (i,j) `det0 + i*du + j*dv`
//     in model coordinates (mm, origin at voxel (0,0,0)).
//   Voxel projection (ST_Tomography.cpp:698-703): camera coordinates of voxel
//     (x,y,z) are cam = A*(x,y,z) + b (FP32, voxel spacing and centring folded
//     in); the pixel is (W-1)/2 + cam.x/(-cam.z) * sdd/ds, likewise in y.
// `layout` selects the volume copy the forward projector gathers from: 0 the
// x-fastest volume, 1 a z-fastest transposed copy, chosen on the host for views
// whose central ray runs more along x than along z, so that a warp's 32 rays
// (consecutive detector columns) sample consecutive addresses.  `staged` marks
// the oblique views (central ray more than 25 degrees off both x and z), whose
// gathers spread over several planes per warp request: the forward projector
// with the SART correction stages their volume slabs into shared memory
// (k_fp_slab.cu) when it can.  `staged16` is the same choice for a BF16-stored
// volume (its gathers and boxes move half the bytes, so the faster projector
// can differ; the autotuner sets both).
struct ViewRec {
    double src[3];
    double det0[3];
    double du[3];
    double dv[3];
    float A[9];
    float b[3];
    int layout;
    int staged;
    int staged16;
    float pad;
};

// Whether a view goes to the slab-staged projector, for a volume stored as T.
template <typename T>
__device__ __forceinline__ bool view_staged(const ViewRec &v) {
    return sizeof(T) == 2 ? v.staged16 != 0 : v.staged != 0;
}

struct GeomDev {
    int nx, ny, nz;
    int W, H;
    int n_views;
    double inv_sp[3];  // 1/spacing (M2V, TypicalRayProducer.cpp:160-169)
    float sd;          // sample distance |spacing| (ST_Tomography.cpp:300), FP32
    float cx, cy;      // (W-1)/2, (H-1)/2
    float sdd_ds;      // sdd / ds
};

// Value a kernel writes to its status word when a bounded wait gave up (a
// TMA copy into shared memory that did not land within about 0.1 s).  The
// host reads it with stt_poll_status / stt_solver_poll_status.
#define STT_WAIT_TIMEOUT_FLAG 1

// The reference clamps with the macros max(a,b) = a>b?a:b, min(a,b) = a<b?a:b
// (ST_Tomography.cpp:167-173); their NaN behaviour (NaN -> the second operand
// of max) is part of the semantics, so fminf/fmaxf are not used for them.
template <typename T>
__device__ __forceinline__ T rmax(T a, T b) { return (a > b) ? a : b; }
template <typename T>
__device__ __forceinline__ T rmin(T a, T b) { return (a < b) ? a : b; }

// Which view a launch works on: a fixed index, or base + perm[slot] read from
// device memory (the solver's per-iteration view order, drawn on the device so
// that a captured CUDA graph replays with a fresh order each time).  `local`
// is the view's index within its frame (its slot in the projection stack).
struct ViewSel {
    int view;
    const int *perm;
    int slot;
    int base;
};

__device__ __forceinline__ int sel_view(const ViewSel &s, int &local) {
    local = s.perm ? __ldg(s.perm + s.slot) : s.view - s.base;
    return s.base + local;
}

// Compensated (Kahan) accumulator for ray sums.  Every operation is rounded
// on its own (no contraction), so kernels that add the same samples in the
// same order get the same bits whatever the compiler fuses around them.
struct Kahan {
    float s, c;
    __device__ __forceinline__ void add(float v) {
        const float y = __fsub_rn(v, c);
        const float t = __fadd_rn(s, y);
        c = __fsub_rn(__fsub_rn(t, s), y);
        s = t;
    }
};

// Ray in voxel-index space: pos(t) = vz + vu * t, t in mm.
struct Ray {
    float vz[3], vu[3];
    float tnear, tfar;
};

// ProduceRay in FP64 (TypicalRayProducer.core.h:32-69): normalised model-space
// direction, volume-space origin/direction, slab clip against [0, dims-1],
// tnear clamped to 0.  Rounded to FP32 for the march.
__device__ __forceinline__ void make_ray(const GeomDev &g, const ViewRec &v, int i, int j, Ray &r) {
    double d[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) d[k] = v.det0[k] + (double)i * v.du[k] + (double)j * v.dv[k] - v.src[k];
    double li = 1.0 / sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
    const int dims[3] = {g.nx, g.ny, g.nz};
    double tmin[3], tmax[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        double vz = v.src[k] * g.inv_sp[k];
        double vu = d[k] * li * g.inv_sp[k];
        double t1 = (0.0 - vz) / vu;
        double t2 = ((double)(dims[k] - 1) - vz) / vu;
        tmin[k] = rmin(t1, t2);
        tmax[k] = rmax(t1, t2);
        r.vz[k] = (float)vz;
        r.vu[k] = (float)vu;
    }
    double tn = rmax(rmax(tmin[0], tmin[1]), tmin[2]);
    tn = rmax(tn, 0.0);
    double tf = rmin(rmin(tmax[0], tmax[1]), tmax[2]);
    r.tnear = (float)tn;
    r.tfar = (float)tf;
}

// Clamped trilinear tap set (S/ImageFormationModel/SingleScalarVolume.core.h:87-120):
// position clamped to [0, dims-1], base truncated, +1 neighbours clamped.
// Element strides of the x, y, z axes: (1, nx, nx*ny) for the volume, or
// (nz*ny, nz, 1) for its z-fastest transposed copy; the values gathered and
// the interpolation order are the same for both.
struct Strides {
    int sx, sy, sz;
};

__device__ __forceinline__ Strides xyz_strides(const GeomDev &g) { return Strides{1, g.nx, g.nx * g.ny}; }
__device__ __forceinline__ Strides zyx_strides(const GeomDev &g) { return Strides{g.nz * g.ny, g.nz, 1}; }

struct Taps {
    long long base;
    int dx, dy, dz;   // neighbour offsets (0 at the upper edge)
    float fx, fy, fz;
};

__device__ __forceinline__ void make_taps(const GeomDev &g, const float p[3], Taps &t, const Strides &st) {
    float px = rmax(rmin(p[0], (float)(g.nx - 1)), 0.0f);
    float py = rmax(rmin(p[1], (float)(g.ny - 1)), 0.0f);
    float pz = rmax(rmin(p[2], (float)(g.nz - 1)), 0.0f);
    int ix = (int)px, iy = (int)py, iz = (int)pz;
    t.fx = px - (float)ix;
    t.fy = py - (float)iy;
    t.fz = pz - (float)iz;
    t.base = (long long)ix * st.sx + (long long)iy * st.sy + (long long)iz * st.sz;
    t.dx = (ix < g.nx - 1) ? st.sx : 0;
    t.dy = (iy < g.ny - 1) ? st.sy : 0;
    t.dz = (iz < g.nz - 1) ? st.sz : 0;
}

__device__ __forceinline__ void make_taps(const GeomDev &g, const float p[3], Taps &t) {
    make_taps(g, p, t, xyz_strides(g));
}

// One stored voxel as float: FP32 as is; BF16 storage (raw 16-bit patterns,
// the upper half of an FP32) widened exactly.
__device__ __forceinline__ float ld_voxel(const float *p) { return __ldg(p); }
__device__ __forceinline__ float ld_voxel(const unsigned short *p) {
    return __uint_as_float((unsigned)__ldg(p) << 16);
}

// Read-write arrays of either storage: a plain load widened to FP32, and a
// store of an FP32 value (BF16: rounded to nearest even by the CUDA
// conversion).  Arithmetic on stored values is always FP32.
__device__ __forceinline__ float ld_stored(const float *p) { return *p; }
__device__ __forceinline__ float ld_stored(const unsigned short *p) { return __uint_as_float((unsigned)*p << 16); }
__device__ __forceinline__ void st_stored(float *p, float v) { *p = v; }
__device__ __forceinline__ void st_stored(unsigned short *p, float v) {
    *p = __bfloat16_as_ushort(__float2bfloat16_rn(v));
}

// The forward projector's sample: the clamped trilinear value of
// SingleScalarVolume.core.h:87-120, lerped x, then y, then z as the reference
// does.  The position is clamped to [0, dims-1] as in make_taps, but the base
// is capped at dims-2, so the +1 neighbours are always one stride away and no
// tap offset is selected per sample.  Where the reference's base is dims-1
// (position exactly dims-1, fraction 0, +1 neighbour collapsed onto the base)
// this base is dims-2 with fraction exactly 1: the lerp then returns the
// dims-1 value exactly, as the reference's does, and the y and z lerps see the
// same operands.
struct FpCell {
    int ix, iy, iz;    // base voxel, each capped at dims-2
    float fx, fy, fz;  // fractions in [0, 1]
};

__device__ __forceinline__ void fp_cell(const GeomDev &g, const float p[3], FpCell &c) {
    const float px = rmax(rmin(p[0], (float)(g.nx - 1)), 0.0f);
    const float py = rmax(rmin(p[1], (float)(g.ny - 1)), 0.0f);
    const float pz = rmax(rmin(p[2], (float)(g.nz - 1)), 0.0f);
    c.ix = min((int)px, g.nx - 2);
    c.iy = min((int)py, g.ny - 2);
    c.iz = min((int)pz, g.nz - 2);
    c.fx = px - (float)c.ix;
    c.fy = py - (float)c.iy;
    c.fz = pz - (float)c.iz;
}

// v[k] is the corner (x + (k&1), y + ((k>>1)&1), z + (k>>2)).  Each lerp
// a*(1-f) + b*f is one explicit multiply and one fused multiply-add, so every
// kernel that interpolates the same corners gets the same bits.
__device__ __forceinline__ float lerp1(float a, float b, float f1, float f) {
    return __fmaf_rn(b, f, __fmul_rn(a, f1));
}

__device__ __forceinline__ float trilerp(const float v[8], const FpCell &c) {
    const float fx1 = __fsub_rn(1.0f, c.fx), fy1 = __fsub_rn(1.0f, c.fy), fz1 = __fsub_rn(1.0f, c.fz);
    const float a = lerp1(v[0], v[1], fx1, c.fx);
    const float b = lerp1(v[2], v[3], fx1, c.fx);
    const float d0 = lerp1(v[4], v[5], fx1, c.fx);
    const float d1 = lerp1(v[6], v[7], fx1, c.fx);
    return lerp1(lerp1(a, b, fy1, c.fy), lerp1(d0, d1, fy1, c.fy), fz1, c.fz);
}

// Two samples' cells and interpolations in the packed FP32x2 instructions of
// sm_100 (one instruction per pair of lanes).  Each lane is rounded as the
// scalar instruction it replaces, so trilerp2 returns bit for bit
// (trilerp(va, ca), trilerp(vb, cb)): 1 - f and p - floor(p) are fused
// multiply-adds with a multiplier of -1 (the product is exact, so the one
// rounding is that of the subtraction).
__device__ __forceinline__ float2 f2(float a, float b) { return make_float2(a, b); }

__device__ __forceinline__ void fp_cell2(const GeomDev &g, const float pa[3], const float pb[3], FpCell &ca,
                                         FpCell &cb) {
    float qa[3], qb[3];
    const float hi[3] = {(float)(g.nx - 1), (float)(g.ny - 1), (float)(g.nz - 1)};
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        qa[k] = rmax(rmin(pa[k], hi[k]), 0.0f);
        qb[k] = rmax(rmin(pb[k], hi[k]), 0.0f);
    }
    ca.ix = min((int)qa[0], g.nx - 2), cb.ix = min((int)qb[0], g.nx - 2);
    ca.iy = min((int)qa[1], g.ny - 2), cb.iy = min((int)qb[1], g.ny - 2);
    ca.iz = min((int)qa[2], g.nz - 2), cb.iz = min((int)qb[2], g.nz - 2);
    const float2 m1 = f2(-1.0f, -1.0f);
    const float2 fx = __ffma2_rn(f2((float)ca.ix, (float)cb.ix), m1, f2(qa[0], qb[0]));
    const float2 fy = __ffma2_rn(f2((float)ca.iy, (float)cb.iy), m1, f2(qa[1], qb[1]));
    const float2 fz = __ffma2_rn(f2((float)ca.iz, (float)cb.iz), m1, f2(qa[2], qb[2]));
    ca.fx = fx.x, cb.fx = fx.y, ca.fy = fy.x, cb.fy = fy.y, ca.fz = fz.x, cb.fz = fz.y;
}

__device__ __forceinline__ float2 lerp2(float2 a, float2 b, float2 f1, float2 f) {
    return __ffma2_rn(b, f, __fmul2_rn(a, f1));
}

__device__ __forceinline__ float2 trilerp2(const float va[8], const float vb[8], const FpCell &ca, const FpCell &cb) {
    const float2 m1 = f2(-1.0f, -1.0f), one = f2(1.0f, 1.0f);
    const float2 fx = f2(ca.fx, cb.fx), fy = f2(ca.fy, cb.fy), fz = f2(ca.fz, cb.fz);
    const float2 fx1 = __ffma2_rn(m1, fx, one), fy1 = __ffma2_rn(m1, fy, one), fz1 = __ffma2_rn(m1, fz, one);
    const float2 a = lerp2(f2(va[0], vb[0]), f2(va[1], vb[1]), fx1, fx);
    const float2 b = lerp2(f2(va[2], vb[2]), f2(va[3], vb[3]), fx1, fx);
    const float2 d0 = lerp2(f2(va[4], vb[4]), f2(va[5], vb[5]), fx1, fx);
    const float2 d1 = lerp2(f2(va[6], vb[6]), f2(va[7], vb[7]), fx1, fx);
    return lerp2(lerp2(a, b, fy1, fy), lerp2(d0, d1, fy1, fy), fz1, fz);
}

// One voxel of an array that the running kernel itself writes elsewhere (the
// persistent sweep): a plain, L1-cached load, ordered after the kernel's own
// barriers, never the read-only ld.global.nc path, which may return data
// older than a write made earlier in the same launch.
template <typename T>
__device__ __forceinline__ float ld_src(const T *p, bool rw) {
    return rw ? ld_stored(p) : ld_voxel(p);
}

// The 8 corners of a cell from a volume array: FAST is its contiguous axis
// (0: x, the volume; 2: z, its transposed copy), whose +1 neighbour is the
// next element.  I is the index type: int when the volume has fewer than
// 2^31 voxels.  RW: the array is written by the same launch (ld_src).
template <int FAST, typename I, typename T, bool RW = false>
__device__ __forceinline__ void fp_corners(const T *src, const Strides &st, const FpCell &c, float v[8]) {
    const I idx = (I)c.ix * st.sx + (I)c.iy * st.sy + (I)c.iz * st.sz;
    if (FAST == 0) {  // rows along x at (y, z), (y+1, z), (y, z+1), (y+1, z+1)
        const I r00 = idx, r10 = idx + st.sy, r01 = idx + st.sz, r11 = r01 + st.sy;
        v[0] = ld_src(src + r00, RW), v[1] = ld_src(src + r00 + 1, RW);
        v[2] = ld_src(src + r10, RW), v[3] = ld_src(src + r10 + 1, RW);
        v[4] = ld_src(src + r01, RW), v[5] = ld_src(src + r01 + 1, RW);
        v[6] = ld_src(src + r11, RW), v[7] = ld_src(src + r11 + 1, RW);
    } else {  // runs along z at (x, y), (x+1, y), (x, y+1), (x+1, y+1)
        const I r00 = idx, r10 = idx + st.sx, r01 = idx + st.sy, r11 = r10 + st.sy;
        v[0] = ld_src(src + r00, RW), v[4] = ld_src(src + r00 + 1, RW);
        v[1] = ld_src(src + r10, RW), v[5] = ld_src(src + r10 + 1, RW);
        v[2] = ld_src(src + r01, RW), v[6] = ld_src(src + r01 + 1, RW);
        v[3] = ld_src(src + r11, RW), v[7] = ld_src(src + r11 + 1, RW);
    }
}

// The same 8 corners through two tld4 gathers of a pitch-linear 2D texture
// whose rows are the array's slices across its slowest axis: for the volume
// (FAST 0) texel (x + nx*y, z); for the z-fastest copy (FAST 2) texel
// (z + nz*y, x).  A gather at texel (u, v) returns {u, u+1} x {v, v+1} (.w =
// (u, v), .z = (u+1, v), .x = (u, v+1), .y = (u+1, v+1)): the fast-axis pair
// of two neighbouring slices; the second gather, one row of `row` texels on,
// is the y+1 pair.  The cell's base is at most dims-2 on every axis, so no
// gather leaves the array or crosses into another row of slices.
// T: the texels' storage; BF16 (unsigned short bits, a 16-bit unsigned
// texture) is widened exactly to FP32 as ld_voxel does.
__device__ __forceinline__ float4 gather_texels(unsigned long long tex, float u, float v, const float *) {
    return tex2Dgather<float4>(tex, u, v, 0);
}
__device__ __forceinline__ float4 gather_texels(unsigned long long tex, float u, float v, const unsigned short *) {
    const ushort4 r = tex2Dgather<ushort4>(tex, u, v, 0);
    return make_float4(__uint_as_float((unsigned)r.x << 16), __uint_as_float((unsigned)r.y << 16),
                       __uint_as_float((unsigned)r.z << 16), __uint_as_float((unsigned)r.w << 16));
}

template <int FAST, typename T = float>
__device__ __forceinline__ void fp_corners_tex(unsigned long long tex, int row, const FpCell &c, float v[8]) {
    const int u = FAST == 0 ? c.ix + row * c.iy : c.iz + row * c.iy;
    const float fv = (float)(FAST == 0 ? c.iz : c.ix) + 1.0f;
    const float4 a = gather_texels(tex, (float)u + 1.0f, fv, (const T *)nullptr);
    const float4 b = gather_texels(tex, (float)(u + row) + 1.0f, fv, (const T *)nullptr);
    if (FAST == 0) {  // u along x, v along z
        v[0] = a.w, v[1] = a.z, v[4] = a.x, v[5] = a.y;
        v[2] = b.w, v[3] = b.z, v[6] = b.x, v[7] = b.y;
    } else {  // u along z, v along x
        v[0] = a.w, v[4] = a.z, v[1] = a.x, v[5] = a.y;
        v[2] = b.w, v[6] = b.z, v[3] = b.x, v[7] = b.y;
    }
}

template <int FAST, typename I, typename T>
__device__ __forceinline__ float fp_sample(const GeomDev &g, const T *__restrict__ src, const Strides &st,
                                           const float p[3]) {
    FpCell c;
    fp_cell(g, p, c);
    float v[8];
    fp_corners<FAST, I>(src, st, c, v);
    return trilerp(v, c);
}

// Corner weights in the order of SingleScalarVolume.core.h:104-105.
__device__ __forceinline__ void tri_weights(const Taps &t, float w[8]) {
    float m0 = 1.0f - t.fx, m1 = 1.0f - t.fy, m2 = 1.0f - t.fz;
    w[0] = m0 * m1 * m2;
    w[1] = t.fx * m1 * m2;
    w[2] = m0 * t.fy * m2;
    w[3] = t.fx * t.fy * m2;
    w[4] = m0 * m1 * t.fz;
    w[5] = t.fx * m1 * t.fz;
    w[6] = m0 * t.fy * t.fz;
    w[7] = t.fx * t.fy * t.fz;
}

__device__ __forceinline__ long long tap_index(const Taps &t, int k) {
    return t.base + ((k & 1) ? t.dx : 0) + ((k & 2) ? t.dy : 0) + ((k & 4) ? t.dz : 0);
}

// The ray-driven backprojection's update of one sample: (c*w_k, w_k) into the
// interleaved accumulators of its 8 corners (x-fastest taps).  Corners 2m
// and 2m+1 are x-neighbours; inside the volume (dx = 1) their accumulators
// are adjacent, and where the first one's address is 16-byte aligned the two
// are one vector atomic instead of two 8-byte ones (the same terms, fewer
// atomics at L2, whose atomic rate bounds the scatter).  The test is on the
// address, not on the index: a frame's accumulators start at acc + f * n,
// which is only 8-byte aligned when f and n are odd.
__device__ __forceinline__ void scatter_corners(float2 *acc, const Taps &t, float c, const float w[8]) {
#pragma unroll
    for (int m = 0; m < 8; m += 2) {
        const long long idx = tap_index(t, m);
        if (t.dx == 1 && !(reinterpret_cast<uintptr_t>(acc + idx) & 15)) {
            atomicAdd(reinterpret_cast<float4 *>(acc + idx), make_float4(c * w[m], w[m], c * w[m + 1], w[m + 1]));
        } else {
            atomicAdd(acc + idx, make_float2(c * w[m], w[m]));
            atomicAdd(acc + idx + t.dx, make_float2(c * w[m + 1], w[m + 1]));
        }
    }
}

// The march of CastingRay (S/ImageFormationModel/RayCaster.core.h:42-188).  The
// DDA over blocks of size dims splits a ray only where it crosses coordinate
// 0.5 on an axis it travels down; each segment restarts at
// ceil((t1-tnear)/sd)*sd + tnear with pos recomputed, then steps t += sd,
// pos += vu*sd.  The entry sample is visited once before the loop and again
// as the first sample of the first segment.  A split point can lie before
// tnear (entry coordinate in [0, 0.5) on a descending axis); the reference then
// restarts at ceil of a negative count and re-walks clamped samples outside the
// box up to the split's far end, and so does this march.  `visit(pos)` is
// called per sample.  Loops are bounded by the segment's own extent
// ((tb - t)/sd + 2 samples), at most 16 segments, and 2^22 samples per ray.
// Splits and steps of the march (RayCaster.core.h:62-128): the per-sample
// step vu*sd, the first split point along each axis and the split spacing.
struct MarchDda {
    float tmax[3], tdelta[3], step[3];
};

__device__ __forceinline__ void march_dda(const GeomDev &g, const Ray &r, const float pos1[3], MarchDda &d) {
    const int dims[3] = {g.nx, g.ny, g.nz};
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        d.step[k] = __fmul_rn(r.vu[k], g.sd);
        const int b = dims[k];
        if (r.vu[k] == 0.0f) {
            d.tmax[k] = r.tfar;
            d.tdelta[k] = 0.0f;
        } else if (r.vu[k] < 0.0f) {
            int blk = ((int)ceilf(pos1[k] - 0.5f) - 1) / b;
            d.tmax[k] = __fdiv_rn(__fsub_rn(__fadd_rn((float)(blk * b), 0.5f), r.vz[k]), r.vu[k]);
            d.tdelta[k] = __fdiv_rn((float)(-b), r.vu[k]);
        } else {
            int blk = ((int)floorf(pos1[k] - 0.5f)) / b;
            d.tmax[k] = __fdiv_rn(__fsub_rn(__fadd_rn((float)((blk + 1) * b), 0.5f), r.vz[k]), r.vu[k]);
            d.tdelta[k] = __fdiv_rn((float)b, r.vu[k]);
        }
    }
}

__device__ __forceinline__ void march_split(MarchDda &d) {
    if (d.tmax[0] < d.tmax[1]) {
        if (d.tmax[0] < d.tmax[2]) d.tmax[0] += d.tdelta[0];
        else d.tmax[2] += d.tdelta[2];
    } else {
        if (d.tmax[1] < d.tmax[2]) d.tmax[1] += d.tdelta[1];
        else d.tmax[2] += d.tdelta[2];
    }
}

// The march, handing the samples of a segment out G at a time where G
// remain: visitg(p) gets consecutive samples p[0..G) (in that order), visit(p)
// the entry sample and the last ones of a segment.  The samples and their
// order are those of march() (t only grows, so the G-th sample inside the
// segment implies the ones before it); a caller that issues all G samples'
// loads before using any keeps G times the loads in flight.
template <int G, typename Visit, typename VisitG>
__device__ __forceinline__ void march_groups(const GeomDev &g, const Ray &r, Visit &&visit, VisitG &&visitg) {
    const float sd = g.sd;
    const float tnear = r.tnear, tfar = r.tfar;
    float t1 = tnear;
    float pos1[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) pos1[k] = __fadd_rn(r.vz[k], __fmul_rn(r.vu[k], t1));
    visit(pos1);
    MarchDda d;
    march_dda(g, r, pos1, d);
    constexpr int kMaxSamples = 1 << 22;
    int budget = kMaxSamples;
    for (int seg = 0; seg < 16 && t1 < tfar && budget > 0; ++seg) {
        float tb = rmin(rmin(d.tmax[0], d.tmax[1]), d.tmax[2]);
        if (tb > tfar) tb = tfar;
        float t = __fadd_rn(__fmul_rn(ceilf(__fdiv_rn(__fsub_rn(t1, tnear), sd)), sd), tnear);
        float pos[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) pos[k] = __fadd_rn(r.vz[k], __fmul_rn(r.vu[k], t));
        // fminf drops a NaN extent; the t < tb test then ends the segment
        const int cap = (int)fminf(ceilf(__fdiv_rn(tb - t, sd)) + 2.0f, (float)budget);
        budget -= cap > 0 ? cap : 0;
        int n = 0;
        // (x, y) and (t, z) advance as packed pairs: the same float additions
        const float2 sxy = make_float2(d.step[0], d.step[1]), stz = make_float2(sd, d.step[2]);
        while (n < cap && t < tb) {
            float2 xy[G], tz[G];  // the group's samples; tz[G-1].x is the time of its last
            xy[0] = make_float2(pos[0], pos[1]);
            tz[0] = make_float2(t, pos[2]);
#pragma unroll
            for (int i = 1; i < G; ++i) {
                xy[i] = __fadd2_rn(xy[i - 1], sxy);
                tz[i] = __fadd2_rn(tz[i - 1], stz);
            }
            if (n + G - 1 < cap && tz[G - 1].x < tb) {
                float p[G][3];
#pragma unroll
                for (int i = 0; i < G; ++i) p[i][0] = xy[i].x, p[i][1] = xy[i].y, p[i][2] = tz[i].y;
                visitg(p);
                const float2 nxy = __fadd2_rn(xy[G - 1], sxy), ntz = __fadd2_rn(tz[G - 1], stz);
                t = ntz.x;
                pos[0] = nxy.x, pos[1] = nxy.y, pos[2] = ntz.y;
                n += G;
            } else {
                visit(pos);
                const float2 nxy = __fadd2_rn(xy[0], sxy), ntz = __fadd2_rn(tz[0], stz);
                t = ntz.x;
                pos[0] = nxy.x, pos[1] = nxy.y, pos[2] = ntz.y;
                ++n;
            }
        }
        march_split(d);
        t1 = tb;
    }
}

template <typename Visit>
__device__ __forceinline__ void march(const GeomDev &g, const Ray &r, Visit &&visit) {
    const float sd = g.sd;
    const float tnear = r.tnear, tfar = r.tfar;
    float t1 = tnear;
    float pos1[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) pos1[k] = __fadd_rn(r.vz[k], __fmul_rn(r.vu[k], t1));
    visit(pos1);
    MarchDda d;
    march_dda(g, r, pos1, d);
    constexpr int kMaxSamples = 1 << 22;
    int budget = kMaxSamples;
    for (int seg = 0; seg < 16 && t1 < tfar && budget > 0; ++seg) {
        float tb = rmin(rmin(d.tmax[0], d.tmax[1]), d.tmax[2]);
        if (tb > tfar) tb = tfar;
        float t = __fadd_rn(__fmul_rn(ceilf(__fdiv_rn(__fsub_rn(t1, tnear), sd)), sd), tnear);
        float pos[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) pos[k] = __fadd_rn(r.vz[k], __fmul_rn(r.vu[k], t));
        // fminf drops a NaN extent; the t < tb test then ends the segment
        const int cap = (int)fminf(ceilf(__fdiv_rn(tb - t, sd)) + 2.0f, (float)budget);
        budget -= cap > 0 ? cap : 0;
        for (int n = 0; n < cap && t < tb; ++n) {
            visit(pos);
            t = __fadd_rn(t, sd);
#pragma unroll
            for (int k = 0; k < 3; ++k) pos[k] = __fadd_rn(pos[k], d.step[k]);
        }
        march_split(d);
        t1 = tb;
    }
}

// march() as a resumable generator, for kernels that interleave the samples
// of many rays with block-wide steps: peek() makes `pos` the next sample (false
// when the ray is done), advance() moves past it.  The same samples in the
// same order, from the same float operations: the entry sample, then each
// segment restarted at ceil((t1 - tnear)/sd)*sd + tnear, with the same caps.
struct MarchGen {
    float vz[3], vu[3];
    MarchDda d;
    float pos[3];
    float tnear, tfar, sd, t1, t, tb;
    int seg, n, cap, budget;
    int phase;  // 0: entry sample pending, 1: in a segment, 2: done

    __device__ __forceinline__ void init(const GeomDev &g, const Ray &r) {
        sd = g.sd;
        tnear = r.tnear;
        tfar = r.tfar;
        t1 = tnear;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            vz[k] = r.vz[k];
            vu[k] = r.vu[k];
            pos[k] = __fadd_rn(vz[k], __fmul_rn(vu[k], t1));
        }
        march_dda(g, r, pos, d);
        seg = 0;
        budget = 1 << 22;
        phase = 0;
    }

    __device__ __forceinline__ void start_segment() {
        if (seg < 16 && t1 < tfar && budget > 0) {
            tb = rmin(rmin(d.tmax[0], d.tmax[1]), d.tmax[2]);
            if (tb > tfar) tb = tfar;
            t = __fadd_rn(__fmul_rn(ceilf(__fdiv_rn(__fsub_rn(t1, tnear), sd)), sd), tnear);
#pragma unroll
            for (int k = 0; k < 3; ++k) pos[k] = __fadd_rn(vz[k], __fmul_rn(vu[k], t));
            cap = (int)fminf(ceilf(__fdiv_rn(tb - t, sd)) + 2.0f, (float)budget);
            budget -= cap > 0 ? cap : 0;
            n = 0;
            phase = 1;
        } else {
            phase = 2;
        }
    }

    __device__ __forceinline__ void end_segment() {
        march_split(d);
        t1 = tb;
        ++seg;
    }

    __device__ __forceinline__ bool peek() {
        while (phase == 1 && !(n < cap && t < tb)) {
            end_segment();
            start_segment();
        }
        return phase != 2;
    }

    __device__ __forceinline__ void advance() {
        if (phase == 0) {  // the entry sample is done; segment 0 starts at tnear
            start_segment();
            return;
        }
        t = __fadd_rn(t, sd);
#pragma unroll
        for (int k = 0; k < 3; ++k) pos[k] = __fadd_rn(pos[k], d.step[k]);
        ++n;
    }
};

// tld4 of the 2x2 texels {u, u+1} x {v, v+1} of one layer of a layered 2D
// texture (coordinate (u+1, v+1), point sampling, clamp addressing):
// .w = (u, v), .z = (u+1, v), .x = (u, v+1), .y = (u+1, v+1).
__device__ __forceinline__ float4 gather_layer(unsigned long long tex, int u, int v, int layer) {
    float4 r;
    asm volatile("tld4.r.a2d.v4.f32.f32 {%0, %1, %2, %3}, [%4, {%5, %6, %7, %7}];"
                 : "=f"(r.x), "=f"(r.y), "=f"(r.z), "=f"(r.w)
                 : "l"(tex), "r"(layer), "f"((float)u + 1.0f), "f"((float)v + 1.0f));
    return r;
}

// Catmull-Rom weights for taps (-1, 0, +1, +2) at fraction d (the cubic of
// ST_Tomography.cpp:183-186 and CImg's _cubic_atX, written in weight form).
__device__ __forceinline__ void cr_weights(float d, float w[4]) {
    float d2 = d * d, d3 = d2 * d;
    w[0] = 0.5f * (-d + 2.0f * d2 - d3);
    w[1] = 1.0f + 0.5f * (-5.0f * d2 + 3.0f * d3);
    w[2] = 0.5f * (d + 4.0f * d2 - 3.0f * d3);
    w[3] = 0.5f * (-d2 + d3);
}

// The ray sum of one forward-projector ray (hit rays only): the Kahan sum of
// its samples times the sample distance.  Samples go G at a time where the
// march allows: all their taps are fetched before any is interpolated.  The
// sum is the same for every G (the samples are added one by one in march
// order).
constexpr int FP_GROUP = 4;

// `corners(k, c, v)` fetches the 8 corners of cell c, the k-th sample of a
// group (0 for a sample on its own): loads from an array, or tld4 gathers of
// its texture (the same values).
template <int G = FP_GROUP, bool PK = false, typename Corners>
__device__ __forceinline__ float fp_ray_sum_with(const GeomDev &g, const Corners &corners, const Ray &r, int *count) {
    Kahan acc{0.0f, 0.0f};
    int n = 0;
    march_groups<G>(
        g, r,
        [&](const float p[3]) {
            FpCell c;
            fp_cell(g, p, c);
            float v[8];
            corners(0, c, v);
            acc.add(__fmul_rn(trilerp(v, c), g.sd));
            ++n;
        },
        [&](const float (*p)[3]) {
            FpCell c[G];
            float v[G][8];
            if constexpr (PK) {  // pairs of samples in the packed FP32x2 instructions
                static_assert(G % 2 == 0, "samples go in packed pairs");
#pragma unroll
                for (int i = 0; i < G; i += 2) {
                    fp_cell2(g, p[i], p[i + 1], c[i], c[i + 1]);
                    corners(i, c[i], v[i]);
                    corners(i + 1, c[i + 1], v[i + 1]);
                }
                const float2 sd2 = make_float2(g.sd, g.sd);
#pragma unroll
                for (int i = 0; i < G; i += 2) {
                    const float2 s = __fmul2_rn(trilerp2(v[i], v[i + 1], c[i], c[i + 1]), sd2);
                    acc.add(s.x);
                    acc.add(s.y);
                }
            } else {
#pragma unroll
                for (int i = 0; i < G; ++i) {
                    fp_cell(g, p[i], c[i]);
                    corners(i, c[i], v[i]);
                }
#pragma unroll
                for (int i = 0; i < G; ++i) acc.add(__fmul_rn(trilerp(v[i], c[i]), g.sd));
            }
            n += G;
        });
    if (count) *count = n;
    return acc.s;
}

__device__ __host__ __forceinline__ unsigned long long splitmix(unsigned long long &s) {
    unsigned long long z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// Seed of frame f's view order in PD iteration `iter` (the reference reseeds
// with time(0) in every SART call, ST_Tomography.cpp:635).  f is the frame's
// index in the whole sequence of `frames`, so that shards of a frame-sharded
// solve draw the orders the unsharded solve would.
__device__ __host__ __forceinline__ unsigned long long frame_seed(unsigned long long seed,
                                                                 unsigned long long iter, int frames,
                                                                 int f) {
    return seed + 0x9E3779B97F4A7C15ull * (iter * (unsigned long long)frames + (unsigned long long)f + 1ull);
}

// The view order of frame f (of a sequence of `frames`) in PD iteration
// `iter`: Fisher-Yates with SplitMix64 (the same stream as stt_permutation).
__device__ __host__ __forceinline__ void view_order(unsigned long long seed, unsigned long long iter, int frames,
                                                    int f, int views, int *p) {
    for (int i = 0; i < views; ++i) p[i] = i;
    unsigned long long s = frame_seed(seed, iter, frames, f);
    for (int i = views - 1; i > 0; --i) {
        const int j = (int)(splitmix(s) % (unsigned long long)(i + 1));
        const int t = p[i];
        p[i] = p[j];
        p[j] = t;
    }
}

// One job of the persistent sweep (k_persist.cu): one frame's SART call (or
// one batch instance's) -- V views in the order perm[0 .. V), each the
// transpose (views that gather along x), the forward projection with the
// correction and the voxel-based backprojection -- then the ROI mask with the
// over-relaxation.  Jobs run in rounds: in its round a job has blocks
// [block0, block0 + nblocks) of the launch, which meet at the job's own
// barrier between phases; a block goes on to its job of the next round when
// its job is done (jobs are independent).  Built on the host; vol, volt,
// stack, xprev and xbar are arrays of the launch's storage (float, or BF16
// bits).
struct SweepJob {
    GeomDev g;
    const ViewRec *views;  // the context's view table
    int *perm;             // V local view indices (drawn by an earlier launch, or by the whole-iteration launch)
    int view_base, V;      // view perm[i] of the job is table entry view_base + perm[i]
    void *vol, *volt;      // the frame's volume and its z-fastest copy
    const void *stack;     // V projections, W*H each, in local view order
    float *raylen, *corr;  // sticky ray lengths and the correction, W*H each
    void *xprev;
    void *xbar;            // over-relaxed X_bar (null: the ROI mask only)
    float alpha, gmax;
    int roi[8], pdcut[8];  // ROI mask cut, primal-dual region cut
    int round, block0, nblocks;
    unsigned *bar;         // [0] arrivals, [1] abort, [2] tile tickets; zeroed before every launch
    double work;           // relative cost, for the host's split of the blocks
    // The whole-iteration launch (k_iter_persistent) also runs, before the
    // SART call, the frame's view order, backward warp + dual step and forward
    // warp + primal step (ST_Tomography.cpp:492-578).
    float sigma, tau, tv_w, tp_w, bc_w, hf;
    int first;                         // the sequence's first frame: no f-1 terms in the primal step
    const void *xbar1;                 // X_bar[f+1] (the job's storage)
    const float *flow, *flow_prev;     // flow[f], flow[f-1]
    float *ytv, *ytp, *ybc;            // the frame's duals
    const float *ytp_prev, *ybc_prev;  // frame f-1's (written by its dual step in the same launch)
    unsigned long long seed;           // the view order: frame frame_seq of frames_total, iteration *counter
    unsigned long long *counter;
    int frame_seq, frames_total;
    int counter_owner;                 // this job advances *counter once every job has read it
};

}  // namespace stt
