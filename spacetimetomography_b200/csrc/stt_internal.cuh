// stt_internal.cuh -- device-side records and helpers shared by the kernels of libstt.so.
//
// Paths cited are relative to the reference project root (gmzang/SpaceTimeTomography);
// S/ = SpaceTimeTomography/.
#pragma once

#ifndef cuda_runtime_h
#include <cuda_runtime.h>
#endif
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
// (consecutive detector columns) sample consecutive addresses.
struct ViewRec {
    double src[3];
    double det0[3];
    double du[3];
    double dv[3];
    float A[9];
    float b[3];
    int layout;
    float pad[3];
};

struct GeomDev {
    int nx, ny, nz;
    int W, H;
    int n_views;
    double inv_sp[3];  // 1/spacing (M2V, TypicalRayProducer.cpp:160-169)
    float sd;          // sample distance |spacing| (ST_Tomography.cpp:300), FP32
    float cx, cy;      // (W-1)/2, (H-1)/2
    float sdd_ds;      // sdd / ds
};

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

// Compensated (Kahan) accumulator for ray sums.
struct Kahan {
    float s, c;
    __device__ __forceinline__ void add(float v) {
        float y = v - c;
        float t = s + y;
        c = (t - s) - y;
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

// x, then y, then z as the reference interpolates.
// One stored voxel as float: FP32 as is; BF16 storage (raw 16-bit patterns,
// the upper half of an FP32) widened exactly.
__device__ __forceinline__ float ld_voxel(const float *p) { return __ldg(p); }
__device__ __forceinline__ float ld_voxel(const unsigned short *p) {
    return __uint_as_float((unsigned)__ldg(p) << 16);
}

template <typename T>
__device__ __forceinline__ float tri_value(const T *__restrict__ vol, const Taps &t) {
    const T *p = vol + t.base;
    float v000 = ld_voxel(p), v100 = ld_voxel(p + t.dx);
    float v010 = ld_voxel(p + t.dy), v110 = ld_voxel(p + t.dy + t.dx);
    float v001 = ld_voxel(p + t.dz), v101 = ld_voxel(p + t.dz + t.dx);
    float v011 = ld_voxel(p + t.dz + t.dy), v111 = ld_voxel(p + t.dz + t.dy + t.dx);
    float fx1 = 1.0f - t.fx;
    float a = v000 * fx1 + v100 * t.fx;
    float b = v010 * fx1 + v110 * t.fx;
    float c = v001 * fx1 + v101 * t.fx;
    float d = v011 * fx1 + v111 * t.fx;
    float fy1 = 1.0f - t.fy;
    a = a * fy1 + b * t.fy;
    c = c * fy1 + d * t.fy;
    return a * (1.0f - t.fz) + c * t.fz;
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
template <typename Visit>
__device__ __forceinline__ void march(const GeomDev &g, const Ray &r, Visit &&visit) {
    const float sd = g.sd;
    const float tnear = r.tnear, tfar = r.tfar;
    float t1 = tnear;
    float pos1[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) pos1[k] = __fadd_rn(r.vz[k], __fmul_rn(r.vu[k], t1));
    visit(pos1);
    const int dims[3] = {g.nx, g.ny, g.nz};
    float tmax[3], tdelta[3], step[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        step[k] = __fmul_rn(r.vu[k], sd);
        const int b = dims[k];
        if (r.vu[k] == 0.0f) {
            tmax[k] = tfar;
            tdelta[k] = 0.0f;
        } else if (r.vu[k] < 0.0f) {
            int blk = ((int)ceilf(pos1[k] - 0.5f) - 1) / b;
            tmax[k] = __fdiv_rn(__fsub_rn(__fadd_rn((float)(blk * b), 0.5f), r.vz[k]), r.vu[k]);
            tdelta[k] = __fdiv_rn((float)(-b), r.vu[k]);
        } else {
            int blk = ((int)floorf(pos1[k] - 0.5f)) / b;
            tmax[k] = __fdiv_rn(__fsub_rn(__fadd_rn((float)((blk + 1) * b), 0.5f), r.vz[k]), r.vu[k]);
            tdelta[k] = __fdiv_rn((float)b, r.vu[k]);
        }
    }
    constexpr int kMaxSamples = 1 << 22;
    int budget = kMaxSamples;
    for (int seg = 0; seg < 16 && t1 < tfar && budget > 0; ++seg) {
        float tb = rmin(rmin(tmax[0], tmax[1]), tmax[2]);
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
            for (int k = 0; k < 3; ++k) pos[k] = __fadd_rn(pos[k], step[k]);
        }
        if (tmax[0] < tmax[1]) {
            if (tmax[0] < tmax[2]) tmax[0] += tdelta[0];
            else tmax[2] += tdelta[2];
        } else {
            if (tmax[1] < tmax[2]) tmax[1] += tdelta[1];
            else tmax[2] += tdelta[2];
        }
        t1 = tb;
    }
}

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

}  // namespace stt
