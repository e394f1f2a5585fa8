// oracle/stt_oracle.cpp -- TEST INFRASTRUCTURE ONLY: the CPU restatement of the
// reconstruction hot path that the CUDA product is checked against.  It is never
// linked into, loaded by, or called from the product (spacetimetomography_b200/);
// only tests/, tests/golden/gen_golden.py and bench.py's CPU-baseline leg use it.
//
// Paths below are relative to the reference project root (gmzang/SpaceTimeTomography):
//   S/ = SpaceTimeTomography/
//
// Pinning: the FP32 flavour of the projector, the ray-BP scatter, the view
// geometry, warping::warp and CImg's cubic sampler are compared bit-for-bit (or
// to within float reassociation) against the reference's own code compiled into
// oracle/_ref (oracle/ref_driver.cpp), and against the committed fixtures in
// tests/golden/.  The SART/primal-dual loop body lives in
// S/ST_Tomo/ST_Tomography.cpp, which needs Eigen, libtiff and GLEW and is not
// compiled here; those lines are restated below and exercised on top of the
// pinned pieces.
//
// Arithmetic: float functions reproduce the reference's float expression order
// (this file is compiled with -ffp-contract=off); where the reference mixes in
// double literals or double members, the same promotions are made.  The double
// flavour is the same algorithm evaluated entirely in FP64, with the view
// geometry built directly in FP64 (the FP64 oracle).

#include "stt_oracle.h"

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

// ---------------------------------------------------------------------------
// Reference macro semantics.  The reference clamps with the Windows-style
// macros max(a,b) = a>b?a:b and min(a,b) = a<b?a:b (ST_Tomography.cpp:167-173,
// TypicalRayProducer.core.h:22-28); their NaN behaviour matters (a NaN voxel
// clamps to 0 in the ray-BP update) so they are kept as written.
template <typename A, typename B>
inline auto rmax(A a, B b) -> decltype(a + b) { return (a > b) ? a : b; }
template <typename A, typename B>
inline auto rmin(A a, B b) -> decltype(a + b) { return (a < b) ? a : b; }

// ---------------------------------------------------------------------------
// FP32 4x4 matrices, column-major, with the reference's element formulas
// (S/Math/Matrix4x4.h:66-90, 294-304; Matrix4x4.cpp:79-148).
struct M4 {
    float e[16];
};

M4 m4_identity() {
    M4 m;
    for (int i = 0; i < 16; ++i) m.e[i] = (i % 5 == 0) ? 1.0f : 0.0f;
    return m;
}

M4 m4_mul(const M4 &A, const M4 &B) {
    M4 R;
    for (int c = 0; c < 4; ++c)
        for (int r = 0; r < 4; ++r)
            R.e[4 * c + r] = A.e[r] * B.e[4 * c] + A.e[4 + r] * B.e[4 * c + 1] +
                             A.e[8 + r] * B.e[4 * c + 2] + A.e[12 + r] * B.e[4 * c + 3];
    return R;
}

void m4_apply(const M4 &M, const float v[4], float out[4]) {
    for (int r = 0; r < 4; ++r)
        out[r] = M.e[r] * v[0] + M.e[4 + r] * v[1] + M.e[8 + r] * v[2] + M.e[12 + r] * v[3];
}

inline float det3f(float a, float b, float c, float d, float e, float f, float g, float h,
                   float i) {
    return a * e * i + b * f * g + c * d * h - c * e * g - a * f * h - b * d * i;
}

// Adjugate / determinant inverse in the reference's term order
// (Matrix4x4::Inverse, Matrix4x4.cpp:80-135).  A singular matrix is left as is.
void m4_inverse(M4 &M) {
    const float *e = M.e;
    float a1 = e[0], b1 = e[1], c1 = e[2], d1 = e[3];
    float a2 = e[4], b2 = e[5], c2 = e[6], d2 = e[7];
    float a3 = e[8], b3 = e[9], c3 = e[10], d3 = e[11];
    float a4 = e[12], b4 = e[13], c4 = e[14], d4 = e[15];
    float k1 = det3f(b2, b3, b4, c2, c3, c4, d2, d3, d4);
    float k2 = det3f(a2, a3, a4, c2, c3, c4, d2, d3, d4);
    float k3 = det3f(a2, a3, a4, b2, b3, b4, d2, d3, d4);
    float k4 = det3f(a2, a3, a4, b2, b3, b4, c2, c3, c4);
    float det = a1 * k1 - b1 * k2 + c1 * k3 - d1 * k4;
    if (det == 0.0f) return;
    float inv = 1.0f / det;
    float o[16];
    o[0] = k1 * inv;
    o[4] = -k2 * inv;
    o[8] = k3 * inv;
    o[12] = -k4 * inv;
    o[1] = -det3f(b1, b3, b4, c1, c3, c4, d1, d3, d4) * inv;
    o[5] = det3f(a1, a3, a4, c1, c3, c4, d1, d3, d4) * inv;
    o[9] = -det3f(a1, a3, a4, b1, b3, b4, d1, d3, d4) * inv;
    o[13] = det3f(a1, a3, a4, b1, b3, b4, c1, c3, c4) * inv;
    o[2] = det3f(b1, b2, b4, c1, c2, c4, d1, d2, d4) * inv;
    o[6] = -det3f(a1, a2, a4, c1, c2, c4, d1, d2, d4) * inv;
    o[10] = det3f(a1, a2, a4, b1, b2, b4, d1, d2, d4) * inv;
    o[14] = -det3f(a1, a2, a4, b1, b2, b4, c1, c2, c4) * inv;
    o[3] = -det3f(b1, b2, b3, c1, c2, c3, d1, d2, d3) * inv;
    o[7] = det3f(a1, a2, a3, c1, c2, c3, d1, d2, d3) * inv;
    o[11] = -det3f(a1, a2, a3, b1, b2, b3, d1, d2, d3) * inv;
    o[15] = det3f(a1, a2, a3, b1, b2, b3, c1, c2, c3) * inv;
    std::memcpy(M.e, o, sizeof(o));
}

M4 m4_translate(float x, float y, float z) {
    M4 m = m4_identity();
    m.e[12] = x;
    m.e[13] = y;
    m.e[14] = z;
    return m;
}

// Quaternion (S/Math/Quaternion.cpp:7-40, Quaternion.h:86-126), FP32.
struct Q4 {
    float x, y, z, w;
};

Q4 q_axis_angle(float ax, float ay, float az, float angle) {
    Q4 q;
    float length = std::sqrt(ax * ax + ay * ay + az * az);
    if (length == 0.0f) return Q4{0.0f, 0.0f, 0.0f, 1.0f};
    float inv = 1.0f / length;
    float xx = ax * inv, yy = ay * inv, zz = az * inv;
    float rad = angle / 2;
    q.w = std::cos(rad);
    float s = std::sin(rad);
    q.x = xx * s;
    q.y = yy * s;
    q.z = zz * s;
    return q;
}

Q4 q_mul(const Q4 &p, const Q4 &q) {
    Q4 r;
    r.w = p.w * q.w - p.x * q.x - p.y * q.y - p.z * q.z;
    r.x = p.w * q.x + p.x * q.w + p.y * q.z - p.z * q.y;
    r.y = p.w * q.y + p.y * q.w + p.z * q.x - p.x * q.z;
    r.z = p.w * q.z + p.z * q.w + p.x * q.y - p.y * q.x;
    return r;
}

M4 q_matrix(const float q4[4]) {
    float x = q4[0], y = q4[1], z = q4[2], w = q4[3];
    M4 mat = m4_identity();
    float *m = mat.e;
    m[0] = 1.0f - 2.0f * (y * y + z * z);
    m[1] = 2.0f * (x * y + z * w);
    m[2] = 2.0f * (z * x - y * w);
    m[3] = 0.0f;
    m[4] = 2.0f * (x * y - z * w);
    m[5] = 1.0f - 2.0f * (z * z + x * x);
    m[6] = 2.0f * (y * z + x * w);
    m[7] = 0.0f;
    m[8] = 2.0f * (z * x + y * w);
    m[9] = 2.0f * (y * z - x * w);
    m[10] = 1.0f - 2.0f * (x * x + y * y);
    m[11] = 0.0f;
    m[12] = m[13] = m[14] = 0.0f;
    m[15] = 1.0f;
    return mat;
}

// ---------------------------------------------------------------------------
// Per-view geometry.
//
// View32 is the reference's FP32 matrix pipeline:
//   Scene::_calculateMatrix (S/ImageFormationModel/Scene.cpp:181-207),
//   TypicalRayProducer::_calculateMatrix (TypicalRayProducer.cpp:142-208),
//   eye from P2M (TypicalRayProducer.core.h:255-258).
// View64 is the same cone-beam geometry in closed form in FP64: the camera is
// T(-ox, -oz, oy - sid) * R_y(theta) applied to model coordinates centred at
// (dims-1)*spacing/2; detector pixel (i,j) sits on the near plane z = -sdd at
// ((i-(W-1)/2)*ds, (j-(H-1)/2)*ds).
struct View32 {
    M4 p2m, m2v, mv, v2m, mvv;
    float eye[4];
    double half_w, half_h;  // Scene::m_halfFrustumWidth/Height (double members)
    float sdd;              // Scene::m_sdd (float member)
    double ds;              // Scene::m_ds (double member)
};

struct View64 {
    double R[9];      // row-major rotation (model -> camera)
    double t[3];      // camera translation
    double ctr[3];    // model centre (dims-1)*sp/2
    double src[3];    // source, model coords (mm)
    double det0[3];   // pixel (0,0) on the detector, model coords
    double du[3], dv[3];
    double sp[3];
};

void make_view32(const orc_geom &g, const orc_view &v, View32 &o) {
    float spf[3] = {(float)g.sx, (float)g.sy, (float)g.sz};
    int dims[3] = {g.nx, g.ny, g.nz};
    // ST_Tomography ctor (ST_Tomography.cpp:229-246), Scene::_calculateCamera (Scene.cpp:77, 131-133)
    o.half_w = (g.W - 1) * g.ds * 0.5f;
    o.half_h = (g.H - 1) * g.ds * 0.5f;
    float m_sid = (float)g.sid;
    float m_sdd = (float)g.sdd;
    float zbase = -1 * m_sid;
    float nearp = m_sdd, farp = 10000.0f;
    float tr[3] = {(float)(-g.off[0]), (float)(-g.off[2]), (float)(+g.off[1])};
    // Scene::_calculateMatrix
    M4 view = m4_mul(m4_mul(m4_translate(tr[0], tr[1], zbase + tr[2]), m4_identity()),
                     q_matrix(v.quat));
    M4 proj = m4_identity();
    float *pm = proj.e;
    pm[0] = (float)(nearp / o.half_w);
    pm[1] = pm[2] = pm[3] = 0.0f;
    pm[4] = 0.0f;
    pm[5] = (float)(nearp / o.half_h);
    pm[6] = pm[7] = pm[8] = pm[9] = 0.0f;
    pm[10] = -(farp + nearp) / (farp - nearp);
    pm[11] = -1.0f;
    pm[12] = pm[13] = 0.0f;
    pm[14] = -2.0f * farp * nearp / (farp - nearp);
    pm[15] = 0.0f;
    // TypicalRayProducer::SetVolSize / _calculateMatrix
    float volsize[3];
    for (int k = 0; k < 3; ++k) volsize[k] = (dims[k] - 1) * spf[k];
    o.mv = m4_mul(view, m4_translate(-volsize[0] * 0.5f, -volsize[1] * 0.5f, -volsize[2] * 0.5f));
    o.m2v = m4_identity();
    o.m2v.e[0] = 1.0f / spf[0];
    o.m2v.e[5] = 1.0f / spf[1];
    o.m2v.e[10] = 1.0f / spf[2];
    o.v2m = o.m2v;
    m4_inverse(o.v2m);
    M4 vp = m4_identity();
    vp.e[0] = 0.5f * (g.W - 1);
    vp.e[5] = 0.5f * (g.H - 1);
    vp.e[10] = 0.5f;
    vp.e[11] = 0.0f;
    vp.e[12] = vp.e[0];
    vp.e[13] = vp.e[5];
    vp.e[14] = vp.e[10];
    vp.e[15] = 1.0f;
    M4 m2p = m4_mul(m4_mul(vp, proj), o.mv);
    o.p2m = m2p;
    m4_inverse(o.p2m);
    o.eye[0] = o.p2m.e[8] / o.p2m.e[11];
    o.eye[1] = o.p2m.e[9] / o.p2m.e[11];
    o.eye[2] = o.p2m.e[10] / o.p2m.e[11];
    o.eye[3] = 1.0f;
    o.mvv = m4_mul(o.mv, o.v2m);  // voxel BP: m_model_view * m_VolumeToModelMatrix (ST_Tomography.cpp:699)
    o.sdd = m_sdd;
    o.ds = g.ds;
}

void make_view64(const orc_geom &g, const orc_view &v, View64 &o) {
    double c = std::cos(v.angle), s = std::sin(v.angle);
    // R_y(theta): the rotation Quaternion(0,1,0,theta).ToMatrix() describes
    double R[9] = {c, 0, s, 0, 1, 0, -s, 0, c};
    std::memcpy(o.R, R, sizeof(R));
    o.t[0] = -g.off[0];
    o.t[1] = -g.off[2];
    o.t[2] = -g.sid + g.off[1];
    int dims[3] = {g.nx, g.ny, g.nz};
    o.sp[0] = g.sx;
    o.sp[1] = g.sy;
    o.sp[2] = g.sz;
    for (int k = 0; k < 3; ++k) o.ctr[k] = (dims[k] - 1) * o.sp[k] * 0.5;
    // model = ctr + R^T (cam - t)
    auto to_model = [&](const double cam[3], double out[3]) {
        double d[3] = {cam[0] - o.t[0], cam[1] - o.t[1], cam[2] - o.t[2]};
        for (int r = 0; r < 3; ++r)
            out[r] = o.ctr[r] + R[0 * 3 + r] * d[0] + R[1 * 3 + r] * d[1] + R[2 * 3 + r] * d[2];
    };
    double zero[3] = {0, 0, 0};
    to_model(zero, o.src);
    double p0[3] = {(0 - (g.W - 1) * 0.5) * g.ds, (0 - (g.H - 1) * 0.5) * g.ds, -g.sdd};
    to_model(p0, o.det0);
    for (int r = 0; r < 3; ++r) {
        o.du[r] = R[0 * 3 + r] * g.ds;
        o.dv[r] = R[1 * 3 + r] * g.ds;
    }
}

// ---------------------------------------------------------------------------
// The ray march (RayCaster.core.h:42-188).  The DDA over blocks of size
// bsize = dims degenerates to split points at coordinate 0.5 on axes that the
// ray crosses in the negative direction; every segment restarts its first
// sample at ceil((t1-tnear)/sd)*sd + tnear with pos recomputed, then steps
// pos += vu*sd.  The entry sample is taken once before the loop and again as
// the first sample of the first segment.
template <typename R, typename Sample>
R cast_ray(const R vz[3], const R vu[3], R tnear, R tfar, R sd, const int dims[3],
           Sample &&sample) {
    R density = 0;
    R t1 = tnear;
    R pos1[3] = {vz[0] + vu[0] * t1, vz[1] + vu[1] * t1, vz[2] + vu[2] * t1};
    R step[3] = {vu[0] * sd, vu[1] * sd, vu[2] * sd};
    R s1 = sample(pos1);
    density += s1 * sd;
    R tmax[3], tdelta[3];
    for (int c = 0; c < 3; ++c) {
        const int b = dims[c];
        if (vu[c] == 0) {
            tmax[c] = tfar;
            tdelta[c] = 0;
        } else if (vu[c] < 0) {
            int blk = ((int)std::ceil(pos1[c] - (R)0.5) - 1) / b;
            tmax[c] = ((R)(blk * b) + (R)0.5 - vz[c]) / vu[c];
            tdelta[c] = (R)(-b) / vu[c];
        } else {
            int blk = ((int)std::floor(pos1[c] - (R)0.5)) / b;
            tmax[c] = ((R)((blk + 1) * b) + (R)0.5 - vz[c]) / vu[c];
            tdelta[c] = (R)b / vu[c];
        }
    }
    while (t1 < tfar) {
        R tb = rmin(rmin(tmax[0], tmax[1]), tmax[2]);
        if (tb > tfar) tb = tfar;
        R t = std::ceil((t1 - tnear) / sd) * sd + tnear;
        R pos[3] = {vz[0] + vu[0] * t, vz[1] + vu[1] * t, vz[2] + vu[2] * t};
        while (t < tb) {
            density += sample(pos) * sd;
            t += sd;
            pos[0] += step[0];
            pos[1] += step[1];
            pos[2] += step[2];
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
    return density;
}

// Clamped trilinear sample setup (SingleScalarVolume.core.h:87-120): position
// clamped to [0, dims-1], base index truncated, upper neighbour clamped.
template <typename R>
struct Tri {
    long idx[8];
    R f[3];
};

template <typename R>
inline void tri_setup(const R pin[3], const int dims[3], Tri<R> &t) {
    int ip[3];
    for (int c = 0; c < 3; ++c) {
        R p = rmax(rmin(pin[c], (R)(dims[c] - 1)), (R)0);
        ip[c] = (int)p;
        t.f[c] = p - ip[c];
    }
    const long nx = dims[0], nxy = (long)dims[0] * dims[1];
    for (int k = 0; k < 8; ++k) {
        int x = ip[0] + (k & 1), y = ip[1] + ((k >> 1) & 1), z = ip[2] + ((k >> 2) & 1);
        x = rmax(rmin(x, dims[0] - 1), 0);
        y = rmax(rmin(y, dims[1] - 1), 0);
        z = rmax(rmin(z, dims[2] - 1), 0);
        t.idx[k] = x + y * nx + z * nxy;
    }
}

// Interpolation order of SingleScalarVolume.core.h:118-141: x, then y, then z.
template <typename R, typename V>
inline R tri_value(const V *vol, const Tri<R> &t) {
    R fx2 = t.f[0], fx1 = (R)1 - fx2;
    R a = (R)vol[t.idx[0]] * fx1 + (R)vol[t.idx[1]] * fx2;
    R b = (R)vol[t.idx[2]] * fx1 + (R)vol[t.idx[3]] * fx2;
    R c = (R)vol[t.idx[4]] * fx1 + (R)vol[t.idx[5]] * fx2;
    R d = (R)vol[t.idx[6]] * fx1 + (R)vol[t.idx[7]] * fx2;
    R fy2 = t.f[1], fy1 = (R)1 - fy2;
    a = a * fy1 + b * fy2;
    c = c * fy1 + d * fy2;
    R fz2 = t.f[2], fz1 = (R)1 - fz2;
    return a * fz1 + c * fz2;
}

// Corner weights in the order of SingleScalarVolume.core.h:104-105.
template <typename R>
inline void tri_weights(const Tri<R> &t, R w[8]) {
    R t0 = t.f[0], t1 = t.f[1], t2 = t.f[2];
    R m0 = (R)1 - t0, m1 = (R)1 - t1, m2 = (R)1 - t2;
    w[0] = m0 * m1 * m2;
    w[1] = t0 * m1 * m2;
    w[2] = m0 * t1 * m2;
    w[3] = t0 * t1 * m2;
    w[4] = m0 * m1 * t2;
    w[5] = t0 * m1 * t2;
    w[6] = m0 * t1 * t2;
    w[7] = t0 * t1 * t2;
}

// Ray setup for pixel (i, j): ProduceRay (TypicalRayProducer.core.h:32-69).
template <typename R>
struct RaySetup {
    R vz[3], vu[3], tnear, tfar;
};

inline void ray_setup32(const View32 &V, const int dims[3], int i, int j, RaySetup<float> &r) {
    float in[4] = {(float)i, (float)j, 0.0f, 1.0f};
    float mp[4];
    m4_apply(V.p2m, in, mp);
    float inv = 1.0f / mp[3];
    for (int k = 0; k < 4; ++k) mp[k] *= inv;
    float dir[4];
    for (int k = 0; k < 4; ++k) dir[k] = mp[k] - V.eye[k];
    float li = 1.0f / std::sqrt(dir[0] * dir[0] + dir[1] * dir[1] + dir[2] * dir[2]);
    dir[0] *= li;
    dir[1] *= li;
    dir[2] *= li;
    float vz4[4], vu4[4];
    m4_apply(V.m2v, V.eye, vz4);
    m4_apply(V.m2v, dir, vu4);
    float tmin[3], tmax[3];
    for (int c = 0; c < 3; ++c) {
        float t1 = (0.0f - vz4[c]) / vu4[c];
        float t2 = ((float)(dims[c] - 1) - vz4[c]) / vu4[c];
        tmin[c] = rmin(t1, t2);
        tmax[c] = rmax(t1, t2);
        r.vz[c] = vz4[c];
        r.vu[c] = vu4[c];
    }
    float tn = rmax(rmax(tmin[0], tmin[1]), tmin[2]);
    r.tnear = rmax(tn, 0.0f);
    r.tfar = rmin(rmin(tmax[0], tmax[1]), tmax[2]);
}

template <typename R>
inline void ray_setup64(const View64 &V, const int dims[3], int i, int j, RaySetup<R> &r) {
    double d[3];
    for (int k = 0; k < 3; ++k) d[k] = V.det0[k] + i * V.du[k] + j * V.dv[k] - V.src[k];
    double li = 1.0 / std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
    double tmin[3], tmax[3];
    double vz[3], vu[3];
    for (int c = 0; c < 3; ++c) {
        vz[c] = V.src[c] / V.sp[c];
        vu[c] = d[c] * li / V.sp[c];
        double t1 = (0.0 - vz[c]) / vu[c];
        double t2 = ((double)(dims[c] - 1) - vz[c]) / vu[c];
        tmin[c] = rmin(t1, t2);
        tmax[c] = rmax(t1, t2);
    }
    double tn = rmax(rmax(tmin[0], tmin[1]), tmin[2]);
    tn = rmax(tn, 0.0);
    double tf = rmin(rmin(tmax[0], tmax[1]), tmax[2]);
    for (int c = 0; c < 3; ++c) {
        r.vz[c] = (R)vz[c];
        r.vu[c] = (R)vu[c];
    }
    r.tnear = (R)tn;
    r.tfar = (R)tf;
}

template <typename R>
R sample_distance(const orc_geom &g) {
    if (sizeof(R) == sizeof(float)) {
        float sx = (float)g.sx, sy = (float)g.sy, sz = (float)g.sz;
        return (R)std::sqrt(sx * sx + sy * sy + sz * sz);
    }
    return (R)std::sqrt(g.sx * g.sx + g.sy * g.sy + g.sz * g.sz);
}

void set_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

// GenerateImage_MT (TypicalRayProducer.core.h:123-225) for one view.
template <typename R>
int fp_impl(const orc_geom &g, int gmode, const orc_view &v, const R *vol, R *img, R *raylen,
            R *weight, int j0 = 0, int j1 = -1) {
    const int dims[3] = {g.nx, g.ny, g.nz};
    View32 V32;
    View64 V64;
    if (gmode == 0) make_view32(g, v, V32);
    else make_view64(g, v, V64);
    const R sd = sample_distance<R>(g);
    if (j1 < 0 || j1 > g.H) j1 = g.H;
#pragma omp parallel for schedule(dynamic, 4)
    for (int j = j0; j < j1; ++j) {
        for (int i = 0; i < g.W; ++i) {
            long pix = i + (long)j * g.W;
            RaySetup<R> rs;
            if (gmode == 0) {
                RaySetup<float> r32;
                ray_setup32(V32, dims, i, j, r32);
                for (int c = 0; c < 3; ++c) {
                    rs.vz[c] = r32.vz[c];
                    rs.vu[c] = r32.vu[c];
                }
                rs.tnear = r32.tnear;
                rs.tfar = r32.tfar;
            } else {
                ray_setup64<R>(V64, dims, i, j, rs);
            }
            R value = 0;
            R count = 0;
            if (rs.tnear < rs.tfar) {
                if (raylen) raylen[pix] = rs.tfar - rs.tnear;
                value = cast_ray<R>(rs.vz, rs.vu, rs.tnear, rs.tfar, sd, dims, [&](const R p[3]) {
                    Tri<R> t;
                    tri_setup(p, dims, t);
                    count += 1;
                    return tri_value<R>(vol, t);
                });
            }
            if (weight) weight[pix] = count;
            if (img) img[pix] = value;
        }
    }
    return 0;
}

// BP-mode march (SingleScalarVolume.core.h:128-143, UpdateContributionSum :73-84):
// with adjoint=false scatters corr*w and w (the reference's ray BP); with
// adjoint=true scatters sd*w*y only (the exact transpose of fp_impl).
template <typename R>
int scatter_impl(const orc_geom &g, int gmode, const orc_view &v, const R *corr, R *contrib,
                 R *wsum, bool adjoint) {
    const int dims[3] = {g.nx, g.ny, g.nz};
    View32 V32;
    View64 V64;
    if (gmode == 0) make_view32(g, v, V32);
    else make_view64(g, v, V64);
    const R sd = sample_distance<R>(g);
    for (int j = 0; j < g.H; ++j) {
        for (int i = 0; i < g.W; ++i) {
            long pix = i + (long)j * g.W;
            RaySetup<R> rs;
            if (gmode == 0) {
                RaySetup<float> r32;
                ray_setup32(V32, dims, i, j, r32);
                for (int c = 0; c < 3; ++c) {
                    rs.vz[c] = r32.vz[c];
                    rs.vu[c] = r32.vu[c];
                }
                rs.tnear = r32.tnear;
                rs.tfar = r32.tfar;
            } else {
                ray_setup64<R>(V64, dims, i, j, rs);
            }
            if (!(rs.tnear < rs.tfar)) continue;
            const R cval = corr[pix];
            cast_ray<R>(rs.vz, rs.vu, rs.tnear, rs.tfar, sd, dims, [&](const R p[3]) {
                Tri<R> t;
                tri_setup(p, dims, t);
                R w[8];
                tri_weights(t, w);
                for (int k = 0; k < 8; ++k) {
                    if (adjoint) {
                        contrib[t.idx[k]] += sd * w[k] * cval;
                    } else {
                        contrib[t.idx[k]] += cval * w[k];
                        wsum[t.idx[k]] += w[k];
                    }
                }
                return (R)0;
            });
        }
    }
    return 0;
}

// Catmull-Rom helpers of ST_Tomography.cpp:183-197 (double literals, so the
// reference evaluates them in double and returns float).
inline float cubic_ref(const float p[4], float x) {
    return p[1] + 0.5 * x * (p[2] - p[0] + x * (2.0 * p[0] - 5.0 * p[1] + 4.0 * p[2] - p[3] +
                                                x * (3.0 * (p[1] - p[2]) + p[3] - p[0])));
}
inline double cubic_d(const double p[4], double x) {
    return p[1] + 0.5 * x * (p[2] - p[0] + x * (2.0 * p[0] - 5.0 * p[1] + 4.0 * p[2] - p[3] +
                                                x * (3.0 * (p[1] - p[2]) + p[3] - p[0])));
}

// Voxel-driven BP (ST_Tomography.cpp:690-730).
template <typename R>
int bp_voxel_impl(const orc_geom &g, int gmode, const orc_view &v, const R *corr, double alpha,
                  R gmax, R *vol) {
    View32 V32;
    View64 V64;
    if (gmode == 0) make_view32(g, v, V32);
    else make_view64(g, v, V64);
    const int W = g.W, H = g.H;
#pragma omp parallel for schedule(static)
    for (int z = 0; z < g.nz; ++z) {
        for (int y = 0; y < g.ny; ++y) {
            for (int x = 0; x < g.nx; ++x) {
                long pos = x + (long)y * g.nx + (long)z * g.nx * g.ny;
                R fpx, fpy;
                int px, py;
                if (gmode == 0) {
                    float vec[4] = {(float)x, (float)y, (float)z, 1.0f};
                    float det[4];
                    m4_apply(V32.mvv, vec, det);
                    float _px = V32.half_w - (det[0] / det[2]) * V32.sdd;
                    float _py = V32.half_h - (det[1] / det[2]) * V32.sdd;
                    _px = _px / V32.ds;
                    _py = _py / V32.ds;
                    px = (int)_px;
                    py = (int)_py;
                    fpx = _px - px;
                    fpy = _py - py;
                } else {
                    double m[3] = {x * V64.sp[0] - V64.ctr[0], y * V64.sp[1] - V64.ctr[1],
                                   z * V64.sp[2] - V64.ctr[2]};
                    double cam[3];
                    for (int r = 0; r < 3; ++r)
                        cam[r] = V64.R[r * 3 + 0] * m[0] + V64.R[r * 3 + 1] * m[1] +
                                 V64.R[r * 3 + 2] * m[2] + V64.t[r];
                    double half_w = (W - 1) * g.ds * 0.5, half_h = (H - 1) * g.ds * 0.5;
                    double _px = (half_w - (cam[0] / cam[2]) * g.sdd) / g.ds;
                    double _py = (half_h - (cam[1] / cam[2]) * g.sdd) / g.ds;
                    px = (int)_px;
                    py = (int)_py;
                    fpx = (R)(_px - px);
                    fpy = (R)(_py - py);
                }
                if (px < 2 || px >= W - 2 || py < 2 || py >= H - 2) continue;
                const R *pc = corr + (long)py * W + px;
                R val;
                if (sizeof(R) == sizeof(float)) {
                    float p[4][4], arr[4];
                    for (int a = 0; a < 4; ++a)
                        for (int b = 0; b < 4; ++b) p[a][b] = (float)pc[(a - 1) + (b - 1) * W];
                    for (int a = 0; a < 4; ++a) arr[a] = cubic_ref(p[a], (float)fpy);
                    val = (R)cubic_ref(arr, (float)fpx);
                    double nv = (double)vol[pos] + alpha * (double)val;
                    vol[pos] = (R)(float)nv;
                } else {
                    double p[4][4], arr[4];
                    for (int a = 0; a < 4; ++a)
                        for (int b = 0; b < 4; ++b) p[a][b] = (double)pc[(a - 1) + (b - 1) * W];
                    for (int a = 0; a < 4; ++a) arr[a] = cubic_d(p[a], (double)fpy);
                    val = (R)cubic_d(arr, (double)fpx);
                    vol[pos] = vol[pos] + (R)alpha * val;
                }
                vol[pos] = rmax(rmin(gmax, vol[pos]), (R)0);
            }
        }
    }
    return 0;
}

template <typename R>
void correction_impl(long n, const R *b, const R *ax, const R *raylen, R *c) {
    // ST_Tomography.cpp:673, Factor = sqrtf(2*SART_lambda) = 1 and pY == 0
    for (long k = 0; k < n; ++k) {
        R num = (R)1 * b[k] - (R)1 * ax[k] - (R)0;
        R den = (R)((R)1 * raylen[k] + 1.0);
        c[k] = num / den;
    }
}

template <typename R>
void bp_ray_update_impl(long n, const R *contrib, const R *wsum, R gmax, R *vol) {
    // ST_Tomography.cpp:746-762; 0/0 = NaN clamps to 0 through the macros
    for (long k = 0; k < n; ++k) {
        R r = (R)((1.0 * contrib[k]) / wsum[k]);
        vol[k] += r;
        vol[k] = rmax(rmin(gmax, vol[k]), (R)0);
    }
}

template <typename R>
int sart_impl(const orc_geom &g, int gmode, const orc_view *views, const int *perm, int nv,
              const R *proj, double alpha, R gmax, int bp_mode, R *vol, R *raylen, const R *roi) {
    const long npix = (long)g.W * g.H;
    const long nvox = (long)g.nx * g.ny * g.nz;
    std::vector<R> img(npix), wt(npix), c(npix);
    std::vector<R> contrib, wsum;
    if (bp_mode) {
        contrib.assign(nvox, 0);
        wsum.assign(nvox, 0);
    }
    for (int i = 0; i < nv; ++i) {
        const int vid = perm[i];
        fp_impl<R>(g, gmode, views[vid], vol, img.data(), raylen, wt.data());
        correction_impl<R>(npix, proj + (long)vid * npix, img.data(), raylen, c.data());
        if (bp_mode == 0) {
            bp_voxel_impl<R>(g, gmode, views[vid], c.data(), alpha, gmax, vol);
        } else {
            std::fill(contrib.begin(), contrib.end(), (R)0);
            std::fill(wsum.begin(), wsum.end(), (R)0);
            scatter_impl<R>(g, gmode, views[vid], c.data(), contrib.data(), wsum.data(), false);
            bp_ray_update_impl<R>(nvox, contrib.data(), wsum.data(), gmax, vol);
            // TypicalRayProducer::Initial (TypicalRayProducer.cpp:78-96)
            std::fill(raylen, raylen + npix, (R)0);
        }
    }
    if (roi)  // ST_Tomography.cpp:793-804
        for (long k = 0; k < nvox; ++k) vol[k] *= roi[k];
    return 0;
}

inline bool roi_out(int i, int j, int k, const int *d, const int *cut) {
    // region test of the PD loops (ST_Tomography.cpp:514, 565, 593)
    return i < cut[0] || i > d[0] - cut[1] || j < cut[2] || j > d[1] - cut[3] || k < cut[4] ||
           k > d[2] - cut[5];
}

template <typename R>
void pd_dual_impl(const int *d, R sigma, R tv_w, R tp_w, R bc_w, R hf, const int *cut,
                  const R *xf, const R *xf1, const R *bw, R *ytv, R *ytp, R *ybc) {
    const long n = (long)d[0] * d[1] * d[2];
    const long sy = d[0], sz = (long)d[0] * d[1];
    // ST_Tomography.cpp:504-505 (whole volume, CImg image arithmetic)
    for (long k = 0; k < n; ++k) {
        ytp[k] += sigma * (xf1[k] - xf[k]);
        ybc[k] += sigma * (bw[k] - xf[k]);
    }
    // ST_Tomography.cpp:509-534 (interior, ROI)
#pragma omp parallel for schedule(static)
    for (int k = 1; k < d[2] - 1; ++k)
        for (int j = 1; j < d[1] - 1; ++j)
            for (int i = 1; i < d[0] - 1; ++i) {
                if (roi_out(i, j, k, d, cut)) continue;
                long p = i + j * sy + k * sz;
                R *y0 = ytv, *y1 = ytv + n, *y2 = ytv + 2 * n;
                y0[p] += sigma * (xf[p + 1] - xf[p]) * hf;
                y1[p] += sigma * (xf[p + sy] - xf[p]) * hf;
                y2[p] += sigma * (xf[p + sz] - xf[p]) * hf;
                y0[p] = rmax(-tv_w, rmin(tv_w, y0[p]));
                y1[p] = rmax(-tv_w, rmin(tv_w, y1[p]));
                y2[p] = rmax(-tv_w, rmin(tv_w, y2[p]));
                ytp[p] = ytp[p] * tp_w / (tp_w + 2 * sigma);
                ybc[p] = rmax(-bc_w, rmin(bc_w, ybc[p]));
            }
}

template <typename R>
void pd_primal_impl(const int *d, R tau, R gmax, const int *cut, int first, const R *ytp_prev,
                    const R *ytp, const R *fw, const R *ybc, const R *ytv, R *vol, R *xprev) {
    const long n = (long)d[0] * d[1] * d[2];
    const long sy = d[0], sz = (long)d[0] * d[1];
    for (long k = 0; k < n; ++k) xprev[k] = vol[k];  // ST_Tomography.cpp:536
    if (first) {                                      // :540-545
        for (long k = 0; k < n; ++k) vol[k] -= tau * (-ytp[k]);
        for (long k = 0; k < n; ++k) vol[k] -= tau * (-ybc[k]);
    } else {  // :546-555 (fw = warp(flow[f-1], Y_bc[f-1], +dt))
        for (long k = 0; k < n; ++k) vol[k] -= tau * (ytp_prev[k] - ytp[k]);
        for (long k = 0; k < n; ++k) vol[k] -= tau * (fw[k] - ybc[k]);
    }
    // :560-578 TV adjoint (-div) and clamp, interior, ROI
#pragma omp parallel for schedule(static)
    for (int k = 1; k < d[2] - 1; ++k)
        for (int j = 1; j < d[1] - 1; ++j)
            for (int i = 1; i < d[0] - 1; ++i) {
                if (roi_out(i, j, k, d, cut)) continue;
                long p = i + j * sy + k * sz;
                const R *y0 = ytv, *y1 = ytv + n, *y2 = ytv + 2 * n;
                R y = -(y0[p] - y0[p - 1] + y1[p] - y1[p - sy] + y2[p] - y2[p - sz]);
                vol[p] -= (tau * y);
                vol[p] = rmax(rmin(gmax, vol[p]), (R)0);
            }
}

template <typename R>
void pd_extrapolate_impl(const int *d, const int *cut, const R *vol, const R *xprev, R *xbar) {
    // ST_Tomography.cpp:586-604
    for (int z = 0; z < d[2]; ++z)
        for (int y = 0; y < d[1]; ++y)
            for (int x = 0; x < d[0]; ++x) {
                if (roi_out(x, y, z, d, cut)) continue;
                long p = x + (long)y * d[0] + (long)z * d[0] * d[1];
                xbar[p] = 2 * vol[p] - xprev[p];
            }
}

// ---------------------------------------------------------------------------
// CImg::_cubic_atXYZ (S/ImageFormationModel/CImg.h:13429-13520): Catmull-Rom
// in x for each (y,z) row, then y, then z; indices clamped to the image;
// the "next" index is x+1 only when dx > 0.
template <typename R>
inline R cr(R p, R c, R n, R a, R d) {
    return c + (R)0.5 * (d * (-p + n) + d * d * (2 * p - 5 * c + 4 * n - a) +
                         d * d * d * (-p + 3 * c - 3 * n + a));
}

template <typename R>
struct Cub {
    int xi[4], yi[4], zi[4];
    R dx, dy, dz;
};

template <typename R>
inline void cub_setup(const int *dim, R fx, R fy, R fz, Cub<R> &s) {
    auto cut = [](R v, R lo, R hi) { return v < lo ? lo : (v > hi ? hi : v); };
    R nf[3] = {cut(fx, (R)0, (R)(dim[0] - 1)), cut(fy, (R)0, (R)(dim[1] - 1)),
               cut(fz, (R)0, (R)(dim[2] - 1))};
    int *ix[3] = {s.xi, s.yi, s.zi};
    R *dd[3] = {&s.dx, &s.dy, &s.dz};
    for (int a = 0; a < 3; ++a) {
        int x = (int)nf[a];
        R d = nf[a] - x;
        *dd[a] = d;
        ix[a][0] = x - 1 < 0 ? 0 : x - 1;
        ix[a][1] = x;
        ix[a][2] = d > 0 ? x + 1 : x;
        ix[a][3] = x + 2 >= dim[a] ? dim[a] - 1 : x + 2;
    }
}

template <typename R, typename V>
inline R cub_value(const int *dim, const V *img, const Cub<R> &s) {
    const long nx = dim[0], nxy = (long)dim[0] * dim[1];
    R zv[4];
    for (int c = 0; c < 4; ++c) {
        R yv[4];
        for (int b = 0; b < 4; ++b) {
            const V *row = img + s.yi[b] * nx + s.zi[c] * nxy;
            yv[b] = cr<R>((R)row[s.xi[0]], (R)row[s.xi[1]], (R)row[s.xi[2]], (R)row[s.xi[3]], s.dx);
        }
        zv[c] = cr<R>(yv[0], yv[1], yv[2], yv[3], s.dy);
    }
    return cr<R>(zv[0], zv[1], zv[2], zv[3], s.dz);
}

// Catmull-Rom basis weights w(d) for taps (p, c, n, a) and their derivatives.
inline void cr_w(double d, double w[4], double dw[4]) {
    w[0] = 0.5 * (-d + 2 * d * d - d * d * d);
    w[1] = 1 + 0.5 * (-5 * d * d + 3 * d * d * d);
    w[2] = 0.5 * (d + 4 * d * d - 3 * d * d * d);
    w[3] = 0.5 * (-d * d + d * d * d);
    dw[0] = 0.5 * (-1 + 4 * d - 3 * d * d);
    dw[1] = 0.5 * (-10 * d + 9 * d * d);
    dw[2] = 0.5 * (1 + 8 * d - 9 * d * d);
    dw[3] = 0.5 * (-2 * d + 3 * d * d);
}

// warping::sample_image (warping.h:49-88): world -> cell grid, clamp to
// [1, dim-2], Catmull-Rom sample clamped to the 8-corner min/max.
// box: aabb extents [0, box[a]] (NULL: the cell grid itself, aabb = [0, dim]).
template <typename R, typename V>
inline R sample_image(const int *dim, const V *img, const R p[3], const R *box = nullptr) {
    R gq[3];
    for (int a = 0; a < 3; ++a) {
        const R ext = box ? box[a] : (R)dim[a];
        R gw = (R)dim[a] * (p[a] - (R)0) / (ext - (R)0);
        gq[a] = (R)(gw - 0.5);
        R hi = (R)(dim[a] - 2);
        R lo = (R)1;
        gq[a] = (gq[a] < hi) ? gq[a] : hi;   // std::min(hi, g)
        gq[a] = (lo < gq[a]) ? gq[a] : lo;   // std::max(lo, g)
    }
    int ix = (int)gq[0], iy = (int)gq[1], iz = (int)gq[2];
    const long nx = dim[0], nxy = (long)dim[0] * dim[1];
    auto at = [&](int x, int y, int z) { return (R)img[x + y * nx + z * nxy]; };
    R mn = at(ix, iy, iz), mx = mn;
    const int cx[7] = {1, 1, 0, 0, 1, 1, 0}, cy[7] = {0, 1, 1, 0, 0, 1, 1},
              cz[7] = {0, 0, 0, 1, 1, 1, 1};
    for (int k = 0; k < 7; ++k) {
        R v = at(ix + cx[k], iy + cy[k], iz + cz[k]);
        mn = (v < mn) ? v : mn;
        mx = (mx < v) ? v : mx;
    }
    Cub<R> s;
    cub_setup<R>(dim, gq[0], gq[1], gq[2], s);
    R val = cub_value<R>(dim, img, s);
    R inner = (val < mx) ? val : mx;
    return (mn < inner) ? inner : mn;
}

// warping::warp / trace (warping.h:100-145): p = cell centre, trace with -dt.
// box: aabb = [0, box] (NULL: [0, dim]); the multiscale flow warps every level
// in full-resolution world units (optical_flow.h:700).
template <typename R>
void warp_impl(const int *dim, const R *vel, const R *src, int nc, R dt, R *out,
               const R *box = nullptr) {
    const long n = (long)dim[0] * dim[1] * dim[2];
#pragma omp parallel for schedule(static)
    for (int k = 0; k < dim[2]; ++k)
        for (int j = 0; j < dim[1]; ++j)
            for (int i = 0; i < dim[0]; ++i) {
                R p[3];
                const int ijk[3] = {i, j, k};
                for (int a = 0; a < 3; ++a) {
                    const R ext = box ? box[a] : (R)dim[a];
                    p[a] = (R)(0 + ((R)ijk[a] + 0.5) * (ext - 0) / (R)dim[a]);
                }
                const R h = -dt;
                R v1[3], p2[3], v2[3], p0[3], q[3];
                for (int c = 0; c < 3; ++c) v1[c] = sample_image<R>(dim, vel + c * n, p, box);
                for (int c = 0; c < 3; ++c) p2[c] = p[c] + h * v1[c];
                for (int c = 0; c < 3; ++c) v2[c] = sample_image<R>(dim, vel + c * n, p2, box);
                for (int c = 0; c < 3; ++c) p0[c] = p2[c] - h * v2[c];
                for (int c = 0; c < 3; ++c) q[c] = p2[c] + (R)(0.5 * (p[c] - p0[c]));
                long o = i + (long)j * dim[0] + (long)k * dim[0] * dim[1];
                for (int c = 0; c < nc; ++c) out[o + c * n] = sample_image<R>(dim, src + c * n, q, box);
            }
}

// ---- VJP of sample_image in FP64 ----------------------------------------
// value v = clamp(cub(g(p)), mn, mx).  d v/d img: Catmull-Rom tensor weights
// when unclamped, else 1 on the arg-min/arg-max corner.  d v/d p: spatial
// gradient of the cubic when unclamped and the coordinate itself was not
// clamped to [1, dim-2], else 0.
struct SampleJ {
    double value;
    double grad[3];     // d value / d p (world)
    long idx[64];
    double w[64];       // d value / d img[idx]
    int nw;
};

void sample_image_j(const int *dim, const double *img, const double p[3], SampleJ &J) {
    double gq[3];
    bool clamped[3];
    for (int a = 0; a < 3; ++a) {
        double g = p[a] - 0.5;
        double lo = 1.0, hi = dim[a] - 2.0;
        clamped[a] = (g < lo) || (g > hi);
        gq[a] = g < lo ? lo : (g > hi ? hi : g);
    }
    int ix = (int)gq[0], iy = (int)gq[1], iz = (int)gq[2];
    const long nx = dim[0], nxy = (long)dim[0] * dim[1];
    auto lin = [&](int x, int y, int z) { return x + y * nx + z * nxy; };
    long imn = lin(ix, iy, iz), imx = imn;
    double mn = img[imn], mx = mn;
    const int cx[7] = {1, 1, 0, 0, 1, 1, 0}, cy[7] = {0, 1, 1, 0, 0, 1, 1},
              cz[7] = {0, 0, 0, 1, 1, 1, 1};
    for (int k = 0; k < 7; ++k) {
        long id = lin(ix + cx[k], iy + cy[k], iz + cz[k]);
        double v = img[id];
        if (v < mn) { mn = v; imn = id; }
        if (mx < v) { mx = v; imx = id; }
    }
    Cub<double> s;
    cub_setup<double>(dim, gq[0], gq[1], gq[2], s);
    double wx[4], wy[4], wz[4], dwx[4], dwy[4], dwz[4];
    cr_w(s.dx, wx, dwx);
    cr_w(s.dy, wy, dwy);
    cr_w(s.dz, wz, dwz);
    double val = 0, gx = 0, gy = 0, gz = 0;
    int n = 0;
    for (int c = 0; c < 4; ++c)
        for (int b = 0; b < 4; ++b)
            for (int a = 0; a < 4; ++a) {
                long id = lin(s.xi[a], s.yi[b], s.zi[c]);
                double v = img[id];
                double w = wx[a] * wy[b] * wz[c];
                val += w * v;
                gx += dwx[a] * wy[b] * wz[c] * v;
                gy += wx[a] * dwy[b] * wz[c] * v;
                gz += wx[a] * wy[b] * dwz[c] * v;
                J.idx[n] = id;
                J.w[n] = w;
                ++n;
            }
    J.nw = n;
    if (val > mx) {
        J.value = mx;
        J.nw = 1;
        J.idx[0] = imx;
        J.w[0] = 1;
        J.grad[0] = J.grad[1] = J.grad[2] = 0;
    } else if (val < mn) {
        J.value = mn;
        J.nw = 1;
        J.idx[0] = imn;
        J.w[0] = 1;
        J.grad[0] = J.grad[1] = J.grad[2] = 0;
    } else {
        J.value = val;
        J.grad[0] = clamped[0] ? 0 : gx;
        J.grad[1] = clamped[1] ? 0 : gy;
        J.grad[2] = clamped[2] ? 0 : gz;
    }
}

void warp_vjp_impl(const int *dim, const double *vel, const double *src, int nc, double dt,
                   const double *out_bar, double *src_bar, double *vel_bar) {
    const long n = (long)dim[0] * dim[1] * dim[2];
    for (int k = 0; k < dim[2]; ++k)
        for (int j = 0; j < dim[1]; ++j)
            for (int i = 0; i < dim[0]; ++i) {
                const double p[3] = {i + 0.5, j + 0.5, k + 0.5};
                const double h = -dt;
                SampleJ J1[3], J2[3];
                double v1[3], p2[3], v2[3], q[3];
                for (int c = 0; c < 3; ++c) {
                    sample_image_j(dim, vel + c * n, p, J1[c]);
                    v1[c] = J1[c].value;
                }
                for (int c = 0; c < 3; ++c) p2[c] = p[c] + h * v1[c];
                for (int c = 0; c < 3; ++c) {
                    sample_image_j(dim, vel + c * n, p2, J2[c]);
                    v2[c] = J2[c].value;
                }
                // q = p2 + 0.5*(p - (p2 - h*v2)) = 0.5*p + 0.5*p2 + 0.5*h*v2
                for (int c = 0; c < 3; ++c) q[c] = 0.5 * p[c] + 0.5 * p2[c] + 0.5 * h * v2[c];
                long o = i + (long)j * dim[0] + (long)k * dim[0] * dim[1];
                double qbar[3] = {0, 0, 0};
                for (int c = 0; c < nc; ++c) {
                    double ob = out_bar[o + c * n];
                    if (ob == 0) continue;
                    SampleJ Jq;
                    sample_image_j(dim, src + c * n, q, Jq);
                    if (src_bar)
                        for (int t = 0; t < Jq.nw; ++t) src_bar[c * n + Jq.idx[t]] += ob * Jq.w[t];
                    for (int a = 0; a < 3; ++a) qbar[a] += ob * Jq.grad[a];
                }
                if (!vel_bar) continue;
                // q depends on p2 (0.5 I + 0.5 h dv2/dp2) and on v2 directly (0.5 h)
                double v2bar[3], p2bar[3];
                for (int c = 0; c < 3; ++c) v2bar[c] = 0.5 * h * qbar[c];
                for (int a = 0; a < 3; ++a) {
                    p2bar[a] = 0.5 * qbar[a];
                    for (int c = 0; c < 3; ++c) p2bar[a] += v2bar[c] * J2[c].grad[a];
                }
                for (int c = 0; c < 3; ++c)
                    for (int t = 0; t < J2[c].nw; ++t) vel_bar[c * n + J2[c].idx[t]] += v2bar[c] * J2[c].w[t];
                // p2 = p + h*v1
                for (int c = 0; c < 3; ++c) {
                    double v1bar = h * p2bar[c];
                    for (int t = 0; t < J1[c].nw; ++t) vel_bar[c * n + J1[c].idx[t]] += v1bar * J1[c].w[t];
                }
            }
}


// ---------------------------------------------------------------------------
// 3D TV-L1/Huber optical flow (S/ST_Tomo/optical_flow.h:83-734) and the CImg
// image operations it calls (S/ImageFormationModel/CImg.h).

// CImg::deriche, order 0, Neumann boundaries (CImg.h:32917-33050).
struct DericheC {
    float a0, a1, a2, a3, b1, b2, coefp, coefn;
};

DericheC deriche_coefs(float sigma) {
    const float nnsigma = sigma < 0.1f ? 0.1f : sigma, alpha = 1.695f / nnsigma,
                ema = (float)std::exp(-alpha), ema2 = (float)std::exp(-2 * alpha), b1 = -2 * ema,
                b2 = ema2;
    const float k = (1 - ema) * (1 - ema) / (1 + 2 * alpha * ema - ema2);
    DericheC c;
    c.a0 = k;
    c.a1 = k * (alpha - 1) * ema;
    c.a2 = k * (alpha + 1) * ema;
    c.a3 = -k * ema2;
    c.b1 = b1;
    c.b2 = b2;
    c.coefp = (c.a0 + c.a1) / (1 + b1 + b2);
    c.coefn = (c.a2 + c.a3) / (1 + b1 + b2);
    return c;
}

// _cimg_deriche_apply on one line of N samples spaced `off` apart.
void deriche_line(float *X, long off, int N, const DericheC &c, std::vector<float> &Y) {
    float xp = X[0], yb = c.coefp * xp, yp = yb;
    for (int m = 0; m < N; ++m) {
        const float xc = X[m * off];
        const float yc = c.a0 * xc + c.a1 * xp - c.b1 * yp - c.b2 * yb;
        Y[m] = yc;
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
        X[m * off] = Y[m] + yc;
    }
}

// CImg::blur(sigma) (CImg.h:33249-33262, 33275-33278): Deriche along x, y, z
// (each axis of extent > 1), in place on nc planar channels.
void blur_impl(const int *d, int nc, float sigma, float *img) {
    if (sigma < 0.1f) return;  // deriche() returns early for order 0
    const DericheC c = deriche_coefs(sigma);
    const long nx = d[0], ny = d[1], nz = d[2], n = nx * ny * nz;
    std::vector<float> Y(std::max(nx, std::max(ny, nz)));
    for (int ch = 0; ch < nc; ++ch) {
        float *I = img + ch * n;
        if (nx > 1)
            for (long z = 0; z < nz; ++z)
                for (long y = 0; y < ny; ++y) deriche_line(I + y * nx + z * nx * ny, 1, (int)nx, c, Y);
        if (ny > 1)
            for (long z = 0; z < nz; ++z)
                for (long x = 0; x < nx; ++x) deriche_line(I + x + z * nx * ny, nx, (int)ny, c, Y);
        if (nz > 1)
            for (long y = 0; y < ny; ++y)
                for (long x = 0; x < nx; ++x) deriche_line(I + x + y * nx, nx * ny, (int)nz, c, Y);
    }
}

// One axis of CImg::get_resize(..., 5) (CImg.h:28432-28560): a shrinking axis
// takes the moving average (resize type 2, :28135-28195); a growing axis is
// Catmull-Rom interpolated with step (old-1)/(new-1), evaluated in double.
void resize_axis_impl(const int *d, int nc, const float *in, int axis, int nn, float *out) {
    int od[3] = {d[0], d[1], d[2]};
    const int old = d[axis];
    od[axis] = nn;
    const long st_in[3] = {1, d[0], (long)d[0] * d[1]};
    const long st_out[3] = {1, od[0], (long)od[0] * od[1]};
    const long nin = (long)d[0] * d[1] * d[2], nout = (long)od[0] * od[1] * od[2];
    // the two coordinates that are not resized
    const int a1 = axis == 0 ? 1 : 0, a2 = axis == 2 ? 1 : 2;
    std::vector<float> acc(nn);
    std::vector<unsigned> off(nn);
    std::vector<double> foff(nn);
    if (nn > old) {
        const double fx = nn > 1 ? (old - 1.0) / (nn - 1) : 0;
        double curr = 0, prev = 0;
        for (int x = 0; x < nn; ++x) {
            foff[x] = curr - (unsigned)curr;
            prev = curr;
            curr = std::min(old - 1.0, curr + fx);
            off[x] = (unsigned)curr - (unsigned)prev;
        }
    }
    for (int ch = 0; ch < nc; ++ch)
        for (int u = 0; u < d[a2]; ++u)
            for (int w = 0; w < d[a1]; ++w) {
                const float *src = in + ch * nin + w * st_in[a1] + u * st_in[a2];
                float *dst = out + ch * nout + w * st_out[a1] + u * st_out[a2];
                const long si = st_in[axis], so = st_out[axis];
                if (nn == old) {
                    for (int t = 0; t < nn; ++t) dst[t * so] = src[t * si];
                } else if (nn < old) {
                    std::fill(acc.begin(), acc.end(), 0.0f);
                    for (unsigned a = (unsigned)old * nn, b = old, c = nn, s = 0, t = 0; a;) {
                        const unsigned dd = std::min(b, c);
                        a -= dd;
                        b -= dd;
                        c -= dd;
                        acc[t] += src[s * si] * dd;
                        if (!b) {
                            acc[t] /= old;
                            ++t;
                            b = old;
                        }
                        if (!c) {
                            ++s;
                            c = nn;
                        }
                    }
                    for (int t = 0; t < nn; ++t) dst[t * so] = acc[t];
                } else {
                    long s = 0;
                    for (int x = 0; x < nn; ++x) {
                        const double t = foff[x], val1 = (double)src[s * si],
                                     val0 = s > 0 ? (double)src[(s - 1) * si] : val1,
                                     val2 = s <= old - 2 ? (double)src[(s + 1) * si] : val1,
                                     val3 = s < old - 2 ? (double)src[(s + 2) * si] : val2,
                                     val = val1 + 0.5f * (t * (-val0 + val2) +
                                                          t * t * (2 * val0 - 5 * val1 + 4 * val2 - val3) +
                                                          t * t * t * (-val0 + 3 * val1 - 3 * val2 + val3));
                        dst[x * so] = (float)(val < -FLT_MAX ? -FLT_MAX : val > FLT_MAX ? FLT_MAX : val);
                        s += off[x];
                    }
                }
            }
}

// get_resize(nx, ny, nz, nc, 5): x, then y, then z.
void resize_impl(const int *d, int nc, const float *in, const int *od, float *out) {
    std::vector<float> a(in, in + (size_t)d[0] * d[1] * d[2] * nc), b;
    int cur[3] = {d[0], d[1], d[2]};
    for (int axis = 0; axis < 3; ++axis) {
        if (od[axis] == cur[axis]) continue;
        int nd[3] = {cur[0], cur[1], cur[2]};
        nd[axis] = od[axis];
        b.assign((size_t)nd[0] * nd[1] * nd[2] * nc, 0.0f);
        resize_axis_impl(cur, nc, a.data(), axis, od[axis], b.data());
        a.swap(b);
        cur[axis] = od[axis];
    }
    std::memcpy(out, a.data(), sizeof(float) * a.size());
}

// get_gradient("xyz", 0): central differences, neighbours clamped (CImg.h:34570-34581).
void gradient_impl(const int *d, const float *I, float *gx, float *gy, float *gz) {
    const long nx = d[0], ny = d[1], nz = d[2];
    for (long z = 0; z < nz; ++z)
        for (long y = 0; y < ny; ++y)
            for (long x = 0; x < nx; ++x) {
                auto at = [&](long i, long j, long k) { return I[i + j * nx + k * nx * ny]; };
                const long p = x + y * nx + z * nx * ny;
                gx[p] = (at(std::min(x + 1, nx - 1), y, z) - at(std::max(x - 1, 0L), y, z)) / 2;
                gy[p] = (at(x, std::min(y + 1, ny - 1), z) - at(x, std::max(y - 1, 0L), z)) / 2;
                gz[p] = (at(x, y, std::min(z + 1, nz - 1)) - at(x, y, std::max(z - 1, 0L))) / 2;
            }
}

// Backward / forward differences of S/ImageFormationModel/tools.cpp:126-192.
inline float dm_(const float *f, long p, int c, int n, long st) {
    if (c > 0 && c < n - 1) return f[p] - f[p - st];
    if (c == 0) return f[p];
    return -f[p - st];
}
inline float dp_(const float *f, long p, int c, int n, long st) {
    return c < n - 1 ? f[p + st] - f[p] : 0.0f;
}

// optical_flow::L1Huber_OF (optical_flow.h:83-623), one thread, so the
// residual sums follow the sequential loop order.  V: 3 channels (in/out),
// Y: Y1|Y2|Y3|Y4 = 10 channels (in/out, written back inside the ROI only, as
// the reference does).  roi = {x0, x1, y0, y1, z0, z1} cut from each face.
// The gradient and ut outside the ROI, which the reference leaves unset, are 0.
// iters, errs (optional, n_warps entries): iterations run per warp and the
// last residual formed in each warp (1 when none was).
void flow_level_impl(const int *d, const float *box, const int *roi, const float *I1, const float *I2,
                     float *V, float *Y, float tol, float lambda, int max_iter, int norm, int n_warps,
                     float huber, int *iters, float *errs) {
    const long nx = d[0], ny = d[1], nz = d[2], n = nx * ny * nz, sy = nx, sz = nx * ny;
    const float sigma1 = std::min(1.0f / 3.0f, std::min(1.0f / 3.0f, 1.0f / 3.0f));
    const float hf = 1.0f / (1.0f + sigma1 * huber / lambda);
    std::vector<float> y(Y, Y + 10 * n), kx(10 * n, 0.0f), kty(3 * n, 0.0f), ktyo(3 * n), vo(3 * n);
    std::vector<float> u(4 * n, 0.0f), tau(3 * n), sig2(n), i2w(n), g(3 * n);
    for (int w = 0; w < n_warps; ++w) {
        warp_impl<float>(d, V, I2, 1, -1.0f, i2w.data(), box);
        gradient_impl(d, i2w.data(), g.data(), g.data() + n, g.data() + 2 * n);
        for (long k = roi[4]; k < nz - roi[5]; ++k)
            for (long j = roi[2]; j < ny - roi[3]; ++j)
                for (long i = roi[0]; i < nx - roi[1]; ++i) {
                    const long p = i + j * sy + k * sz;
                    u[p] = g[p];
                    u[n + p] = g[n + p];
                    u[2 * n + p] = g[2 * n + p];
                    u[3 * n + p] = i2w[p] - I1[p] - u[p] * V[p] - u[n + p] * V[n + p] - u[2 * n + p] * V[2 * n + p];
                }
        for (long p = 0; p < n; ++p) {
            for (int c = 0; c < 3; ++c) tau[c * n + p] = 1.0f / (4.0f / 1.0f + std::fabs(u[c * n + p]));
            sig2[p] = 1.0f / (std::fabs(u[p]) + std::fabs(u[n + p]) + std::fabs(u[2 * n + p]));
        }
        int it = 0;
        float err = 1.0f, pr = 0.0f, dr = 0.0f;
        while (err > tol && it <= max_iter) {
            ++it;
            const bool res = it % 50 == 0;
            if (res) pr = dr = 0.0f;
            for (long k = roi[4]; k < nz - roi[5]; ++k)
                for (long j = roi[2]; j < ny - roi[3]; ++j)
                    for (long i = roi[0]; i < nx - roi[1]; ++i) {
                        const long p = i + j * sy + k * sz;
                        if (res)
                            for (int c = 0; c < 3; ++c) {
                                vo[c * n + p] = V[c * n + p];
                                ktyo[c * n + p] = kty[c * n + p];
                            }
                        for (int c = 0; c < 3; ++c) {
                            const float *yc = y.data() + 3 * c * n;
                            kty[c * n + p] = -1.0f * dm_(yc, p, (int)i, (int)nx, 1) -
                                             1.0f * dm_(yc + n, p, (int)j, (int)ny, sy) -
                                             1.0f * dm_(yc + 2 * n, p, (int)k, (int)nz, sz) + u[c * n + p] * y[9 * n + p];
                        }
                        for (int c = 0; c < 3; ++c) V[c * n + p] -= tau[c * n + p] * kty[c * n + p];
                        if (res) {
                            float s = 0.0f;
                            for (int c = 0; c < 3; ++c) {
                                const float t = std::fabs((vo[c * n + p] - V[c * n + p]) / tau[c * n + p] -
                                                          ktyo[c * n + p] + kty[c * n + p]);
                                s = c == 0 ? t : s + t;
                            }
                            pr += s;
                        }
                    }
            for (long k = 0; k < nz; ++k)
                for (long j = 0; j < ny; ++j)
                    for (long i = 0; i < nx; ++i) {
                        const long p = i + j * sy + k * sz;
                        float yold[10], kold[10], yt[9];
                        for (int q = 0; q < 10; ++q) {
                            yold[q] = y[q * n + p];
                            kold[q] = kx[q * n + p];
                        }
                        for (int c = 0; c < 3; ++c) {
                            const float *vc = V + c * n;
                            kx[(3 * c) * n + p] = 1.0f * dp_(vc, p, (int)i, (int)nx, 1);
                            kx[(3 * c + 1) * n + p] = 1.0f * dp_(vc, p, (int)j, (int)ny, sy);
                            kx[(3 * c + 2) * n + p] = 1.0f * dp_(vc, p, (int)k, (int)nz, sz);
                        }
                        kx[9 * n + p] = u[p] * V[p] + u[n + p] * V[n + p] + u[2 * n + p] * V[2 * n + p];
                        for (int q = 0; q < 9; ++q) {
                            const float kq = kx[q * n + p];
                            yt[q] = (y[q * n + p] + sigma1 * (kq + kq - kold[q]));
                            if (norm == 4) yt[q] = yt[q] * hf;
                        }
                        for (int c = 0; c < 3; ++c) {
                            const float *t = yt + 3 * c;
                            const float dv = std::max(1.0f, std::sqrt(t[0] * t[0] + t[1] * t[1] + t[2] * t[2]) / lambda);
                            for (int a = 0; a < 3; ++a) y[(3 * c + a) * n + p] = t[a] / dv;
                        }
                        const float k4 = kx[9 * n + p];
                        y[9 * n + p] = std::max(-1.0f, std::min(1.0f, y[9 * n + p] + sig2[p] * (k4 + k4 - kold[9] + u[3 * n + p])));
                        if (res) {
                            float s = 0.0f;
                            for (int q = 0; q < 9; ++q) {
                                const float t = std::fabs((yold[q] - y[q * n + p]) / sigma1 - kold[q] + kx[q * n + p]);
                                s = q == 0 ? t : s + t;
                            }
                            s = s + std::fabs((yold[9] - y[9 * n + p]) / sig2[p] - kold[9] + k4);
                            dr += s;
                        }
                    }
            if (res) err = (dr * dr + pr * pr) / (float)n;
        }
        if (iters) iters[w] = it;
        if (errs) errs[w] = err;
    }
    for (long k = roi[4]; k < nz - roi[5]; ++k)
        for (long j = roi[2]; j < ny - roi[3]; ++j)
            for (long i = roi[0]; i < nx - roi[1]; ++i) {
                const long p = i + j * sy + k * sz;
                for (int q = 0; q < 10; ++q) Y[q * n + p] = y[q * n + p];
            }
}

// optical_flow::L1Huber_OF_MultiScale3D (optical_flow.h:630-734).  Returns the
// finest-level flow in Vout; Yin (10 channels, NULL = zeros) is the dual start.
void flow_multiscale_impl(const int *d, const float *I1, const float *I2, const float *Vin, const float *Yin,
                          float *Vout, float tol, float lambda, int max_iter, int norm, int n_warps, float eta,
                          float sigma, int scales, float huber, const int *cut) {
    const long n = (long)d[0] * d[1] * d[2];
    std::vector<float> b1(I1, I1 + n), b2(I2, I2 + n);
    blur_impl(d, 1, sigma, b1.data());
    blur_impl(d, 1, sigma, b2.data());
    std::vector<float> y0(10 * n, 0.0f);
    if (Yin) std::memcpy(y0.data(), Yin, sizeof(float) * 10 * n);
    struct Level {
        int d[3];
        std::vector<float> i1, i2, v, y;
    };
    std::vector<Level> L(scales);
    float t_eta = 1.0f;
    for (int s = 0; s < scales; ++s) {
        Level &l = L[scales - 1 - s];  // coarse first after the reverse
        for (int a = 0; a < 3; ++a) l.d[a] = (int)((float)d[a] * t_eta);
        const long m = (long)l.d[0] * l.d[1] * l.d[2];
        l.i1.resize(m);
        l.i2.resize(m);
        l.v.resize(3 * m);
        l.y.resize(10 * m);
        resize_impl(d, 1, b1.data(), l.d, l.i1.data());
        resize_impl(d, 1, b2.data(), l.d, l.i2.data());
        resize_impl(d, 3, Vin, l.d, l.v.data());
        resize_impl(d, 10, y0.data(), l.d, l.y.data());
        t_eta = t_eta * eta;
    }
    const float box[3] = {(float)d[0], (float)d[1], (float)d[2]};
    for (int s = 0; s < scales; ++s) {
        Level &l = L[s];
        int roi[6];
        for (int q = 0; q < 6; ++q) roi[q] = (int)((float)cut[q] * ((float)l.d[q / 2] / (float)d[q / 2]));
        flow_level_impl(l.d, box, roi, l.i1.data(), l.i2.data(), l.v.data(), l.y.data(), tol, lambda, max_iter,
                        norm, n_warps, huber, nullptr, nullptr);
        if (s < scales - 1) {
            Level &nx = L[s + 1];
            resize_impl(l.d, 3, l.v.data(), nx.d, nx.v.data());
            resize_impl(l.d, 10, l.y.data(), nx.d, nx.y.data());
        }
    }
    std::memcpy(Vout, L[scales - 1].v.data(), sizeof(float) * 3 * n);
}

}  // namespace

// ---------------------------------------------------------------------------
extern "C" {

void orc_view_from_round(double start_deg, int k, orc_view *v) {
    // InitViews (ST_Tomography.cpp:894-912), RotateVolume (:865-884); the
    // start angle is read from lds.txt into a float (:264-268).
    const float sdeg = (float)start_deg;
    const double a0 = sdeg * 3.1415926 / 180;
    const double step = (360.0 / 10) * 3.1415926 / 180;
    Q4 q = q_mul(q_axis_angle(0.0f, 1.0f, 0.0f, (float)(1.0 * a0)), Q4{0, 0, 0, 1});
    for (int i = 0; i < k; ++i) q = q_mul(q_axis_angle(0.0f, 1.0f, 0.0f, (float)(1.0 * step)), q);
    v->quat[0] = q.x;
    v->quat[1] = q.y;
    v->quat[2] = q.z;
    v->quat[3] = q.w;
    v->angle = a0 + k * step;
}

void orc_view_from_angle(double angle, orc_view *v) {
    Q4 q = q_mul(q_axis_angle(0.0f, 1.0f, 0.0f, (float)angle), Q4{0, 0, 0, 1});
    v->quat[0] = q.x;
    v->quat[1] = q.y;
    v->quat[2] = q.z;
    v->quat[3] = q.w;
    v->angle = angle;
}

void orc_view_matrices_f32(const orc_geom *g, const orc_view *v, float *out) {
    View32 V;
    make_view32(*g, *v, V);
    std::memcpy(out, V.p2m.e, 64);
    std::memcpy(out + 16, V.m2v.e, 64);
    std::memcpy(out + 32, V.mv.e, 64);
    std::memcpy(out + 48, V.v2m.e, 64);
}

int orc_fp_f32(const orc_geom *g, int gmode, const orc_view *v, const float *vol, float *img,
               float *raylen, float *weight, int nthreads) {
    set_threads(nthreads);
    return fp_impl<float>(*g, gmode, *v, vol, img, raylen, weight);
}

int orc_fp_rows_f64(const orc_geom *g, const orc_view *v, const double *vol, int row0, int row1, double *img,
                    int nthreads) {
    set_threads(nthreads);
    if (row0 < 0 || row1 < row0) return -1;
    return fp_impl<double>(*g, 1, *v, vol, img, nullptr, nullptr, row0, row1);
}

int orc_fp_rows_f32(const orc_geom *g, int gmode, const orc_view *v, const float *vol, int row0, int row1,
                    float *img, int nthreads) {
    set_threads(nthreads);
    if (row0 < 0 || row1 < row0) return -1;
    return fp_impl<float>(*g, gmode, *v, vol, img, nullptr, nullptr, row0, row1);
}

int orc_fp_f64(const orc_geom *g, const orc_view *v, const double *vol, double *img,
               double *raylen, double *weight, int nthreads) {
    set_threads(nthreads);
    return fp_impl<double>(*g, 1, *v, vol, img, raylen, weight);
}

int orc_bp_ray_scatter_f32(const orc_geom *g, int gmode, const orc_view *v, const float *corr,
                           float *contrib, float *wsum) {
    return scatter_impl<float>(*g, gmode, *v, corr, contrib, wsum, false);
}

int orc_fp_adjoint_f64(const orc_geom *g, const orc_view *v, const double *proj_bar,
                       double *vol_bar) {
    return scatter_impl<double>(*g, 1, *v, proj_bar, vol_bar, nullptr, true);
}

int orc_fp_adjoint_f32(const orc_geom *g, int gmode, const orc_view *v, const float *proj_bar,
                       float *vol_bar) {
    return scatter_impl<float>(*g, gmode, *v, proj_bar, vol_bar, nullptr, true);
}

int orc_bp_voxel_f32(const orc_geom *g, int gmode, const orc_view *v, const float *corr,
                     double alpha, float gmax, float *vol, int nthreads) {
    set_threads(nthreads);
    return bp_voxel_impl<float>(*g, gmode, *v, corr, alpha, gmax, vol);
}

int orc_bp_voxel_f64(const orc_geom *g, const orc_view *v, const double *corr, double alpha,
                     double gmax, double *vol, int nthreads) {
    set_threads(nthreads);
    return bp_voxel_impl<double>(*g, 1, *v, corr, alpha, gmax, vol);
}

void orc_correction_f32(int n, const float *b, const float *ax, const float *raylen, float *c) {
    correction_impl<float>(n, b, ax, raylen, c);
}

void orc_bp_ray_update_f32(long n, const float *contrib, const float *wsum, float gmax,
                           float *vol) {
    bp_ray_update_impl<float>(n, contrib, wsum, gmax, vol);
}

int orc_sart_f32(const orc_geom *g, int gmode, const orc_view *views, const int *perm, int nv,
                 const float *proj, double alpha, float gmax, int bp_mode, float *vol,
                 float *raylen_state, const float *roi, int nthreads) {
    set_threads(nthreads);
    return sart_impl<float>(*g, gmode, views, perm, nv, proj, alpha, gmax, bp_mode, vol,
                            raylen_state, roi);
}

int orc_sart_f64(const orc_geom *g, const orc_view *views, const int *perm, int nv,
                 const double *proj, double alpha, double gmax, int bp_mode, double *vol,
                 double *raylen_state, const double *roi, int nthreads) {
    set_threads(nthreads);
    return sart_impl<double>(*g, 1, views, perm, nv, proj, alpha, gmax, bp_mode, vol,
                             raylen_state, roi);
}

void orc_roi_mask_f32(const int *d, const int *cut, float *roi) {
    // ST_Tomography.cpp:303-329 (note the literal 7 in the j test of :324)
    for (int k = 0; k < d[2]; k++)
        for (int j = 0; j < d[1]; j++)
            for (int i = 0; i < d[0]; i++) {
                float r = 1.0f;
                if (((i < cut[6]) && (k < cut[7])) || ((i < cut[6]) && (k > (d[2] - cut[7])))) r = 0.0f;
                if (((i > (d[0] - cut[6])) && (k < cut[7])) || ((i > (d[0] - cut[6])) && (k > (d[2] - cut[7])))) r = 0.0f;
                if (((k < cut[6]) && (i < cut[7])) || ((k < cut[6]) && (i > (d[0] - cut[7])))) r = 0.0f;
                if (((k > (d[2] - cut[6])) && (i < cut[7])) || ((k > (d[2] - cut[6])) && (i > (d[0] - cut[7])))) r = 0.0f;
                if (i < cut[0] || i > d[0] - cut[1] || j < cut[2] || j > d[1] - 7 || k < cut[4] || k > d[2] - cut[5]) r = 0.0f;
                roi[i + (long)j * d[0] + (long)k * d[0] * d[1]] = r;
            }
}

void orc_permutation(unsigned long long seed, int n, int *perm) {
    // SplitMix64 (Steele, Lea, Flood 2014) driving a Fisher-Yates shuffle.
    uint64_t s = seed;
    auto next = [&s]() {
        uint64_t z = (s += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    };
    for (int i = 0; i < n; ++i) perm[i] = i;
    for (int i = n - 1; i > 0; --i) {
        int j = (int)(next() % (uint64_t)(i + 1));
        std::swap(perm[i], perm[j]);
    }
}

void orc_pd_dual_f32(const int *dims, const orc_pd_params *p, const float *xbar_f,
                     const float *xbar_f1, const float *bw, float *ytv, float *ytp, float *ybc) {
    pd_dual_impl<float>(dims, p->sigma, p->tv_w, p->tp_w, p->bc_w, p->huber_factor, p->cut,
                        xbar_f, xbar_f1, bw, ytv, ytp, ybc);
}

void orc_pd_primal_f32(const int *dims, const orc_pd_params *p, int first_frame,
                       const float *ytp_prev, const float *ytp, const float *fw,
                       const float *ybc, const float *ytv, float *vol, float *xprev) {
    pd_primal_impl<float>(dims, p->tau, p->gmax, p->cut, first_frame, ytp_prev, ytp, fw, ybc,
                          ytv, vol, xprev);
}

void orc_pd_extrapolate_f32(const int *dims, const int *cut, const float *vol,
                            const float *xprev, float *xbar) {
    pd_extrapolate_impl<float>(dims, cut, vol, xprev, xbar);
}

// pp = {sigma, tau, tv_w, tp_w, bc_w, huber_factor, gmax}
void orc_pd_dual_f64(const int *dims, const double *pp, const int *cut, const double *xbar_f,
                     const double *xbar_f1, const double *bw, double *ytv, double *ytp,
                     double *ybc) {
    pd_dual_impl<double>(dims, pp[0], pp[2], pp[3], pp[4], pp[5], cut, xbar_f, xbar_f1, bw, ytv,
                         ytp, ybc);
}

void orc_pd_primal_f64(const int *dims, const double *pp, const int *cut, int first_frame,
                       const double *ytp_prev, const double *ytp, const double *fw,
                       const double *ybc, const double *ytv, double *vol, double *xprev) {
    pd_primal_impl<double>(dims, pp[1], pp[6], cut, first_frame, ytp_prev, ytp, fw, ybc, ytv, vol,
                           xprev);
}

void orc_pd_extrapolate_f64(const int *dims, const int *cut, const double *vol,
                            const double *xprev, double *xbar) {
    pd_extrapolate_impl<double>(dims, cut, vol, xprev, xbar);
}

void orc_warp_f32(const int *dim, const float *vel, const float *src, int nc, float dt,
                  float *out, int nthreads) {
    set_threads(nthreads);
    warp_impl<float>(dim, vel, src, nc, dt, out);
}

void orc_warp_f64(const int *dim, const double *vel, const double *src, int nc, double dt,
                  double *out, int nthreads) {
    set_threads(nthreads);
    warp_impl<double>(dim, vel, src, nc, dt, out);
}

void orc_warp_vjp_f64(const int *dim, const double *vel, const double *src, int nc, double dt,
                      const double *out_bar, double *src_bar, double *vel_bar) {
    warp_vjp_impl(dim, vel, src, nc, dt, out_bar, src_bar, vel_bar);
}

float orc_cubic_at_f32(const int *dim, const float *img, float x, float y, float z) {
    Cub<float> s;
    cub_setup<float>(dim, x, y, z, s);
    return cub_value<float>(dim, img, s);
}

double orc_cubic_at_f64(const int *dim, const double *img, double x, double y, double z) {
    Cub<double> s;
    cub_setup<double>(dim, x, y, z, s);
    return cub_value<double>(dim, img, s);
}

void orc_warp_box_f32(const int *dim, const float *box, const float *vel, const float *src, int nc,
                      float dt, float *out, int nthreads) {
    set_threads(nthreads);
    warp_impl<float>(dim, vel, src, nc, dt, out, box);
}

void orc_blur_f32(const int *dim, int nc, float sigma, float *img) { blur_impl(dim, nc, sigma, img); }

void orc_resize_f32(const int *dim, int nc, const float *in, const int *odim, float *out) {
    resize_impl(dim, nc, in, odim, out);
}

void orc_gradient_f32(const int *dim, const float *img, float *gx, float *gy, float *gz) {
    gradient_impl(dim, img, gx, gy, gz);
}

void orc_flow_level_f32(const int *dim, const float *box, const int *roi, const float *I1, const float *I2,
                        float *V, float *Y, float tol, float lambda, int max_iter, int norm, int n_warps,
                        float huber, int *iters, float *errs) {
    set_threads(1);
    flow_level_impl(dim, box, roi, I1, I2, V, Y, tol, lambda, max_iter, norm, n_warps, huber, iters, errs);
}

void orc_flow_multiscale_f32(const int *dim, const float *I1, const float *I2, const float *Vin,
                             const float *Yin, float *Vout, float tol, float lambda, int max_iter,
                             int norm, int n_warps, float eta, float sigma, int scales, float huber,
                             const int *cut) {
    set_threads(1);
    flow_multiscale_impl(dim, I1, I2, Vin, Yin, Vout, tol, lambda, max_iter, norm, n_warps, eta, sigma,
                         scales, huber, cut);
}

}  // extern "C"
