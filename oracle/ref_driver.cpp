// oracle/ref_driver.cpp -- TEST INFRASTRUCTURE ONLY.
//
// C entry points around the reference's own, unmodified CPU code, so that the
// oracle restatement (oracle/stt_oracle.cpp) and the golden fixtures can be
// checked against the real thing.  oracle/Makefile compiles this file together
// with the reference sources where they lie (SpaceTimeTomography/ImageFormationModel,
// SpaceTimeTomography/Math, SpaceTimeTomography/ST_Tomo) into oracle/_ref/libstt_ref.so.
// Nothing in the product links or loads this library; only tests/, the
// fixture generator and bench.py's CPU-baseline leg do.
//
// What is called (reference paths relative to the project root):
//   - the forward projector:   GenerateImage_GetCorrections
//       SpaceTimeTomography/ImageFormationModel/TypicalRayProducer.core.h:230-268,
//       CastingRay RayCaster.core.h:42-188, T_VolumeAccess SingleScalarVolume.core.h:41-146
//   - the ray-driven BP scatter: the same march with VolumeData::SetProjectionMode(1)
//       (SingleScalarVolume.core.h:73-84,128-143)
//   - the view geometry: Scene::_calculateCamera / _calculateMatrix (Scene.cpp:69-138,181-207),
//       TypicalRayProducer::_calculateMatrix (TypicalRayProducer.cpp:142-208)
//   - warping::warp (ST_Tomo/warping.h:116-145) and CImg::cubic_atXYZ
//   - optical_flow::L1Huber_OF / L1Huber_OF_MultiScale3D (ST_Tomo/optical_flow.h:83-734)
//
// The Scene subclass below sets the same members that the ST_Tomography
// constructor and SetData set (ST_Tomography.cpp:229-246, 290), and composes
// the view quaternion as InitViews/RotateVolume do (ST_Tomography.cpp:865-934).

#include <cmath>
#include <cstring>
#include <cstdio>
#include <iostream>
#include <algorithm>
#include <functional>
#include <omp.h>

#include "VolumeData.h"
#include "Scene.h"
#include "RayCaster.h"
#include "TypicalRayProducer.h"
#include "Quaternion.h"

// ST_Tomography.cpp:167-173 defines these macros before it includes the core
// headers, whose clamps mix float and int arguments.
#ifndef max
#define max(a, b) (((a) > (b)) ? (a) : (b))
#endif
#ifndef min
#define min(a, b) (((a) < (b)) ? (a) : (b))
#endif

#include "SingleScalarVolume.core.h"
#include "RayCaster.core.h"
#include "TypicalRayProducer.core.h"

#undef max
#undef min
#include "optical_flow.h"
#include "warping.h"

namespace {

struct RefGeom {
    int dims[3];
    float sp[3];
    int W, H;
    double ds, sid, sdd;
    double oxyz[3];
};

class RefScene : public Scene {
public:
    explicit RefScene(const RefGeom &g) {
        // ST_Tomography::ST_Tomography (ST_Tomography.cpp:229-246)
        m_halfFrustumWidth = (g.W - 1) * g.ds * 0.5f;
        m_halfFrustumHeight = (g.H - 1) * g.ds * 0.5f;
        m_sid = g.sid;
        m_sdd = g.sdd;
        m_ds = g.ds;
        m_ViewPort[0] = g.W;
        m_ViewPort[1] = g.H;
        m_Translate[0] = -g.oxyz[0];
        m_Translate[2] = +g.oxyz[1];
        m_Translate[1] = -g.oxyz[2];
        // ST_Tomography::SetData -> SetSize3DModified (Scene.cpp:140-179)
        SetSize3DModified();
        // InitViews calls _calculateCamera once (ST_Tomography.cpp:915-919)
        _calculateCamera();
    }
    void Render() override {}

    // InitViews (ST_Tomography.cpp:894-912) then RotateVolume k times (:865-884).
    static Quaternion view_rotation(double start_deg, int k) {
        Quaternion ident;
        Vector4 v;
        v[0] = 0;
        v[1] = 1;
        v[2] = v[3] = 0.0f;
        double length = v.Length();
        v *= 1.0f / length;
        double a0 = (float)start_deg * 3.1415926 / 180;  // m_startDegree is float
        Quaternion q = Quaternion(v[0], v[1], v[2], length * a0) * ident;
        double step = (360.0 / 10) * 3.1415926 / 180;
        for (int i = 0; i < k; ++i) q = Quaternion(v[0], v[1], v[2], length * step) * q;
        return q;
    }
};

void copy_mat(const Matrix4x4 &m, float *out) {
    for (int i = 0; i < 16; ++i) out[i] = m.ele[i];
}

// Runs one march of the reference projector in forward (bp_mode=0) or
// backprojection (bp_mode=1) mode.
int run_view(const RefGeom &g, double start_deg, int k, const float *vol,
             const float *corr, int bp_mode, float *image, float *raylen,
             float *weight, float *contrib, float *wsum, float *mats) {
    RefScene scene(g);
    VolumeData vd;
    vd.SetDimensions(g.dims);
    vd.SetSpacings(g.sp);
    size_t nvox = (size_t)g.dims[0] * g.dims[1] * g.dims[2];
    if (vol)
        vd.m_Volumelist.insert(CImg<float>(vol, g.dims[0], g.dims[1], g.dims[2], 1));
    else
        vd.m_Volumelist.insert(CImg<float>(g.dims[0], g.dims[1], g.dims[2], 1, 0.0f));
    TypicalRayProducer rp(g.dims[0], g.dims[1], g.dims[2], g.W, g.H, g.ds,
                          bp_mode ? "Raybased" : "Voxelbased");
    rp.SetVolSize(g.dims, g.sp);
    rp.SetViewPort(g.W, g.H);
    RayCaster rc;
    rc.SetSampleDistance(std::sqrt(g.sp[0] * g.sp[0] + g.sp[1] * g.sp[1] + g.sp[2] * g.sp[2]));
    scene.m_Rotation = RefScene::view_rotation(start_deg, k);
    scene._calculateMatrix();
    rp.SetViewMatrix(scene.GetViewMatrix());
    rp.SetProjectionMatrix(scene.GetProjectionMatrix());
    if (corr) std::memcpy(rp.GetCorrection(), corr, sizeof(float) * g.W * g.H);
    vd.SetProjectionMode(bp_mode != 0);
    int bsz[3] = {g.dims[0], g.dims[1], g.dims[2]};
    if (!SingleScalarVolumePrepare(&vd, &rp, 0)) return -1;
    if (!RayCasterPrepare(&rc, bsz)) return -2;
    GenerateImage_GetCorrections(&rp);
    size_t npix = (size_t)g.W * g.H;
    if (image) std::memcpy(image, rp.GetImageData(), sizeof(float) * npix);
    if (raylen) std::memcpy(raylen, rp.GetImageRaylength(), sizeof(float) * npix);
    if (weight) std::memcpy(weight, rp.GetWeightOfImage(), sizeof(float) * npix);
    if (contrib) std::memcpy(contrib, rp.GetContributions(), sizeof(float) * nvox);
    if (wsum) std::memcpy(wsum, rp.GetTotalWeight(), sizeof(float) * nvox);
    if (mats) {
        copy_mat(rp.GetPixelsToModelMatrix(), mats);
        copy_mat(rp.GetModelToVolumeMatrix(), mats + 16);
        copy_mat(rp.m_model_view, mats + 32);
        copy_mat(rp.m_VolumeToModelMatrix, mats + 48);
        copy_mat(scene.GetViewMatrix(), mats + 64);
        copy_mat(scene.GetProjectionMatrix(), mats + 80);
    }
    delete va;
    va = 0;
    // buffers the reference's destructor does not free (TypicalRayProducer.cpp:69-73)
    delete[] rp.m_imageraylength;
    delete[] rp.m_Correction;
    delete[] rp.m_EachVoxel_TotalWeight;
    delete[] rp.m_Voxel_Contributions;
    return 0;
}

RefGeom make_geom(const int *dims, const float *sp, int W, int H, double ds,
                  double sid, double sdd, const double *oxyz) {
    RefGeom g;
    for (int i = 0; i < 3; ++i) {
        g.dims[i] = dims[i];
        g.sp[i] = sp[i];
        g.oxyz[i] = oxyz ? oxyz[i] : 0.0;
    }
    g.W = W;
    g.H = H;
    g.ds = ds;
    g.sid = sid;
    g.sdd = sdd;
    return g;
}

}  // namespace

extern "C" {

// Forward projection of one view, view k of a round that starts at start_deg.
// image/raylen/weight: W*H floats each (any may be NULL). mats (optional): 96
// floats = P2M, M2V, model-view, volume-to-model, view, projection matrices.
int ref_fp_view(const int *dims, const float *sp, int W, int H, double ds,
                double sid, double sdd, const double *oxyz, double start_deg,
                int k, const float *vol, float *image, float *raylen,
                float *weight, float *mats, int nthreads) {
    if (nthreads > 0) omp_set_num_threads(nthreads);
    RefGeom g = make_geom(dims, sp, W, H, ds, sid, sdd, oxyz);
    return run_view(g, start_deg, k, vol, nullptr, 0, image, raylen, weight,
                    nullptr, nullptr, mats);
}

// Ray-driven backprojection scatter of one view: contrib[v] = sum c*w,
// wsum[v] = sum w, in the reference's sequential order (one thread).
int ref_bp_ray_view(const int *dims, const float *sp, int W, int H, double ds,
                    double sid, double sdd, const double *oxyz,
                    double start_deg, int k, const float *corr, float *contrib,
                    float *wsum, float *raylen) {
    omp_set_num_threads(1);
    RefGeom g = make_geom(dims, sp, W, H, ds, sid, sdd, oxyz);
    return run_view(g, start_deg, k, nullptr, corr, 1, nullptr, raylen,
                    nullptr, contrib, wsum, nullptr);
}

// View rotation quaternion (x, y, z, w) as InitViews/RotateVolume build it.
void ref_view_quaternion(double start_deg, int k, float *xyzw) {
    Quaternion q = RefScene::view_rotation(start_deg, k);
    xyzw[0] = q.x;
    xyzw[1] = q.y;
    xyzw[2] = q.z;
    xyzw[3] = q.w;
}

// warping::warp on a cell-centred grid with aabb = [0,dim] (ST_Tomography.cpp:330-335).
// vel: 3 planar channels; src/out: nc planar channels (CImg layout).
void ref_warp(const int *dim, const float *vel, const float *src, int nc,
              float dt, float *out) {
    CImg<float> V(vel, dim[0], dim[1], dim[2], 3);
    CImg<float> S(src, dim[0], dim[1], dim[2], nc);
    float aabb[6] = {0.0f, (float)dim[0], 0.0f, (float)dim[1], 0.0f, (float)dim[2]};
    CImg<float> O = warping::warp(dim, aabb, V, S, dt);
    std::memcpy(out, O.data(), sizeof(float) * O.size());
}

// warping::warp with aabb = [0, box] over a dim grid (the multiscale flow's case).
void ref_warp_box(const int *dim, const float *box, const float *vel, const float *src, int nc,
                  float dt, float *out) {
    CImg<float> V(vel, dim[0], dim[1], dim[2], 3);
    CImg<float> S(src, dim[0], dim[1], dim[2], nc);
    float aabb[6] = {0.0f, box[0], 0.0f, box[1], 0.0f, box[2]};
    CImg<float> O = warping::warp(dim, aabb, V, S, dt);
    std::memcpy(out, O.data(), sizeof(float) * O.size());
}

// CImg::cubic_atXYZ at n points (px, py, pz), channel 0.
void ref_cubic_at(const int *dim, const float *img, int n, const float *px,
                  const float *py, const float *pz, float *out) {
    CImg<float> I(img, dim[0], dim[1], dim[2], 1);
    for (int i = 0; i < n; ++i) out[i] = I.cubic_atXYZ(px[i], py[i], pz[i], 0);
}

// CImg::get_gradient("xyz", 0): central differences, Neumann boundary.
void ref_gradient(const int *dim, const float *img, float *gx, float *gy, float *gz) {
    CImg<float> I(img, dim[0], dim[1], dim[2], 1);
    CImgList<float> G = I.get_gradient("xyz", 0);
    size_t n = I.size();
    std::memcpy(gx, G[0].data(), sizeof(float) * n);
    std::memcpy(gy, G[1].data(), sizeof(float) * n);
    std::memcpy(gz, G[2].data(), sizeof(float) * n);
}

// CImg::get_blur(sigma) (Deriche, Neumann) of an nc-channel volume.
void ref_blur(const int *dim, int nc, const float *img, float sigma, float *out) {
    CImg<float> I(img, dim[0], dim[1], dim[2], nc);
    CImg<float> O = I.get_blur(sigma);
    std::memcpy(out, O.data(), sizeof(float) * O.size());
}

// CImg::get_resize(nx, ny, nz, nc, 5) (cubic interpolation) of an nc-channel volume.
void ref_resize_cubic(const int *dim, int nc, const float *img, const int *odim, float *out) {
    CImg<float> I(img, dim[0], dim[1], dim[2], nc);
    CImg<float> O = I.get_resize(odim[0], odim[1], odim[2], nc, 5);
    std::memcpy(out, O.data(), sizeof(float) * O.size());
}

// optical_flow::L1Huber_OF (one pyramid level).  V: 3 planar channels, Y1..Y3:
// 3 channels, Y4: 1 channel; all updated in place.  aabb = [0,adim].
void ref_flow_level(const int *dim, const int *adim, const float *I1, const float *I2,
                    float *V, float *Y1, float *Y2, float *Y3, float *Y4,
                    float tol, float lambda, int max_iter, int norm, int nwarps,
                    float huber, const int *roi, int nthreads) {
    if (nthreads > 0) omp_set_num_threads(nthreads);
    int d[3] = {dim[0], dim[1], dim[2]};
    size_t n = (size_t)d[0] * d[1] * d[2];
    CImg<float> A(I1, d[0], d[1], d[2], 1), B(I2, d[0], d[1], d[2], 1);
    CImg<float> v(V, d[0], d[1], d[2], 3), y1(Y1, d[0], d[1], d[2], 3),
        y2(Y2, d[0], d[1], d[2], 3), y3(Y3, d[0], d[1], d[2], 3), y4(Y4, d[0], d[1], d[2], 1);
    float aabb[6] = {0.0f, (float)adim[0], 0.0f, (float)adim[1], 0.0f, (float)adim[2]};
    for (int i = 0; i < 6; ++i) ROI[i] = roi[i];
    optical_flow::L1Huber_OF<float>(d, A, B, v, y1, y2, y3, y4, tol, lambda, max_iter,
                                    norm, nwarps, aabb, huber);
    std::memcpy(V, v.data(), sizeof(float) * n * 3);
    std::memcpy(Y1, y1.data(), sizeof(float) * n * 3);
    std::memcpy(Y2, y2.data(), sizeof(float) * n * 3);
    std::memcpy(Y3, y3.data(), sizeof(float) * n * 3);
    std::memcpy(Y4, y4.data(), sizeof(float) * n);
}

// optical_flow::L1Huber_OF_MultiScale3D; returns the finest-level flow in Vout.
void ref_flow_multiscale(const int *dim, const float *I1, const float *I2,
                         const float *Vin, float *Vout, float tol, float lambda,
                         int max_iter, int norm, int nwarps, float eta,
                         float sigma, int scales, float huber, const int *cut,
                         int nthreads) {
    if (nthreads > 0) omp_set_num_threads(nthreads);
    int d[3] = {dim[0], dim[1], dim[2]};
    CImg<float> A(I1, d[0], d[1], d[2], 1), B(I2, d[0], d[1], d[2], 1);
    CImg<float> v(Vin, d[0], d[1], d[2], 3);
    CImg<float> y1(d[0], d[1], d[2], 3, 0.0f), y2(d[0], d[1], d[2], 3, 0.0f),
        y3(d[0], d[1], d[2], 3, 0.0f), y4(d[0], d[1], d[2], 1, 0.0f);
    int c[8];
    for (int i = 0; i < 8; ++i) c[i] = cut[i];
    CImg<float> out = optical_flow::L1Huber_OF_MultiScale3D<float>(
        d, A, B, v, y1, y2, y3, y4, tol, lambda, max_iter, norm, nwarps, eta, sigma,
        scales, huber, c);
    std::memcpy(Vout, out.data(), sizeof(float) * out.size());
}

}  // extern "C"
