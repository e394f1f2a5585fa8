/* oracle/stt_oracle.h -- TEST INFRASTRUCTURE ONLY (the checker, never the product).
 *
 * C entry points of the CPU restatement of SpaceTimeTomography's
 * reconstruction hot path (oracle/stt_oracle.cpp).  Every function exists in an
 * FP32 flavour (`_f32`, the reference's own float arithmetic, used to pin the
 * restatement against the compiled reference) and most in an FP64 flavour
 * (`_f64`, the FP64 oracle the CUDA path is graded against).
 *
 * Only tests/, tests/golden/ and bench.py's CPU-baseline leg load this library.
 * Layouts follow the reference: volumes x-fastest (idx = x + y*nx + z*nx*ny),
 * detector images m-fastest (idx = m + n*W), multi-channel volumes planar
 * (CImg (x,y,z,c) order).
 */
#ifndef STT_ORACLE_H
#define STT_ORACLE_H
#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_geom {
    int nx, ny, nz;       /* volume dims (voxels) */
    double sx, sy, sz;    /* voxel spacing (mm) */
    int W, H;             /* detector pixels */
    double ds;            /* detector pixel spacing (mm) */
    double sid, sdd;      /* source-isocentre / source-detector distance (mm) */
    double off[3];        /* --oxyz volume-centre offset (mm) */
} orc_geom;

/* Per-view description.  gmode 0: the reference's FP32 matrix pipeline driven
 * by the float quaternion `quat` (x,y,z,w); gmode 1: FP64 geometry from
 * `angle` (radians about +y). */
typedef struct orc_view {
    double angle;
    float quat[4];
} orc_view;

/* The reference's view quaternion for view k of a round starting at start_deg
 * (InitViews/RotateVolume, ST_Tomography.cpp:887-934); also fills angle. */
void orc_view_from_round(double start_deg, int k, orc_view *v);
/* A single rotation by `angle` radians (explicit angle lists). */
void orc_view_from_angle(double angle, orc_view *v);

/* The 16-float matrices of the reference pipeline for one view:
 * out[0..15] P2M, [16..31] M2V, [32..47] model-view, [48..63] V2M. */
void orc_view_matrices_f32(const orc_geom *g, const orc_view *v, float *out);

/* Forward projection (TypicalRayProducer.core.h:123-268, RayCaster.core.h:42-188).
 * raylen is sticky: written only where the ray hits the volume, as in
 * the reference.  weight = sample count.  Any output may be NULL. */
int orc_fp_f32(const orc_geom *g, int gmode, const orc_view *v, const float *vol,
               float *img, float *raylen, float *weight, int nthreads);
int orc_fp_f64(const orc_geom *g, const orc_view *v, const double *vol,
               double *img, double *raylen, double *weight, int nthreads);

/* orc_fp_f64 on detector rows [row0, row1) only (img is the full W*H image;
 * other rows are left as they are): a band of a view whose full FP64
 * projection would take minutes. */
int orc_fp_rows_f64(const orc_geom *g, const orc_view *v, const double *vol, int row0, int row1,
                    double *img, int nthreads);
/* The same band in the reference's FP32 arithmetic (orc_fp_f32). */
int orc_fp_rows_f32(const orc_geom *g, int gmode, const orc_view *v, const float *vol, int row0, int row1,
                    float *img, int nthreads);

/* Ray-driven BP scatter (SingleScalarVolume.core.h:73-84,128-143): adds
 * c[pix]*w to contrib and w to wsum, sequentially in pixel order. */
int orc_bp_ray_scatter_f32(const orc_geom *g, int gmode, const orc_view *v,
                           const float *corr, float *contrib, float *wsum);
/* Exact adjoint of orc_fp: vol_bar += A^T proj_bar (sd * w_i * y, first sample twice). */
int orc_fp_adjoint_f64(const orc_geom *g, const orc_view *v, const double *proj_bar,
                       double *vol_bar);
int orc_fp_adjoint_f32(const orc_geom *g, int gmode, const orc_view *v,
                       const float *proj_bar, float *vol_bar);

/* Voxel-driven BP (ST_Tomography.cpp:690-730): vol = clamp(vol + alpha*bicubic(c)).
 * alpha is a double, as the reference's m_alpha (:91): the update is formed in
 * double and rounded to float once. */
int orc_bp_voxel_f32(const orc_geom *g, int gmode, const orc_view *v, const float *corr,
                     double alpha, float gmax, float *vol, int nthreads);
int orc_bp_voxel_f64(const orc_geom *g, const orc_view *v, const double *corr,
                     double alpha, double gmax, double *vol, int nthreads);

/* SART correction (ST_Tomography.cpp:667-676 with pY == 0): c = (b - Ax)/(L + 1). */
void orc_correction_f32(int n, const float *b, const float *ax, const float *raylen, float *c);

/* Ray-BP normalisation (ST_Tomography.cpp:746-762): vol = clamp(vol + contrib/wsum), 0/0 -> 0. */
void orc_bp_ray_update_f32(long n, const float *contrib, const float *wsum, float gmax,
                           float *vol);

/* One SART call for one frame (ST_Tomography.cpp:616-808): views in the order
 * perm[0..nv-1]; proj holds nv_total images (W*H each) indexed by view id;
 * bp_mode 0 voxel-based, 1 ray-based; raylen_state is the producer's sticky
 * ray-length buffer (W*H, caller-owned, zero at construction); roi (optional)
 * multiplies the volume after the sweep. */
int orc_sart_f32(const orc_geom *g, int gmode, const orc_view *views, const int *perm, int nv,
                 const float *proj, double alpha, float gmax, int bp_mode, float *vol,
                 float *raylen_state, const float *roi, int nthreads);
int orc_sart_f64(const orc_geom *g, const orc_view *views, const int *perm, int nv,
                 const double *proj, double alpha, double gmax, int bp_mode, double *vol,
                 double *raylen_state, const double *roi, int nthreads);

/* ROI mask (ST_Tomography.cpp:303-329) with cut[8]. */
void orc_roi_mask_f32(const int *dims, const int *cut, float *roi);

/* Seeded view permutation used in place of srand(time(0)) + random_shuffle
 * (ST_Tomography.cpp:635-642): SplitMix64 stream, Fisher-Yates. */
void orc_permutation(unsigned long long seed, int n, int *perm);

/* Primal-dual steps for frame f (ST_Tomography.cpp:503-604).  bw is the
 * backward-warped X_bar[f+1] and fw the forward-warped Y_bc[f-1] (NULL for f == 0). */
typedef struct orc_pd_params {
    float sigma, tau, tv_w, tp_w, bc_w, huber_factor, gmax;
    int cut[8];
} orc_pd_params;
void orc_pd_dual_f32(const int *dims, const orc_pd_params *p, const float *xbar_f,
                     const float *xbar_f1, const float *bw, float *ytv, float *ytp, float *ybc);
void orc_pd_primal_f32(const int *dims, const orc_pd_params *p, int first_frame,
                       const float *ytp_prev, const float *ytp, const float *fw,
                       const float *ybc, const float *ytv, float *vol, float *xprev);
void orc_pd_extrapolate_f32(const int *dims, const int *cut, const float *vol,
                            const float *xprev, float *xbar);
void orc_pd_dual_f64(const int *dims, const double *pp, const int *cut, const double *xbar_f,
                     const double *xbar_f1, const double *bw, double *ytv, double *ytp, double *ybc);
void orc_pd_primal_f64(const int *dims, const double *pp, const int *cut, int first_frame,
                       const double *ytp_prev, const double *ytp, const double *fw,
                       const double *ybc, const double *ytv, double *vol, double *xprev);
void orc_pd_extrapolate_f64(const int *dims, const int *cut, const double *vol,
                            const double *xprev, double *xbar);

/* warping::warp (ST_Tomo/warping.h:49-145) with aabb = [0,dim]: vel 3 planar
 * channels, src/out nc planar channels. */
void orc_warp_f32(const int *dim, const float *vel, const float *src, int nc, float dt,
                  float *out, int nthreads);
void orc_warp_f64(const int *dim, const double *vel, const double *src, int nc, double dt,
                  double *out, int nthreads);
/* Vector-Jacobian product of orc_warp_f64: src_bar += J_src^T out_bar,
 * vel_bar += J_vel^T out_bar (either may be NULL).  The 8-corner min/max clamp
 * and the [1, dim-2] coordinate clamp are differentiated piecewise. */
void orc_warp_vjp_f64(const int *dim, const double *vel, const double *src, int nc,
                      double dt, const double *out_bar, double *src_bar, double *vel_bar);

/* CImg::_cubic_atXYZ (CImg.h:13429-13520) at one point, float and double. */
float orc_cubic_at_f32(const int *dim, const float *img, float x, float y, float z);
double orc_cubic_at_f64(const int *dim, const double *img, double x, double y, double z);

/* warping::warp with aabb = [0, box] over a dim grid (the multiscale flow
 * warps every pyramid level in full-resolution units, optical_flow.h:700). */
void orc_warp_box_f32(const int *dim, const float *box, const float *vel, const float *src, int nc,
                      float dt, float *out, int nthreads);

/* CImg::blur(sigma) (Deriche, Neumann) in place on nc planar channels. */
void orc_blur_f32(const int *dim, int nc, float sigma, float *img);
/* CImg::get_resize(odim, nc, 5): moving average on shrinking axes, Catmull-Rom
 * on growing ones, x then y then z. */
void orc_resize_f32(const int *dim, int nc, const float *in, const int *odim, float *out);
/* CImg::get_gradient("xyz", 0): central differences, Neumann. */
void orc_gradient_f32(const int *dim, const float *img, float *gx, float *gy, float *gz);
/* optical_flow::L1Huber_OF (optical_flow.h:83-623) on one level, one thread.
 * V: 3 channels, Y: 10 channels (Y1|Y2|Y3|Y4), both in/out; roi = {x0,x1,y0,y1,z0,z1};
 * box: aabb extents; iters, errs (optional): iterations run per warp and its last residual. */
void orc_flow_level_f32(const int *dim, const float *box, const int *roi, const float *I1, const float *I2,
                        float *V, float *Y, float tol, float lambda, int max_iter, int norm, int n_warps,
                        float huber, int *iters, float *errs);
/* optical_flow::L1Huber_OF_MultiScale3D (optical_flow.h:630-734); cut: 6 ints. */
void orc_flow_multiscale_f32(const int *dim, const float *I1, const float *I2, const float *Vin,
                             const float *Yin, float *Vout, float tol, float lambda, int max_iter,
                             int norm, int n_warps, float eta, float sigma, int scales, float huber,
                             const int *cut);

#ifdef __cplusplus
}
#endif
#endif
