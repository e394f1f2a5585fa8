// stt_kernels.h -- host-side launch wrappers of the kernels in k_*.cu.
#pragma once

#include <cuda.h>
#include <cuda_runtime.h>

namespace stt {

struct ViewRec;
struct GeomDev;
struct ViewSel;

struct PdParams {
    float sigma, tau, tv_w, tp_w, bc_w, hf, gmax;
    int cut[8];
};

// Multiprocessor count of the current device (cached per device).
int sm_count();
int grid_stride_blocks(long long n, int threads);

// Launch shapes of the tunable kernels, picked by the autotuner (stt_tune.cu).
// Variant 0 of each is the default; all variants of a kernel give the same
// bits (they change which thread or block computes what, never a value's
// arithmetic).
//   fp:   the gather forward projector k_fp_corr: detector tile, samples
//         in flight and, for variants 10 and 11, corners fetched as two tld4
//         texture gathers per sample instead of eight loads (fp_variant_name);
//   slab: the box of the slab-staged projector (slab_variant_name);
//   bp:   the column length of the voxel backprojection, and whether each
//         column's voxels are first prefetched into L2 (bp_variant_name);
//   ray:  the scatter of the ray-driven backprojection (ray_variant_name):
//         0 one global vector atomic per corner, 1 a shared-memory box per
//         slab (volumes below 2^31 voxels).  Its sums differ in float order
//         only (as any two atomic runs do), not in their terms.
// Which views the slab kernel projects is the per-view ViewRec::staged flag.
constexpr int kFpVariants = 12, kSlabVariants = 8, kBpVariants = 5, kRayVariants = 2;
struct Tuning {
    int fp = 0, slab = 0, bp = 0, ray = 0;
    int fp16 = 0;  // the BF16-stored volume's gather form (fp16_variant_name)
};
const char *fp_variant_name(int v);
const char *slab_variant_name(int v);
const char *bp_variant_name(int v);
const char *ray_variant_name(int v);
// The scatter an untuned context uses: the slab box from 2^26 voxels on (at
// 512^3 it is the faster form; at 256^3 and below the global scatter is).
int default_ray_variant(const GeomDev &g);

cudaError_t launch_fp(const GeomDev &g, const ViewRec *views, const float *vol, const float *vol_t, int view0,
                      int nviews, float *proj, float *raylen, float *weight, cudaStream_t s);
// Slab-staged forward projector (k_fp_slab.cu) for the views marked `staged`:
// the same outputs as the gather form bit for bit, the volume read through
// TMA boxes.  The tensor maps cover the volume and its z-fastest copy (vol_t
// may be null: then every view gathers from vol) with the box of slab variant
// `variant`; make_fp_slab_maps returns false where the form does not apply (x
// or z extent not a multiple of 4, an array not 16-byte aligned, 2^31 voxels
// or more).  `status` (may be null) is set to 1 if a box copy did not land
// within the wait limit.
struct FpSlabMaps {
    CUtensorMap x, z;
    int ok, has_z, variant;
    int esize;  // bytes per voxel: 4 (FP32) or 2 (BF16)
};
bool make_fp_slab_maps(const GeomDev &g, const float *vol, const float *vol_t, FpSlabMaps &m, int variant = 0);
// BF16 storage: the scalar boxes (variant & 3); x and z extents multiples of 8.
bool make_fp_slab_maps(const GeomDev &g, const unsigned short *vol, const unsigned short *vol_t, FpSlabMaps &m,
                       int variant = 0);
// A 4D FP32 tensor map over nc planar volumes (x fastest, then y, z, plane)
// with the given box (x, y, z, plane); false where TMA cannot address them
// (nx not a multiple of 4, ptr not 16-byte aligned, box row not 16 bytes).
bool encode_planes_map(CUtensorMap *m, const float *ptr, int nx, int ny, int nz, int nc, const unsigned box[4]);
cudaError_t launch_fp_corr_slab(const GeomDev &g, const ViewRec *views, const FpSlabMaps &m, const float *vol,
                                const float *vol_t, const ViewSel &sel, const float *b_stack, float *raylen_state,
                                float *corr, cudaStream_t s, unsigned long long corr_surf, int *status);
cudaError_t launch_fp_corr_slab(const GeomDev &g, const ViewRec *views, const FpSlabMaps &m,
                                const unsigned short *vol, const unsigned short *vol_t, const ViewSel &sel,
                                const unsigned short *b_stack, float *raylen_state, float *corr, cudaStream_t s,
                                unsigned long long corr_surf, int *status);
// Texture objects of the gather variants that fetch corners with tld4: the
// volume as a pitch-linear 2D texture whose rows are its z slices (width
// nx*ny texels, nz rows) and its z-fastest copy likewise (rows the x slices;
// z = 0 without a copy); FP32 texels, or for a BF16-stored volume 16-bit
// unsigned texels holding its bits.  Point sampling returns stored values
// exactly, so the samples are those of the loads they replace.
// make_fp_tex returns false (and creates nothing) where the device's limits
// on linear 2D textures do not admit the arrays: a row of more than the
// maximum width or pitch, more rows than the maximum height, a base not
// aligned to the texture alignment.  The caller owns the objects
// (destroy_fp_tex).
struct FpTex {
    unsigned long long x = 0, z = 0;
    int ok = 0;
    int esize = 0;  // bytes per texel: 4 (FP32) or 2 (BF16)
};
bool is_tex_fp_variant(int fp_variant);
bool make_fp_tex(const GeomDev &g, const float *vol, const float *vol_t, FpTex &t);
bool make_fp_tex(const GeomDev &g, const unsigned short *vol, const unsigned short *vol_t, FpTex &t);
// Whether make_fp_tex admits `vol` (esize bytes per voxel) and a z-fastest
// copy at an aligned base on this device (checks the limits only; creates
// nothing).
bool fp_tex_fits(const GeomDev &g, const void *vol, int esize);
void destroy_fp_tex(FpTex &t);
// Forward projection of one view fused with the SART correction.  With usable
// slab maps, staged views run in the slab-staged kernel and the others in the
// gather kernel (both are launched; each leaves the other's views alone).
// `fp_variant` selects the gather kernel's launch shape; a texture variant
// (is_tex_fp_variant) without usable `tex` runs the load-based variant of the
// same shape, which gives the same bits.
cudaError_t launch_fp_corr(const GeomDev &g, const ViewRec *views, const float *vol, const float *vol_t,
                           const ViewSel &sel, const float *b_stack, float *raylen_state, float *corr,
                           cudaStream_t s, unsigned long long corr_surf = 0, const FpSlabMaps *maps = nullptr,
                           int *status = nullptr, int fp_variant = 0, const FpTex *tex = nullptr);
cudaError_t launch_transpose(const GeomDev &g, const float *in, float *out, cudaStream_t s);
cudaError_t launch_fp_bf16(const GeomDev &g, const ViewRec *views, const unsigned short *vol,
                           const unsigned short *vol_t, int view0, int nviews, float *proj, float *raylen,
                           float *weight, cudaStream_t s);
cudaError_t launch_transpose_bf16(const GeomDev &g, const unsigned short *in, unsigned short *out, cudaStream_t s);
cudaError_t launch_transpose_for_view(const GeomDev &g, const ViewRec *views, const ViewSel &sel, const float *in,
                                      float *out, cudaStream_t s);
cudaError_t launch_transpose_for_view(const GeomDev &g, const ViewRec *views, const ViewSel &sel,
                                      const unsigned short *in, unsigned short *out, cudaStream_t s);

// BF16 storage (the raw upper halves of FP32 values; the solver's
// stt_solve_cfg.storage): the overloads below on unsigned short arrays read
// stored values widened exactly to FP32, compute as their FP32 forms do, and
// round what they store to nearest even.  Duals, flows, corrections and
// accumulators stay FP32.
// The fused forward projection of a BF16 volume against a BF16 sinogram:
// with usable BF16 slab maps the staged views run in the slab kernel (BF16
// boxes), the others in the gather kernel; without them every view gathers.
// The gather kernel loads its corners (fp_variant16 0: 32x4 rays, 4 samples
// in flight) or, with usable BF16 textures `tex`, gathers them with tld4
// (fp_variant16 1: warps of 8x4 rays, 8 samples in flight in packed pairs);
// the same bits either way.
constexpr int kFp16Variants = 2;
const char *fp16_variant_name(int v);
cudaError_t launch_fp_corr(const GeomDev &g, const ViewRec *views, const unsigned short *vol,
                           const unsigned short *vol_t, const ViewSel &sel, const unsigned short *b_stack,
                           float *raylen_state, float *corr, cudaStream_t s, unsigned long long corr_surf = 0,
                           const FpSlabMaps *maps = nullptr, int *status = nullptr, int fp_variant16 = 0,
                           const FpTex *tex = nullptr);
cudaError_t launch_correction(long long n, const unsigned short *b, const float *ax, const float *raylen,
                              float *corr, cudaStream_t s);
cudaError_t launch_correction(long long n, const float *b, const float *ax, const float *raylen,
                              float *corr, cudaStream_t s);
// Ray-driven backprojection: the scatter into acc (interleaved contribution,
// weight), then vol += contribution/weight and acc cleared.  The scatter is
// ray variant `ray_variant` (-1: default_ray_variant): a global atomic per
// corner, or a shared-memory box per slab (k_bp_slab.cu, below 2^31 voxels).
cudaError_t launch_bp_ray(const GeomDev &g, const ViewRec *views, const ViewSel &sel, const float *corr,
                          float2 *acc, float *vol, float gmax, cudaStream_t s, int ray_variant = -1);
cudaError_t launch_bp_ray(const GeomDev &g, const ViewRec *views, const ViewSel &sel, const float *corr,
                          float2 *acc, unsigned short *vol, float gmax, cudaStream_t s, int ray_variant = -1);
cudaError_t launch_bp_ray_scatter_slab(const GeomDev &g, const ViewRec *views, const ViewSel &sel, const float *corr,
                                       float2 *acc, cudaStream_t s);
cudaError_t launch_bp_ray_scatter(const GeomDev &g, const ViewRec *views, const ViewSel &sel, const float *corr,
                                  float2 *acc, float *contrib, float *wsum, cudaStream_t s, int ray_variant = -1);
cudaError_t launch_fp_adjoint(const GeomDev &g, const ViewRec *views, int view0, int nviews,
                              const float *proj_bar, float *vol_bar, cudaStream_t s);
// The gather ceiling (k_project.cu): one view's rays sampled at the
// projector's step with its gathers and interpolation and none of its march
// control; `host_view` is the view's record (its layout picks vol_t).  With
// `tex` (made over vol and vol_t) the corners are tld4 gathers in packed pairs.
cudaError_t launch_gather_ceiling(const GeomDev &g, const ViewRec *views, const ViewRec &host_view, int view,
                                  const float *vol, const float *vol_t, int packed, float *out, int *count,
                                  cudaStream_t s, const FpTex *tex = nullptr);
cudaError_t launch_fill_zero(float *p, long long n, cudaStream_t s);
cudaError_t launch_dot_f64(long long n, const float *a, const float *b, double *out, cudaStream_t s);
cudaError_t launch_scale_inv_sqrt(long long n, float *x, const double *norm2, cudaStream_t s);
cudaError_t launch_fill_seeded(long long n, unsigned long long seed, float *x, cudaStream_t s);

// The persistent sweep (k_persist.cu): the SART calls of all jobs (frames or
// batch instances, SweepJob in stt_internal.cuh) in one cooperative launch of
// `nblocks` blocks, jobs_d a device array sorted by block0.  bf16: the jobs'
// storage; wide: some job's volume has 2^31 voxels or more.
struct SweepJob;
// Blocks of the launch that can be resident at once on the current device (0
// on error): the most a launch may have.
int sweep_max_blocks(bool bf16, bool wide);
// Orders the jobs into rounds (largest first, at most nblocks jobs a round:
// one round unless there are more jobs than blocks) and splits the nblocks
// over each round's jobs in proportion to their work: sets round, block0 and
// nblocks and sorts the array by round.  Returns the number of rounds.
int sweep_plan(SweepJob *jobs, int njobs, int nblocks);
cudaError_t launch_sweep_persistent(const SweepJob *jobs_d, int njobs, int nblocks, bool bf16, bool wide,
                                    int *status, cudaStream_t s);
// The whole primal-dual iteration of every job (view order, warps, dual and
// primal steps, then the SART call) in one cooperative launch; one round (at
// most nblocks jobs); gbar: two words zeroed before the launch, like the
// jobs' barrier words.
cudaError_t launch_iter_persistent(const SweepJob *jobs_d, int njobs, int nblocks, bool bf16, bool wide,
                                   unsigned *gbar, int *status, cudaStream_t s);

// The correction image held as a one-layer layered CUDA array: the texture
// object the column backprojection gathers from (tld4) and the surface object
// the fused forward projection writes (launch_fp_corr's corr_surf).
struct CorrTex {
    cudaArray_t arr = nullptr;
    unsigned long long tex = 0, surf = 0;
    int W = 0, H = 0;
};
cudaError_t make_corr_tex(int W, int H, CorrTex &o);
void free_corr_tex(CorrTex &o);

// Voxel-driven backprojection; with the correction as a texture (corr_tex)
// the column walk of bp variant `bp_variant` runs, else the per-voxel form.
cudaError_t launch_bp_voxel(const GeomDev &g, const ViewRec *views, const ViewSel &sel, const float *corr,
                            float *vol, float alpha, float gmax, cudaStream_t s, unsigned long long corr_tex = 0,
                            int bp_variant = 0);
cudaError_t launch_bp_voxel(const GeomDev &g, const ViewRec *views, const ViewSel &sel, const float *corr,
                            unsigned short *vol, float alpha, float gmax, cudaStream_t s,
                            unsigned long long corr_tex = 0, int bp_variant = 0);
// Sets the solver's device-side iteration counter (stream-ordered, no host memory read).
cudaError_t launch_set_counter(unsigned long long *counter, unsigned long long v, cudaStream_t s);
// View orders of `frames` local frames (at most 1024), local frame f being
// frame frame0 + f of a sequence of `total`; advances *counter.
cudaError_t launch_make_perm(unsigned long long seed, unsigned long long *counter, int frames, int total,
                             int frame0, int views, int *perm, cudaStream_t s);
cudaError_t launch_pd_dual(const int *dims, const PdParams &p, const float *xf, const float *xf1,
                           const float *bw, float *ytv, float *ytp, float *ybc, cudaStream_t s);
cudaError_t launch_pd_dual(const int *dims, const PdParams &p, const unsigned short *xf, const unsigned short *xf1,
                           const float *bw, float *ytv, float *ytp, float *ybc, cudaStream_t s);
cudaError_t launch_pd_primal(const int *dims, const PdParams &p, int first, const float *ytp_prev,
                             const float *ytp, const float *fw, const float *ybc, const float *ytv,
                             float *vol, float *xprev, cudaStream_t s);
cudaError_t launch_pd_primal(const int *dims, const PdParams &p, int first, const float *ytp_prev,
                             const float *ytp, const float *fw, const float *ybc, const float *ytv,
                             unsigned short *vol, unsigned short *xprev, cudaStream_t s);
cudaError_t launch_pd_extrapolate(const int *dims, const int *cut, const float *vol,
                                  const float *xprev, float *xbar, cudaStream_t s);
cudaError_t launch_pd_extrapolate(const int *dims, const int *cut, const unsigned short *vol,
                                  const unsigned short *xprev, unsigned short *xbar, cudaStream_t s);
cudaError_t launch_roi_apply(const int *dims, const int *roi_cut, const int *pd_cut, float *vol,
                             const float *xprev, float *xbar, cudaStream_t s);
cudaError_t launch_roi_apply(const int *dims, const int *roi_cut, const int *pd_cut, unsigned short *vol,
                             const unsigned short *xprev, unsigned short *xbar, cudaStream_t s);
cudaError_t launch_roi_mask(const int *dims, const int *cut, float *roi, cudaStream_t s);

// ---- optical flow (k_flow.cu) ----
struct FlowRoi {
    int x0, x1, y0, y1, z0, z1;  // cut from each face
};

struct DericheCoef {
    float a0, a1, a2, a3, b1, b2, coefp, coefn;
};

// One axis of a CImg resize: mode 0 = moving average (shrinking), mode 1 =
// Catmull-Rom (growing) with the per-output (source index, fraction) table
// written by launch_resize_table.
struct ResizeAxis {
    int axis, mode, nc;
    int ix, iy, iz;  // input extents
    int ox, oy, oz;  // output extents (differ from the input along `axis` only)
    int old_n, new_n;
    const int *src;
    const double *frac;
};

cudaError_t launch_warp_box(const int *dim, const float *box, const float *vel, const float *src, int nc,
                            float dt, float *out, cudaStream_t s);
cudaError_t launch_flow_setup(const int *d, const FlowRoi &roi, const float *i2w, const float *i1,
                              const float *v, float *u, float *tau, float *sig2, float *k4prev, cudaStream_t s);
cudaError_t launch_flow_primal(const int *d, const FlowRoi &roi, const float *y, const float *u,
                               const float *tau, const float *v_in, float *v_out, float *kty, int flags,
                               double *resid, const int *done, cudaStream_t s);
cudaError_t launch_flow_dual(const int *d, const float *v, const float *v_old, const float *u, const float *sig2,
                             const float *k4prev, float *y, float sigma1, float hf, float lambda, int huber,
                             int flags, double *resid, const int *done, cudaStream_t s);
cudaError_t launch_flow_settle(long long n3, const int *iters, const float *v_b, float *v_a, cudaStream_t s);
cudaError_t launch_flow_check(double *resid, long long n, float tol, int it, int is_resid, int is_last,
                              int *done, int *iters, float *err, cudaStream_t s);
cudaError_t launch_flow_reset(int *done, double *resid, int *iters, float *err, cudaStream_t s);
cudaError_t launch_deriche(const int *d, int nc, int axis, const DericheCoef &c, float *img, float *tmp,
                           cudaStream_t s);
cudaError_t launch_resize_table(int old_n, int new_n, int *src, double *frac, cudaStream_t s);
cudaError_t launch_resize_axis(const ResizeAxis &ra, const float *in, float *out, cudaStream_t s);
cudaError_t launch_gradient(const int *d, const float *img, float *g, cudaStream_t s);
cudaError_t launch_copy_roi(const int *d, int nc, const FlowRoi &roi, const float *src, float *dst,
                            cudaStream_t s);

// `status` (may be null: then a per-device word read by warp_poll_status) is
// set when the staged kernel's bounded wait for its velocity box gave up.
cudaError_t launch_warp(const int *dim, const float *vel, const float *src, int nc, float dt,
                        float *out, cudaStream_t s, int *status = nullptr);
// The warp of a BF16-stored source (taps widened to FP32; FP32 flow and output).
cudaError_t launch_warp(const int *dim, const float *vel, const unsigned short *src, int nc, float dt,
                        float *out, cudaStream_t s, int *status = nullptr);
// Reads and clears the per-device status word of warps launched without one
// (synchronises `s`); *flag is non-zero if a bounded wait gave up.
cudaError_t warp_poll_status(int *flag, cudaStream_t s);
cudaError_t launch_warp_vjp(const int *dim, const float *vel, const float *src, int nc, float dt,
                            const float *out_bar, float *src_bar, float *vel_bar, cudaStream_t s);

}  // namespace stt
