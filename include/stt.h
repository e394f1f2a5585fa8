/* include/stt.h -- C ABI of libstt.so, the B200 (sm_100a) implementation of
 * SpaceTimeTomography's reconstruction hot path.
 *
 * Conventions
 *   - Every entry point returns stt_status; STT_OK is 0.  Nothing throws across
 *     the ABI.  stt_last_error() returns the message of the last failure on a
 *     context (a pointer valid until the next call on that context).
 *   - All array arguments are DEVICE pointers owned by the caller, except where
 *     a comment says "host".  Layouts follow the reference: volumes x-fastest
 *     (idx = x + y*nx + z*nx*ny, CImg (x,y,z) order), detector images
 *     m-fastest (idx = m + n*W), multi-channel volumes planar (CImg (x,y,z,c)),
 *     projection stacks view-major (idx = m + n*W + v*W*H).
 *   - `stream` is a cudaStream_t passed as void*; NULL is the legacy default
 *     stream.  Calls only enqueue work; nothing synchronises unless stated.
 *   - A context is used by one host thread at a time; different contexts may
 *     be used concurrently.  A context owns its geometry tables and the scratch
 *     accumulators of the ray-driven backprojector.
 *
 * Reference interfaces replaced (paths relative to the reference project root
 * gmzang/SpaceTimeTomography, S/ = SpaceTimeTomography/):
 *   forward projector  GenerateImage_GetCorrections  S/ImageFormationModel/TypicalRayProducer.core.h:230
 *                      + SingleScalarVolumePrepare    S/ImageFormationModel/SingleScalarVolume.core.h:195
 *                      + RayCasterPrepare             S/ImageFormationModel/RayCaster.core.h:191
 *   geometry           TypicalRayProducer ctor / SetVolSize / SetViewMatrix / SetProjectionMatrix
 *                      S/ImageFormationModel/TypicalRayProducer.h:11-24, Scene::_calculateMatrix Scene.cpp:181,
 *                      ST_Tomography::InitViews S/ST_Tomo/ST_Tomography.cpp:887
 *   SART               ST_Tomography::SART        S/ST_Tomo/ST_Tomography.cpp:616-808
 *   primal-dual steps  ST_Tomography::Render      S/ST_Tomo/ST_Tomography.cpp:492-607
 *   warp               warping::warp              S/ST_Tomo/warping.h:116-145
 *   optical flow       optical_flow::L1Huber_OF_MultiScale3D / L1Huber_OF
 *                                                 S/ST_Tomo/optical_flow.h:83-734
 */
#ifndef STT_H
#define STT_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum stt_status {
    STT_OK = 0,
    STT_ERR_INVALID = 1,      /* bad argument (null pointer, size, geometry) */
    STT_ERR_CUDA = 2,         /* a CUDA runtime call or kernel launch failed */
    STT_ERR_NOMEM = 3,        /* device allocation failed */
    STT_ERR_STATE = 4,        /* call out of order (e.g. no geometry set) */
    STT_ERR_UNSUPPORTED = 5,  /* option not available in this build */
    STT_ERR_TIMEOUT = 6       /* a bounded device-side wait gave up */
} stt_status;

typedef struct stt_ctx stt_ctx;

/* Scan geometry.  Replaces the TypicalRayProducer constructor arguments
 * (TypicalRayProducer.h:11), VolumeData::SetSpacings, the Scene members set by
 * the ST_Tomography constructor (ST_Tomography.cpp:200-246) and the per-view
 * quaternions of InitViews (:887-934).  The per-view ray and voxel projections
 * are built on the host in FP64.
 *   angles_rad: HOST array of n_views rotation angles about +y (radians);
 *   stt_views_from_rounds() builds the reference's "rounds x 10 views 36 deg
 *   apart" lists. */
typedef struct stt_geometry {
    int nx, ny, nz;        /* volume dimensions (voxels)             -f        */
    double sx, sy, sz;     /* voxel spacing (mm)                      -c        */
    int W, H;              /* detector size (pixels)                  -u        */
    double ds;             /* detector pixel spacing (mm)             -d        */
    double sid, sdd;       /* source-isocentre, source-detector (mm)  -g, -j    */
    double off[3];         /* volume-centre offset (mm)               --oxyz    */
    int n_views;
    const double *angles_rad;
} stt_geometry;

/* Context lifetime.  device: CUDA ordinal. */
stt_status stt_create(stt_ctx **ctx, int device);
stt_status stt_destroy(stt_ctx *ctx);
const char *stt_last_error(const stt_ctx *ctx);
/* Library version string, e.g. "stt 0.1.0 sm_100a". */
const char *stt_version(void);

/* Bounded device-side waits.  No counterpart in the reference (CPU code, no
 * device waits).  The TMA-staged kernels (the slab forward projector of
 * stt_fp_correction / stt_sart_sweep / the solver, the staged warp) wait for
 * their shared-memory copies for at most about 0.1 s.  A copy that does not
 * land in time is an error: the kernel takes those taps from global memory
 * instead (the same result), waits once more, again bounded, so that no block
 * exits with a copy still writing into its shared memory, and raises a status
 * flag.  stt_poll_status synchronises `stream` and returns STT_ERR_TIMEOUT
 * (message in stt_last_error) if a launch of this context raised the flag
 * since the last poll, clearing it; otherwise STT_OK.  stt_solver_poll_status
 * and stt_batch_poll_status do the same for a solver or a batch, and
 * stt_warp_poll_status for stt_warp / stt_warp_box calls on the current
 * device. */
stt_status stt_poll_status(stt_ctx *ctx, void *stream);
stt_status stt_warp_poll_status(void *stream);

/* Host helper: angles (radians) of the reference's view list.  Round r of
 * `rounds` starts at start_deg[r] (host); views k = 0..views_per_round-1 sit
 * step_deg apart; angles_out (host) receives rounds*views_per_round values.
 * The start angle is rounded through float and pi is 3.1415926 as in
 * ST_Tomography.cpp:264-268, 871, 899. */
stt_status stt_views_from_rounds(int rounds, const double *start_deg, int views_per_round,
                                 double step_deg, double *angles_out);

/* Low-discrepancy start angles (degrees) of the acquisition scripts
 * (low discrepancy sequence/Low_discrepency_squence.m:38-67): van der Corput in
 * base p, Ns segments, a reference angle 0 every Nz entries.  out (host) gets n values. */
stt_status stt_lds_angles(int n, int Ns, int p, int Nz, double *out);

/* Set (or replace) the geometry and view list. Allocates the context's device
 * tables and resets the launch choices below to their defaults. */
stt_status stt_set_geometry(stt_ctx *ctx, const stt_geometry *g);

/* ---- launch choices and the autotuner ------------------------------------
 * No counterpart in the reference (a CPU program with fixed OpenMP loops
 * over detector rows, TypicalRayProducer.core.h:168, and voxels,
 * ST_Tomography.cpp:690).  The forward projector with the SART correction
 * (stt_fp_correction, stt_sart_sweep, the solver) and the solver's voxel
 * backprojection come in launch variants that give the same bits:
 *   fp_variant   the gather projector's detector tile and samples in flight;
 *                variants 10 and 11 fetch a sample's 8 corners as two tld4
 *                gathers of the FP32 volume bound as a pitch-linear 2D texture
 *                (the context keeps one texture object per array it is given,
 *                until stt_destroy; where the device's texture limits do not
 *                admit the array, the load-based variant of the same shape runs);
 *   slab_variant the box the slab-staged projector stages with TMA;
 *   bp_variant   the column length of the voxel backprojection (solver), and
 *                whether each column's voxels are first prefetched into L2
 *                (for volumes larger than L2);
 *   staged_bins  bit b set: views whose central ray is 5b to 5b+5 degrees off
 *                the nearest of the x and z axes (bit 8: 40 to 45) are
 *                projected by the slab-staged kernel, the others by the gather
 *                kernel (the slab form needs x and z extents that are multiples
 *                of 4 and a 16-byte aligned volume; elsewhere every view gathers).
 * stt_autotune times every variant with CUDA events on this context's
 * geometry (one representative view per off-axis class, weighted by the views
 * in the class; scratch volumes it allocates and frees), keeps the fastest,
 * and caches the choice per device and geometry shape for later contexts.  It
 * synchronises `stream` and rewrites the context's view table, so call it
 * (and stt_set_tuning) while no launch of this context is in flight; launches
 * enqueued after it use the choice, and a solver uses the choice current when
 * it is created (stt_solve_cfg.autotune runs the tuner then).  out (may be
 * NULL) receives the choice and the timings (microseconds per launch, 0 where
 * a variant was not timed).  stt_get_tuning reads the current choice;
 * stt_set_tuning sets one (a variant out of range is STT_ERR_INVALID). */
typedef struct stt_tuning {
    int fp_variant, slab_variant, bp_variant;
    unsigned staged_bins;
    int tuned;       /* 0: the defaults; 1: set by stt_autotune or stt_set_tuning */
    int from_cache;  /* stt_autotune: the choice came from the cache (nothing timed) */
    float fp_us[12], slab_us[8], bp_us[8];
    int ray_variant;  /* the ray-driven backprojection's scatter (kernel 3 of stt_tuning_variant_name);
                         untuned: the shared-memory slab box from 2^26 voxels on, else global atomics */
    float ray_us[2];
    unsigned staged_bins_bf16;  /* staged_bins for a BF16-stored volume (stt_solve_cfg.storage,
                                   stt_sart_sweep_typed): its gathers and boxes move half the bytes */
    int fp_variant_bf16;  /* the gather projector's form for a BF16-stored volume (kernel 4 of
                             stt_tuning_variant_name): 0 loads, 1 tld4 gathers of 16-bit textures
                             (where the device's texture limits admit the volume; else loads) */
    float fp16_us[2];
} stt_tuning;
stt_status stt_autotune(stt_ctx *ctx, stt_tuning *out, void *stream);
stt_status stt_get_tuning(const stt_ctx *ctx, stt_tuning *out);
stt_status stt_set_tuning(stt_ctx *ctx, const stt_tuning *t);
/* Whether the tld4 gather variants (fp_variant 10, 11) bind `vol` on this
 * device: *ok = 1 when the device's limits on pitch-linear 2D textures admit
 * the volume (nx*ny texels a row, nz rows, its base aligned) and its z-fastest
 * copy; 0 when those variants run as their load-based forms for it. */
stt_status stt_fp_texture_ok(stt_ctx *ctx, const float *vol, int *ok);
/* The same for a volume stored as `dtype` (STT_DTYPE_BF16: 16-bit texels,
 * the gather form fp_variant_bf16 1). */
stt_status stt_fp_texture_ok_typed(stt_ctx *ctx, const void *vol, int dtype, int *ok);
/* Description of variant `variant` of kernel `kernel` (0 gather projector,
 * 1 slab-staged projector, 2 voxel backprojection, 3 ray backprojection
 * scatter, 4 gather projector of a BF16-stored volume); NULL when out of
 * range. */
const char *stt_tuning_variant_name(int kernel, int variant);

/* ---- forward projector (TypicalRayProducer.core.h:123-268) ---------------
 * Projects views [view0, view0+nviews) of `vol`.
 *   proj   : nviews*W*H line integrals (sum of f*sd, entry sample counted twice)
 *   raylen : optional W*H*nviews ray lengths (tfar - tnear, mm); written only
 *            where the ray hits the volume, as the reference does
 *   weight : optional W*H*nviews sample counts */
stt_status stt_fp(stt_ctx *ctx, const float *vol, float *proj, float *raylen, float *weight,
                  int view0, int nviews, void *stream);

/* Forward projection of a volume stored in FP32 or BF16 (`vol` points to
 * nx*ny*nz elements of `dtype`; BF16 = the upper 16 bits of an FP32, rounded
 * by the caller).  BF16 halves the volume's memory and cache footprint; taps
 * are widened exactly to FP32 and the march and sums are FP32, so the result
 * equals stt_fp of the widened volume.  Against the FP32 volume it carries
 * the BF16 rounding of the voxels (relative 2^-9 each), i.e. about 1e-3
 * relative L2 per projection.  Not in the reference (CImg<float> only). */
typedef enum stt_dtype { STT_DTYPE_F32 = 0, STT_DTYPE_BF16 = 1 } stt_dtype;
stt_status stt_fp_typed(stt_ctx *ctx, const void *vol, int dtype, float *proj, float *raylen, float *weight,
                        int view0, int nviews, void *stream);

/* Forward projection of one view fused with the SART correction
 * (ST_Tomography.cpp:667-676): corr = (b - Ax) / (L + 1), where L is the
 * sticky ray-length state (W*H, updated where the ray hits).  Views whose
 * central ray is more than 25 degrees off both x and z are projected with the
 * volume staged into shared memory by TMA when nx and nz are multiples of 4
 * and vol is 16-byte aligned; the result is the same bits either way. */
stt_status stt_fp_correction(stt_ctx *ctx, const float *vol, const float *b, float *raylen_state,
                             float *corr, int view, void *stream);

/* Exact adjoint of stt_fp: vol_bar += A^T proj_bar over views [view0, view0+nviews).
 * Scatter with float atomics (order-nondeterministic). */
stt_status stt_fp_vjp(stt_ctx *ctx, const float *proj_bar, float *vol_bar, int view0, int nviews,
                      void *stream);

/* ---- backprojectors ------------------------------------------------------
 * Voxel-driven (ST_Tomography.cpp:690-730): vol = clamp(vol + alpha *
 * bicubic(corr at the voxel's projection), 0, gmax); voxels projecting
 * outside [2, W-2) x [2, H-2) are left unchanged.  Deterministic.  From
 * 2^23 voxels on, corr is first copied (on `stream`) into a texture the
 * context owns, which the column walk of the tuned bp_variant gathers from
 * (stt_sart_sweep writes it from the projector directly, at every size);
 * calls of one context that overlap on different streams race on that copy.
 * The result is the same either way. */
stt_status stt_bp_voxel(stt_ctx *ctx, const float *corr, float *vol, double alpha, float gmax,
                        int view, void *stream);
/* stt_bp_voxel on a volume stored as `dtype` (STT_DTYPE_BF16: each voxel is
 * read widened to FP32, updated as in FP32 and stored rounded to nearest
 * even; the correction stays FP32). */
stt_status stt_bp_voxel_typed(stt_ctx *ctx, const float *corr, void *vol, int dtype, double alpha, float gmax,
                              int view, void *stream);

/* Ray-driven (ST_Tomography.cpp:733-764, SingleScalarVolume.core.h:73-84):
 * scatters corr*w and w along every ray into the context's accumulators, then
 * vol = clamp(vol + contrib/weight, 0, gmax) with 0/0 -> 0 and the
 * accumulators reset.  Atomics: result is order-nondeterministic in the last bits. */
stt_status stt_bp_ray(stt_ctx *ctx, const float *corr, float *vol, float gmax, int view,
                      void *stream);
/* stt_bp_ray on a volume stored as `dtype` (FP32 accumulators; BF16: the
 * normalised update is added in FP32 and stored rounded to nearest even). */
stt_status stt_bp_ray_typed(stt_ctx *ctx, const float *corr, void *vol, int dtype, float gmax, int view,
                            void *stream);

/* The backprojection mode of the reference's projector on its own: one
 * march of view `view` scattering contrib[v] += c*w and wsum[v] += w for the
 * 8 trilinear corners of every sample (SingleScalarVolume.core.h:128-143 with
 * VolumeData::SetProjectionMode(1)); contrib and wsum (nx*ny*nz floats each)
 * accumulate, as the producer's accumulators do until Initial()
 * (TypicalRayProducer.cpp:78-96).  Atomic float adds: the summation order,
 * not the terms, differs from the reference's sequential loop. */
stt_status stt_bp_ray_scatter(stt_ctx *ctx, const float *corr, float *contrib, float *wsum, int view,
                              void *stream);

/* The gather ceiling of the forward projector (a measurement; no
 * counterpart in the reference).  Every ray of view `view` takes as many
 * samples as its clip length holds, at the projector's step from its entry
 * point, with the projector's cell, 8-corner gather and trilinear
 * interpolation (packed bit 0: pairs of samples in packed FP32x2
 * instructions; bit 1: packed pairs with the corners as tld4 texture gathers,
 * as fp_variant 10 and 11 fetch them, STT_ERR_UNSUPPORTED where
 * stt_fp_texture_ok says no) and none of the march's control (no block
 * splits, no per-sample bound checks, a plain sum).  out[W*H] receives the
 * sums times the step, count[W*H] (may be NULL) the samples per ray.  Timed
 * against stt_fp, it says how far the projector is from the rate its gathers
 * alone reach.  Volumes below 2^31 voxels. */
stt_status stt_gather_ceiling(stt_ctx *ctx, const float *vol, int view, int packed, float *out, int *count,
                              void *stream);

/* Ray-driven backprojection that allocates no device memory.  No counterpart
 * in the reference: it is stt_bp_ray for callers that cannot let a library
 * call cudaMalloc (a plugin whose host application owns all device memory, a
 * real-time loop that cannot take cudaMalloc's synchronisation).  Its
 * accumulators live in a fixed array compiled into libstt.so,
 * STT_BP_RAY_NOALLOC_MAX_VOXELS float2 entries (16 MiB per GPU that loads the
 * library, held until exit); larger volumes are rejected with
 * STT_ERR_INVALID.  Calls on one device share that array: calls that overlap
 * on the GPU race, so serialise them.  Every call clears the part it uses
 * first.  The first call on a device looks up the array's device address;
 * make it before any stream capture.  Same arguments and result as stt_bp_ray. */
#define STT_BP_RAY_NOALLOC_MAX_VOXELS (1 << 21)
stt_status stt_bp_ray_noalloc(stt_ctx *ctx, const float *corr, float *vol, float gmax, int view,
                              void *stream);

/* ---- SART (ST_Tomography.cpp:616-808) -------------------------------------
 * One SART call for one frame: for i in 0..nperm-1, view = view_offset +
 * perm[i] (perm is HOST): FP + correction, then backprojection (bp_mode 0
 * voxel-based with alpha, 1 ray-based).  proj_stack holds the frame's
 * projections indexed by perm values (W*H each).  raylen_state: W*H sticky
 * ray lengths (zero it once at start; ray-based mode re-zeroes it after every
 * view as TypicalRayProducer::Initial does).  If roi_cut (HOST, 8 ints) is not
 * NULL the ROI mask of ST_Tomography.cpp:303-329 is applied at the end. */
stt_status stt_sart_sweep(stt_ctx *ctx, float *vol, const float *proj_stack, const int *perm,
                          int nperm, int view_offset, double alpha, float gmax, int bp_mode,
                          float *raylen_state, const int *roi_cut, void *stream);
/* stt_sart_sweep with the volume and the projection stack both stored as
 * `dtype`.  STT_DTYPE_BF16: the forward projector gathers from the BF16
 * volume (taps widened exactly to FP32; FP32 march, Kahan sums and
 * correction), every view's backprojection stores its update rounded to
 * nearest even, and every view gathers (no slab staging).  The ray-length
 * state, the corrections and the accumulators stay FP32. */
stt_status stt_sart_sweep_typed(stt_ctx *ctx, void *vol, int dtype, const void *proj_stack, const int *perm,
                                int nperm, int view_offset, double alpha, float gmax, int bp_mode,
                                float *raylen_state, const int *roi_cut, void *stream);

/* Host helper: the seeded view permutation that replaces srand(time(0)) +
 * random_shuffle (ST_Tomography.cpp:635-642): SplitMix64 + Fisher-Yates. */
stt_status stt_permutation(unsigned long long seed, int n, int *perm_out);

/* One SART view (the body of the loop at ST_Tomography.cpp:651-764): forward
 * projection of view `view` fused with the correction against its projection
 * b (W*H), then the backprojection (bp_mode 0 voxel-based with alpha, 1
 * ray-based); stt_sart_sweep with a one-view order, no ROI mask. */
stt_status stt_sart_view(stt_ctx *ctx, float *vol, const float *b, int view, double alpha, float gmax, int bp_mode,
                         float *raylen_state, void *stream);

/* Operator norm of the forward projector by power iteration on A^T A (the
 * exact adjoint stt_fp_vjp), over all views of the geometry, from a seeded
 * positive start vector; dot products and norms in FP64.  norm_A = sqrt of the
 * last Rayleigh quotient (a lower bound that converges to ||A||_2); norm_K =
 * sqrt(norm_A^2 + 12), the bound for K = [A; grad] with the 3D forward-
 * difference gradient (||grad||^2 <= 12); sigma = tau = 0.99 / norm_K satisfy
 * sigma*tau*||K||^2 < 1 for a Chambolle-Pock iteration on K.  rel_change: the
 * last iteration's relative change of the quotient.  Synchronises `stream`.
 * The reference fixes these steps instead (L = 8, ST_Tomography.cpp:98-102). */
typedef struct stt_opnorm {
    double norm_A, norm_K, sigma, tau;
    int iterations;
    double rel_change;
} stt_opnorm;
stt_status stt_opnorm_power_iter(stt_ctx *ctx, int n_iter, unsigned long long seed, stt_opnorm *out,
                                 void *stream);

/* ---- primal-dual steps (ST_Tomography.cpp:492-604) -------------------------
 * Parameters as the reference uses them: sigma = CP_sigma, tau = CP_tau,
 * tv_w = TV_w, tp_w = TP_w, bc_w = BC_w, huber_factor = m_huberfactor,
 * gmax = G_Max; cut = the ROI cut[8] (ST_Tomography.cpp:114). */
typedef struct stt_pd_params {
    float sigma, tau, tv_w, tp_w, bc_w, huber_factor, gmax;
    int cut[8];
} stt_pd_params;

/* Dual step of frame f (:504-534).  bw = warp(flow[f], xbar[f+1], -1).
 * ytv: 3 planar channels.  All arrays nx*ny*nz (dims from the geometry). */
stt_status stt_pd_dual(stt_ctx *ctx, const stt_pd_params *p, const float *xbar_f,
                       const float *xbar_f1, const float *bw, float *ytv, float *ytp, float *ybc,
                       void *stream);
/* Primal step of frame f (:536-578).  first_frame != 0 uses ytp/ybc only;
 * otherwise fw = warp(flow[f-1], ybc[f-1], +1) and ytp_prev = ytp[f-1].
 * Writes xprev = vol (before the update). */
stt_status stt_pd_primal(stt_ctx *ctx, const stt_pd_params *p, int first_frame,
                         const float *ytp_prev, const float *ytp, const float *fw,
                         const float *ybc, const float *ytv, float *vol, float *xprev,
                         void *stream);
/* Over-relaxation (:586-604): xbar = 2*vol - xprev inside the ROI box. */
stt_status stt_pd_extrapolate(stt_ctx *ctx, const int *cut, const float *vol, const float *xprev,
                              float *xbar, void *stream);
/* ROI mask (:303-329): roi = 0/1 per voxel; cut is HOST int[8]. */
stt_status stt_roi_mask(stt_ctx *ctx, const int *cut, float *roi, void *stream);

/* ---- warp (ST_Tomo/warping.h:49-145) ---------------------------------------
 * Semi-Lagrangian warp on the cell-centred grid with aabb = [0, dim]:
 * out(x) = clamped-Catmull-Rom(src, trace(x, -dt)), nc planar channels.
 * vel: 3 planar channels.  dim (HOST) is independent of the geometry. */
stt_status stt_warp(const int *dim, const float *vel, const float *src, int nc, float dt,
                    float *out, void *stream);
/* stt_warp of a source stored as `dtype` (STT_DTYPE_BF16: taps widened
 * exactly to FP32); the flow and the output are FP32. */
stt_status stt_warp_typed(const int *dim, const float *vel, const void *src, int dtype, int nc, float dt,
                          float *out, void *stream);
/* Vector-Jacobian product of stt_warp: src_bar += J_src^T out_bar and
 * vel_bar += J_vel^T out_bar (either may be NULL; both accumulate with atomics). */
stt_status stt_warp_vjp(const int *dim, const float *vel, const float *src, int nc, float dt,
                        const float *out_bar, float *src_bar, float *vel_bar, void *stream);

/* Warp with aabb = [0, box] over a dim grid (warping.h:11-145 with a general
 * bounding box), sampling with CImg's nested Catmull-Rom arithmetic in the
 * reference's operation order: the result equals warping::warp bit for bit.
 * The multiscale flow warps each pyramid level in full-size units this way
 * (optical_flow.h:700).  dim and box are HOST arrays. */
stt_status stt_warp_box(const int *dim, const float *box, const float *vel, const float *src, int nc,
                        float dt, float *out, void *stream);
/* CImg::get_gradient("xyz", 0) (CImg.h:34570-34581): central differences with
 * Neumann boundaries; grad = 3 planes (d/dx, d/dy, d/dz). */
stt_status stt_image_gradient(const int *dim, const float *img, float *grad, void *stream);

/* ---- optical flow (ST_Tomo/optical_flow.h:83-734) --------------------------
 * 3D TV-L1 / Huber optical flow by preconditioned primal-dual iterations with
 * warping, on a pyramid of Deriche-blurred images, as
 * optical_flow::L1Huber_OF_MultiScale3D (:630-734) and L1Huber_OF (:83-623).
 * Fields are planar x-fastest volumes: I1 and I2 one plane each, V 3 planes
 * (flow in voxel units of the full-size grid), Y 10 planes (Y1|Y2|Y3: dual
 * variables of the gradients of the three flow components, Y4: dual of the
 * data term).
 * Stopping rule (optical_flow.h:305-495): the primal-dual residual is formed
 * every 50 iterations and a warp stops once it is not above tol, else after
 * max_iter + 1 iterations.  The residual is summed with atomics (the
 * reference's sum is a racy OpenMP loop), so the iteration a warp stops at can
 * differ from the reference's only when the residual is within rounding of
 * tol; everything else follows the reference's float arithmetic exactly.
 * Outside the ROI the reference reads gradient arrays that it never set; they
 * are 0 here (this reaches only Y4 outside the ROI, not V).
 * The reference's Render uses tol 0.1, lambda 1.2, huber 1, eta 0.65,
 * sigma 0.5, max_iter 3000, norm 4, 3 warps, 3 scales (ST_Tomography.cpp:440-456). */
typedef struct stt_flow_params {
    float tol;      /* residual threshold */
    float lambda;   /* weight of the TV term: radius of the dual ball */
    float huber;    /* Huber epsilon (norm 4) */
    float eta;      /* pyramid factor per level */
    float sigma;    /* Deriche blur of I1 and I2 before the pyramid */
    int max_iter;   /* a warp runs at most max_iter + 1 iterations */
    int norm;       /* 4: Huber-regularised TV; anything else: TV */
    int n_warps;    /* re-linearisations per level */
    int scales;     /* pyramid levels */
    int cut[6];     /* ROI at full size: cut from x-, x+, y-, y+, z-, z+ faces */
} stt_flow_params;

typedef struct stt_flow stt_flow;

/* Allocates every buffer of a multiscale solve for volumes of size dims
 * (HOST int[3]) on `device`: about 200 bytes per voxel. */
stt_status stt_flow_create(int device, const int *dims, const stt_flow_params *p, stt_flow **out);
const char *stt_flow_last_error(const stt_flow *f);
stt_status stt_flow_destroy(stt_flow *f);
/* L1Huber_OF_MultiScale3D: V holds the initial flow and receives the
 * finest-level flow; Y0 (10 planes, NULL = zeros) is the initial dual.
 * This and stt_flow_level enqueue their work on `stream`; to stop enqueuing a
 * warp's iterations once its residual check has stopped it, they keep at most
 * 200 of a warp's iterations queued ahead of the device and wait for it
 * (an event of `stream`) past that.  While `stream` is being captured every
 * iteration is enqueued and nothing waits. */
stt_status stt_flow_multiscale(stt_flow *f, const float *I1, const float *I2, float *V, const float *Y0,
                               void *stream);
/* L1Huber_OF on one level of size dim (HOST, each extent >= 3 and at most the
 * created size), aabb = [0, box] (HOST float[3]), roi (HOST int[6], same order
 * as cut).  V and Y are updated in place; Y only inside the ROI. */
stt_status stt_flow_level(stt_flow *f, const int *dim, const float *box, const int *roi, const float *I1,
                          const float *I2, float *V, float *Y, void *stream);
/* Iterations run by each (level, warp) of the last solve, coarse level
 * first, and the last residual of each (HOST arrays of *n_entries, either may
 * be NULL).  Synchronises the device. */
stt_status stt_flow_stats(stt_flow *f, int *n_entries, int *iters, float *err);
/* CImg::blur(sigma) (Deriche, order 0, Neumann; CImg.h:32917-33050) in place
 * on nc planes of size dim, each at most the created volume. */
stt_status stt_flow_blur(stt_flow *f, const int *dim, int nc, float sigma, float *img, void *stream);
/* CImg::get_resize(odim, nc, 5) (CImg.h:28432-28560): moving average along
 * shrinking axes, Catmull-Rom along growing ones, x then y then z.  Every
 * intermediate plane is at most the created volume; in != out. */
stt_status stt_flow_resize(stt_flow *f, const int *dim, int nc, const float *in, const int *odim, float *out,
                           void *stream);

/* ---- space-time primal-dual solver (ST_Tomography::Render, ST_Tomography.cpp:492-607) ----
 * One call to stt_solver_iterate runs one primal-dual iteration over all
 * frames: for every frame the backward warp + dual step, the forward warp +
 * primal step, SART(f) over its views, the ROI mask and the over-relaxation.
 * Frame f uses views [f*V, (f+1)*V) of the context's geometry and its V
 * projections at proj + f*V*W*H.  The view order of each SART call is a
 * seeded permutation (stt_solver_frame_order gives it on the host).
 * State arrays are caller-owned device memory, nx*ny*nz floats per volume:
 *   vol   (F+1) volumes, vol[F] the duplicated last frame (VolumeData.cpp:124-126)
 *   xbar  (F+1)  over-relaxed volumes X_bar (initialise to vol)
 *   xprev  F     previous primal iterate X_prev
 *   ytv   F*3    TV dual (planar channels), ytp F, ybc F
 *   flow  F*3    flow[f]: motion from frame f to f+1 (planar channels)
 *   proj  F*V*H*W measured projections */
typedef enum stt_solve_mode {
    STT_SOLVE_PLAIN = 0,      /* per-view launches from a host loop, sync per view */
    STT_SOLVE_STREAMS = 1,    /* batched: fused launches, one stream per frame */
    STT_SOLVE_GRAPH = 2,      /* batched, captured once into a CUDA graph and replayed */
    /* The whole iteration in ONE persistent cooperative launch: every
     * frame's view order, backward warp + dual step, then (after a barrier
     * of the grid) its forward warp + primal step, SART call (all views:
     * transpose, projection + correction, backprojection), ROI mask and
     * over-relaxation, the frames side by side on their share of the
     * resident blocks; the launch is captured into a CUDA graph and
     * replayed (enqueued directly where the runtime cannot capture a
     * cooperative launch: stt_solver_persistent_info).  A sharded solve
     * (halo) runs its phase 0 as launches and its phase 1's SART calls as
     * one launch.  Voxel-based backprojection only (bp_mode 0).  The same
     * bits as the other batched modes; inside one launch the arrays it
     * writes are gathered with plain loads (the texture and read-only caches
     * are not coherent with the launch's own writes), so on volumes that the
     * texture gathers serve well it is slower than STT_SOLVE_GRAPH. */
    STT_SOLVE_PERSISTENT = 3
} stt_solve_mode;

typedef struct stt_solve_cfg {
    int n_frames, views_per_frame;
    int bp_mode;               /* 0 voxel-based (alpha), 1 ray-based */
    double alpha;              /* SART step of the voxel-based BP (-a) */
    stt_pd_params pd;          /* sigma, tau, weights, gmax, PD region cut */
    int roi_cut[8];            /* cut of the ROI mask applied after each SART call */
    unsigned long long seed;   /* view-order seed */
    int mode;                  /* stt_solve_mode */
    /* Frame sharding across GPUs: when `halo` is set, local frame 0 is not the
     * sequence's first frame; its primal step uses ytp_halo/ybc_halo/flow_halo
     * (the previous shard's last frame) and xbar[F] holds the next shard's
     * X_bar[0].  The caller exchanges them between the two phases. */
    int halo;
    /* Place of these frames in the whole sequence (frame sharding): local
     * frame f is frame frame_offset + f of total_frames (0 = n_frames).  The
     * view order of each frame is drawn from its place in the sequence, so
     * shards draw the orders the unsharded solve would. */
    int frame_offset;
    int total_frames;
    /* Non-zero: stt_solver_create runs stt_autotune on the context first
     * (unless it is tuned already). */
    int autotune;
    /* Storage of the primal volumes and the sinogram (stt_dtype).
     * STT_DTYPE_BF16: state.vol, xbar, xprev and proj point to arrays of BF16
     * values (the upper 16 bits of an FP32; pass them cast to float*), half
     * the memory of FP32.  Every kernel widens what it reads exactly to FP32,
     * computes in FP32 as the FP32 solve does, and rounds what it stores to
     * nearest even; the duals (ytv, ytp, ybc), the flow and all scratch stay
     * FP32, and the forward projector gathers for every view (no slab
     * staging).  A result then carries the BF16 rounding of every stored
     * update. */
    int storage;
} stt_solve_cfg;

typedef struct stt_pd_state {
    float *vol, *xbar, *xprev, *ytv, *ytp, *ybc;
    const float *flow, *proj;
    const float *ytp_halo, *ybc_halo, *flow_halo;  /* only read when cfg.halo is set */
} stt_pd_state;

typedef struct stt_solver stt_solver;

stt_status stt_solver_create(stt_ctx *ctx, const stt_solve_cfg *cfg, const stt_pd_state *state,
                             stt_solver **out);
/* Enqueue n_iters iterations on `stream` (the plain mode synchronises it). */
stt_status stt_solver_iterate(stt_solver *s, int n_iters, void *stream);
/* One phase of one iteration: phase 0 = view order + every frame's backward
 * warp and dual step; phase 1 = every frame's forward warp, primal step,
 * SART, ROI mask and over-relaxation.  Phase 0 then phase 1 equals one
 * stt_solver_iterate step; sharded solves exchange halos in between. */
stt_status stt_solver_iterate_phase(stt_solver *s, int phase, void *stream);
/* Makes the next iteration iteration number `iter` (its view orders are those
 * of that iteration); 0 restarts the sequence of orders.  Enqueued on
 * `stream` (iterations enqueued after it on that stream see it). */
stt_status stt_solver_set_iteration(stt_solver *s, unsigned long long iter, void *stream);
/* Kernel launches per iteration and iterations run so far. */
stt_status stt_solver_stats(const stt_solver *s, long long *launches_per_iter,
                            unsigned long long *iterations);
/* STT_SOLVE_PERSISTENT: blocks of the persistent launch, and whether the
 * iteration is a replayed graph (1) or enqueued directly (0; the runtime
 * refused to capture the cooperative launch).  Zeros in the other modes. */
stt_status stt_solver_persistent_info(const stt_solver *s, int *blocks, int *graph);
const char *stt_solver_last_error(const stt_solver *s);
/* See stt_poll_status. */
stt_status stt_solver_poll_status(stt_solver *s, void *stream);
stt_status stt_solver_destroy(stt_solver *s);
/* Host copy of the view order frame `frame` of a sequence of n_frames uses in
 * iteration `iter` (HOST perm_out); for a shard, frame and n_frames are its
 * frame_offset + local frame and total_frames. */
stt_status stt_solver_frame_order(unsigned long long seed, unsigned long long iter, int n_frames,
                                  int frame, int views, int *perm_out);

/* ---- batched independent instances (config 4 of the survey's scope) ------
 * Many single-frame reconstructions of uneven size solved together.  Each
 * instance is a one-frame primal-dual TV + SART solve -- the iteration of
 * ST_Tomography::Render with one frame (ST_Tomography.cpp:492-607; its
 * temporal and brightness-constancy weights are forced to 0) -- on its own
 * context (geometry, views [0, n_views)) and stream.  stt_batch_iterate runs
 * one iteration of every instance concurrently (STT_SOLVE_STREAMS) or as one
 * captured CUDA graph (STT_SOLVE_GRAPH); after it each instance's `vol` holds
 * its current volume.  The batch owns the instances' solver state (13 volumes
 * each); `vol` and `proj` stay the caller's and must outlive the batch. */
typedef struct stt_instance {
    stt_ctx *ctx;
    float *vol;           /* nx*ny*nz: start volume in, current volume out */
    const float *proj;    /* n_views projections (view-major, W*H each) */
    int n_views;
    int bp_mode;          /* 0 voxel-based (alpha), 1 ray-based */
    double alpha;
    stt_pd_params pd;     /* sigma, tau, tv_w, huber_factor, gmax, cut (tp_w, bc_w ignored) */
    int roi_cut[8];
    unsigned long long seed;
    int autotune;         /* non-zero: tune the instance's context at stt_batch_create (stt_autotune) */
    int storage;          /* stt_dtype of vol and proj (and of the instance's primal state): see
                             stt_solve_cfg.storage */
} stt_instance;

/* When any instance asks for autotuning, stt_batch_create also chooses, for
 * the batch as a whole, between the instances' tuned split of the views
 * between the two forward projectors and every view gathering: it times one
 * batched iteration each way (results not written to the instances' vol),
 * keeps the faster (when it is the gather, each instance's context keeps a
 * staged mask of 0 for its storage: stt_get_tuning shows it), and starts the
 * solve from the untouched start volumes with fresh solvers.  Instances tuned alone on an idle GPU favour the
 * slab-staged projector, whose shared memory limits how many of the other
 * instances' blocks run beside it.  stt_batch_staging reports the choice: timed
 * (0 when no instance asked for tuning or no view was staged), all_gather, and
 * the two iteration times in ms (any pointer may be NULL). */
typedef struct stt_batch stt_batch;
stt_status stt_batch_create(const stt_instance *instances, int n, int mode, stt_batch **out);
stt_status stt_batch_staging(const stt_batch *b, int *timed, int *all_gather, float *ms_split, float *ms_gather);
stt_status stt_batch_iterate(stt_batch *b, int n_iters, void *stream);
const char *stt_batch_last_error(const stt_batch *b);
/* See stt_poll_status: polls every instance's solver. */
stt_status stt_batch_poll_status(stt_batch *b, void *stream);
stt_status stt_batch_destroy(stt_batch *b);

/* Volume size (nx, ny, nz) of a context's geometry (HOST int[3]). */
stt_status stt_ctx_dims(const stt_ctx *ctx, int *dims);

#ifdef __cplusplus
}
#endif
#endif /* STT_H */
