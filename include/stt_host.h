/* include/stt_host.h -- host-pointer entry points of libstt_facade.so, the
 * layer between the reference's C++ interfaces and the device-pointer C ABI
 * of include/stt.h.  Every array here is HOST memory; each call stages its
 * inputs to the device, runs the libstt kernels on device 0 (or the device set
 * with stt_host_set_device) and copies the results back, synchronously.
 * Return value: 0 on success, else an stt_status code; stt_host_last_error()
 * gives the message (thread-local).
 *
 * Reference interfaces served (paths relative to gmzang/SpaceTimeTomography,
 * S/ = SpaceTimeTomography/):
 *   stt_host_warp            warping::warp                         S/ST_Tomo/warping.h:116-145
 *   stt_host_flow_level      optical_flow::L1Huber_OF              S/ST_Tomo/optical_flow.h:83-623
 *   stt_host_flow_multiscale optical_flow::L1Huber_OF_MultiScale3D S/ST_Tomo/optical_flow.h:630-734
 *   stt_tiff_read/_write     CImg(const char*) / CImg::save_tiff (float stacks, one page per z slice),
 *                            used for the projection stack and volumes (S/ST_Tomo/ST_Tomography.cpp:355, 805)
 *   stt_analyze_write/_read  CImg::save_analyze for the flow field (S/ST_Tomo/ST_Tomography.cpp:467)
 */
#ifndef STT_HOST_H
#define STT_HOST_H

#include "stt.h"

#ifdef __cplusplus
extern "C" {
#endif

const char *stt_host_last_error(void);
int stt_host_set_device(int device);

/* warping::warp(dim, aabb, vel, src, dt): aabb = {x0, x1, y0, y1, z0, z1}
 * with x0 = y0 = z0 = 0 (the only form the reference uses); vel 3 planes,
 * src/out nc planes of dim[0]*dim[1]*dim[2] floats. */
int stt_host_warp(const int *dim, const float *aabb, const float *vel, const float *src, int nc, float dt,
                  float *out);

/* L1Huber_OF on one level: V (3 planes) and Y (10 planes: Y1|Y2|Y3|Y4) in/out;
 * aabb as above; roi = {x0, x1, y0, y1, z0, z1}; iters (optional, n_warps
 * entries) receives the iterations run per warp. */
int stt_host_flow_level(const int *dim, const float *aabb, const int *roi, const float *I1, const float *I2,
                        float *V, float *Y, float tol, float lambda, int max_iter, int norm, int n_warps,
                        float huber, int *iters);

/* L1Huber_OF_MultiScale3D: Vin (3 planes, initial flow), Y0 (10 planes or
 * NULL), Vout (3 planes) receives the finest-level flow; cut: at least 6 ints. */
int stt_host_flow_multiscale(const int *dim, const float *I1, const float *I2, const float *Vin,
                             const float *Y0, float *Vout, float tol, float lambda, int max_iter, int norm,
                             int n_warps, float eta, float sigma, int scales, float huber, const int *cut);

/* Uncompressed baseline TIFF, one page per z slice.  stt_tiff_read accepts
 * 8/16/32-bit unsigned or signed integer and 32/64-bit float samples, one
 * sample per pixel, strips or tiles absent (strips only), either byte order;
 * it returns a malloc'ed x-fastest float array (free with stt_host_free).
 * stt_tiff_write writes 32-bit IEEE float pages, little endian. */
int stt_tiff_read(const char *path, int *w, int *h, int *d, float **data);
int stt_tiff_write(const char *path, int w, int h, int d, const float *data);

/* Analyze 7.5 pair (path ends in .hdr; the data goes to the matching .img):
 * dim = {4, w, h, d, c}, 32-bit float, little endian, planar channels. */
int stt_analyze_write(const char *hdr_path, int w, int h, int d, int c, const float *data);
int stt_analyze_read(const char *hdr_path, int *w, int *h, int *d, int *c, float **data);

void stt_host_free(void *p);

/* ---- the space-time primal-dual solve on host buffers ---------------------
 * Replaces ST_Tomography::Render's image phase (S/ST_Tomo/ST_Tomography.cpp:
 * 475-607: per frame the backward warp and dual step, the forward warp and
 * primal step, SART(f), the ROI mask and the over-relaxation), for callers
 * whose volumes, flows and projections live in host memory, as they do in the
 * reference (CImg lists, VolumeData.h:97-98, ST_Tomography.cpp:355).
 *
 * stt_host_solver_create: geometry and solve configuration as for
 * stt_set_geometry / stt_solver_create (cfg->halo must be 0, cfg->storage
 * STT_DTYPE_F32; use STT_SOLVE_GRAPH); `slots` (1..8) complete copies of the device state are
 * allocated on the current stt_host_set_device device, so that with 2 slots a
 * step's upload and the previous step's read-back overlap a step's compute.
 * With cfg->autotune the launch choices are timed on this geometry once, when
 * the first slot's solver is created (the others share the context). 
 *
 * stt_host_solver_submit: one step on the next slot (waiting first for that
 * slot's previous step if it is still pending): uploads vol (F volumes, x
 * fastest; the last is duplicated on the device as VolumeData.cpp:124-126
 * does), flow (F x 3 planar volumes) and proj (F x V images, view-major),
 * sets X_bar = vol and zero duals, runs n_iters iterations from the first
 * view order, and copies the F volumes back into vol_out (HOST, may be NULL).
 * It only enqueues: the host buffers must stay valid and vol_out unread until
 * stt_host_solver_wait has completed the step.  Page-locked buffers
 * (cudaHostAlloc / cudaHostRegister) make the copies asynchronous.
 *
 * stt_host_solver_wait: completes the oldest pending step (its vol_out is
 * filled); returns STT_ERR_TIMEOUT if a bounded device-side wait of that step
 * gave up (see stt_poll_status).  stt_host_solver_pending: steps submitted and
 * not yet waited for. */
typedef struct stt_host_solver stt_host_solver;
int stt_host_solver_create(const stt_geometry *g, const stt_solve_cfg *cfg, int slots, stt_host_solver **out);
int stt_host_solver_submit(stt_host_solver *h, const float *vol, const float *flow, const float *proj, int n_iters,
                           float *vol_out);
int stt_host_solver_wait(stt_host_solver *h);
int stt_host_solver_pending(const stt_host_solver *h);
int stt_host_solver_destroy(stt_host_solver *h);

#ifdef __cplusplus
}
#endif
#endif /* STT_HOST_H */
