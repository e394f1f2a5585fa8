// stt_kernels.h -- host-side launch wrappers of the kernels in k_*.cu.
#pragma once

#include <cuda_runtime.h>

namespace stt {

struct ViewRec;
struct GeomDev;
struct ViewSel;

struct PdParams {
    float sigma, tau, tv_w, tp_w, bc_w, hf, gmax;
    int cut[8];
};

int grid_stride_blocks(long long n, int threads);

cudaError_t launch_fp(const GeomDev &g, const ViewRec *views, const float *vol, const float *vol_t, int view0,
                      int nviews, float *proj, float *raylen, float *weight, cudaStream_t s);
cudaError_t launch_fp_corr(const GeomDev &g, const ViewRec *views, const float *vol, const float *vol_t,
                           const ViewSel &sel, const float *b_stack, float *raylen_state, float *corr,
                           cudaStream_t s);
cudaError_t launch_transpose(const GeomDev &g, const float *in, float *out, cudaStream_t s);
cudaError_t launch_transpose_for_view(const GeomDev &g, const ViewRec *views, const ViewSel &sel, const float *in,
                                      float *out, cudaStream_t s);
cudaError_t launch_correction(long long n, const float *b, const float *ax, const float *raylen,
                              float *corr, cudaStream_t s);
cudaError_t launch_bp_ray(const GeomDev &g, const ViewRec *views, const ViewSel &sel, const float *corr,
                          float2 *acc, float *vol, float gmax, cudaStream_t s);
cudaError_t launch_fp_adjoint(const GeomDev &g, const ViewRec *views, int view0, int nviews,
                              const float *proj_bar, float *vol_bar, cudaStream_t s);
cudaError_t launch_fill_zero(float *p, long long n, cudaStream_t s);

cudaError_t launch_bp_voxel(const GeomDev &g, const ViewRec *views, const ViewSel &sel, const float *corr,
                            float *vol, float alpha, float gmax, cudaStream_t s);
cudaError_t launch_make_perm(unsigned long long seed, unsigned long long *counter, int frames,
                             int views, int *perm, cudaStream_t s);
cudaError_t launch_pd_dual(const int *dims, const PdParams &p, const float *xf, const float *xf1,
                           const float *bw, float *ytv, float *ytp, float *ybc, cudaStream_t s);
cudaError_t launch_pd_primal(const int *dims, const PdParams &p, int first, const float *ytp_prev,
                             const float *ytp, const float *fw, const float *ybc, const float *ytv,
                             float *vol, float *xprev, cudaStream_t s);
cudaError_t launch_pd_extrapolate(const int *dims, const int *cut, const float *vol,
                                  const float *xprev, float *xbar, cudaStream_t s);
cudaError_t launch_roi_apply(const int *dims, const int *roi_cut, const int *pd_cut, float *vol,
                             const float *xprev, float *xbar, cudaStream_t s);
cudaError_t launch_roi_mask(const int *dims, const int *cut, float *roi, cudaStream_t s);

cudaError_t launch_warp(const int *dim, const float *vel, const float *src, int nc, float dt,
                        float *out, cudaStream_t s);
cudaError_t launch_warp_vjp(const int *dim, const float *vel, const float *src, int nc, float dt,
                            const float *out_bar, float *src_bar, float *vel_bar, cudaStream_t s);

}  // namespace stt
