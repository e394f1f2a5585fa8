// optical_flow.h -- drop-in for S/ST_Tomo/optical_flow.h (gmzang/
// SpaceTimeTomography): L1Huber_OF (:84-85) and L1Huber_OF_MultiScale3D
// (:631-633) with the reference's signatures, run on libstt's sm_100a kernels
// through the host staging calls of stt_host.h.  The level solver's region of
// interest is the global ROI[6] as in the reference (:24).  `image` is
// CImg<float> or stt::Image.  Results equal the reference's bit for bit; the
// one exception is when a warp's residual check lands within rounding of
// tol (the reference sums that residual in a racy OpenMP loop).
#ifndef OPTICAL_FLOW_H
#define OPTICAL_FLOW_H

#include <stdexcept>
#include <vector>

#include "stt_host.h"

namespace optical_flow {

inline int ROI[6] = {1, 1, 1, 1, 1, 1};

namespace detail {
template <typename image>
std::vector<float> pack_duals(const image &Y1, const image &Y2, const image &Y3, const image &Y4, size_t n) {
    std::vector<float> y(10 * n);
    const image *ys[4] = {&Y1, &Y2, &Y3, &Y4};
    size_t at = 0;
    for (int q = 0; q < 4; ++q) {
        const size_t m = (q < 3 ? 3 : 1) * n;
        const float *s = ys[q]->data();
        for (size_t k = 0; k < m; ++k) y[at + k] = s[k];
        at += m;
    }
    return y;
}
}  // namespace detail

template <typename real, typename image>
void L1Huber_OF(int *dim, const image &image1, const image &image2, image &_inputV, image &_inputY1,
                image &_inputY2, image &_inputY3, image &_inputY4, float _tol, float _lambda, int _maxIterations,
                int _norm, int _numberOfWarps, real *_aabb, float huber) {
    const size_t n = (size_t)dim[0] * dim[1] * dim[2];
    std::vector<float> y = detail::pack_duals(_inputY1, _inputY2, _inputY3, _inputY4, n);
    const float box[6] = {(float)_aabb[0], (float)_aabb[1], (float)_aabb[2],
                          (float)_aabb[3], (float)_aabb[4], (float)_aabb[5]};
    if (stt_host_flow_level(dim, box, ROI, image1.data(), image2.data(), _inputV.data(), y.data(), _tol, _lambda,
                            _maxIterations, _norm, _numberOfWarps, huber, nullptr) != 0)
        throw std::runtime_error(stt_host_last_error());
    image *ys[4] = {&_inputY1, &_inputY2, &_inputY3, &_inputY4};
    size_t at = 0;
    for (int q = 0; q < 4; ++q) {
        const size_t m = (q < 3 ? 3 : 1) * n;
        float *d = ys[q]->data();
        for (size_t k = 0; k < m; ++k) d[k] = y[at + k];
        at += m;
    }
}

template <typename real, typename image>
image L1Huber_OF_MultiScale3D(int *dim, const image &image1, const image &image2, image &_inputV, image &_inputY1,
                              image &_inputY2, image &_inputY3, image &_inputY4, real _tol, real _lambda,
                              int _maxIterations, int _norm, int _numberOfWarps, real eta, real sigma, int scales,
                              real _huber, int *cut) {
    const size_t n = (size_t)dim[0] * dim[1] * dim[2];
    std::vector<float> y = detail::pack_duals(_inputY1, _inputY2, _inputY3, _inputY4, n);
    image out(dim[0], dim[1], dim[2], 3, 0.0f);
    if (stt_host_flow_multiscale(dim, image1.data(), image2.data(), _inputV.data(), y.data(), out.data(),
                                 (float)_tol, (float)_lambda, _maxIterations, _norm, _numberOfWarps, (float)eta,
                                 (float)sigma, scales, (float)_huber, cut) != 0)
        throw std::runtime_error(stt_host_last_error());
    return out;
}

}  // namespace optical_flow

#endif
