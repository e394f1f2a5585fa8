// warping.h -- drop-in for S/ST_Tomo/warping.h (gmzang/SpaceTimeTomography):
// the same warping::warp signature (:116-117), computed by libstt's sm_100a
// warp kernel (bit-identical to the reference's float arithmetic) through the
// host staging call of stt_host.h.  `image` is CImg<float> or stt::Image; the
// bounding box must start at the origin, as every reference call has it.
#ifndef WARPING_H
#define WARPING_H

#include <stdexcept>

#include "stt_host.h"

namespace warping {

template <typename real, typename image>
image warp(const int *dim, const real *aabb, const image &vel, const image &src, real dt) {
    const float box[6] = {(float)aabb[0], (float)aabb[1], (float)aabb[2],
                          (float)aabb[3], (float)aabb[4], (float)aabb[5]};
    image out(dim[0], dim[1], dim[2], src.spectrum(), 0.0f);
    if (stt_host_warp(dim, box, vel.data(), src.data(), src.spectrum(), (float)dt, out.data()) != 0)
        throw std::runtime_error(stt_host_last_error());
    return out;
}

}  // namespace warping

#endif
