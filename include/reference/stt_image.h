// stt_image.h -- the host image container of the drop-in headers in this
// directory: a dense float volume with channels, laid out as CImg<float> lays
// its data out (x fastest, then y, z, and channel planes last; data()[x + y*w
// + z*w*h + c*w*h*d]).  It carries just what the reference's hot-path
// interfaces touch (S/ImageFormationModel/CImg.h is not part of this build);
// the templates in warping.h and optical_flow.h accept it or a CImg<float>.
#ifndef STT_REFERENCE_IMAGE_H
#define STT_REFERENCE_IMAGE_H

#include <algorithm>
#include <cstddef>
#include <vector>

namespace stt {

class Image {
public:
    Image() = default;
    Image(int w, int h, int d = 1, int c = 1, float value = 0.0f)
        : w_(w), h_(h), d_(d), c_(c), v_((size_t)w * h * d * c, value) {}
    int width() const { return w_; }
    int height() const { return h_; }
    int depth() const { return d_; }
    int spectrum() const { return c_; }
    size_t size() const { return v_.size(); }
    bool is_empty() const { return v_.empty(); }
    float *data() { return v_.data(); }
    const float *data() const { return v_.data(); }
    float &operator()(int x, int y = 0, int z = 0, int c = 0) { return v_[index(x, y, z, c)]; }
    float operator()(int x, int y = 0, int z = 0, int c = 0) const { return v_[index(x, y, z, c)]; }
    Image &fill(float value) {
        std::fill(v_.begin(), v_.end(), value);
        return *this;
    }
    float max() const { return v_.empty() ? 0.0f : *std::max_element(v_.begin(), v_.end()); }
    float min() const { return v_.empty() ? 0.0f : *std::min_element(v_.begin(), v_.end()); }
    // Slices [z0, z1) along z, as one piece of CImg::get_split('z', n).
    Image get_slices(int z0, int z1) const {
        Image out(w_, h_, z1 - z0, c_);
        const size_t plane = (size_t)w_ * h_;
        for (int c = 0; c < c_; ++c)
            std::copy(v_.begin() + ((size_t)c * d_ + z0) * plane, v_.begin() + ((size_t)c * d_ + z1) * plane,
                      out.v_.begin() + (size_t)c * (z1 - z0) * plane);
        return out;
    }

private:
    size_t index(int x, int y, int z, int c) const {
        return (size_t)x + (size_t)w_ * ((size_t)y + (size_t)h_ * ((size_t)z + (size_t)d_ * c));
    }
    int w_ = 0, h_ = 0, d_ = 0, c_ = 0;
    std::vector<float> v_;
};

}  // namespace stt

#endif
