// facade_dropin_check.cpp -- test driver for the drop-in headers of
// include/reference/: written the way reference code calls the reference's
// interfaces (warping::warp, optical_flow::L1Huber_OF[_MultiScale3D],
// TypicalRayProducer + SingleScalarVolumePrepare + RayCasterPrepare +
// GenerateImage_GetCorrections), on stt::Image.  tests/test_gpu_facade.py
// compiles it, feeds it raw float32 files and compares its outputs with the
// oracle.  Test infrastructure only.
//
//   facade_dropin_check warp      DIR nx ny nz nc dt bx by bz
//   facade_dropin_check flowlevel DIR nx ny nz bx by bz r0..r5 tol lambda iters norm warps huber
//   facade_dropin_check flowms    DIR nx ny nz c0..c5 tol lambda iters norm warps eta sigma scales huber
//   facade_dropin_check project   DIR nx ny nz sx sy sz W H
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <stdexcept>
#include <string>
#include <vector>

#include "RayCaster.core.h"
#include "SingleScalarVolume.core.h"
#include "TypicalRayProducer.core.h"
#include "optical_flow.h"
#include "warping.h"

namespace {

std::string g_dir;

void load(const char *name, float *dst, size_t n) {
    FILE *f = std::fopen((g_dir + "/" + name).c_str(), "rb");
    if (!f || std::fread(dst, sizeof(float), n, f) != n) throw std::runtime_error(std::string("cannot read ") + name);
    std::fclose(f);
}

void save(const char *name, const float *src, size_t n) {
    FILE *f = std::fopen((g_dir + "/" + name).c_str(), "wb");
    if (!f || std::fwrite(src, sizeof(float), n, f) != n) throw std::runtime_error(std::string("cannot write ") + name);
    std::fclose(f);
}

int run(int argc, char **argv) {
    const std::string mode = argv[1];
    g_dir = argv[2];
    auto I = [&](int k) { return std::atoi(argv[k]); };
    auto F = [&](int k) { return (float)std::atof(argv[k]); };
    int dim[3] = {I(3), I(4), I(5)};
    const size_t n = (size_t)dim[0] * dim[1] * dim[2];
    if (mode == "warp") {
        const int nc = I(6);
        stt::Image vel(dim[0], dim[1], dim[2], 3), src(dim[0], dim[1], dim[2], nc);
        load("vel.raw", vel.data(), vel.size());
        load("src.raw", src.data(), src.size());
        const float aabb[6] = {0.0f, F(8), 0.0f, F(9), 0.0f, F(10)};
        stt::Image out = warping::warp(dim, aabb, vel, src, F(7));
        save("out.raw", out.data(), out.size());
    } else if (mode == "flowlevel") {
        stt::Image I1(dim[0], dim[1], dim[2]), I2(dim[0], dim[1], dim[2]), V(dim[0], dim[1], dim[2], 3);
        stt::Image Y1(dim[0], dim[1], dim[2], 3), Y2(dim[0], dim[1], dim[2], 3), Y3(dim[0], dim[1], dim[2], 3),
            Y4(dim[0], dim[1], dim[2], 1);
        load("I1.raw", I1.data(), n);
        load("I2.raw", I2.data(), n);
        load("V.raw", V.data(), 3 * n);
        std::vector<float> y(10 * n);
        load("Y.raw", y.data(), 10 * n);
        std::memcpy(Y1.data(), y.data(), 12 * n);
        std::memcpy(Y2.data(), y.data() + 3 * n, 12 * n);
        std::memcpy(Y3.data(), y.data() + 6 * n, 12 * n);
        std::memcpy(Y4.data(), y.data() + 9 * n, 4 * n);
        float aabb[6] = {0.0f, F(6), 0.0f, F(7), 0.0f, F(8)};
        for (int q = 0; q < 6; ++q) optical_flow::ROI[q] = I(9 + q);
        optical_flow::L1Huber_OF<float>(dim, I1, I2, V, Y1, Y2, Y3, Y4, F(15), F(16), I(17), I(18), I(19), aabb,
                                        F(20));
        std::memcpy(y.data(), Y1.data(), 12 * n);
        std::memcpy(y.data() + 3 * n, Y2.data(), 12 * n);
        std::memcpy(y.data() + 6 * n, Y3.data(), 12 * n);
        std::memcpy(y.data() + 9 * n, Y4.data(), 4 * n);
        save("V_out.raw", V.data(), 3 * n);
        save("Y_out.raw", y.data(), 10 * n);
    } else if (mode == "flowms") {
        stt::Image I1(dim[0], dim[1], dim[2]), I2(dim[0], dim[1], dim[2]), V(dim[0], dim[1], dim[2], 3);
        stt::Image Y1(dim[0], dim[1], dim[2], 3), Y2(dim[0], dim[1], dim[2], 3), Y3(dim[0], dim[1], dim[2], 3),
            Y4(dim[0], dim[1], dim[2], 1);
        load("I1.raw", I1.data(), n);
        load("I2.raw", I2.data(), n);
        load("V.raw", V.data(), 3 * n);
        int cut[8] = {I(6), I(7), I(8), I(9), I(10), I(11), 0, 0};
        stt::Image out = optical_flow::L1Huber_OF_MultiScale3D<float>(dim, I1, I2, V, Y1, Y2, Y3, Y4, F(12), F(13),
                                                                      I(14), I(15), I(16), F(17), F(18), I(19), F(20),
                                                                      cut);
        save("V_out.raw", out.data(), out.size());
    } else if (mode == "project") {
        const float sp[3] = {F(6), F(7), F(8)};
        const int W = I(9), H = I(10);
        float view[16], proj[16];
        load("view.raw", view, 16);
        load("proj.raw", proj, 16);
        VolumeData data(dim[0], dim[1], dim[2], sp[0], sp[1], sp[2], nullptr);
        load("vol.raw", data.m_Volumelist[0].data(), n);
        TypicalRayProducer producer(dim[0], dim[1], dim[2], W, H, 1.0, "Raybased");
        RayCaster caster;
        producer.SetVolSize(dim, sp);
        producer.SetViewMatrix(view);
        producer.SetProjectionMatrix(proj);
        producer.UpdateMatrixAndBounds();
        data.SetProjectionMode(0);
        if (!SingleScalarVolumePrepare(&data, &producer, 0) || !RayCasterPrepare(&caster, dim))
            throw std::runtime_error("prepare failed");
        GenerateImage_GetCorrections(&producer);
        save("img.raw", producer.GetImageData(), (size_t)W * H);
        save("rl.raw", producer.GetImageRaylength(), (size_t)W * H);
        save("wt.raw", producer.GetWeightOfImage(), (size_t)W * H);
        load("corr.raw", producer.GetCorrection(), (size_t)W * H);
        data.SetProjectionMode(1);
        producer.Initial();
        if (!SingleScalarVolumePrepare(&data, &producer, 0)) throw std::runtime_error("prepare failed");
        GenerateImage_GetCorrections(&producer);
        save("contrib.raw", producer.GetContributions(), n);
        save("wsum.raw", producer.GetTotalWeight(), n);
        const float angle = (float)producer.ViewAngle();
        save("angle.raw", &angle, 1);
    } else {
        throw std::runtime_error("unknown mode " + mode);
    }
    return 0;
}

}  // namespace

int main(int argc, char **argv) {
    if (argc < 3) {
        std::fprintf(stderr, "usage: facade_dropin_check MODE DIR ...\n");
        return 1;
    }
    try {
        return run(argc, argv);
    } catch (const std::exception &e) {
        std::fprintf(stderr, "facade_dropin_check: %s\n", e.what());
        return 2;
    }
}
