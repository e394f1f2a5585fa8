// stt_ctx.h -- the context behind the opaque stt_ctx handle of include/stt.h
// (private to libstt.so: stt_capi.cu owns it; the solver reads its launch
// choices; the autotuner stt_tune.cu sets them and rewrites the view table).
#pragma once

#include <string>
#include <vector>

#include "stt.h"
#include "stt_internal.cuh"
#include "stt_kernels.h"

struct stt_ctx {
    int device = 0;
    std::string err;
    bool has_geom = false;
    stt::GeomDev g{};
    double sp[3] = {1, 1, 1};
    stt_geometry geom{};              // the last geometry set (its angles pointer is not kept)
    std::vector<stt::ViewRec> views_h;
    std::vector<float> off_axis_deg;  // per view: angle of the central ray off the nearest of x and z
    stt::ViewRec *views_d = nullptr;
    size_t views_cap = 0;
    float2 *acc = nullptr;  // ray-BP accumulators (contrib, weight) per voxel
    size_t acc_n = 0;
    float *corr = nullptr;  // W*H correction image used by stt_sart_sweep
    size_t corr_n = 0;
    // The correction as a texture for the column backprojection of
    // stt_sart_sweep and stt_bp_voxel (made on first use at the geometry's
    // W x H; tex 0 where it could not be made: the per-voxel load form runs).
    stt::CorrTex corr_tex{};
    float *volt = nullptr;  // z-fastest copy of the volume for views gathering along x
    size_t volt_n = 0;
    unsigned short *volt16 = nullptr;  // the same for a BF16-stored volume
    size_t volt16_n = 0;
    float *pw = nullptr;  // power iteration: x, A^T A x, and a chunk of projections
    size_t pw_n = 0;
    double *pwd = nullptr;  // power iteration: FP64 sums
    size_t pwd_n = 0;
    int *status = nullptr;  // raised by a bounded device-side wait that gave up (stt_poll_status)
    size_t status_n = 0;
    // Launch choices (stt_autotune / stt_set_tuning).  staged_bins: bit b set =
    // views 5b..5b+5 degrees off the nearest axis use the slab-staged projector
    // (0x1E0, 25-45 degrees, is the rule build_view applies by default).
    stt::Tuning tuning{};
    unsigned staged_bins = 0x1E0u;
    unsigned staged_bins16 = 0x1E0u;  // the same for a BF16-stored volume (ViewRec::staged16)
    bool tuned = false;
    stt_tuning report{};
    // Texture objects of the tld4 gather variants for the arrays the entry
    // points were given, keyed by the arrays and the dimensions (at most
    // kFpTexCache; past that the load-based variant of the same shape runs).
    // Kept until stt_destroy, so a stream capture of an entry point that
    // bound one stays valid.
    struct FpTexEntry {
        const void *vol, *volt;
        int nx, ny, nz, esize;
        stt::FpTex tex;
    };
    static constexpr int kFpTexCache = 32;
    std::vector<FpTexEntry> fp_tex;
};

namespace stt {
// Off-axis class of a view: 0..8, 5-degree classes (40-45 degrees in 8).
inline int off_axis_bin(float deg) {
    int b = (int)(deg / 5.0f);
    return b < 0 ? 0 : (b > 8 ? 8 : b);
}
// Applies ctx->staged_bins and staged_bins16 to every view (host and device tables).
stt_status apply_staged_bins(stt_ctx *ctx);
// The textures of the tuned gather variant for (vol, vol_t) when it is a tld4
// variant (created on first use, cached in the context); nullptr otherwise.
const FpTex *ctx_fp_tex(stt_ctx *ctx, const float *vol, const float *vol_t);
// The same whatever the tuned variant (nullptr only when the cache is full).
const FpTex *ctx_fp_tex_any(stt_ctx *ctx, const float *vol, const float *vol_t);
// The BF16 volume's textures when the tuned BF16 gather form is the tld4 one.
const FpTex *ctx_fp_tex(stt_ctx *ctx, const unsigned short *vol, const unsigned short *vol_t);
}  // namespace stt
