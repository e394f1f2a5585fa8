// stt_tune.cu -- the project-written autotuner of the launch choices
// (include/stt.h: stt_autotune, stt_get_tuning, stt_set_tuning).
//
// What it picks, for one context's geometry (volume, detector, distances,
// view list):
//   * the gather projector's launch variant (detector tile of a block,
//     samples in flight per ray, corners by loads or by tld4 texture gathers,
//     fp_variant_name);
//   * the slab-staged projector's TMA box (slab_variant_name);
//   * for every 5-degree class of views (the central ray's angle off the
//     nearest of the x and z axes), which of the two projectors runs them;
//   * the voxel backprojection's column length (bp_variant_name).
// Every variant of a kernel gives the same bits, so the choice changes only
// the time.  One representative view per class is timed with CUDA events
// (one warm-up launch, then the fastest of three rounds of three); classes
// are weighted by their number of views.  Choices are cached per device and
// geometry shape.
//
// The loops these launches tile are the reference's row loop of the projector
// (S/ImageFormationModel/TypicalRayProducer.core.h:168) and voxel loop of the
// backprojection (S/ST_Tomo/ST_Tomography.cpp:690).
#include <cmath>
#include <cstdio>
#include <cstring>
#include <map>
#include <mutex>
#include <string>

#include "stt.h"
#include "stt_ctx.h"
#include "stt_internal.cuh"
#include "stt_kernels.h"

namespace {

std::mutex g_cache_mu;
std::map<std::string, stt_tuning> g_cache;

std::string shape_key(const stt_ctx *ctx) {
    const stt_geometry &g = ctx->geom;
    int counts[9] = {0};  // the view classes present, and their sizes, shape the choice too
    for (float a : ctx->off_axis_deg) ++counts[stt::off_axis_bin(a)];
    char buf[512];
    std::snprintf(buf, sizeof buf, "dev%d %dx%dx%d sp%.4g,%.4g,%.4g det%dx%d ds%.4g sid%.5g sdd%.5g off%.3g,%.3g,%.3g",
                  ctx->device, g.nx, g.ny, g.nz, g.sx, g.sy, g.sz, g.W, g.H, g.ds, g.sid, g.sdd, g.off[0], g.off[1],
                  g.off[2]);
    std::string key(buf);
    for (int b = 0; b < 9; ++b) key += " " + std::to_string(counts[b]);
    return key;
}

// Device scratch of one tuning run, released on every return path.
struct Scratch {
    float *vol = nullptr, *volt = nullptr, *b = nullptr, *rl = nullptr, *corr = nullptr;
    float2 *acc = nullptr;
    unsigned short *vol16 = nullptr, *volt16 = nullptr, *b16 = nullptr;  // BF16 copies for the BF16 choice
    stt::ViewRec *tv = nullptr;
    cudaArray_t arr = nullptr;
    cudaTextureObject_t tex = 0;
    stt::FpTex fptex;    // the textures of the tld4 gather variants over vol and volt
    stt::FpTex fptex16;  // the same over vol16 and volt16
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    ~Scratch() {
        stt::destroy_fp_tex(fptex);
        stt::destroy_fp_tex(fptex16);
        cudaFree(vol);
        cudaFree(volt);
        cudaFree(b);
        cudaFree(rl);
        cudaFree(corr);
        cudaFree(acc);
        cudaFree(vol16);
        cudaFree(volt16);
        cudaFree(b16);
        cudaFree(tv);
        if (tex) cudaDestroyTextureObject(tex);
        if (arr) cudaFreeArray(arr);
        if (e0) cudaEventDestroy(e0);
        if (e1) cudaEventDestroy(e1);
    }
};

// Microseconds of one launch of fn(): after one warm-up launch, the fastest of
// three rounds of three launches (the least disturbed round: choices between
// variants a few percent apart must not follow the noise).
template <typename Fn>
cudaError_t time_us(Scratch &sc, cudaStream_t s, Fn &&fn, float &us) {
    cudaError_t e = fn();
    if (e != cudaSuccess) return e;
    float best = 3.0e38f;
    for (int round = 0; round < 3; ++round) {
        if ((e = cudaEventRecord(sc.e0, s)) != cudaSuccess) return e;
        for (int r = 0; r < 3; ++r)
            if ((e = fn()) != cudaSuccess) return e;
        if ((e = cudaEventRecord(sc.e1, s)) != cudaSuccess) return e;
        if ((e = cudaEventSynchronize(sc.e1)) != cudaSuccess) return e;
        float ms = 0.0f;
        if ((e = cudaEventElapsedTime(&ms, sc.e0, sc.e1)) != cudaSuccess) return e;
        best = ms < best ? ms : best;
    }
    us = 1000.0f * best / 3.0f;
    return cudaSuccess;
}

}  // namespace

namespace stt {

stt_status apply_staged_bins(stt_ctx *ctx) {
    for (size_t v = 0; v < ctx->views_h.size(); ++v) {
        const int b = off_axis_bin(ctx->off_axis_deg[v]);
        ctx->views_h[v].staged = ((ctx->staged_bins >> b) & 1u) ? 1 : 0;
        ctx->views_h[v].staged16 = ((ctx->staged_bins16 >> b) & 1u) ? 1 : 0;
    }
    if (!ctx->views_h.empty() &&
        cudaMemcpy(ctx->views_d, ctx->views_h.data(), sizeof(ViewRec) * ctx->views_h.size(), cudaMemcpyHostToDevice) !=
            cudaSuccess) {
        cudaGetLastError();
        ctx->err = "cudaMemcpy(view table) failed";
        return STT_ERR_CUDA;
    }
    return STT_OK;
}

const FpTex *ctx_fp_tex(stt_ctx *ctx, const float *vol, const float *vol_t) {
    return is_tex_fp_variant(ctx->tuning.fp) ? ctx_fp_tex_any(ctx, vol, vol_t) : nullptr;
}

namespace {
template <typename T>
const FpTex *cached_tex(stt_ctx *ctx, const T *vol, const T *vol_t) {
    const GeomDev &g = ctx->g;
    const int es = (int)sizeof(T);
    for (const auto &e : ctx->fp_tex)
        if (e.vol == vol && e.volt == vol_t && e.nx == g.nx && e.ny == g.ny && e.nz == g.nz && e.esize == es)
            return &e.tex;
    if ((int)ctx->fp_tex.size() >= stt_ctx::kFpTexCache) return nullptr;
    stt_ctx::FpTexEntry e{vol, vol_t, g.nx, g.ny, g.nz, es, FpTex{}};
    make_fp_tex(g, vol, vol_t, e.tex);  // where it fails, tex.ok = 0 is cached too: the loads run
    ctx->fp_tex.push_back(e);
    return &ctx->fp_tex.back().tex;
}
}  // namespace

const FpTex *ctx_fp_tex_any(stt_ctx *ctx, const float *vol, const float *vol_t) {
    return cached_tex(ctx, vol, vol_t);
}

const FpTex *ctx_fp_tex(stt_ctx *ctx, const unsigned short *vol, const unsigned short *vol_t) {
    return ctx->tuning.fp16 == 1 ? cached_tex(ctx, vol, vol_t) : nullptr;
}

}  // namespace stt

extern "C" {

const char *stt_tuning_variant_name(int kernel, int variant) {
    const char *s = kernel == 0 ? stt::fp_variant_name(variant)
                    : kernel == 1 ? stt::slab_variant_name(variant)
                    : kernel == 2 ? stt::bp_variant_name(variant)
                    : kernel == 3 ? stt::ray_variant_name(variant)
                    : kernel == 4 ? stt::fp16_variant_name(variant) : "?";
    return s[0] == '?' ? nullptr : s;
}

stt_status stt_get_tuning(const stt_ctx *ctx, stt_tuning *out) {
    if (!ctx || !out) return STT_ERR_INVALID;
    if (!ctx->has_geom) return STT_ERR_STATE;
    *out = ctx->report;
    out->fp_variant = ctx->tuning.fp;
    out->slab_variant = ctx->tuning.slab;
    out->bp_variant = ctx->tuning.bp;
    out->ray_variant = ctx->tuning.ray;
    out->fp_variant_bf16 = ctx->tuning.fp16;
    out->staged_bins = ctx->staged_bins;
    out->staged_bins_bf16 = ctx->staged_bins16;
    out->tuned = ctx->tuned ? 1 : 0;
    return STT_OK;
}

stt_status stt_set_tuning(stt_ctx *ctx, const stt_tuning *t) {
    if (!ctx || !t) return STT_ERR_INVALID;
    if (!ctx->has_geom) return STT_ERR_STATE;
    if (t->fp_variant < 0 || t->fp_variant >= stt::kFpVariants || t->slab_variant < 0 ||
        t->slab_variant >= stt::kSlabVariants || t->bp_variant < 0 || t->bp_variant >= stt::kBpVariants ||
        t->ray_variant < 0 || t->ray_variant >= stt::kRayVariants || (t->staged_bins >> 9) != 0 ||
        (t->staged_bins_bf16 >> 9) != 0 || t->fp_variant_bf16 < 0 || t->fp_variant_bf16 >= stt::kFp16Variants) {
        ctx->err = "stt_set_tuning: a variant or staged_bins out of range";
        return STT_ERR_INVALID;
    }
    if (cudaSetDevice(ctx->device) != cudaSuccess) {
        cudaGetLastError();
        ctx->err = "cudaSetDevice failed";
        return STT_ERR_CUDA;
    }
    ctx->tuning.fp = t->fp_variant;
    ctx->tuning.slab = t->slab_variant;
    ctx->tuning.bp = t->bp_variant;
    ctx->tuning.ray = t->ray_variant;
    ctx->tuning.fp16 = t->fp_variant_bf16;
    ctx->staged_bins = t->staged_bins;
    ctx->staged_bins16 = t->staged_bins_bf16;
    ctx->tuned = true;
    ctx->report = *t;
    ctx->report.tuned = 1;
    return stt::apply_staged_bins(ctx);
}

stt_status stt_autotune(stt_ctx *ctx, stt_tuning *out, void *stream) {
    if (!ctx) return STT_ERR_INVALID;
    if (!ctx->has_geom) {
        ctx->err = "no geometry set (call stt_set_geometry)";
        return STT_ERR_STATE;
    }
    if (ctx->views_h.empty()) {
        ctx->err = "stt_autotune: the geometry has no views";
        return STT_ERR_INVALID;
    }
    if (cudaSetDevice(ctx->device) != cudaSuccess) {
        cudaGetLastError();
        ctx->err = "cudaSetDevice failed";
        return STT_ERR_CUDA;
    }
    const std::string key = shape_key(ctx);
    {
        std::lock_guard<std::mutex> lock(g_cache_mu);
        auto it = g_cache.find(key);
        if (it != g_cache.end()) {
            stt_tuning t = it->second;
            t.from_cache = 1;
            stt_status st = stt_set_tuning(ctx, &t);
            if (st) return st;
            if (out) *out = ctx->report;
            return STT_OK;
        }
    }
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    const stt::GeomDev &g = ctx->g;
    const size_t n = (size_t)g.nx * g.ny * g.nz, npix = (size_t)g.W * g.H;
    Scratch sc;
    auto fail = [&](cudaError_t e, const char *where) {
        cudaGetLastError();
        ctx->err = std::string("stt_autotune: ") + where + ": " + cudaGetErrorString(e);
        return e == cudaErrorMemoryAllocation ? STT_ERR_NOMEM : STT_ERR_CUDA;
    };
    cudaError_t e = cudaSuccess;
    if ((e = cudaMalloc(&sc.vol, n * sizeof(float))) || (e = cudaMalloc(&sc.volt, n * sizeof(float))) ||
        (e = cudaMalloc(&sc.b, npix * sizeof(float))) || (e = cudaMalloc(&sc.rl, npix * sizeof(float))) ||
        (e = cudaMalloc(&sc.corr, npix * sizeof(float))) || (e = cudaMalloc(&sc.tv, 2 * sizeof(stt::ViewRec))) ||
        (e = cudaEventCreate(&sc.e0)) || (e = cudaEventCreate(&sc.e1)))
        return fail(e, "scratch");
    {  // the correction as a one-layer texture, as the solver's backprojection reads it
        cudaChannelFormatDesc cd = cudaCreateChannelDesc<float>();
        if ((e = cudaMalloc3DArray(&sc.arr, &cd, make_cudaExtent(g.W, g.H, 1), cudaArrayLayered)))
            return fail(e, "texture array");
        cudaResourceDesc rd{};
        rd.resType = cudaResourceTypeArray;
        rd.res.array.array = sc.arr;
        cudaTextureDesc td{};
        td.addressMode[0] = td.addressMode[1] = td.addressMode[2] = cudaAddressModeClamp;
        td.filterMode = cudaFilterModePoint;
        td.readMode = cudaReadModeElementType;
        if ((e = cudaCreateTextureObject(&sc.tex, &rd, &td, nullptr))) return fail(e, "texture object");
    }
    // the times do not depend on the values; these are positive and typical enough
    if ((e = stt::launch_fill_seeded((long long)n, 7, sc.vol, s)) || (e = stt::launch_transpose(g, sc.vol, sc.volt, s)) ||
        (e = cudaMemsetAsync(sc.b, 0, npix * sizeof(float), s)) || (e = cudaMemsetAsync(sc.rl, 0, npix * sizeof(float), s)))
        return fail(e, "scratch fill");
    // one representative view per class, and the class sizes
    int rep[9], count[9];
    for (int b = 0; b < 9; ++b) rep[b] = -1, count[b] = 0;
    for (size_t v = 0; v < ctx->views_h.size(); ++v) {
        const int b = stt::off_axis_bin(ctx->off_axis_deg[v]);
        if (rep[b] < 0) rep[b] = (int)v;
        ++count[b];
    }
    float tg[stt::kFpVariants][9] = {}, ts[stt::kSlabVariants][9] = {};
    float t_idle = 0.0f;  // a slab launch on a view it does not project (returns at once)
    stt::FpSlabMaps maps[stt::kSlabVariants];
    bool maps_ok[stt::kSlabVariants] = {};
    bool slab_ok = false;
    for (int sv = 0; sv < stt::kSlabVariants; ++sv)
        slab_ok |= maps_ok[sv] = stt::make_fp_slab_maps(g, sc.vol, sc.volt, maps[sv], sv);
    stt::make_fp_tex(g, sc.vol, sc.volt, sc.fptex);  // where it fails, ok = 0 and the tld4 variants are skipped
    for (int b = 0; b < 9; ++b) {
        if (rep[b] < 0) continue;
        stt::ViewRec two[2] = {ctx->views_h[rep[b]], ctx->views_h[rep[b]]};
        two[0].staged = 0;
        two[1].staged = 1;
        if ((e = cudaMemcpyAsync(sc.tv, two, sizeof two, cudaMemcpyHostToDevice, s)) || (e = cudaStreamSynchronize(s)))
            return fail(e, "view copy");
        const stt::ViewSel gather_sel{0, nullptr, 0, 0}, slab_sel{1, nullptr, 0, 1};
        for (int fv = 0; fv < stt::kFpVariants; ++fv) {
            if (stt::is_tex_fp_variant(fv) && !sc.fptex.ok) {
                tg[fv][b] = 3.0e38f;  // no textures on this geometry: never chosen
                continue;
            }
            e = time_us(sc, s, [&] {
                return stt::launch_fp_corr(g, sc.tv, sc.vol, sc.volt, gather_sel, sc.b, sc.rl, sc.corr, s, 0, nullptr,
                                           ctx->status, fv, &sc.fptex);
            }, tg[fv][b]);
            if (e) return fail(e, "gather projector");
        }
        if (slab_ok && t_idle == 0.0f) {
            int sv0 = 0;
            while (!maps_ok[sv0]) ++sv0;
            e = time_us(sc, s, [&] {
                return stt::launch_fp_corr_slab(g, sc.tv, maps[sv0], sc.vol, sc.volt, gather_sel, sc.b, sc.rl, sc.corr,
                                                s, 0, ctx->status);
            }, t_idle);
            if (e) return fail(e, "idle slab launch");
        }
        for (int sv = 0; sv < stt::kSlabVariants; ++sv) {
            if (!maps_ok[sv]) continue;
            e = time_us(sc, s, [&] {
                return stt::launch_fp_corr_slab(g, sc.tv, maps[sv], sc.vol, sc.volt, slab_sel, sc.b, sc.rl, sc.corr, s,
                                                0, ctx->status);
            }, ts[sv][b]);
            if (e) return fail(e, "slab projector");
        }
    }
    // the gather variant with the least time over all views; then the box
    // whose per-class minimum with it is least; then the class choices
    stt_tuning t{};
    double best = 1e300;
    for (int fv = 0; fv < stt::kFpVariants; ++fv) {
        if (stt::is_tex_fp_variant(fv) && !sc.fptex.ok) continue;  // not timed: fp_us stays 0
        double tot = 0.0, w = 0.0;
        for (int b = 0; b < 9; ++b)
            if (rep[b] >= 0) tot += (double)count[b] * tg[fv][b], w += count[b];
        t.fp_us[fv] = (float)(tot / w);
        if (tot < best) best = tot, t.fp_variant = fv;
    }
    if (slab_ok) {
        best = 1e300;
        for (int sv = 0; sv < stt::kSlabVariants; ++sv) {
            if (!maps_ok[sv]) continue;
            double tot = 0.0, w = 0.0, slab_only = 0.0;
            for (int b = 0; b < 9; ++b) {
                if (rep[b] < 0) continue;
                tot += (double)count[b] * std::fmin(tg[t.fp_variant][b], ts[sv][b]);
                slab_only += (double)count[b] * ts[sv][b];
                w += count[b];
            }
            t.slab_us[sv] = (float)(slab_only / w);
            if (tot < best) best = tot, t.slab_variant = sv;
        }
        for (int b = 0; b < 9; ++b) {
            if (rep[b] >= 0) {
                if (ts[t.slab_variant][b] < tg[t.fp_variant][b]) t.staged_bins |= 1u << b;
            } else {
                t.staged_bins |= 0x1E0u & (1u << b);  // a class without views keeps the default rule
            }
        }
        // With any view staged, every view launches both kernels and the one
        // with nothing to do costs an idle launch; gathering every view is one
        // launch.  Keep the split only where it wins with that cost counted.
        double split = 0.0, gather_all = 0.0;
        for (int b = 0; b < 9; ++b) {
            if (rep[b] < 0) continue;
            const double own = ((t.staged_bins >> b) & 1u) ? ts[t.slab_variant][b] : tg[t.fp_variant][b];
            split += (double)count[b] * (own + t_idle);
            gather_all += (double)count[b] * tg[t.fp_variant][b];
        }
        if (split >= gather_all) t.staged_bins = 0;
    } else {
        t.staged_bins = 0x1E0u;  // irrelevant: without slab maps every view gathers
    }
    // BF16 storage: per class the gather kernel's two forms (loads, and tld4
    // gathers of 16-bit textures where they bind) and the slab kernel's BF16
    // box (the box just chosen); a BF16 volume's gathers move half the bytes,
    // so the faster projector can differ from the FP32 choice
    t.staged_bins_bf16 = 0x1E0u;  // irrelevant where the BF16 maps do not apply
    t.fp_variant_bf16 = 0;
    {
        if ((e = cudaMalloc(&sc.vol16, n * sizeof(unsigned short))) ||
            (e = cudaMalloc(&sc.volt16, n * sizeof(unsigned short))) ||
            (e = cudaMalloc(&sc.b16, npix * sizeof(unsigned short))) ||
            (e = cudaMemsetAsync(sc.vol16, 0x3F, n * sizeof(unsigned short), s)) ||  // 0x3F3F: about 0.75
            (e = cudaMemsetAsync(sc.volt16, 0x3F, n * sizeof(unsigned short), s)) ||
            (e = cudaMemsetAsync(sc.b16, 0, npix * sizeof(unsigned short), s)))
            return fail(e, "BF16 scratch");
        stt::make_fp_tex(g, sc.vol16, sc.volt16, sc.fptex16);  // where it fails, ok = 0: loads only
        stt::FpSlabMaps m16;
        const bool maps16 = stt::make_fp_slab_maps(g, sc.vol16, sc.volt16, m16, t.slab_variant);
        float tg16[stt::kFp16Variants][9] = {}, ts16[9] = {};
        float t_idle16 = 0.0f;
        for (int b = 0; b < 9; ++b) {
            if (rep[b] < 0) continue;
            stt::ViewRec two[2] = {ctx->views_h[rep[b]], ctx->views_h[rep[b]]};
            two[0].staged16 = 0;
            two[1].staged16 = 1;
            if ((e = cudaMemcpyAsync(sc.tv, two, sizeof two, cudaMemcpyHostToDevice, s)) ||
                (e = cudaStreamSynchronize(s)))
                return fail(e, "view copy");
            for (int fv = 0; fv < stt::kFp16Variants; ++fv) {
                if (fv == 1 && !sc.fptex16.ok) continue;
                e = time_us(sc, s, [&] {
                    return stt::launch_fp_corr(g, sc.tv, sc.vol16, sc.volt16, stt::ViewSel{0, nullptr, 0, 0}, sc.b16,
                                               sc.rl, sc.corr, s, 0, nullptr, ctx->status, fv, &sc.fptex16);
                }, tg16[fv][b]);
                if (e) return fail(e, "BF16 gather projector");
            }
            if (!maps16) continue;
            e = time_us(sc, s, [&] {
                return stt::launch_fp_corr_slab(g, sc.tv, m16, sc.vol16, sc.volt16, stt::ViewSel{1, nullptr, 0, 1},
                                                sc.b16, sc.rl, sc.corr, s, 0, ctx->status);
            }, ts16[b]);
            if (e) return fail(e, "BF16 slab projector");
            if (t_idle16 == 0.0f) {
                e = time_us(sc, s, [&] {
                    return stt::launch_fp_corr_slab(g, sc.tv, m16, sc.vol16, sc.volt16, stt::ViewSel{0, nullptr, 0, 0},
                                                    sc.b16, sc.rl, sc.corr, s, 0, ctx->status);
                }, t_idle16);
                if (e) return fail(e, "idle BF16 slab launch");
            }
        }
        // the gather form with the least time over all views, then the classes
        // the slab kernel takes from it
        double best16 = 1e300;
        for (int fv = 0; fv < stt::kFp16Variants; ++fv) {
            if (fv == 1 && !sc.fptex16.ok) continue;  // not timed: fp16_us stays 0
            double tot = 0.0, w = 0.0;
            for (int b = 0; b < 9; ++b)
                if (rep[b] >= 0) tot += (double)count[b] * tg16[fv][b], w += count[b];
            t.fp16_us[fv] = (float)(tot / w);
            if (tot < best16) best16 = tot, t.fp_variant_bf16 = fv;
        }
        if (maps16) {
            t.staged_bins_bf16 = 0;
            double split = 0.0, gather_all = 0.0;
            for (int b = 0; b < 9; ++b) {
                if (rep[b] < 0) {
                    t.staged_bins_bf16 |= 0x1E0u & (1u << b);
                    continue;
                }
                const float tg = tg16[t.fp_variant_bf16][b];
                if (ts16[b] < tg) t.staged_bins_bf16 |= 1u << b;
                split += (double)count[b] * (std::fmin(ts16[b], tg) + t_idle16);
                gather_all += (double)count[b] * tg;
            }
            if (split >= gather_all) t.staged_bins_bf16 = 0;  // (as for FP32 above)
        }
    }
    // voxel backprojection: the column lengths on the views of the first and last classes present
    if ((e = cudaMemcpy2DToArrayAsync(sc.arr, 0, 0, sc.corr, g.W * sizeof(float), g.W * sizeof(float), g.H,
                                      cudaMemcpyDeviceToDevice, s)))
        return fail(e, "texture fill");
    {
        int vb[2] = {-1, -1};
        for (int b = 0; b < 9; ++b)
            if (rep[b] >= 0) {
                if (vb[0] < 0) vb[0] = rep[b];
                vb[1] = rep[b];
            }
        best = 1e300;
        for (int bv = 0; bv < stt::kBpVariants; ++bv) {
            float tot = 0.0f;
            for (int k = 0; k < 2; ++k) {
                const stt::ViewRec one = ctx->views_h[vb[k]];
                if ((e = cudaMemcpyAsync(sc.tv, &one, sizeof one, cudaMemcpyHostToDevice, s)) ||
                    (e = cudaStreamSynchronize(s)))
                    return fail(e, "view copy");
                float us = 0.0f;
                e = time_us(sc, s, [&] {
                    return stt::launch_bp_voxel(g, sc.tv, stt::ViewSel{0, nullptr, 0, 0}, sc.corr, sc.vol, 0.3f,
                                                1e30f, s, sc.tex, bv);
                }, us);
                if (e) return fail(e, "voxel backprojection");
                tot += us;
            }
            t.bp_us[bv] = tot / 2.0f;
            if (tot < best) best = tot, t.bp_variant = bv;
        }
    }
    // ray backprojection: both scatters (with the update) on the view of the largest class
    {
        int vb = -1;
        for (int b = 0; b < 9; ++b)
            if (rep[b] >= 0 && (vb < 0 || count[b] > count[stt::off_axis_bin(ctx->off_axis_deg[vb])])) vb = rep[b];
        const stt::ViewRec one = ctx->views_h[vb];
        if ((e = cudaMalloc(&sc.acc, n * sizeof(float2))) || (e = cudaMemsetAsync(sc.acc, 0, n * sizeof(float2), s)) ||
            (e = cudaMemcpyAsync(sc.tv, &one, sizeof one, cudaMemcpyHostToDevice, s)) || (e = cudaStreamSynchronize(s)))
            return fail(e, "ray backprojection scratch");
        const bool slab_ok_ray = n < (1ull << 31);
        best = 1e300;
        for (int rv = 0; rv < stt::kRayVariants; ++rv) {
            if (rv == 1 && !slab_ok_ray) continue;
            float us = 0.0f;
            e = time_us(sc, s, [&] {
                return stt::launch_bp_ray(g, sc.tv, stt::ViewSel{0, nullptr, 0, 0}, sc.corr, sc.acc, sc.vol, 1e30f, s,
                                          rv);
            }, us);
            if (e) return fail(e, "ray backprojection");
            t.ray_us[rv] = us;
            if (us < best) best = us, t.ray_variant = rv;
        }
    }
    if ((e = cudaStreamSynchronize(s))) return fail(e, "synchronize");
    stt_status st = stt_set_tuning(ctx, &t);
    if (st) return st;
    {
        std::lock_guard<std::mutex> lock(g_cache_mu);
        g_cache[key] = ctx->report;
    }
    if (out) *out = ctx->report;
    return STT_OK;
}

}  // extern "C"
