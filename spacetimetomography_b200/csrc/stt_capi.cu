// stt_capi.cu -- the C ABI of libstt.so (declared in include/stt.h): context,
// FP64 view geometry, argument checking and kernel dispatch.
//
// Reference paths are relative to gmzang/SpaceTimeTomography (S/ = SpaceTimeTomography/).
#include <cmath>
#include <cstdint>
#include <cstring>
#include <string>
#include <vector>

#include "stt.h"
#include "stt_ctx.h"
#include "stt_internal.cuh"
#include "stt_kernels.h"

namespace {

thread_local std::string g_thread_err;

stt_status fail(stt_ctx *ctx, stt_status st, const std::string &msg) {
    if (ctx) ctx->err = msg;
    else g_thread_err = msg;
    return st;
}

stt_status cuda_fail(stt_ctx *ctx, cudaError_t e, const char *where) {
    return fail(ctx, STT_ERR_CUDA, std::string(where) + ": " + cudaGetErrorString(e));
}

// A failed CUDA call: its error is read and cleared (cudaGetLastError), so a
// non-sticky error does not resurface in a later, unrelated launch check.
#define STT_CUDA(ctx, call, where)                          \
    do {                                                    \
        cudaError_t e_ = (call);                            \
        if (e_ != cudaSuccess) {                            \
            cudaGetLastError();                             \
            return cuda_fail(ctx, e_, where);               \
        }                                                   \
    } while (0)

cudaStream_t S(void *s) { return reinterpret_cast<cudaStream_t>(s); }

long long nvox(const stt_ctx *c) { return (long long)c->g.nx * c->g.ny * c->g.nz; }

stt_status need_geom(stt_ctx *ctx) {
    if (!ctx) return fail(nullptr, STT_ERR_INVALID, "null context");
    if (!ctx->has_geom) return fail(ctx, STT_ERR_STATE, "no geometry set (call stt_set_geometry)");
    return STT_OK;
}

stt_status set_device(stt_ctx *ctx) {
    STT_CUDA(ctx, cudaSetDevice(ctx->device), "cudaSetDevice");
    return STT_OK;
}

// Per-view FP64 geometry.  Camera = T(-ox, -oz, oy - sid) * R_y(theta) applied
// to model coordinates centred at (dims-1)*spacing/2 (Scene::_calculateMatrix
// Scene.cpp:187-188, TypicalRayProducer::_calculateMatrix
// TypicalRayProducer.cpp:146-147, ST_Tomography ctor :244-246).  Detector
// pixel (i,j) lies on the near plane z = -sdd at ((i-(W-1)/2)ds, (j-(H-1)/2)ds)
// (ViewToPixels and the frustum of Scene.cpp:194-206, TypicalRayProducer.cpp:174-194).
void build_view(const stt_geometry &g, double theta, stt::ViewRec &v) {
    const double c = std::cos(theta), s = std::sin(theta);
    const double R[3][3] = {{c, 0, s}, {0, 1, 0}, {-s, 0, c}};
    const double t[3] = {-g.off[0], -g.off[2], -g.sid + g.off[1]};
    const double sp[3] = {g.sx, g.sy, g.sz};
    const int dims[3] = {g.nx, g.ny, g.nz};
    double ctr[3];
    for (int k = 0; k < 3; ++k) ctr[k] = (dims[k] - 1) * sp[k] * 0.5;
    auto to_model = [&](const double cam[3], double out[3]) {
        const double d[3] = {cam[0] - t[0], cam[1] - t[1], cam[2] - t[2]};
        for (int r = 0; r < 3; ++r) out[r] = ctr[r] + R[0][r] * d[0] + R[1][r] * d[1] + R[2][r] * d[2];
    };
    const double zero[3] = {0, 0, 0};
    to_model(zero, v.src);
    const double p0[3] = {-(g.W - 1) * 0.5 * g.ds, -(g.H - 1) * 0.5 * g.ds, -g.sdd};
    to_model(p0, v.det0);
    for (int r = 0; r < 3; ++r) {
        v.du[r] = R[0][r] * g.ds;
        v.dv[r] = R[1][r] * g.ds;
    }
    // voxel (x,y,z) -> camera: R * (diag(sp) * x - ctr) + t
    for (int r = 0; r < 3; ++r) {
        double b = t[r];
        for (int q = 0; q < 3; ++q) {
            v.A[r * 3 + q] = (float)(R[r][q] * sp[q]);
            b -= R[r][q] * ctr[q];
        }
        v.b[r] = (float)b;
    }
    // gather from the z-fastest copy when the central ray runs more along x than z
    v.layout = std::fabs(s) > std::fabs(c) ? 1 : 0;
    v.staged = std::fmin(std::fabs(s), std::fabs(c)) > 0.4226 ? 1 : 0;  // sin 25 degrees
    v.staged16 = v.staged;
    v.pad = 0.0f;
}

template <typename T>
stt_status ensure(stt_ctx *ctx, T *&ptr, size_t &cap, size_t n, const char *what) {
    if (cap >= n && ptr) return STT_OK;
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    cap = 0;
    cudaError_t e = cudaMalloc((void **)&ptr, n * sizeof(T));
    if (e != cudaSuccess) {
        ptr = nullptr;
        return fail(ctx, STT_ERR_NOMEM, std::string("cudaMalloc(") + what + "): " + cudaGetErrorString(e));
    }
    cap = n;
    return STT_OK;
}

}  // namespace

extern "C" {

const char *stt_version(void) { return "stt 0.1.0 sm_100a"; }

stt_status stt_create(stt_ctx **out, int device) {
    if (!out) return fail(nullptr, STT_ERR_INVALID, "null output pointer");
    *out = nullptr;
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess) return cuda_fail(nullptr, e, "cudaGetDeviceCount");
    if (device < 0 || device >= n) return fail(nullptr, STT_ERR_INVALID, "device ordinal out of range");
    stt_ctx *ctx = new stt_ctx();
    ctx->device = device;
    *out = ctx;
    return STT_OK;
}

stt_status stt_destroy(stt_ctx *ctx) {
    if (!ctx) return STT_OK;
    cudaSetDevice(ctx->device);
    if (ctx->views_d) cudaFree(ctx->views_d);
    if (ctx->acc) cudaFree(ctx->acc);
    if (ctx->corr) cudaFree(ctx->corr);
    if (ctx->volt) cudaFree(ctx->volt);
    cudaFree(ctx->volt16);
    cudaFree(ctx->pw);
    cudaFree(ctx->pwd);
    cudaFree(ctx->status);
    for (auto &e : ctx->fp_tex) stt::destroy_fp_tex(e.tex);
    stt::free_corr_tex(ctx->corr_tex);
    delete ctx;
    return STT_OK;
}

stt_status stt_ctx_dims(const stt_ctx *ctx, int *dims) {
    if (!ctx || !dims) return STT_ERR_INVALID;
    if (!ctx->has_geom) return STT_ERR_STATE;
    dims[0] = ctx->g.nx;
    dims[1] = ctx->g.ny;
    dims[2] = ctx->g.nz;
    return STT_OK;
}

const char *stt_last_error(const stt_ctx *ctx) {
    return ctx ? ctx->err.c_str() : g_thread_err.c_str();
}

stt_status stt_views_from_rounds(int rounds, const double *start_deg, int views_per_round,
                                 double step_deg, double *angles_out) {
    if (rounds < 0 || views_per_round < 0 || (rounds > 0 && (!start_deg || !angles_out)))
        return fail(nullptr, STT_ERR_INVALID, "bad arguments to stt_views_from_rounds");
    // InitViews / RotateVolume (ST_Tomography.cpp:887-934): start angle read as
    // float, pi = 3.1415926, each following view 36 degrees further.
    const double step = step_deg * 3.1415926 / 180;
    for (int r = 0; r < rounds; ++r) {
        const double a0 = (double)(float)start_deg[r] * 3.1415926 / 180;
        for (int k = 0; k < views_per_round; ++k) angles_out[r * views_per_round + k] = a0 + k * step;
    }
    return STT_OK;
}

stt_status stt_lds_angles(int n, int Ns, int p, int Nz, double *out) {
    if (n < 0 || Ns <= 0 || p < 2 || Nz <= 0 || (n > 0 && !out))
        return fail(nullptr, STT_ERR_INVALID, "bad arguments to stt_lds_angles");
    // Low_discrepency_squence.m:38-67: van der Corput radical inverse of i in
    // base p, scaled to one segment of 360/Ns degrees, repeated over the Ns
    // segments; an extra 0 every Nz entries.
    int len = 0;
    long long i = 0;
    while (len < n) {
        if (len > 0 && len % Nz == 0) out[len++] = 0.0;
        if (len >= n) break;
        long long b = i++;
        double r = 0.0, q = 1.0 / p;
        while (b != 0) {
            r += (double)(b % p) * q;
            q /= p;
            b /= p;
        }
        r = 360.0 * r / Ns;
        for (int k = 0; len < n && k < Ns; ++k) out[len++] = r + k * 360.0 / Ns;
    }
    return STT_OK;
}

stt_status stt_permutation(unsigned long long seed, int n, int *perm) {
    if (n < 0 || (n > 0 && !perm)) return fail(nullptr, STT_ERR_INVALID, "bad arguments to stt_permutation");
    // SplitMix64 (Steele, Lea, Flood 2014) driving a Fisher-Yates shuffle.
    uint64_t s = seed;
    auto next = [&s]() {
        uint64_t z = (s += 0x9E3779B97F4A7C15ull);
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    };
    for (int i = 0; i < n; ++i) perm[i] = i;
    for (int i = n - 1; i > 0; --i) {
        int j = (int)(next() % (uint64_t)(i + 1));
        int tmp = perm[i];
        perm[i] = perm[j];
        perm[j] = tmp;
    }
    return STT_OK;
}

stt_status stt_set_geometry(stt_ctx *ctx, const stt_geometry *g) {
    if (!ctx || !g) return fail(ctx, STT_ERR_INVALID, "null argument");
    if (g->nx < 2 || g->ny < 2 || g->nz < 2) return fail(ctx, STT_ERR_INVALID, "volume dims must be >= 2");
    if (g->W < 5 || g->H < 5) return fail(ctx, STT_ERR_INVALID, "detector must be at least 5x5");
    if (!(g->sx > 0 && g->sy > 0 && g->sz > 0 && g->ds > 0))
        return fail(ctx, STT_ERR_INVALID, "spacings must be positive");
    if (!(g->sdd > 0 && g->sid > 0 && std::isfinite(g->sid) && std::isfinite(g->sdd)))
        return fail(ctx, STT_ERR_INVALID, "sid and sdd must be positive and finite");
    if ((long long)g->nx * g->ny * g->nz > (1LL << 34))
        return fail(ctx, STT_ERR_INVALID, "volume too large");
    if (g->n_views < 0 || (g->n_views > 0 && !g->angles_rad))
        return fail(ctx, STT_ERR_INVALID, "n_views > 0 needs angles_rad");
    // The source must lie outside the volume so that every voxel projects in
    // front of it (cam.z < 0 in the voxel-driven backprojector).
    const double hx = (g->nx - 1) * g->sx * 0.5, hy = (g->ny - 1) * g->sy * 0.5, hz = (g->nz - 1) * g->sz * 0.5;
    const double off = std::sqrt(g->off[0] * g->off[0] + g->off[1] * g->off[1] + g->off[2] * g->off[2]);
    if (g->sid <= std::sqrt(hx * hx + hy * hy + hz * hz) + off)
        return fail(ctx, STT_ERR_INVALID, "sid must exceed the volume half-diagonal plus the offset");
    stt_status st = set_device(ctx);
    if (st) return st;
    if (!ctx->status) {
        if ((st = ensure(ctx, ctx->status, ctx->status_n, 4, "status word"))) return st;
        STT_CUDA(ctx, cudaMemset(ctx->status, 0, 4 * sizeof(int)), "cudaMemset(status word)");
    }
    ctx->views_h.resize(g->n_views);
    ctx->off_axis_deg.resize(g->n_views);
    for (int v = 0; v < g->n_views; ++v) {
        build_view(*g, g->angles_rad[v], ctx->views_h[v]);
        const double s = std::fabs(std::sin(g->angles_rad[v])), c = std::fabs(std::cos(g->angles_rad[v]));
        ctx->off_axis_deg[v] = (float)(std::atan2(std::fmin(s, c), std::fmax(s, c)) * 180.0 / M_PI);
    }
    // a new geometry starts from the default launch choices
    ctx->geom = *g;
    ctx->geom.angles_rad = nullptr;
    ctx->tuning = stt::Tuning{};
    ctx->staged_bins = ctx->staged_bins16 = 0x1E0u;
    ctx->tuned = false;
    ctx->report = stt_tuning{};
    if (g->n_views > 0) {
        st = ensure(ctx, ctx->views_d, ctx->views_cap, (size_t)g->n_views, "view table");
        if (st) return st;
        STT_CUDA(ctx, cudaMemcpy(ctx->views_d, ctx->views_h.data(), sizeof(stt::ViewRec) * g->n_views,
                                 cudaMemcpyHostToDevice),
                 "cudaMemcpy(view table)");
    }
    stt::GeomDev &d = ctx->g;
    d.nx = g->nx;
    d.ny = g->ny;
    d.nz = g->nz;
    d.W = g->W;
    d.H = g->H;
    d.n_views = g->n_views;
    d.inv_sp[0] = 1.0 / g->sx;
    d.inv_sp[1] = 1.0 / g->sy;
    d.inv_sp[2] = 1.0 / g->sz;
    // ST_Tomography.cpp:300: sqrt of the float spacings, stored as float
    const float fx = (float)g->sx, fy = (float)g->sy, fz = (float)g->sz;
    d.sd = std::sqrt(fx * fx + fy * fy + fz * fz);
    d.cx = (float)((g->W - 1) * 0.5);
    d.cy = (float)((g->H - 1) * 0.5);
    d.sdd_ds = (float)(g->sdd / g->ds);
    ctx->sp[0] = g->sx;
    ctx->sp[1] = g->sy;
    ctx->sp[2] = g->sz;
    ctx->tuning.ray = stt::default_ray_variant(d);  // (depends on the volume size just set)
    ctx->has_geom = true;
    return STT_OK;
}

// When a view in [view0, view0+nviews) gathers from the z-fastest copy,
// refresh the context's copy of `vol` and return it in *volt.
}  // extern "C"

// The z-fastest copy of the volume when a view in [view0, view0 + nviews)
// gathers along x (FP32 and BF16 storage).
static stt_status transposed_if_needed(stt_ctx *ctx, const float *vol, int view0, int nviews, cudaStream_t s,
                                       const float **volt) {
    *volt = nullptr;
    bool any = false;
    for (int v = view0; v < view0 + nviews && !any; ++v) any = ctx->views_h[v].layout == 1;
    if (!any) return STT_OK;
    stt_status st = ensure(ctx, ctx->volt, ctx->volt_n, (size_t)nvox(ctx), "transposed volume");
    if (st) return st;
    STT_CUDA(ctx, stt::launch_transpose(ctx->g, vol, ctx->volt, s), "k_transpose launch");
    *volt = ctx->volt;
    return STT_OK;
}

static stt_status transposed_if_needed(stt_ctx *ctx, const unsigned short *vol, int view0, int nviews,
                                       cudaStream_t s, const unsigned short **volt) {
    *volt = nullptr;
    bool any = false;
    for (int v = view0; v < view0 + nviews && !any; ++v) any = ctx->views_h[v].layout == 1;
    if (!any) return STT_OK;
    stt_status st = ensure(ctx, ctx->volt16, ctx->volt16_n, (size_t)nvox(ctx), "transposed BF16 volume");
    if (st) return st;
    STT_CUDA(ctx, stt::launch_transpose_bf16(ctx->g, vol, ctx->volt16, s), "k_transpose launch");
    *volt = ctx->volt16;
    return STT_OK;
}

// The staged-class mask for a volume of this storage (0: no view is staged).
static unsigned staged_mask(const stt_ctx *ctx, const float *) { return ctx->staged_bins; }
static unsigned staged_mask(const stt_ctx *ctx, const unsigned short *) { return ctx->staged_bins16; }

extern "C" {

static stt_status check_views(stt_ctx *ctx, int view0, int nviews) {
    if (view0 < 0 || nviews < 0 || view0 + nviews > ctx->g.n_views)
        return fail(ctx, STT_ERR_INVALID, "view range outside the geometry's view list");
    return STT_OK;
}

stt_status stt_fp(stt_ctx *ctx, const float *vol, float *proj, float *raylen, float *weight,
                  int view0, int nviews, void *stream) {
    stt_status st = need_geom(ctx);
    if (st) return st;
    if (!vol || !proj) return fail(ctx, STT_ERR_INVALID, "null vol or proj");
    if ((st = check_views(ctx, view0, nviews))) return st;
    if (nviews == 0) return STT_OK;
    if ((st = set_device(ctx))) return st;
    const float *volt = nullptr;
    if ((st = transposed_if_needed(ctx, vol, view0, nviews, S(stream), &volt))) return st;
    STT_CUDA(ctx, stt::launch_fp(ctx->g, ctx->views_d, vol, volt, view0, nviews, proj, raylen, weight, S(stream)),
             "k_fp launch");
    return STT_OK;
}

stt_status stt_fp_typed(stt_ctx *ctx, const void *vol, int dtype, float *proj, float *raylen, float *weight,
                        int view0, int nviews, void *stream) {
    if (dtype == STT_DTYPE_F32)
        return stt_fp(ctx, static_cast<const float *>(vol), proj, raylen, weight, view0, nviews, stream);
    stt_status st = need_geom(ctx);
    if (st) return st;
    if (dtype != STT_DTYPE_BF16) return fail(ctx, STT_ERR_INVALID, "dtype must be STT_DTYPE_F32 or STT_DTYPE_BF16");
    if (!vol || !proj) return fail(ctx, STT_ERR_INVALID, "null vol or proj");
    if ((st = check_views(ctx, view0, nviews))) return st;
    if (nviews == 0) return STT_OK;
    if ((st = set_device(ctx))) return st;
    const unsigned short *v16 = static_cast<const unsigned short *>(vol);
    const unsigned short *vt16 = nullptr;
    bool any = false;
    for (int v = view0; v < view0 + nviews && !any; ++v) any = ctx->views_h[v].layout == 1;
    if (any) {
        if ((st = ensure(ctx, ctx->volt16, ctx->volt16_n, (size_t)nvox(ctx), "transposed BF16 volume"))) return st;
        STT_CUDA(ctx, stt::launch_transpose_bf16(ctx->g, v16, ctx->volt16, S(stream)), "k_transpose launch");
        vt16 = ctx->volt16;
    }
    STT_CUDA(ctx, stt::launch_fp_bf16(ctx->g, ctx->views_d, v16, vt16, view0, nviews, proj, raylen, weight,
                                      S(stream)),
             "k_fp launch");
    return STT_OK;
}

stt_status stt_fp_correction(stt_ctx *ctx, const float *vol, const float *b, float *raylen_state,
                             float *corr, int view, void *stream) {
    stt_status st = need_geom(ctx);
    if (st) return st;
    if (!vol || !b || !corr) return fail(ctx, STT_ERR_INVALID, "null vol, b or corr");
    if ((st = check_views(ctx, view, 1))) return st;
    if ((st = set_device(ctx))) return st;
    const stt::ViewSel sel{view, nullptr, 0, view};
    const float *volt = nullptr;
    if ((st = transposed_if_needed(ctx, vol, view, 1, S(stream), &volt))) return st;
    stt::FpSlabMaps maps{};  // ok = 0: every view gathers, one launch
    if (staged_mask(ctx, vol)) stt::make_fp_slab_maps(ctx->g, vol, volt, maps, ctx->tuning.slab);
    STT_CUDA(ctx, stt::launch_fp_corr(ctx->g, ctx->views_d, vol, volt, sel, b, raylen_state, corr, S(stream), 0, &maps,
                                      ctx->status, ctx->tuning.fp, stt::ctx_fp_tex(ctx, vol, volt)),
             "k_fp_corr launch");
    return STT_OK;
}

stt_status stt_fp_texture_ok_typed(stt_ctx *ctx, const void *vol, int dtype, int *ok) {
    stt_status st = need_geom(ctx);
    if (st) return st;
    if (!vol || !ok) return fail(ctx, STT_ERR_INVALID, "null vol or ok");
    if (dtype != STT_DTYPE_F32 && dtype != STT_DTYPE_BF16) return fail(ctx, STT_ERR_INVALID, "unknown dtype");
    if ((st = set_device(ctx))) return st;
    *ok = stt::fp_tex_fits(ctx->g, vol, dtype == STT_DTYPE_BF16 ? 2 : 4) ? 1 : 0;
    return STT_OK;
}

stt_status stt_fp_texture_ok(stt_ctx *ctx, const float *vol, int *ok) {
    return stt_fp_texture_ok_typed(ctx, vol, STT_DTYPE_F32, ok);
}

stt_status stt_gather_ceiling(stt_ctx *ctx, const float *vol, int view, int packed, float *out, int *count,
                              void *stream) {
    stt_status st = need_geom(ctx);
    if (st) return st;
    if (!vol || !out) return fail(ctx, STT_ERR_INVALID, "null vol or out");
    if ((st = check_views(ctx, view, 1))) return st;
    if ((long long)ctx->g.nx * ctx->g.ny * ctx->g.nz >= (1LL << 31))
        return fail(ctx, STT_ERR_UNSUPPORTED, "the gather ceiling takes volumes below 2^31 voxels");
    if ((st = set_device(ctx))) return st;
    const float *volt = nullptr;
    if ((st = transposed_if_needed(ctx, vol, view, 1, S(stream), &volt))) return st;
    const stt::FpTex *tex = nullptr;
    if (packed & 2) {  // tld4 corners
        tex = stt::ctx_fp_tex_any(ctx, vol, volt);
        if (!tex || !tex->ok)
            return fail(ctx, STT_ERR_UNSUPPORTED, "the device's texture limits do not admit this volume");
    }
    STT_CUDA(ctx, stt::launch_gather_ceiling(ctx->g, ctx->views_d, ctx->views_h[view], view, vol, volt, packed & 1, out,
                                             count, S(stream), tex),
             "k_gather_ceiling launch");
    return STT_OK;
}

stt_status stt_fp_vjp(stt_ctx *ctx, const float *proj_bar, float *vol_bar, int view0, int nviews,
                      void *stream) {
    stt_status st = need_geom(ctx);
    if (st) return st;
    if (!proj_bar || !vol_bar) return fail(ctx, STT_ERR_INVALID, "null proj_bar or vol_bar");
    if ((st = check_views(ctx, view0, nviews))) return st;
    if (nviews == 0) return STT_OK;
    if ((st = set_device(ctx))) return st;
    STT_CUDA(ctx, stt::launch_fp_adjoint(ctx->g, ctx->views_d, view0, nviews, proj_bar, vol_bar, S(stream)),
             "k_fp_adjoint launch");
    return STT_OK;
}

}  // extern "C"

static void ensure_corr_tex(stt_ctx *ctx);

// The caller's correction copied into the context's texture (stream-ordered,
// W*H*4 bytes) for the column backprojection; 0 (the per-voxel load form)
// for volumes under 2^23 voxels, or where the texture cannot be made or the
// copy fails.  Measured per view, copy included: 256^3 / 512^2 102 us against
// 130 us for the load form; 128^3 / 128^2 18.3 us against 13.9 us.
static unsigned long long bp_corr_texture(stt_ctx *ctx, const float *corr, cudaStream_t s) {
    if ((long long)ctx->g.nx * ctx->g.ny * ctx->g.nz < (1LL << 23)) return 0;
    ensure_corr_tex(ctx);
    if (!ctx->corr_tex.tex) return 0;
    const size_t row = (size_t)ctx->g.W * sizeof(float);
    if (cudaMemcpy2DToArrayAsync(ctx->corr_tex.arr, 0, 0, corr, row, row, ctx->g.H, cudaMemcpyDeviceToDevice, s) !=
        cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    return ctx->corr_tex.tex;
}

extern "C" {

stt_status stt_bp_voxel(stt_ctx *ctx, const float *corr, float *vol, double alpha, float gmax,
                        int view, void *stream) {
    stt_status st = need_geom(ctx);
    if (st) return st;
    if (!corr || !vol) return fail(ctx, STT_ERR_INVALID, "null corr or vol");
    if ((st = check_views(ctx, view, 1))) return st;
    if ((st = set_device(ctx))) return st;
    const stt::ViewSel sel{view, nullptr, 0, view};
    const unsigned long long tex = bp_corr_texture(ctx, corr, S(stream));
    STT_CUDA(ctx, stt::launch_bp_voxel(ctx->g, ctx->views_d, sel, corr, vol, (float)alpha, gmax, S(stream), tex,
                                       ctx->tuning.bp),
             "k_bp_voxel launch");
    return STT_OK;
}

stt_status stt_bp_voxel_typed(stt_ctx *ctx, const float *corr, void *vol, int dtype, double alpha, float gmax,
                              int view, void *stream) {
    if (dtype == STT_DTYPE_F32) return stt_bp_voxel(ctx, corr, static_cast<float *>(vol), alpha, gmax, view, stream);
    stt_status st = need_geom(ctx);
    if (st) return st;
    if (dtype != STT_DTYPE_BF16) return fail(ctx, STT_ERR_INVALID, "dtype must be STT_DTYPE_F32 or STT_DTYPE_BF16");
    if (!corr || !vol) return fail(ctx, STT_ERR_INVALID, "null corr or vol");
    if ((st = check_views(ctx, view, 1))) return st;
    if ((st = set_device(ctx))) return st;
    const stt::ViewSel sel{view, nullptr, 0, view};
    const unsigned long long tex = bp_corr_texture(ctx, corr, S(stream));
    STT_CUDA(ctx, stt::launch_bp_voxel(ctx->g, ctx->views_d, sel, corr, static_cast<unsigned short *>(vol),
                                       (float)alpha, gmax, S(stream), tex, ctx->tuning.bp),
             "k_bp_voxel launch");
    return STT_OK;
}

static stt_status ensure_acc(stt_ctx *ctx, cudaStream_t s) {
    const size_t n = (size_t)nvox(ctx);
    if (ctx->acc && ctx->acc_n >= n) return STT_OK;
    stt_status st = ensure(ctx, ctx->acc, ctx->acc_n, n, "ray-BP accumulators");
    if (st) return st;
    STT_CUDA(ctx, cudaMemsetAsync(ctx->acc, 0, n * sizeof(float2), s), "cudaMemsetAsync(accumulators)");
    return STT_OK;
}

stt_status stt_bp_ray(stt_ctx *ctx, const float *corr, float *vol, float gmax, int view, void *stream) {
    stt_status st = need_geom(ctx);
    if (st) return st;
    if (!corr || !vol) return fail(ctx, STT_ERR_INVALID, "null corr or vol");
    if ((st = check_views(ctx, view, 1))) return st;
    if ((st = set_device(ctx))) return st;
    if ((st = ensure_acc(ctx, S(stream)))) return st;
    const stt::ViewSel sel{view, nullptr, 0, view};
    STT_CUDA(ctx, stt::launch_bp_ray(ctx->g, ctx->views_d, sel, corr, ctx->acc, vol, gmax, S(stream), ctx->tuning.ray),
             "k_bp_ray launch");
    return STT_OK;
}

stt_status stt_bp_ray_typed(stt_ctx *ctx, const float *corr, void *vol, int dtype, float gmax, int view,
                            void *stream) {
    if (dtype == STT_DTYPE_F32) return stt_bp_ray(ctx, corr, static_cast<float *>(vol), gmax, view, stream);
    stt_status st = need_geom(ctx);
    if (st) return st;
    if (dtype != STT_DTYPE_BF16) return fail(ctx, STT_ERR_INVALID, "dtype must be STT_DTYPE_F32 or STT_DTYPE_BF16");
    if (!corr || !vol) return fail(ctx, STT_ERR_INVALID, "null corr or vol");
    if ((st = check_views(ctx, view, 1))) return st;
    if ((st = set_device(ctx))) return st;
    if ((st = ensure_acc(ctx, S(stream)))) return st;
    const stt::ViewSel sel{view, nullptr, 0, view};
    STT_CUDA(ctx, stt::launch_bp_ray(ctx->g, ctx->views_d, sel, corr, ctx->acc, static_cast<unsigned short *>(vol),
                                     gmax, S(stream), ctx->tuning.ray),
             "k_bp_ray launch");
    return STT_OK;
}

stt_status stt_bp_ray_scatter(stt_ctx *ctx, const float *corr, float *contrib, float *wsum, int view,
                              void *stream) {
    stt_status st = need_geom(ctx);
    if (st) return st;
    if (!corr || !contrib || !wsum) return fail(ctx, STT_ERR_INVALID, "null corr, contrib or wsum");
    if ((st = check_views(ctx, view, 1))) return st;
    if ((st = set_device(ctx))) return st;
    if ((st = ensure_acc(ctx, S(stream)))) return st;
    const stt::ViewSel sel{view, nullptr, 0, view};
    STT_CUDA(ctx, stt::launch_bp_ray_scatter(ctx->g, ctx->views_d, sel, corr, ctx->acc, contrib, wsum, S(stream),
                                             ctx->tuning.ray),
             "k_bp_ray_scatter launch");
    return STT_OK;
}

}  // extern "C"

// The fused forward projection of one view of a sweep: FP32 through the tuned
// gather variant and, where its maps apply, the slab-staged kernel; BF16
// through the gather kernel and the slab kernel's BF16 boxes.
// The context's texture copy of a W x H correction for the column
// backprojection, made on first use (kept until stt_destroy or a detector of
// another size); where it cannot be made, corr_tex.tex stays 0 and the
// per-voxel load form runs (the same bits).
static void ensure_corr_tex(stt_ctx *ctx) {
    if (ctx->corr_tex.tex && ctx->corr_tex.W == ctx->g.W && ctx->corr_tex.H == ctx->g.H) return;
    // another detector size: launches enqueued earlier (on any stream) may still
    // gather from the old texture, so the device drains before it is destroyed
    if (ctx->corr_tex.tex && cudaDeviceSynchronize() != cudaSuccess) cudaGetLastError();
    stt::free_corr_tex(ctx->corr_tex);
    if (stt::make_corr_tex(ctx->g.W, ctx->g.H, ctx->corr_tex) != cudaSuccess) cudaGetLastError();
}

// surf: also write the correction into the context's texture copy (0: not).
static cudaError_t sweep_fp_corr(stt_ctx *ctx, const float *vol, const float *volt, const stt::ViewSel &sel,
                                 const float *stack, float *rl, cudaStream_t s, unsigned long long surf) {
    stt::FpSlabMaps maps{};  // ok = 0: every view gathers, one launch
    if (staged_mask(ctx, vol)) stt::make_fp_slab_maps(ctx->g, vol, volt, maps, ctx->tuning.slab);
    return stt::launch_fp_corr(ctx->g, ctx->views_d, vol, volt, sel, stack, rl, ctx->corr, s, surf, &maps,
                               ctx->status, ctx->tuning.fp, stt::ctx_fp_tex(ctx, vol, volt));
}

static cudaError_t sweep_fp_corr(stt_ctx *ctx, const unsigned short *vol, const unsigned short *volt,
                                 const stt::ViewSel &sel, const unsigned short *stack, float *rl, cudaStream_t s,
                                 unsigned long long surf) {
    stt::FpSlabMaps maps{};  // ok = 0: every view gathers, one launch
    if (staged_mask(ctx, vol)) stt::make_fp_slab_maps(ctx->g, vol, volt, maps, ctx->tuning.slab);
    return stt::launch_fp_corr(ctx->g, ctx->views_d, vol, volt, sel, stack, rl, ctx->corr, s, surf, &maps,
                               ctx->status, ctx->tuning.fp16, stt::ctx_fp_tex(ctx, vol, volt));
}

template <typename T>
static stt_status sart_sweep_t(stt_ctx *ctx, T *vol, const T *proj_stack, const int *perm, int nperm,
                               int view_offset, double alpha, float gmax, int bp_mode, float *raylen_state,
                               const int *roi_cut, void *stream);

extern "C" {

stt_status stt_sart_sweep(stt_ctx *ctx, float *vol, const float *proj_stack, const int *perm,
                          int nperm, int view_offset, double alpha, float gmax, int bp_mode,
                          float *raylen_state, const int *roi_cut, void *stream) {
    return sart_sweep_t(ctx, vol, proj_stack, perm, nperm, view_offset, alpha, gmax, bp_mode, raylen_state, roi_cut,
                        stream);
}

stt_status stt_sart_sweep_typed(stt_ctx *ctx, void *vol, int dtype, const void *proj_stack, const int *perm,
                                int nperm, int view_offset, double alpha, float gmax, int bp_mode,
                                float *raylen_state, const int *roi_cut, void *stream) {
    if (dtype == STT_DTYPE_F32)
        return sart_sweep_t(ctx, static_cast<float *>(vol), static_cast<const float *>(proj_stack), perm, nperm,
                            view_offset, alpha, gmax, bp_mode, raylen_state, roi_cut, stream);
    if (dtype == STT_DTYPE_BF16)
        return sart_sweep_t(ctx, static_cast<unsigned short *>(vol), static_cast<const unsigned short *>(proj_stack),
                            perm, nperm, view_offset, alpha, gmax, bp_mode, raylen_state, roi_cut, stream);
    return fail(ctx, STT_ERR_INVALID, "dtype must be STT_DTYPE_F32 or STT_DTYPE_BF16");
}

}  // extern "C"

template <typename T>
static stt_status sart_sweep_t(stt_ctx *ctx, T *vol, const T *proj_stack, const int *perm, int nperm,
                               int view_offset, double alpha, float gmax, int bp_mode, float *raylen_state,
                               const int *roi_cut, void *stream) {
    stt_status st = need_geom(ctx);
    if (st) return st;
    if (!vol || !proj_stack || (nperm > 0 && !perm)) return fail(ctx, STT_ERR_INVALID, "null argument");
    if (bp_mode != 0 && bp_mode != 1) return fail(ctx, STT_ERR_INVALID, "bp_mode must be 0 or 1");
    if (bp_mode == 0 && !raylen_state)
        return fail(ctx, STT_ERR_INVALID, "voxel-based SART needs the sticky ray-length state");
    for (int i = 0; i < nperm; ++i)
        if (perm[i] < 0 || view_offset + perm[i] >= ctx->g.n_views || view_offset + perm[i] < 0)
            return fail(ctx, STT_ERR_INVALID, "perm entry outside the view list");
    if ((st = set_device(ctx))) return st;
    cudaStream_t s = S(stream);
    const size_t npix = (size_t)ctx->g.W * ctx->g.H;
    if ((st = ensure(ctx, ctx->corr, ctx->corr_n, npix, "correction image"))) return st;
    if (bp_mode == 1 && (st = ensure_acc(ctx, s))) return st;
    if (bp_mode == 0) ensure_corr_tex(ctx);
    for (int i = 0; i < nperm; ++i) {
        const stt::ViewSel sel{view_offset + perm[i], nullptr, 0, view_offset};
        const T *volt = nullptr;
        if ((st = transposed_if_needed(ctx, vol, view_offset + perm[i], 1, s, &volt))) return st;
        // ray-based mode: TypicalRayProducer::Initial zeroes the ray lengths
        // after every view, so missed rays see L = 0 (no sticky state)
        STT_CUDA(ctx, sweep_fp_corr(ctx, vol, volt, sel, proj_stack, bp_mode == 0 ? raylen_state : nullptr, s,
                                    bp_mode == 0 ? ctx->corr_tex.surf : 0),
                 "k_fp_corr launch");
        if (bp_mode == 0)
            STT_CUDA(ctx, stt::launch_bp_voxel(ctx->g, ctx->views_d, sel, ctx->corr, vol, (float)alpha, gmax, s,
                                               ctx->corr_tex.tex, ctx->tuning.bp),
                     "k_bp_voxel launch");
        else
            STT_CUDA(ctx, stt::launch_bp_ray(ctx->g, ctx->views_d, sel, ctx->corr, ctx->acc, vol, gmax, s,
                                             ctx->tuning.ray),
                     "k_bp_ray launch");
    }
    if (bp_mode == 1 && raylen_state)
        STT_CUDA(ctx, cudaMemsetAsync(raylen_state, 0, npix * sizeof(float), s), "cudaMemsetAsync(raylen)");
    if (roi_cut) {
        const int d[3] = {ctx->g.nx, ctx->g.ny, ctx->g.nz};
        STT_CUDA(ctx, stt::launch_roi_apply(d, roi_cut, nullptr, vol, (const T *)nullptr, (T *)nullptr, s),
                 "k_roi_apply launch");
    }
    return STT_OK;
}

extern "C" {

stt_status stt_sart_view(stt_ctx *ctx, float *vol, const float *b, int view, double alpha, float gmax, int bp_mode,
                         float *raylen_state, void *stream) {
    const int first = 0;
    return stt_sart_sweep(ctx, vol, b, &first, 1, view, alpha, gmax, bp_mode, raylen_state, nullptr, stream);
}

stt_status stt_opnorm_power_iter(stt_ctx *ctx, int n_iter, unsigned long long seed, stt_opnorm *out, void *stream) {
    stt_status st = need_geom(ctx);
    if (st) return st;
    if (!out || n_iter < 1) return fail(ctx, STT_ERR_INVALID, "null out or n_iter < 1");
    if ((st = set_device(ctx))) return st;
    cudaStream_t s = S(stream);
    const long long n = nvox(ctx);
    const long long npix = (long long)ctx->g.W * ctx->g.H;
    const int nv = ctx->g.n_views;
    const int chunk = nv < 32 ? nv : 32;  // projections held at once
    if ((st = ensure(ctx, ctx->pw, ctx->pw_n, (size_t)(2 * n + chunk * npix), "power-iteration vectors"))) return st;
    if ((st = ensure(ctx, ctx->pwd, ctx->pwd_n, (size_t)(3 * n_iter), "power-iteration sums"))) return st;
    float *x = ctx->pw, *ax = ctx->pw + n, *y = ctx->pw + 2 * n;
    STT_CUDA(ctx, cudaMemsetAsync(ctx->pwd, 0, 3 * n_iter * sizeof(double), s), "clear sums");
    STT_CUDA(ctx, stt::launch_fill_seeded(n, seed, x, s), "k_fill_seeded");
    STT_CUDA(ctx, stt::launch_dot_f64(n, x, x, ctx->pwd, s), "k_dot_f64");
    STT_CUDA(ctx, stt::launch_scale_inv_sqrt(n, x, ctx->pwd, s), "k_scale_inv_sqrt");
    for (int it = 0; it < n_iter; ++it) {
        double *sums = ctx->pwd + 3 * it;  // [0] unused at it > 0; [1] <x, A^T A x>; [2] |A^T A x|^2
        STT_CUDA(ctx, stt::launch_fill_zero(ax, n, s), "k_fill_zero");
        for (int v0 = 0; v0 < nv; v0 += chunk) {
            const int k = nv - v0 < chunk ? nv - v0 : chunk;
            if ((st = stt_fp(ctx, x, y, nullptr, nullptr, v0, k, stream))) return st;
            if ((st = stt_fp_vjp(ctx, y, ax, v0, k, stream))) return st;
        }
        STT_CUDA(ctx, stt::launch_dot_f64(n, x, ax, sums + 1, s), "k_dot_f64");
        STT_CUDA(ctx, stt::launch_dot_f64(n, ax, ax, sums + 2, s), "k_dot_f64");
        STT_CUDA(ctx, cudaMemcpyAsync(x, ax, n * sizeof(float), cudaMemcpyDeviceToDevice, s), "copy");
        STT_CUDA(ctx, stt::launch_scale_inv_sqrt(n, x, sums + 2, s), "k_scale_inv_sqrt");
    }
    std::vector<double> h(3 * n_iter);
    STT_CUDA(ctx, cudaMemcpyAsync(h.data(), ctx->pwd, h.size() * sizeof(double), cudaMemcpyDeviceToHost, s),
             "read sums");
    STT_CUDA(ctx, cudaStreamSynchronize(s), "cudaStreamSynchronize");
    const double lam = h[3 * (n_iter - 1) + 1];  // Rayleigh quotient of A^T A at a unit vector
    const double prev = n_iter > 1 ? h[3 * (n_iter - 2) + 1] : lam;
    out->norm_A = std::sqrt(lam > 0.0 ? lam : 0.0);
    out->norm_K = std::sqrt(out->norm_A * out->norm_A + 12.0);
    out->sigma = 0.99 / out->norm_K;
    out->tau = 0.99 / out->norm_K;
    out->iterations = n_iter;
    out->rel_change = lam > 0.0 ? std::fabs(lam - prev) / lam : 0.0;
    return STT_OK;
}

static stt::PdParams to_pd(const stt_pd_params *p) {
    stt::PdParams q;
    q.sigma = p->sigma;
    q.tau = p->tau;
    q.tv_w = p->tv_w;
    q.tp_w = p->tp_w;
    q.bc_w = p->bc_w;
    q.hf = p->huber_factor;
    q.gmax = p->gmax;
    for (int i = 0; i < 8; ++i) q.cut[i] = p->cut[i];
    return q;
}

stt_status stt_pd_dual(stt_ctx *ctx, const stt_pd_params *p, const float *xbar_f, const float *xbar_f1,
                       const float *bw, float *ytv, float *ytp, float *ybc, void *stream) {
    stt_status st = need_geom(ctx);
    if (st) return st;
    if (!p || !xbar_f || !xbar_f1 || !bw || !ytv || !ytp || !ybc) return fail(ctx, STT_ERR_INVALID, "null argument");
    if ((st = set_device(ctx))) return st;
    const int d[3] = {ctx->g.nx, ctx->g.ny, ctx->g.nz};
    STT_CUDA(ctx, stt::launch_pd_dual(d, to_pd(p), xbar_f, xbar_f1, bw, ytv, ytp, ybc, S(stream)), "k_pd_dual launch");
    return STT_OK;
}

stt_status stt_pd_primal(stt_ctx *ctx, const stt_pd_params *p, int first_frame, const float *ytp_prev,
                         const float *ytp, const float *fw, const float *ybc, const float *ytv, float *vol,
                         float *xprev, void *stream) {
    stt_status st = need_geom(ctx);
    if (st) return st;
    if (!p || !ytp || !ybc || !ytv || !vol || !xprev) return fail(ctx, STT_ERR_INVALID, "null argument");
    if (!first_frame && (!ytp_prev || !fw)) return fail(ctx, STT_ERR_INVALID, "ytp_prev and fw needed after frame 0");
    if ((st = set_device(ctx))) return st;
    const int d[3] = {ctx->g.nx, ctx->g.ny, ctx->g.nz};
    STT_CUDA(ctx, stt::launch_pd_primal(d, to_pd(p), first_frame ? 1 : 0, ytp_prev, ytp, fw, ybc, ytv, vol, xprev,
                                        S(stream)),
             "k_pd_primal launch");
    return STT_OK;
}

stt_status stt_pd_extrapolate(stt_ctx *ctx, const int *cut, const float *vol, const float *xprev, float *xbar,
                              void *stream) {
    stt_status st = need_geom(ctx);
    if (st) return st;
    if (!cut || !vol || !xprev || !xbar) return fail(ctx, STT_ERR_INVALID, "null argument");
    if ((st = set_device(ctx))) return st;
    const int d[3] = {ctx->g.nx, ctx->g.ny, ctx->g.nz};
    STT_CUDA(ctx, stt::launch_pd_extrapolate(d, cut, vol, xprev, xbar, S(stream)), "k_pd_extrapolate launch");
    return STT_OK;
}

stt_status stt_roi_mask(stt_ctx *ctx, const int *cut, float *roi, void *stream) {
    stt_status st = need_geom(ctx);
    if (st) return st;
    if (!cut || !roi) return fail(ctx, STT_ERR_INVALID, "null argument");
    if ((st = set_device(ctx))) return st;
    const int d[3] = {ctx->g.nx, ctx->g.ny, ctx->g.nz};
    STT_CUDA(ctx, stt::launch_roi_mask(d, cut, roi, S(stream)), "k_roi_mask launch");
    return STT_OK;
}

static stt_status check_warp_args(const int *dim, const float *vel, const float *src, int nc) {
    if (!dim || !vel || !src) return fail(nullptr, STT_ERR_INVALID, "null argument");
    if (dim[0] < 4 || dim[1] < 4 || dim[2] < 4)
        return fail(nullptr, STT_ERR_INVALID, "warp needs every dimension >= 4");
    if (nc < 1) return fail(nullptr, STT_ERR_INVALID, "nc must be >= 1");
    if ((long long)dim[0] * dim[1] * dim[2] * (nc > 3 ? nc : 3) >= (1LL << 31))
        return fail(nullptr, STT_ERR_INVALID, "warp volume too large for 32-bit tap offsets");
    return STT_OK;
}

// Records an error on a context for code outside this file (not part of the public header).
stt_status stt_internal_set_error(stt_ctx *ctx, stt_status st, const char *msg) {
    return fail(ctx, st, msg ? msg : "");
}

// Solver access to the context's geometry (not part of the public header).
stt_status stt_internal_geom(stt_ctx *ctx, const void **geom, const void **views) {
    stt_status st = need_geom(ctx);
    if (st) return st;
    if ((st = set_device(ctx))) return st;
    *geom = &ctx->g;
    *views = ctx->views_d;
    return STT_OK;
}

stt_status stt_poll_status(stt_ctx *ctx, void *stream) {
    stt_status st = need_geom(ctx);
    if (st) return st;
    if ((st = set_device(ctx))) return st;
    int flag = 0;
    STT_CUDA(ctx, cudaMemcpyAsync(&flag, ctx->status, sizeof(int), cudaMemcpyDeviceToHost, S(stream)),
             "read status word");
    STT_CUDA(ctx, cudaStreamSynchronize(S(stream)), "cudaStreamSynchronize");
    if (!flag) return STT_OK;
    STT_CUDA(ctx, cudaMemsetAsync(ctx->status, 0, sizeof(int), S(stream)), "clear status word");
    STT_CUDA(ctx, cudaStreamSynchronize(S(stream)), "cudaStreamSynchronize");
    return fail(ctx, STT_ERR_TIMEOUT,
                "a bounded device-side wait gave up: a TMA copy into shared memory did not land within about "
                "0.1 s (the results were computed from global memory instead)");
}

stt_status stt_warp_poll_status(void *stream) {
    int flag = 0;
    STT_CUDA(nullptr, stt::warp_poll_status(&flag, S(stream)), "warp status word");
    if (!flag) return STT_OK;
    return fail(nullptr, STT_ERR_TIMEOUT,
                "a bounded device-side wait of a staged warp gave up: its velocity box did not land within about "
                "0.1 s (the warp read global memory instead)");
}

stt_status stt_warp(const int *dim, const float *vel, const float *src, int nc, float dt, float *out,
                    void *stream) {
    stt_status st = check_warp_args(dim, vel, src, nc);
    if (st) return st;
    if (!out) return fail(nullptr, STT_ERR_INVALID, "null out");
    STT_CUDA(nullptr, stt::launch_warp(dim, vel, src, nc, dt, out, S(stream)), "k_warp launch");
    return STT_OK;
}

stt_status stt_warp_typed(const int *dim, const float *vel, const void *src, int dtype, int nc, float dt, float *out,
                          void *stream) {
    if (dtype == STT_DTYPE_F32) return stt_warp(dim, vel, static_cast<const float *>(src), nc, dt, out, stream);
    if (dtype != STT_DTYPE_BF16) return fail(nullptr, STT_ERR_INVALID, "dtype must be STT_DTYPE_F32 or STT_DTYPE_BF16");
    // the argument checks of the FP32 form (they read no element of src)
    stt_status st = check_warp_args(dim, vel, static_cast<const float *>(src), nc);
    if (st) return st;
    if (!out) return fail(nullptr, STT_ERR_INVALID, "null out");
    STT_CUDA(nullptr, stt::launch_warp(dim, vel, static_cast<const unsigned short *>(src), nc, dt, out, S(stream)),
             "k_warp launch");
    return STT_OK;
}

stt_status stt_warp_vjp(const int *dim, const float *vel, const float *src, int nc, float dt,
                        const float *out_bar, float *src_bar, float *vel_bar, void *stream) {
    stt_status st = check_warp_args(dim, vel, src, nc);
    if (st) return st;
    if (!out_bar) return fail(nullptr, STT_ERR_INVALID, "null out_bar");
    STT_CUDA(nullptr, stt::launch_warp_vjp(dim, vel, src, nc, dt, out_bar, src_bar, vel_bar, S(stream)),
             "k_warp_vjp launch");
    return STT_OK;
}

}  // extern "C"
