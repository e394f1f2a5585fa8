// oracle/ref_st_driver.cpp -- TEST INFRASTRUCTURE ONLY.
//
// Runs the reference's own ST_Tomography class (SpaceTimeTomography/ST_Tomo/
// ST_Tomography.cpp, unmodified) so that the oracle's restatement of its loops
// (oracle/stt_oracle.cpp: the SART correction, the voxel- and ray-driven
// backprojection, the primal-dual dual/primal steps, the ROI mask and the
// over-relaxation) can be checked against the real thing.  oracle/Makefile
// compiles this file with ST_Tomography.cpp and the projector, scene and math
// sources where they lie into oracle/_ref/libstt_ref_st.so, with the
// compile-only stand-ins of oracle/shims (Eigen's MatrixXf, a libtiff that
// drops what is written, no-op GL calls).  Nothing in the product links or
// loads this library.
//
// The reference takes its inputs from files and globals, and this driver
// provides them:
//   - the per-frame start angles come from "lds.txt" in the working directory
//     (ST_Tomography.cpp:258-269): written into `workdir` first;
//   - the projection stack is read by SetData through CImg (:355): written as a
//     .cimg file, which CImg reads without libtiff;
//   - the volumes and flows are VolumeData's public lists (VolumeData.h:97-98),
//     filled directly (the reference reads them from TIFF files, :103-129);
//   - the ROI cut, the joint-iteration count and G_Max are globals
//     (ST_Tomography.cpp:95, 114, 82) set before / after SetData.
// Three C library calls are wrapped at link time (-Wl,--wrap):
//   - time(): SART seeds its view shuffle with srand(time(0)) (:635); the
//     wrapped clock is a counter, so the run is repeatable;
//   - srand(): every seed the reference draws with is logged, so that
//     ref_st_shuffle() can return the view order each SART call used;
//   - exit(): Render ends with exit(0) (:611); while Render runs, the wrapper
//     jumps back to ref_st_run instead of ending the process.
#include <csetjmp>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <ctime>
#include <string>
#include <vector>

#include <omp.h>
#include <unistd.h>

#include "ST_Tomography.h"
#include "VolumeData.h"

using cimg_library::CImg;
using cimg_library::CImgList;

// Globals of ST_Tomography.cpp (external linkage there).
extern int cut[];
extern int Joint_iter;
extern float G_Max;
extern CImgList<float> Projslist, X_bar, X_prev, Y_tv, Y_tp, Y_bc;
int myrandom(int i);

extern "C" {
time_t __real_time(time_t *t);
void __real_srand(unsigned seed);
void __real_exit(int code) __attribute__((noreturn));
}

namespace {

time_t g_clock = 1000;
std::vector<unsigned> g_seeds;
bool g_in_render = false;
std::jmp_buf g_render_exit;
double g_run_seconds = 0.0;

// Render's view of the scene: AbstractScene::Render is public.
void run_render(ST_Tomography *st) { static_cast<AbstractScene *>(st)->Render(); }

}  // namespace

extern "C" {

time_t __wrap_time(time_t *t) {
    const time_t v = g_clock++;
    if (t) *t = v;
    return v;
}

void __wrap_srand(unsigned seed) {
    g_seeds.push_back(seed);
    __real_srand(seed);
}

void __wrap_exit(int code) {
    if (g_in_render) std::longjmp(g_render_exit, 1);
    __real_exit(code);
}

struct ref_st_cfg {
    int dims[3];
    float sp[3];
    int W, H;
    double ds, sid, sdd;
    double oxyz[3];
    int nframes, nrounds;  // views per frame: 10 * nrounds (main.cpp:148)
    int bp_mode;           // 0 voxel-based, 1 ray-based (--bp)
    double alpha;          // -a
    double tv_w, tp_w, bc_w, huber;  // -l, -k, -e, --huber (ST_Tomography ctor d3..d6)
    int cut[8];            // ROI cut (the global of ST_Tomography.cpp:114)
    int joint_iters;       // Joint_iter (:95); Render only
    float gmax;            // > 0: overrides G_Max after SetData (:356-357)
    int threads;           // OpenMP threads (1: the racy ray-BP scatter becomes sequential)
};

// Wall time of the SART calls (mode 0) or of Render (mode 1) in the last
// ref_st_run, without the scene set-up around them.
double ref_st_last_run_seconds(void) { return g_run_seconds; }

// The view order the reference's SART draws after srand(seed): the two
// random_shuffle calls of ST_Tomography.cpp:636-642.
void ref_st_shuffle(unsigned seed, int n, int *out) {
    __real_srand(seed);
    std::vector<int> v;
    for (int i = 0; i < n; ++i) v.push_back(i);
    std::random_shuffle(v.begin(), v.end());
    std::random_shuffle(v.begin(), v.end(), myrandom);
    for (int i = 0; i < n; ++i) out[i] = v[i];
}

// Builds the reference's scene from the inputs and runs it.
//   mode 0: SART(f) once for every frame f in order (ST_Tomography.cpp:616-808);
//   mode 1: Render(), the joint loop (:397-614), with cfg->joint_iters outer
//           iterations: flow phase every iteration, image phase (two
//           primal-dual passes over all frames) from the second on.
// Inputs: start_deg[nframes * nrounds] (the lds.txt rows), proj W*H*(V*F)
// (frame f's V projections are slices f*V .. f*V+V-1), vols F volumes (the
// duplicated last frame is added here, VolumeData.cpp:124-126), flows F
// 3-channel fields (planar; the reference keeps F of them, VolumeData.cpp).
// Outputs (any may be null): vol F volumes, xbar F+1, xprev F+1, ytv (F+1)*3,
// ytp F+1, ybc F+1, flow F*3; seeds: every srand seed (up to *n_seeds in, the
// count out); gmax_out: the G_Max the run used.
int ref_st_run(const ref_st_cfg *c, const float *start_deg, const char *workdir, const float *proj,
               const float *vols, const float *flows, int mode, float *vol_out, float *xbar_out,
               float *xprev_out, float *ytv_out, float *ytp_out, float *ybc_out, float *flow_out,
               unsigned *seeds, int *n_seeds, float *gmax_out) {
    const int F = c->nframes, V = 10 * c->nrounds;
    const size_t n = (size_t)c->dims[0] * c->dims[1] * c->dims[2];
    char cwd[4096];
    if (!getcwd(cwd, sizeof cwd)) return -1;
    if (chdir(workdir) != 0) return -2;
    int rc = 0;
    ST_Tomography *st = nullptr;
    VolumeData *vd = nullptr;
    try {
        omp_set_num_threads(c->threads > 0 ? c->threads : 1);
        FILE *lf = std::fopen("lds.txt", "w");
        if (!lf) throw -3;
        for (int f = 0; f < F; ++f) {
            for (int r = 0; r < c->nrounds; ++r) std::fprintf(lf, "%.9g ", (double)start_deg[f * c->nrounds + r]);
            std::fprintf(lf, "\n");
        }
        std::fclose(lf);
        CImg<float>(proj, c->W, c->H, V * F, 1).save_cimg("proj.cimg");
        for (int k = 0; k < 8; ++k) cut[k] = c->cut[k];
        Joint_iter = c->joint_iters;
        Projslist.assign();  // SetData appends to it (:355)

        vd = new VolumeData;
        int dims[3] = {c->dims[0], c->dims[1], c->dims[2]};
        float sp[3] = {c->sp[0], c->sp[1], c->sp[2]};
        vd->SetDimensions(dims);
        vd->SetSpacings(sp);
        for (int f = 0; f < F; ++f) vd->m_Volumelist.insert(CImg<float>(vols + f * n, dims[0], dims[1], dims[2], 1));
        vd->m_Volumelist.insert(CImg<float>(vols + (F - 1) * n, dims[0], dims[1], dims[2], 1));
        for (int f = 0; f < F; ++f)
            vd->m_Flowlist.insert(CImg<float>(flows + f * 3 * n, dims[0], dims[1], dims[2], 3));

        int imgwh[2] = {c->W, c->H};
        double oxyz[3] = {c->oxyz[0], c->oxyz[1], c->oxyz[2]};
        std::vector<const char *> inputs(F, "proj.cimg");
        std::vector<double> startdg(F, 0.0);
        st = new ST_Tomography(0.0, 0.0, c->tv_w, c->tp_w, c->bc_w, c->huber, "sart_out", imgwh, V, 1, 1, c->alpha,
                               c->sid, inputs.data(), oxyz, c->sdd, c->ds, "ATV",
                               c->bp_mode ? "Raybased" : "Voxelbased", dims, F, startdg.data(), c->nrounds);
        st->SetData(vd);
        // GLUT's reshape callback, which runs before the first display
        // (GLUTSceneContainer.cpp:108-113): the producer's viewport is set here
        st->Resize(c->W, c->H);
        if (c->gmax > 0.0f) G_Max = c->gmax;
        if (gmax_out) *gmax_out = G_Max;
        g_seeds.clear();
        const double t0 = omp_get_wtime();
        if (mode == 0) {
            for (int f = 0; f < F; ++f) st->SART(f);
        } else {
            g_in_render = true;
            if (setjmp(g_render_exit) == 0) run_render(st);
            g_in_render = false;
        }
        g_run_seconds = omp_get_wtime() - t0;
        auto put = [&](float *dst, const CImgList<float> &L, int count, int nc) {
            if (!dst) return;
            for (int f = 0; f < count; ++f) std::memcpy(dst + f * nc * n, L[f].data(), sizeof(float) * nc * n);
        };
        put(vol_out, vd->m_Volumelist, F, 1);
        put(xbar_out, X_bar, F + 1, 1);
        put(xprev_out, X_prev, F + 1, 1);
        put(ytv_out, Y_tv, F + 1, 3);
        put(ytp_out, Y_tp, F + 1, 1);
        put(ybc_out, Y_bc, F + 1, 1);
        put(flow_out, vd->m_Flowlist, F, 3);
        if (n_seeds) {
            const int cap = *n_seeds;
            for (int k = 0; k < (int)g_seeds.size() && k < cap; ++k) seeds[k] = g_seeds[k];
            *n_seeds = (int)g_seeds.size();
        }
    } catch (int e) {
        rc = e;
    } catch (...) {
        rc = -4;
    }
    g_in_render = false;
    // The reference's globals outlive the scene; empty them for the next run.
    Projslist.assign();
    X_bar.assign();
    X_prev.assign();
    Y_tv.assign();
    Y_tp.assign();
    Y_bc.assign();
    delete st;
    delete vd;
    if (chdir(cwd) != 0 && rc == 0) rc = -5;
    return rc;
}

}  // extern "C"
