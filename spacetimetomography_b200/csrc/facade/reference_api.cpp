// reference_api.cpp -- the classes and free functions of include/reference/,
// which keep the reference's names and calls (gmzang/SpaceTimeTomography,
// S/ = SpaceTimeTomography/) and run them on libstt's C ABI.
#include <cuda_runtime_api.h>
#include <sys/stat.h>

#include <cerrno>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iostream>
#include <stdexcept>
#include <string>
#include <vector>

#include "RayCaster.core.h"
#include "ST_Tomography.h"
#include "SingleScalarVolume.core.h"
#include "TypicalRayProducer.core.h"
#include "VolumeData.h"
#include "stt.h"
#include "stt_host.h"

namespace {

void check_stt(int st, stt_ctx *ctx, const char *what) {
    if (st != STT_OK) throw std::runtime_error(std::string(what) + ": " + stt_last_error(ctx));
}

void check_cuda(cudaError_t e, const char *what) {
    if (e != cudaSuccess) throw std::runtime_error(std::string(what) + ": " + cudaGetErrorString(e));
}

template <typename T>
T *dev_alloc(size_t n) {
    void *p = nullptr;
    check_cuda(cudaMalloc(&p, std::max<size_t>(n, 1) * sizeof(T)), "cudaMalloc");
    return static_cast<T *>(p);
}

stt::Image read_tiff(const std::string &path) {
    int w = 0, h = 0, d = 0;
    float *data = nullptr;
    if (stt_tiff_read(path.c_str(), &w, &h, &d, &data) != 0) throw std::runtime_error(stt_host_last_error());
    stt::Image img(w, h, d, 1);
    std::memcpy(img.data(), data, sizeof(float) * img.size());
    stt_host_free(data);
    return img;
}

// mkdir -p of the directory part of `path`.
void make_parent_dirs(const std::string &path) {
    for (size_t at = path.find('/', 1); at != std::string::npos; at = path.find('/', at + 1)) {
        const std::string dir = path.substr(0, at);
        if (mkdir(dir.c_str(), 0755) != 0 && errno != EEXIST)
            throw std::runtime_error("cannot create directory " + dir + ": " + std::strerror(errno));
    }
}

void write_tiff(const std::string &path, const stt::Image &img) {
    make_parent_dirs(path);
    if (stt_tiff_write(path.c_str(), img.width(), img.height(), img.depth() * img.spectrum(), img.data()) != 0)
        throw std::runtime_error(stt_host_last_error());
}

// The reference's ROI mask (ST_Tomography.cpp:303-329), including its literal
// 7 in the y test.
const int kCut[8] = {8, 8, 8, 45, 8, 8, 30, 20};

}  // namespace

// ===========================================================================
// VolumeData (S/ImageFormationModel/VolumeData.cpp)

VolumeData::VolumeData() = default;

VolumeData::VolumeData(int d1, int d2, int d3, float sp1, float sp2, float sp3, float *data) {
    m_Dims[0] = m_volX = d1;
    m_Dims[1] = m_volY = d2;
    m_Dims[2] = m_volZ = d3;
    m_Spacings[0] = sp1;
    m_Spacings[1] = sp2;
    m_Spacings[2] = sp3;
    m_nframes = 1;
    stt::Image v(d1, d2, d3, 1);
    if (data) std::memcpy(v.data(), data, sizeof(float) * v.size());
    m_Volumelist = {v, v};
    m_Flowlist = {stt::Image(d1, d2, d3, 3)};
}

VolumeData::~VolumeData() = default;

void VolumeData::Clean() {
    m_Volumelist.clear();
    m_Flowlist.clear();
}

void VolumeData::GetDimensions(int *dims) const { std::memcpy(dims, m_Dims, sizeof(m_Dims)); }
void VolumeData::SetDimensions(const int *dims) { std::memcpy(m_Dims, dims, sizeof(m_Dims)); }
void VolumeData::GetSpacings(float *spacings) const { std::memcpy(spacings, m_Spacings, sizeof(m_Spacings)); }
void VolumeData::SetSpacings(const float *spacings) { std::memcpy(m_Spacings, spacings, sizeof(m_Spacings)); }

stt::Image VolumeData::GetData(int iframe) { return m_Volumelist.at(iframe); }

void VolumeData::SetData(std::vector<stt::Image> _vol_list) { m_Volumelist = std::move(_vol_list); }

void VolumeData::setParas(int *vols, double vs, int nframes) {
    m_volX = vols[0];
    m_volY = vols[1];
    m_volZ = vols[2];
    Vol_Spacing = vs;
    m_nframes = nframes;
}

void VolumeData::_allocate() {
    m_Volumelist.assign(m_nframes + 1, stt::Image(m_Dims[0], m_Dims[1], m_Dims[2], 1));
    m_Flowlist.assign(m_nframes, stt::Image(m_Dims[0], m_Dims[1], m_Dims[2], 3));
}

void VolumeData::ReadStructuredFile() {
    m_Dims[0] = m_volX;
    m_Dims[1] = m_volY;
    m_Dims[2] = m_volZ;
    m_Spacings[0] = m_Spacings[1] = m_Spacings[2] = (float)Vol_Spacing;
    m_Flowlist.assign(m_nframes, stt::Image(m_Dims[0], m_Dims[1], m_Dims[2], 3));
    m_Volumelist.clear();
    for (int i = 0; i < m_nframes; ++i) {
        char name[64];
        std::snprintf(name, sizeof(name), "/rose.-%03d-frame-9iter.tiff", i);
        stt::Image v = read_tiff(m_InputDir + name);
        if (v.width() != m_Dims[0] || v.height() != m_Dims[1] || v.depth() != m_Dims[2])
            throw std::runtime_error(m_InputDir + name + ": size differs from the volume size given");
        m_Volumelist.push_back(std::move(v));
    }
    m_Volumelist.push_back(m_Volumelist[m_nframes - 1]);
}

// ===========================================================================
// TypicalRayProducer (S/ImageFormationModel/TypicalRayProducer.{h,cpp,core.h})

TypicalRayProducer::TypicalRayProducer(int volX, int volY, int volZ, int imgW, int imgH, double ds, const char *_bp)
    : m_ds(ds) {
    (void)_bp;
    m_ViewPort[0] = imgW;
    m_ViewPort[1] = imgH;
    m_VolDims[0] = volX;
    m_VolDims[1] = volY;
    m_VolDims[2] = volZ;
    for (int a = 0; a < 3; ++a) m_VolSize[a] = (float)(m_VolDims[a] - 1) * m_VolSpacings[a];
    for (int k = 0; k < 16; ++k) m_ViewMatrix[k] = m_ProjectionMatrix[k] = (k % 5 == 0) ? 1.0f : 0.0f;
    const size_t npix = (size_t)imgW * imgH;
    m_ImageData.assign(npix, 0.0f);
    m_WeightOfImage.assign(npix, 0.0f);
    m_imageraylength.assign(npix, 0.0f);
    m_CorrectionStore.assign(npix, 0.0f);
    m_Correction = m_CorrectionStore.data();
    check_stt(stt_create(&m_ctx, 0), nullptr, "stt_create");
}

TypicalRayProducer::~TypicalRayProducer() {
    for (float *p : {d_vol, d_img, d_rl, d_wt, d_corr, d_contrib, d_wsum}) cudaFree(p);
    stt_destroy(m_ctx);
}

void TypicalRayProducer::SetViewPort(int width, int height) {
    m_ViewPort[0] = width;
    m_ViewPort[1] = height;
    const size_t npix = (size_t)width * height;
    m_ImageData.assign(npix, 0.0f);
    m_WeightOfImage.assign(npix, 0.0f);
    m_imageraylength.assign(npix, 0.0f);
    m_CorrectionStore.assign(npix, 0.0f);
    m_Correction = m_CorrectionStore.data();
    m_geometry_set = false;
}

void TypicalRayProducer::SetVolSize(const int volDims[3], const float volSpacings[3]) {
    for (int a = 0; a < 3; ++a) {
        m_VolDims[a] = volDims[a];
        m_VolSpacings[a] = volSpacings[a];
        m_VolSize[a] = (float)(volDims[a] - 1) * volSpacings[a];  // TypicalRayProducer.cpp:116-118
    }
    m_geometry_set = false;
}

void TypicalRayProducer::GetVolSize(int volDims[3], float volSpacings[3]) {
    for (int a = 0; a < 3; ++a) {
        volDims[a] = m_VolDims[a];
        volSpacings[a] = m_VolSpacings[a];
    }
}

void TypicalRayProducer::SetViewMatrix(const float *view) {
    std::memcpy(m_ViewMatrix, view, sizeof(m_ViewMatrix));
    m_geometry_set = false;
}

void TypicalRayProducer::SetProjectionMatrix(const float *projection) {
    std::memcpy(m_ProjectionMatrix, projection, sizeof(m_ProjectionMatrix));
    m_geometry_set = false;
}

// The scene's matrices (Scene.cpp:181-207): view = T(t) * R_y(theta) with
// t = (-ox, -oz, oy - sid), projection = the frustum with near plane sdd and
// half widths (W-1)ds/2, (H-1)ds/2.  Only oy - sid enters the geometry, so oy
// is folded into sid.
void TypicalRayProducer::UpdateMatrixAndBounds() {
    const float *V = m_ViewMatrix, *P = m_ProjectionMatrix;
    const double c = V[0], s = V[8];
    const double tol = 1e-4;
    if (std::fabs(V[5] - 1.0) > tol || std::fabs(V[1]) > tol || std::fabs(V[4]) > tol || std::fabs(V[6]) > tol ||
        std::fabs(V[9]) > tol || std::fabs(V[2] + s) > tol || std::fabs(V[10] - c) > tol ||
        std::fabs(c * c + s * s - 1.0) > 10 * tol)
        throw std::runtime_error("TypicalRayProducer: the view matrix is not a unit-scale rotation about y");
    if (P[11] != -1.0f || P[15] != 0.0f || P[0] <= 0.0f || P[5] <= 0.0f)
        throw std::runtime_error("TypicalRayProducer: the projection matrix is not a perspective frustum");
    const double n = (double)P[14] / ((double)P[10] - 1.0);
    const double hw = n / P[0];
    m_theta = std::atan2(s, c);
    m_off[0] = -(double)V[12];
    m_off[2] = -(double)V[13];
    m_off[1] = 0.0;
    m_sid = -(double)V[14];
    m_sdd = n;
    if (m_ViewPort[0] > 1) m_ds = 2.0 * hw / (m_ViewPort[0] - 1);
    m_geometry_set = false;
    SetViewAngle(m_theta, m_sid, m_sdd, m_off);
}

void TypicalRayProducer::SetViewAngle(double theta_rad, double sid, double sdd, const double offset[3]) {
    m_theta = theta_rad;
    m_sid = sid;
    m_sdd = sdd;
    for (int a = 0; a < 3; ++a) m_off[a] = offset[a];
    stt_geometry g{};
    g.nx = m_VolDims[0];
    g.ny = m_VolDims[1];
    g.nz = m_VolDims[2];
    g.sx = m_VolSpacings[0];
    g.sy = m_VolSpacings[1];
    g.sz = m_VolSpacings[2];
    g.W = m_ViewPort[0];
    g.H = m_ViewPort[1];
    g.ds = m_ds;
    g.sid = m_sid;
    g.sdd = m_sdd;
    for (int a = 0; a < 3; ++a) g.off[a] = m_off[a];
    g.n_views = 1;
    g.angles_rad = &m_theta;
    check_stt(stt_set_geometry(m_ctx, &g), m_ctx, "stt_set_geometry");
    m_geometry_set = true;
}

void TypicalRayProducer::GetImageInUseSize(int imageSize[2]) {
    imageSize[0] = m_ViewPort[0];
    imageSize[1] = m_ViewPort[1];
}

void TypicalRayProducer::GetImageOrigin(int imageOrigin[2]) { imageOrigin[0] = imageOrigin[1] = 0; }

void TypicalRayProducer::_ensure_device() {
    const size_t n = (size_t)m_VolDims[0] * m_VolDims[1] * m_VolDims[2];
    const size_t npix = (size_t)m_ViewPort[0] * m_ViewPort[1];
    if (d_vol_n != n) {
        for (float **p : {&d_vol, &d_contrib, &d_wsum}) {
            cudaFree(*p);
            *p = dev_alloc<float>(n);
        }
        check_cuda(cudaMemset(d_contrib, 0, n * sizeof(float)), "clear contributions");
        check_cuda(cudaMemset(d_wsum, 0, n * sizeof(float)), "clear weights");
        d_vol_n = n;
    }
    if (d_img_n != npix) {
        for (float **p : {&d_img, &d_rl, &d_wt, &d_corr}) {
            cudaFree(*p);
            *p = dev_alloc<float>(npix);
        }
        d_img_n = npix;
    }
}

void TypicalRayProducer::Initial() {
    m_Voxel_Contributions.clear();
    m_EachVoxel_TotalWeight.clear();
    if (d_vol_n) {
        check_cuda(cudaMemset(d_contrib, 0, d_vol_n * sizeof(float)), "clear contributions");
        check_cuda(cudaMemset(d_wsum, 0, d_vol_n * sizeof(float)), "clear weights");
    }
    m_scatter_dirty = false;
}

void TypicalRayProducer::_runForward(const float *vol_host, int frame) {
    (void)frame;
    if (!m_geometry_set) UpdateMatrixAndBounds();
    _ensure_device();
    const size_t npix = (size_t)m_ViewPort[0] * m_ViewPort[1];
    check_cuda(cudaMemcpy(d_vol, vol_host, d_vol_n * sizeof(float), cudaMemcpyHostToDevice), "upload volume");
    check_cuda(cudaMemcpy(d_rl, m_imageraylength.data(), npix * sizeof(float), cudaMemcpyHostToDevice),
               "upload ray lengths");
    check_stt(stt_fp(m_ctx, d_vol, d_img, d_rl, d_wt, 0, 1, nullptr), m_ctx, "stt_fp");
    check_cuda(cudaMemcpy(m_ImageData.data(), d_img, npix * sizeof(float), cudaMemcpyDeviceToHost), "image");
    check_cuda(cudaMemcpy(m_imageraylength.data(), d_rl, npix * sizeof(float), cudaMemcpyDeviceToHost), "ray length");
    check_cuda(cudaMemcpy(m_WeightOfImage.data(), d_wt, npix * sizeof(float), cudaMemcpyDeviceToHost), "weight");
}

void TypicalRayProducer::_runBackward() {
    if (!m_geometry_set) UpdateMatrixAndBounds();
    _ensure_device();
    const size_t npix = (size_t)m_ViewPort[0] * m_ViewPort[1];
    check_cuda(cudaMemcpy(d_corr, m_Correction, npix * sizeof(float), cudaMemcpyHostToDevice), "upload correction");
    check_stt(stt_bp_ray_scatter(m_ctx, d_corr, d_contrib, d_wsum, 0, nullptr), m_ctx, "stt_bp_ray_scatter");
    m_scatter_dirty = true;
}

void TypicalRayProducer::_download_scatter() {
    if (!d_vol_n) {
        m_Voxel_Contributions.assign((size_t)m_VolDims[0] * m_VolDims[1] * m_VolDims[2], 0.0f);
        m_EachVoxel_TotalWeight = m_Voxel_Contributions;
        return;
    }
    m_Voxel_Contributions.resize(d_vol_n);
    m_EachVoxel_TotalWeight.resize(d_vol_n);
    check_cuda(cudaMemcpy(m_Voxel_Contributions.data(), d_contrib, d_vol_n * 4, cudaMemcpyDeviceToHost), "contrib");
    check_cuda(cudaMemcpy(m_EachVoxel_TotalWeight.data(), d_wsum, d_vol_n * 4, cudaMemcpyDeviceToHost), "weights");
    m_scatter_dirty = false;
}

float *TypicalRayProducer::GetContributions() {
    if (m_scatter_dirty || m_Voxel_Contributions.empty()) _download_scatter();
    return m_Voxel_Contributions.data();
}

float *TypicalRayProducer::GetTotalWeight() {
    if (m_scatter_dirty || m_EachVoxel_TotalWeight.empty()) _download_scatter();
    return m_EachVoxel_TotalWeight.data();
}

// ===========================================================================
// free functions of the .core.h files

namespace {
struct Binding {
    const float *vol = nullptr;
    bool backward = false;
};
thread_local Binding g_binding;
}  // namespace

bool SingleScalarVolumePrepare(VolumeData *volume, TypicalRayProducer *producer, int frame) {
    if (!volume || !producer) return false;
    if (frame < 0 || frame >= (int)volume->m_Volumelist.size()) return false;
    const stt::Image &v = volume->m_Volumelist[frame];
    if (v.width() != producer->m_VolDims[0] || v.height() != producer->m_VolDims[1] ||
        v.depth() != producer->m_VolDims[2])
        return false;
    g_binding.vol = v.data();
    g_binding.backward = volume->GetProjectionMode();
    producer->_frame = frame;
    return true;
}

bool RayCasterPrepare(RayCaster *caster, int dims[3]) {
    (void)dims;
    return caster != nullptr;
}

void GenerateImage_GetCorrections(TypicalRayProducer *producer) {
    if (!producer) return;
    if (g_binding.backward) producer->_runBackward();
    else if (g_binding.vol) producer->_runForward(g_binding.vol, producer->_frame);
    else throw std::runtime_error("GenerateImage_GetCorrections: no volume bound (SingleScalarVolumePrepare)");
}

// ===========================================================================
// ST_Tomography (S/ST_Tomo/ST_Tomography.cpp)

struct ST_Tomography::Device {
    stt_ctx *ctx = nullptr;
    stt_solver *solver = nullptr;
    stt_flow *flow = nullptr;
    cudaStream_t stream = nullptr;
    size_t n = 0;
    float *vol = nullptr, *xbar = nullptr, *xprev = nullptr, *ytv = nullptr, *ytp = nullptr, *ybc = nullptr,
          *flowv = nullptr, *proj = nullptr, *raylen = nullptr, *tmp = nullptr;
    ~Device() {
        if (solver) stt_solver_destroy(solver);
        if (flow) stt_flow_destroy(flow);
        for (float *p : {vol, xbar, xprev, ytv, ytp, ybc, flowv, proj, raylen, tmp}) cudaFree(p);
        if (stream) cudaStreamDestroy(stream);
        if (ctx) stt_destroy(ctx);
    }
};

ST_Tomography::ST_Tomography(double d1, double d2, double d3, double d4, double d5, double d6, const char *outputfile,
                             int *imgwh, int projNo, int iters, int sartiters, double alp, double sid,
                             const char **projsfile, double *oxyz, double sdd, double ds, const char *_prior,
                             const char *_bp, int *volxyz, int nframes, double *startdg, int nrounds)
    : m_nframes(nframes), m_nrounds(nrounds), m_projno(projNo), m_W(imgwh[0]), m_H(imgwh[1]), m_alpha(alp),
      m_sid(sid), m_sdd(sdd), m_ds(ds) {
    (void)d1;
    (void)d2;
    (void)iters;
    (void)sartiters;
    (void)startdg;
    for (int a = 0; a < 3; ++a) {
        m_vol[a] = volxyz[a];
        m_oxyz[a] = oxyz ? oxyz[a] : 0.0;
    }
    // ST_Tomography.cpp:214-227; CP_sigma = 0.9 / (L * CP_tau) with L = 8, CP_tau = 1 (:98-102)
    const float cp_sigma = 0.9f / (8.0f * 1.0f);
    m_tv_w = (float)d3;
    m_tp_w = (float)d4;
    m_bc_w = (float)d5;
    m_huberfactor = 1.0f / (1.0f + cp_sigma * (float)d6 / (float)d3);
    m_bp_mode = (_bp && std::strcmp(_bp, "Raybased") == 0) ? 1 : 0;
    m_prior = _prior ? _prior : "ATV";
    m_output = outputfile ? outputfile : "Test/test";
    m_proj_file = (projsfile && projsfile[0]) ? projsfile[0] : "proj";
    m_idxSART.assign(nframes, 1);
    SetLdsFile("lds.txt");
}

// Start angles, frame-major, one per round (ST_Tomography.cpp:258-276).
void ST_Tomography::SetLdsFile(const std::string &path) {
    m_lds_file = path;
    m_startDegree.assign(m_nframes, std::vector<float>(m_nrounds, 0.0f));
    std::ifstream lds(m_lds_file);
    if (lds) {
        for (int i = 0; i < m_nframes; ++i)
            for (int r = 0; r < m_nrounds; ++r) lds >> m_startDegree[i][r];
    } else {
        std::cerr << "ST_Tomography: " << m_lds_file
                  << " not found; using the van der Corput start angles it is generated from\n";
        std::vector<double> seq((size_t)10 * m_nframes * m_nrounds);
        check_stt(stt_lds_angles((int)seq.size(), 10, 2, 10000, seq.data()), nullptr, "stt_lds_angles");
        for (int i = 0; i < m_nframes; ++i)
            for (int r = 0; r < m_nrounds; ++r) m_startDegree[i][r] = (float)seq[(size_t)10 * (i * m_nrounds + r)];
    }
    if (m_Data) InitViews();
    m_dev.reset();
}

ST_Tomography::~ST_Tomography() = default;

void ST_Tomography::SetBackGroundColor(float r, float g, float b) {
    m_bg[0] = r;
    m_bg[1] = g;
    m_bg[2] = b;
}
void ST_Tomography::GetBackGroundColor(float &r, float &g, float &b) {
    r = m_bg[0];
    g = m_bg[1];
    b = m_bg[2];
}
void ST_Tomography::SetSurfaceColor(float r, float g, float b) {
    m_surface[0] = r;
    m_surface[1] = g;
    m_surface[2] = b;
}
void ST_Tomography::GetSurfaceColor(float &r, float &g, float &b) {
    r = m_surface[0];
    g = m_surface[1];
    b = m_surface[2];
}
void ST_Tomography::SetLightDirection(float x, float y, float z) {
    m_light_dir[0] = x;
    m_light_dir[1] = y;
    m_light_dir[2] = z;
}
void ST_Tomography::SetLightColor(float r, float g, float b) {
    m_light_color[0] = r;
    m_light_color[1] = g;
    m_light_color[2] = b;
}
void ST_Tomography::Resize(int width, int height) {
    m_W = width;
    m_H = height;
}

void ST_Tomography::GetSize3D(float size[3]) {
    float sp[3] = {1, 1, 1};
    if (m_Data) m_Data->GetSpacings(sp);
    for (int a = 0; a < 3; ++a) size[a] = m_vol[a] * sp[a];
}

// InitViews / RotateVolume (ST_Tomography.cpp:865-934): per frame, rounds of
// 10 views 36 degrees apart from each round's start angle.
void ST_Tomography::InitViews() {
    m_angles.assign(m_nframes, {});
    for (int i = 0; i < m_nframes; ++i) {
        std::vector<double> starts(m_startDegree[i].begin(), m_startDegree[i].end());
        std::vector<double> a((size_t)10 * m_nrounds);
        check_stt(stt_views_from_rounds(m_nrounds, starts.data(), 10, 36.0, a.data()), nullptr,
                  "stt_views_from_rounds");
        a.resize(std::min<size_t>(a.size(), (size_t)m_projno));
        m_angles[i] = a;
    }
}

bool ST_Tomography::RotateVolume(int i) { return i >= 0 && i < m_nframes; }

std::vector<double> ST_Tomography::ViewAngles(int f) const { return m_angles.at(f); }

void ST_Tomography::SetData(VolumeData *data) {
    m_Data = data;
    if (!data) return;
    int dims[3];
    data->GetDimensions(dims);
    for (int a = 0; a < 3; ++a) m_vol[a] = dims[a];
    if ((int)data->m_Volumelist.size() < m_nframes + 1 || (int)data->m_Flowlist.size() < m_nframes)
        throw std::runtime_error("SetData: the volume list needs nframes + 1 volumes and nframes flows");
    // the projection stack, split along z into the frames (ST_Tomography.cpp:355-357)
    m_projs = read_tiff(m_proj_file);
    if (m_projs.width() != m_W || m_projs.height() != m_H || m_projs.depth() != m_projno * m_nframes)
        throw std::runtime_error(m_proj_file + ": expected " + std::to_string(m_W) + " x " + std::to_string(m_H) +
                                 " x " + std::to_string(m_projno * m_nframes) + " (W x H x views*frames)");
    m_gmax = m_projs.get_slices(0, m_projno).max() / 4.0f;
    InitViews();
    m_dev.reset();
}

void ST_Tomography::_ensure_device() {
    if (m_dev) return;
    check_cuda(cudaSetDevice(m_device), "cudaSetDevice");
    std::unique_ptr<Device> d(new Device);
    const int F = m_nframes, V = m_projno;
    const size_t n = (size_t)m_vol[0] * m_vol[1] * m_vol[2];
    const size_t npix = (size_t)m_W * m_H;
    d->n = n;
    check_cuda(cudaStreamCreateWithFlags(&d->stream, cudaStreamNonBlocking), "cudaStreamCreate");
    check_stt(stt_create(&d->ctx, m_device), nullptr, "stt_create");
    std::vector<double> all;
    for (int f = 0; f < F; ++f) all.insert(all.end(), m_angles[f].begin(), m_angles[f].end());
    float sp[3] = {1, 1, 1};
    if (m_Data) m_Data->GetSpacings(sp);
    stt_geometry g{};
    g.nx = m_vol[0];
    g.ny = m_vol[1];
    g.nz = m_vol[2];
    g.sx = sp[0];
    g.sy = sp[1];
    g.sz = sp[2];
    g.W = m_W;
    g.H = m_H;
    g.ds = m_ds;
    g.sid = m_sid;
    g.sdd = m_sdd;
    for (int a = 0; a < 3; ++a) g.off[a] = m_oxyz[a];
    g.n_views = (int)all.size();
    g.angles_rad = all.data();
    check_stt(stt_set_geometry(d->ctx, &g), d->ctx, "stt_set_geometry");
    d->vol = dev_alloc<float>((F + 1) * n);
    d->xbar = dev_alloc<float>((F + 1) * n);
    d->xprev = dev_alloc<float>(F * n);
    d->ytv = dev_alloc<float>(3 * F * n);
    d->ytp = dev_alloc<float>(F * n);
    d->ybc = dev_alloc<float>(F * n);
    d->flowv = dev_alloc<float>(3 * F * n);
    d->proj = dev_alloc<float>((size_t)F * V * npix);
    d->raylen = dev_alloc<float>(npix);
    d->tmp = dev_alloc<float>(n);
    for (float *p : {d->xbar, d->xprev, d->ytv, d->ytp, d->ybc})
        check_cuda(cudaMemset(p, 0, sizeof(float) * n * (p == d->ytv ? 3 * F : (p == d->xbar ? F + 1 : F))),
                   "clear state");
    check_cuda(cudaMemset(d->raylen, 0, sizeof(float) * npix), "clear ray lengths");
    check_cuda(cudaMemcpy(d->proj, m_projs.data(), sizeof(float) * F * V * npix, cudaMemcpyHostToDevice),
               "upload projections");
    for (int f = 0; f <= F; ++f)
        check_cuda(cudaMemcpy(d->vol + f * n, m_Data->m_Volumelist[f].data(), sizeof(float) * n,
                              cudaMemcpyHostToDevice),
                   "upload volume");
    for (int f = 0; f < F; ++f)
        check_cuda(cudaMemcpy(d->flowv + 3 * f * n, m_Data->m_Flowlist[f].data(), sizeof(float) * 3 * n,
                              cudaMemcpyHostToDevice),
                   "upload flow");
    stt_solve_cfg cfg{};
    cfg.n_frames = F;
    cfg.views_per_frame = V;
    cfg.bp_mode = m_bp_mode;
    cfg.alpha = m_alpha;
    cfg.pd.sigma = 0.9f / 8.0f;
    cfg.pd.tau = 1.0f;
    cfg.pd.tv_w = m_tv_w;
    cfg.pd.tp_w = m_tp_w;
    cfg.pd.bc_w = m_bc_w;
    cfg.pd.huber_factor = m_huberfactor;
    cfg.pd.gmax = m_gmax;
    std::memcpy(cfg.pd.cut, kCut, sizeof(kCut));
    std::memcpy(cfg.roi_cut, kCut, sizeof(kCut));
    cfg.seed = m_seed;
    cfg.mode = STT_SOLVE_GRAPH;
    cfg.autotune = 1;  // the launch choices timed on this geometry (stt_autotune) before the graph is captured
    stt_pd_state st{};
    st.vol = d->vol;
    st.xbar = d->xbar;
    st.xprev = d->xprev;
    st.ytv = d->ytv;
    st.ytp = d->ytp;
    st.ybc = d->ybc;
    st.flow = d->flowv;
    st.proj = d->proj;
    check_stt(stt_solver_create(d->ctx, &cfg, &st, &d->solver), d->ctx, "stt_solver_create");
    if (F > 1) {
        stt_flow_params fp{};
        fp.tol = 0.1f;  // ST_Tomography.cpp:440-456
        fp.lambda = 1.2f;
        fp.huber = 1.0f;
        fp.eta = 0.65f;
        fp.sigma = 0.5f;
        fp.max_iter = m_flow_iters;
        fp.norm = 4;
        fp.n_warps = 3;
        fp.scales = 3;
        std::memcpy(fp.cut, kCut, sizeof(fp.cut));
        if (stt_flow_create(m_device, m_vol, &fp, &d->flow) != STT_OK)
            throw std::runtime_error(std::string("stt_flow_create: ") + stt_last_error(nullptr));
    }
    m_dev = std::move(d);
}

void ST_Tomography::_download_volume(int f, stt::Image &out) {
    _ensure_device();
    out = stt::Image(m_vol[0], m_vol[1], m_vol[2], 1);
    check_cuda(cudaStreamSynchronize(m_dev->stream), "sync");
    check_cuda(cudaMemcpy(out.data(), m_dev->vol + f * m_dev->n, sizeof(float) * m_dev->n, cudaMemcpyDeviceToHost),
               "download volume");
}

stt::Image ST_Tomography::Volume(int f) {
    stt::Image v;
    _download_volume(f, v);
    return v;
}

// The file SART(f) writes: <output>-<frame %03d>-frame-<call count>iter.tiff
// (ST_Tomography.cpp:770-806).
void ST_Tomography::_save_frame(int f) {
    if (m_save_mode == SAVE_ALL) {
        stt::Image v;
        _download_volume(f, v);
        char buf[32];
        std::snprintf(buf, sizeof(buf), "-%03d-frame-%d", f, m_idxSART[f]);
        write_tiff(m_output + buf + "iter.tiff", v);
    }
    m_idxSART[f]++;
}

void ST_Tomography::SART(int iframes) {
    _ensure_device();
    const int V = m_projno;
    const size_t npix = (size_t)m_W * m_H;
    std::vector<int> perm(V);
    check_stt(stt_solver_frame_order(m_seed, 1000000ULL + (unsigned long long)m_idxSART[iframes], m_nframes, iframes,
                                     V, perm.data()),
              nullptr, "stt_solver_frame_order");
    check_stt(stt_sart_sweep(m_dev->ctx, m_dev->vol + iframes * m_dev->n, m_dev->proj + (size_t)iframes * V * npix,
                             perm.data(), V, iframes * V, m_alpha, m_gmax, m_bp_mode, m_dev->raylen, kCut,
                             m_dev->stream),
              m_dev->ctx, "stt_sart_sweep");
    check_cuda(cudaStreamSynchronize(m_dev->stream), "sync");
    _save_frame(iframes);
}

// The flow half of the joint loop (ST_Tomography.cpp:421-470): for every pair
// of consecutive frames, the multiscale flow warm-started from the current
// flow, then the warped second frame and the flow field written out.
void ST_Tomography::_flow_step(int out_iter) {
    Device &d = *m_dev;
    const size_t n = d.n;
    const float box[3] = {(float)m_vol[0], (float)m_vol[1], (float)m_vol[2]};
    for (int f = 0; f + 1 < m_nframes; ++f) {
        float *V = d.flowv + 3 * f * n;
        if (stt_flow_multiscale(d.flow, d.vol + f * n, d.vol + (f + 1) * n, V, nullptr, d.stream) != STT_OK)
            throw std::runtime_error(std::string("stt_flow_multiscale: ") + stt_flow_last_error(d.flow));
        if (m_save_mode == SAVE_NONE) continue;
        check_stt(stt_warp_box(m_vol, box, V, d.vol + (f + 1) * n, 1, -1.0f, d.tmp, d.stream), nullptr,
                  "stt_warp_box");
        check_cuda(cudaStreamSynchronize(d.stream), "sync");
        stt::Image warped(m_vol[0], m_vol[1], m_vol[2], 1), field(m_vol[0], m_vol[1], m_vol[2], 3);
        check_cuda(cudaMemcpy(warped.data(), d.tmp, sizeof(float) * n, cudaMemcpyDeviceToHost), "download warp");
        check_cuda(cudaMemcpy(field.data(), V, sizeof(float) * 3 * n, cudaMemcpyDeviceToHost), "download flow");
        char base[160];
        std::snprintf(base, sizeof(base), "%s/%03d.%03d.%03d.frame%02d.iter%02d", m_flow_dir.c_str(), m_vol[0],
                      m_vol[1], m_vol[2], f, out_iter);
        write_tiff(std::string(base) + ".tiff", warped);
        const std::string hdr = std::string(base) + ".field.hdr";
        if (stt_analyze_write(hdr.c_str(), m_vol[0], m_vol[1], m_vol[2], 3, field.data()) != 0)
            throw std::runtime_error(stt_host_last_error());
    }
}

// ST_Tomography::Render (ST_Tomography.cpp:398-611): joint iterations of the
// flow step and, from the second on, primal-dual passes over all frames
// (dual, primal, SART, ROI mask, over-relaxation per frame).
void ST_Tomography::Render() {
    if (!m_Data) throw std::runtime_error("Render: SetData first");
    _ensure_device();
    Device &d = *m_dev;
    const size_t n = d.n;
    for (int out_iter = 0; out_iter < m_joint_iter; ++out_iter) {
        if (d.flow) _flow_step(out_iter);
        if (out_iter == 0) continue;
        for (int pass = 0; pass < m_pd_passes; ++pass) {
            if (out_iter == 1 && pass == 0)  // X_bar starts at the volumes (:494-500)
                check_cuda(cudaMemcpyAsync(d.xbar, d.vol, sizeof(float) * (m_nframes + 1) * n,
                                           cudaMemcpyDeviceToDevice, d.stream),
                           "init X_bar");
            check_stt(stt_solver_iterate(d.solver, 1, d.stream), d.ctx, "stt_solver_iterate");
            const bool last = out_iter == m_joint_iter - 1 && pass == m_pd_passes - 1;
            const int keep = m_save_mode;
            if (m_save_mode == SAVE_LAST) m_save_mode = last ? SAVE_ALL : SAVE_NONE;
            for (int f = 0; f < m_nframes; ++f) _save_frame(f);
            m_save_mode = keep;
        }
    }
    check_cuda(cudaStreamSynchronize(d.stream), "sync");
    for (int f = 0; f <= m_nframes; ++f) _download_volume(f, m_Data->m_Volumelist[f]);
    for (int f = 0; f < m_nframes; ++f)
        check_cuda(cudaMemcpy(m_Data->m_Flowlist[f].data(), d.flowv + 3 * f * n, sizeof(float) * 3 * n,
                              cudaMemcpyDeviceToHost),
                   "download flow");
}
