// ST_Tomography.h -- drop-in for S/ST_Tomo/ST_Tomography.h (gmzang/
// SpaceTimeTomography): the space-time reconstruction scene, headless.  The
// constructor takes the reference's 23 arguments (:27-29) and reads the start
// angles from lds.txt as the reference does (ST_Tomography.cpp:258-276);
// SetData reads the projection stack and builds the views; Render runs the
// joint loop of ST_Tomography.cpp:398-611 (optical flow between consecutive
// frames, then primal-dual iterations whose data term is SART) on the GPU
// and writes the same TIFF and Analyze files.  The OpenGL scene it derives
// from in the reference is not needed: the view geometry is built in FP64 by
// libstt, and the colour/light/iso-value setters only store their values.
//
// Differences from the reference, all deliberate:
//   - SART's view order is a seeded permutation (SetSeed), not
//     std::random_shuffle seeded with time(0) (ST_Tomography.cpp:627-634);
//   - the frames of one primal-dual iteration run as one batched, graph-
//     captured GPU iteration; the per-frame SART output files are written
//     after it, with the same names and contents;
//   - the loop counts the reference hard-codes (20 joint iterations, 2
//     primal-dual passes, 3000 flow iterations) are settable;
//   - a missing lds.txt falls back to the van der Corput angles the file is
//     generated from (Low_discrepency_squence.m), with a warning, instead of
//     reading nothing.
#ifndef STT_REFERENCE_ST_TOMOGRAPHY_H
#define STT_REFERENCE_ST_TOMOGRAPHY_H

#include <memory>
#include <string>
#include <vector>

#include "VolumeData.h"
#include "stt_image.h"

class RayCaster;
class TypicalRayProducer;

class ST_Tomography {
public:
    // d1 sigma, d2 tau (both accepted and unused, as in the reference), d3 TV
    // weight, d4 temporal-prior weight, d5 brightness-constancy weight, d6
    // Huber epsilon; imgwh detector W, H; projNo views per frame (10 per
    // round); iters / sartiters accepted and unused (the reference's loop
    // counts are fixed); alp SART step; projsfile[0] the projection stack;
    // oxyz volume-centre offset; _bp "Raybased" or voxel-based; volxyz volume
    // size; startdg unused (lds.txt holds the start angles); nrounds rounds of
    // 10 views per frame.
    ST_Tomography(double d1, double d2, double d3, double d4, double d5, double d6, const char *outputfile,
                  int *imgwh, int projNo, int iters, int sartiters, double alp, double sid, const char **projsfile,
                  double *oxyz, double sdd, double ds, const char *_prior, const char *_bp, int *volxyz,
                  int nframes, double *startdg, int nrounds);
    virtual ~ST_Tomography();

    void InitViews();
    bool RotateVolume(int i);
    void SetData(VolumeData *data);
    // One SART call for frame iframe (ST_Tomography.cpp:616-808) on the
    // current device state, then the ROI mask and the TIFF output.
    void SART(int iframes);

    void SetBackGroundColor(float r, float g, float b);
    void GetBackGroundColor(float &r, float &g, float &b);
    void SetIsovalue(float isovalue) { m_isovalue = isovalue; }
    float GetIsovalue() { return m_isovalue; }
    void SetSurfaceColor(float r, float g, float b);
    void GetSurfaceColor(float &r, float &g, float &b);
    void SetLightDirection(float x, float y, float z);
    void SetLightIntensity(float intensity) { m_light_intensity = intensity; }
    void SetLightColor(float r, float g, float b);
    void SetAmbient(float value) { m_ambient = value; }
    float GetAmbient() { return m_ambient; }
    void SetDiffuse(float value) { m_diffuse = value; }
    float GetDiffuse() { return m_diffuse; }
    void SetSpecular(float value) { m_specular = value; }
    float GetSpecular() { return m_specular; }
    void SetSpecularPower(float value) { m_specular_power = value; }
    float GetSpecularPower() { return m_specular_power; }
    void SetSampleDistance(float sd) { m_sample_distance = sd; }
    float GetSampleDistance() { return m_sample_distance; }

    virtual void Init() {}
    virtual void Resize(int width, int height);
    // The joint flow + reconstruction loop.  Public here: there is no GLUT
    // window to call it.
    virtual void Render();

    // ---- not in the reference ----
    void SetJointIterations(int n) { m_joint_iter = n; }
    void SetPrimalDualPasses(int n) { m_pd_passes = n; }
    void SetFlowIterations(int n) { m_flow_iters = n; }
    void SetSeed(unsigned long long seed) { m_seed = seed; }
    void SetDevice(int device) { m_device = device; }
    // Re-reads the start angles from `path` (the constructor reads lds.txt).
    void SetLdsFile(const std::string &path);
    enum SaveMode { SAVE_ALL = 0, SAVE_LAST = 1, SAVE_NONE = 2 };
    void SetSaveMode(int mode) { m_save_mode = mode; }
    void SetFlowDirectory(const std::string &dir) { m_flow_dir = dir; }
    int Frames() const { return m_nframes; }
    // Start angles read (or generated) per frame and round, degrees.
    const std::vector<std::vector<float>> &StartDegrees() const { return m_startDegree; }
    // View angles of frame f (radians, FP64), in view-index order.
    std::vector<double> ViewAngles(int f) const;
    // Host copy of frame f's current volume.
    stt::Image Volume(int f);
    float GMax() const { return m_gmax; }

protected:
    virtual void RenderContent(int iframe) { (void)iframe; }
    virtual void GetSize3D(float size[3]);

private:
    struct Device;
    void _ensure_device();
    void _download_volume(int f, stt::Image &out);
    void _save_frame(int f);
    void _flow_step(int out_iter);

    int m_nframes, m_nrounds, m_projno, m_W, m_H, m_vol[3];
    double m_alpha, m_sid, m_sdd, m_ds, m_oxyz[3];
    float m_tv_w, m_tp_w, m_bc_w, m_huberfactor, m_gmax = 10.0f;
    int m_bp_mode;
    std::string m_output, m_proj_file, m_prior;
    std::vector<std::vector<float>> m_startDegree;
    std::vector<std::vector<double>> m_angles;  // per frame, per view
    std::vector<int> m_idxSART;
    VolumeData *m_Data = nullptr;
    stt::Image m_projs;                          // W x H x (projNo * nframes)

    int m_joint_iter = 20, m_pd_passes = 2, m_flow_iters = 3000, m_save_mode = SAVE_ALL, m_device = 0;
    unsigned long long m_seed = 20181203ULL;
    std::string m_lds_file = "lds.txt", m_flow_dir = "FlowOutput";
    float m_bg[3] = {0, 0, 0}, m_surface[3] = {1, 1, 1}, m_light_dir[3] = {0, 0, 1}, m_light_color[3] = {1, 1, 1};
    float m_isovalue = 0.5f, m_light_intensity = 1.0f, m_ambient = 0.1f, m_diffuse = 0.7f, m_specular = 0.2f,
          m_specular_power = 10.0f, m_sample_distance = 1.0f;
    std::unique_ptr<Device> m_dev;
};

#endif
