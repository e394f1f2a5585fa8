// TypicalRayProducer.h -- drop-in for S/ImageFormationModel/TypicalRayProducer.h
// (gmzang/SpaceTimeTomography): the per-view producer of rays and its image
// buffers (:11-44, 73).  The view is given as the reference gives it, by the
// scene's view and projection matrices (16 floats each, column-major; a
// reference Matrix4x4 converts to const float*); UpdateMatrixAndBounds reads
// the rotation about y, the translation and the frustum out of them and sets
// libstt's FP64 geometry.  The march runs on the GPU; the buffers returned by
// the getters are host copies, filled by GenerateImage_GetCorrections.
#ifndef STT_REFERENCE_TYPICALRAYPRODUCER_H
#define STT_REFERENCE_TYPICALRAYPRODUCER_H

#include <vector>

struct stt_ctx;

class TypicalRayProducer {
public:
    TypicalRayProducer(int volX, int volY, int volZ, int imgW, int imgH, double ds, const char *_bp);
    virtual ~TypicalRayProducer();
    // Clears the backprojection accumulators (TypicalRayProducer.cpp:78-96).
    void Initial();
    void SetBackProjectionMode() { m_BackProjection = true; }
    bool IsBackProjectionMode() { return m_BackProjection; }
    void SetViewPort(int width, int height);
    void SetVolSize(const int volDims[3], const float volSpacings[3]);
    void GetVolSize(int volDims[3], float volSpacings[3]);
    void SetViewMatrix(const float *view);
    void SetProjectionMatrix(const float *projection);
    // Throws std::runtime_error if the matrices are not a rotation about y
    // with unit scale and a symmetric frustum.
    void UpdateMatrixAndBounds();
    void GetImageInUseSize(int imageSize[2]);
    void GetImageOrigin(int imageOrigin[2]);
    float *GetTotalWeight();
    float *GetImageData() { return m_ImageData.data(); }
    float *GetWeightOfImage() { return m_WeightOfImage.data(); }
    float *GetImageRaylength() { return m_imageraylength.data(); }
    float *GetContributions();
    float *GetCorrection() { return m_Correction; }
    void RenderImage() {}  // the reference draws the image with OpenGL; nothing to draw here

    // Not in the reference: the view in the form libstt uses.
    void SetViewAngle(double theta_rad, double sid, double sdd, const double offset[3]);
    double ViewAngle() const { return m_theta; }
    stt_ctx *Context() { return m_ctx; }

    int m_ViewPort[2];
    int m_VolDims[3];
    float m_VolSpacings[3] = {1.0f, 1.0f, 1.0f};
    float m_VolSize[3];
    float m_ViewMatrix[16];
    float m_ProjectionMatrix[16];
    float *m_Correction;  // W*H host array the caller fills before a backprojection-mode call

    // used by the free functions of the .core.h headers
    void _runForward(const float *vol_host, int frame);
    void _runBackward();
    int _frame = -1;

private:
    void _download_scatter();
    stt_ctx *m_ctx = nullptr;
    bool m_BackProjection = false;
    double m_ds, m_theta = 0.0, m_sid = 600.0, m_sdd = 1000.0, m_off[3] = {0, 0, 0};
    bool m_geometry_set = false;
    std::vector<float> m_ImageData, m_WeightOfImage, m_imageraylength, m_CorrectionStore;
    std::vector<float> m_Voxel_Contributions, m_EachVoxel_TotalWeight;
    bool m_scatter_dirty = false;
    float *d_vol = nullptr, *d_img = nullptr, *d_rl = nullptr, *d_wt = nullptr, *d_corr = nullptr,
          *d_contrib = nullptr, *d_wsum = nullptr;
    size_t d_vol_n = 0, d_img_n = 0;
    void _ensure_device();
};

#endif
