// VolumeData.h -- drop-in for S/ImageFormationModel/VolumeData.h (gmzang/
// SpaceTimeTomography): the frame list of a space-time reconstruction.  Same
// members and calls as the reference (:30-100); the lists hold stt::Image
// (CImg layout) instead of CImgList<float>.
#ifndef STT_REFERENCE_VOLUMEDATA_H
#define STT_REFERENCE_VOLUMEDATA_H

#include <string>
#include <vector>

#include "stt_image.h"

class VolumeData {
public:
    VolumeData();
    VolumeData(int d1, int d2, int d3, float sp1, float sp2, float sp3, float *data);
    virtual ~VolumeData();

    void Clean();
    void GetDimensions(int *dims) const;
    void SetDimensions(const int *dims);
    void GetSpacings(float *spacings) const;
    void SetSpacings(const float *spacings);
    void SetProjectionMode(bool mode) { m_IsBackProjectMode = mode; }
    bool GetProjectionMode() { return m_IsBackProjectMode; }
    stt::Image GetData(int iframe);
    void SetData(std::vector<stt::Image> _vol_list);
    // volume size (3 ints), voxel spacing, frame count (VolumeData.cpp setParas)
    void setParas(int *vols, double vs, int nframes);
    // Reads <input_dir>/rose.-%03d-frame-9iter.tiff for every frame, appends a
    // copy of the last one (the reference's n+1 guard, VolumeData.cpp:103-129)
    // and zeroes the flow list.  Throws std::runtime_error on a missing or
    // mis-sized file.
    void ReadStructuredFile();
    void _allocate();

    bool m_IsBackProjectMode = false;
    int m_Dims[3] = {0, 0, 0};
    float m_Spacings[3] = {1.0f, 1.0f, 1.0f};
    int m_volX = 0, m_volY = 0, m_volZ = 0;
    double Vol_Spacing = 1.0;
    std::vector<stt::Image> m_Volumelist;  // m_nframes + 1 volumes
    std::vector<stt::Image> m_Flowlist;    // m_nframes flows, 3 channels
    int m_nframes = 0;
    std::string m_InputDir = "Input";      // not in the reference: where ReadStructuredFile looks
};

#endif
