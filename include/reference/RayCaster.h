// RayCaster.h -- drop-in for S/ImageFormationModel/RayCaster.h: the sample
// distance of the ray march (:16-17).  The march itself runs in libstt.
#ifndef STT_REFERENCE_RAYCASTER_H
#define STT_REFERENCE_RAYCASTER_H

class RayCaster {
public:
    RayCaster() = default;
    virtual ~RayCaster() = default;
    void SetSampleDistance(float sd) { m_SampleDistance = sd; }
    float GetSampleDistance() const { return m_SampleDistance; }

private:
    float m_SampleDistance = 1.0f;
};

#endif
