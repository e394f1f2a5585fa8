// TypicalRayProducer.core.h -- drop-in for
// S/ImageFormationModel/TypicalRayProducer.core.h:230: one march of the
// current view over the bound frame.  Forward mode fills GetImageData,
// GetImageRaylength (rays that hit only) and GetWeightOfImage; backprojection
// mode (VolumeData::SetProjectionMode(1) before SingleScalarVolumePrepare)
// scatters GetCorrection() into GetContributions / GetTotalWeight.
#ifndef STT_REFERENCE_TYPICALRAYPRODUCER_CORE_H
#define STT_REFERENCE_TYPICALRAYPRODUCER_CORE_H

#include "TypicalRayProducer.h"

void GenerateImage_GetCorrections(TypicalRayProducer *producer);

#endif
