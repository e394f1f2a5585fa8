// SingleScalarVolume.core.h -- drop-in for the entry point of
// S/ImageFormationModel/SingleScalarVolume.core.h:195: binds frame `frame` of
// the volume list (and the volume's projection mode) to the producer.
#ifndef STT_REFERENCE_SINGLESCALARVOLUME_CORE_H
#define STT_REFERENCE_SINGLESCALARVOLUME_CORE_H

#include "TypicalRayProducer.h"
#include "VolumeData.h"

bool SingleScalarVolumePrepare(VolumeData *volume, TypicalRayProducer *producer, int frame);

#endif
