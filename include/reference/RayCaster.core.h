// RayCaster.core.h -- drop-in for S/ImageFormationModel/RayCaster.core.h:191.
#ifndef STT_REFERENCE_RAYCASTER_CORE_H
#define STT_REFERENCE_RAYCASTER_CORE_H

#include "RayCaster.h"

bool RayCasterPrepare(RayCaster *caster, int dims[3]);

#endif
