// Kernel instantiations for R = 3 (2R disparities per lane); see dispatch.h.
#include "launchers.cuh"

DS_DEFINE_R(3)
DS_DEFINE_BATCH_R(3)
