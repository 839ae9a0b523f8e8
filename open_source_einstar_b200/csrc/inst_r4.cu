// Kernel instantiations for R = 4 (2R disparities per lane); see dispatch.h.
#include "launchers.cuh"

DS_DEFINE_R(4)
DS_DEFINE_BATCH_R(4)
