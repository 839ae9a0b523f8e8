// Kernel instantiations for R = 8 (2R disparities per lane); see dispatch.h.
#include "launchers.cuh"

DS_DEFINE_R(8)
DS_DEFINE_BATCH_R(8)
