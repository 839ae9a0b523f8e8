// Kernel instantiations for R = 1 (2R disparities per lane); see dispatch.h.
#include "launchers.cuh"

DS_DEFINE_R(1)
DS_DEFINE_BATCH_R(1)
