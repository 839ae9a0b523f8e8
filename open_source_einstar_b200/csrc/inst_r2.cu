// Kernel instantiations for R = 2 (2R disparities per lane); see dispatch.h.
#include "launchers.cuh"

DS_DEFINE_R(2)
DS_DEFINE_BATCH_R(2)
