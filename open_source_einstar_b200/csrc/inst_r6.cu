// Kernel instantiations for R = 6 (2R disparities per lane); see dispatch.h.
#include "launchers.cuh"

DS_DEFINE_R(6)
DS_DEFINE_BATCH_R(6)
