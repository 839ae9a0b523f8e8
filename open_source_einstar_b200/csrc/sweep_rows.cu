// Row sweep kernel (horizontal path pair, WTA and L-R check) launchers.
#include "sweep_launch.cuh"

namespace ds {

template <int R, int SEG, bool SL, bool PD>
static cudaError_t rows_frame(const dsk::SweepArgs& a, cudaStream_t st) {
    dsk::k_sweep_rows<R, SEG, SL, PD, kSweepPF><<<sweep_row_blocks(a.h, SEG), dsk::kSweepRowThreads, 0, st>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_sweep_rows(const KernelCfg& cfg, bool slant, bool pad, const dsk::SweepArgs& a, cudaStream_t st) {
#define DS_CALL(R, SEG, SL, PD) rows_frame<R, SEG, SL, PD>(a, st)
    DS_SWEEP_DISPATCH(cfg, slant, pad, DS_CALL);
#undef DS_CALL
}

}  // namespace ds
