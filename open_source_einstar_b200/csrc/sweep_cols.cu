// Column sweep kernel (vertical path pair) launchers.
#include "sweep_launch.cuh"

namespace ds {

template <int R, int SEG, bool SL, bool PD>
static cudaError_t cols_frame(const dsk::SweepArgs& a, cudaStream_t st) {
    dsk::k_sweep_cols<R, SEG, SL, PD, kSweepPF><<<sweep_col_blocks(a.w, SEG), dsk::kSweepColThreads, 0, st>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_sweep_cols(const KernelCfg& cfg, bool slant, bool pad, const dsk::SweepArgs& a, cudaStream_t st) {
#define DS_CALL(R, SEG, SL, PD) cols_frame<R, SEG, SL, PD>(a, st)
    DS_SWEEP_DISPATCH(cfg, slant, pad, DS_CALL);
#undef DS_CALL
}

}  // namespace ds
