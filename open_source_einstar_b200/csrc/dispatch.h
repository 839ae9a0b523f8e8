// Host-side launch of the SGM kernels for one kernel configuration. The kernels are templates over the
// per-lane register count R (2R disparities per lane), the segment width SEG (lanes per scanline / per
// pixel), the census word, the path-value storage type and cost materialisation; each R is
// instantiated in its own translation unit (inst_r*.cu) so that the library builds in parallel.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

namespace dsk {
struct PathArgs;
struct WtaArgs;
struct CostArgs;
struct SweepArgs;
struct WtaRowArgs;
}  // namespace dsk

namespace ds {

// A kernel configuration: 2R disparities per lane, SEG lanes per scanline (16: two lines per warp).
struct KernelCfg {
    int R = 2;
    int seg = 32;
    bool materialize = false;  // cost volume written once and read by every direction
    int paths_warps = 4;       // warps per block of the path kernel
    int prefetch = 4;          // steps of inputs in flight per scanline (4 or 8)
    int wta_threads = 256;     // threads per block of the WTA kernel
    bool fused = true;         // 4 paths as the two sweep kernels (k_sweep_cols, k_sweep_rows with the WTA)
    int horz_warps = 4;        // (kept in the configuration; the sweep kernels have fixed block shapes)
    int dp() const { return seg * 2 * R; }
};

// Configurations that have kernels: SEG 16 with R in {1,2,3,4}; SEG 32 with R in {1,2,3,4,6,8}.
bool cfg_supported(int R, int seg);

// Library-internal bookkeeping shared by the translation units that launch kernels.
void set_global_error(const char* message);  // the text ds_last_global_error() returns
void count_launches(int n);                    // kernels launched (ds_kernel_launches)

// Returns a CUDA error (cudaSuccess on success). `c64`: 64-bit census words; `wide`: u16 path values.
cudaError_t launch_paths(const KernelCfg& cfg, bool c64, bool wide, const dsk::PathArgs& a, int ndirs, int max_lines,
                         cudaStream_t st);
cudaError_t launch_wta(const KernelCfg& cfg, bool wide, const dsk::WtaArgs& a, int rows, size_t smem, cudaStream_t st);
cudaError_t launch_costs(const KernelCfg& cfg, bool c64, const dsk::CostArgs& a, cudaStream_t st);
// Sweep kernels (sweep_kernels.cuh): the vertical pair into S, then the horizontal pair with the WTA and the
// L-R check. `pad`: nd < the slab disparities; `slant`: the k-2 / k+2 neighbours.
cudaError_t launch_sweep_cols(const KernelCfg& cfg, bool slant, bool pad, const dsk::SweepArgs& a, cudaStream_t st);
cudaError_t launch_sweep_rows(const KernelCfg& cfg, bool slant, bool pad, const dsk::SweepArgs& a, cudaStream_t st);

// Row-sweep WTA of the per-direction path (wta_kernels.cuh): lane slab shapes, the chunks of a row of width w
// (columns per chunk, log2 of the chunk count, key sets), and the launches.
bool wta_rows_shape(int dp, int& R, int& seg);
bool wta_rows_layout(int w, int dp, int& chunk, int& lg_chunks, int& sets);
cudaError_t launch_wta_rows(const dsk::WtaRowArgs& a, cudaStream_t st);

struct BatchGroupDev;
cudaError_t launch_wta_rows_batch(int dp, bool pad, const dsk::WtaRowArgs* args, const BatchGroupDev& g, cudaStream_t st);

// Persistent batch launches (one launch walks the blocks of every pair of a kernel-variant group).
cudaError_t launch_paths_batch(const KernelCfg& cfg, bool c64, bool wide, const dsk::PathArgs* args, const BatchGroupDev& g,
                               cudaStream_t st);
cudaError_t launch_wta_batch(const KernelCfg& cfg, bool wide, int ndirs, const dsk::WtaArgs* args, const BatchGroupDev& g,
                             size_t smem, cudaStream_t st);
cudaError_t launch_costs_batch(const KernelCfg& cfg, bool c64, const dsk::CostArgs* args, const BatchGroupDev& g,
                               cudaStream_t st);

#define DS_DECLARE_R(R)                                                                                              \
    cudaError_t launch_paths_r##R(const KernelCfg&, bool, bool, const dsk::PathArgs&, int, int, cudaStream_t);      \
    cudaError_t launch_wta_r##R(const KernelCfg&, bool, const dsk::WtaArgs&, int, size_t, cudaStream_t);              \
    cudaError_t launch_costs_r##R(const KernelCfg&, bool, const dsk::CostArgs&, cudaStream_t);                      \
    cudaError_t launch_paths_batch_r##R(const KernelCfg&, bool, bool, const dsk::PathArgs*, const BatchGroupDev&,    \
                                        cudaStream_t);                                                               \
    cudaError_t launch_wta_batch_r##R(const KernelCfg&, bool, int, const dsk::WtaArgs*, const BatchGroupDev&, size_t,\
                                      cudaStream_t);                                                                 \
    cudaError_t launch_costs_batch_r##R(const KernelCfg&, bool, const dsk::CostArgs*, const BatchGroupDev&, cudaStream_t);
DS_DECLARE_R(1)
DS_DECLARE_R(2)
DS_DECLARE_R(3)
DS_DECLARE_R(4)
DS_DECLARE_R(6)
DS_DECLARE_R(8)
#undef DS_DECLARE_R

}  // namespace ds
