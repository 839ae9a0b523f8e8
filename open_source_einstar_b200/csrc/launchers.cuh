// Template launchers behind dispatch.h, instantiated per R by inst_r*.cu.
#pragma once

#include "batch_common.cuh"
#include "dispatch.h"
#include "stereo_kernels.cuh"

namespace ds {

template <int R, int SEG, typename CW, typename ST, bool MAT>
cudaError_t paths_t(const KernelCfg& cfg, const dsk::PathArgs& a, int ndirs, int max_lines, cudaStream_t st) {
    const int lines_per_block = cfg.paths_warps * (32 / SEG);
    dim3 grid((max_lines + lines_per_block - 1) / lines_per_block, ndirs);
    if (cfg.prefetch == 8) dsk::k_paths<R, SEG, CW, ST, MAT, 8><<<grid, cfg.paths_warps * 32, 0, st>>>(a);
    else dsk::k_paths<R, SEG, CW, ST, MAT, 4><<<grid, cfg.paths_warps * 32, 0, st>>>(a);
    return cudaGetLastError();
}

template <int R, int SEG>
cudaError_t paths_seg(const KernelCfg& cfg, bool c64, bool wide, const dsk::PathArgs& a, int ndirs, int max_lines,
                      cudaStream_t st) {
    if (cfg.materialize) {
        return wide ? paths_t<R, SEG, uint32_t, uint16_t, true>(cfg, a, ndirs, max_lines, st)
                    : paths_t<R, SEG, uint32_t, uint8_t, true>(cfg, a, ndirs, max_lines, st);
    }
    if (c64) {
        return wide ? paths_t<R, SEG, uint64_t, uint16_t, false>(cfg, a, ndirs, max_lines, st)
                    : paths_t<R, SEG, uint64_t, uint8_t, false>(cfg, a, ndirs, max_lines, st);
    }
    return wide ? paths_t<R, SEG, uint32_t, uint16_t, false>(cfg, a, ndirs, max_lines, st)
                : paths_t<R, SEG, uint32_t, uint8_t, false>(cfg, a, ndirs, max_lines, st);
}

template <int R, int SEG, typename ST>
cudaError_t wta_t(const KernelCfg& cfg, const dsk::WtaArgs& a, int rows, size_t smem, cudaStream_t st) {
    auto k = a.ndirs == 8 ? dsk::k_wta<R, SEG, ST, 8> : dsk::k_wta<R, SEG, ST, 4>;
    if (smem > 48 * 1024) {
        const cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
        if (e != cudaSuccess) return e;
    }
    k<<<rows, cfg.wta_threads, smem, st>>>(a);
    return cudaGetLastError();
}

template <int R, int SEG, typename CW>
cudaError_t costs_t(const dsk::CostArgs& a, cudaStream_t st) {
    const long px = static_cast<long>(a.w) * a.h;
    const long px_per_block = 8 * (32 / SEG);
    dsk::k_costs<R, SEG, CW><<<static_cast<unsigned>((px + px_per_block - 1) / px_per_block), 256, 0, st>>>(a);
    return cudaGetLastError();
}

}  // namespace ds

// SEG 16 exists for R <= 4 only.
#define DS_SEG_SWITCH(R, CALL16, CALL32) \
    if (cfg.seg == 16) {                 \
        if constexpr (R <= 4) return CALL16; \
        return cudaErrorInvalidValue;    \
    }                                    \
    return CALL32;

#define DS_DEFINE_R(R)                                                                                               \
    namespace ds {                                                                                                   \
    cudaError_t launch_paths_r##R(const KernelCfg& cfg, bool c64, bool wide, const dsk::PathArgs& a, int ndirs,      \
                                  int max_lines, cudaStream_t st) {                                                  \
        if (cfg.seg == 8) {                                                                                          \
            if constexpr (R == 4 || R == 6 || R == 8) return paths_seg<R, 8>(cfg, c64, wide, a, ndirs, max_lines, st); \
            return cudaErrorInvalidValue;                                                                            \
        }                                                                                                            \
        DS_SEG_SWITCH(R, (paths_seg<R, (R <= 4 ? 16 : 32)>(cfg, c64, wide, a, ndirs, max_lines, st)),               \
                      (paths_seg<R, 32>(cfg, c64, wide, a, ndirs, max_lines, st)))                                   \
    }                                                                                                                \
    cudaError_t launch_wta_r##R(const KernelCfg& cfg, bool wide, const dsk::WtaArgs& a, int rows, size_t smem,       \
                                cudaStream_t st) {                                                                   \
        if (cfg.seg == 8)                                                                                            \
            return wide ? wta_t<R, 8, uint16_t>(cfg, a, rows, smem, st) : wta_t<R, 8, uint8_t>(cfg, a, rows, smem, st); \
        if (cfg.seg == 16)                                                                                           \
            return wide ? wta_t<R, 16, uint16_t>(cfg, a, rows, smem, st) : wta_t<R, 16, uint8_t>(cfg, a, rows, smem, st); \
        return wide ? wta_t<R, 32, uint16_t>(cfg, a, rows, smem, st) : wta_t<R, 32, uint8_t>(cfg, a, rows, smem, st); \
    }                                                                                                                \
    cudaError_t launch_costs_r##R(const KernelCfg& cfg, bool c64, const dsk::CostArgs& a, cudaStream_t st) {         \
        DS_SEG_SWITCH(R,                                                                                             \
                      (c64 ? costs_t<R, (R <= 4 ? 16 : 32), uint64_t>(a, st) : costs_t<R, (R <= 4 ? 16 : 32), uint32_t>(a, st)), \
                      (c64 ? costs_t<R, 32, uint64_t>(a, st) : costs_t<R, 32, uint32_t>(a, st)))                     \
    }                                                                                                                \
    }

// ------------------------------------------------------------------------------------------------
// Persistent batch launches: one grid-strided kernel walks the virtual blocks of every pair of a group
// (pairs sharing one kernel variant); prefix[i] is the first virtual block of group pair i.

namespace dsk {

// The per-pair arguments of the current virtual block are staged in shared memory, so that the stage
// bodies read them as cheaply as kernel parameters.
template <int R, int SEG, typename CW, typename ST, bool MAT, int PF>
__global__ void __launch_bounds__(256) kb_paths(const PathArgs* __restrict__ args, const int* __restrict__ pairs,
                                                const int* __restrict__ prefix, const int* __restrict__ gx, int n, int total) {
    __shared__ PathArgs sa;
    int cur = -1;
    for (int v = blockIdx.x; v < total; v += gridDim.x) {
        const int i = batch_find(prefix, n, v);
        const int lb = v - __ldg(prefix + i), g = __ldg(gx + i);
        const int p = __ldg(pairs + i);
        if (p != cur) {
            __syncthreads();
            if (threadIdx.x == 0) sa = args[p];
            __syncthreads();
            cur = p;
        }
        paths_body<R, SEG, CW, ST, MAT, PF>(sa, sa.p2_table, lb % g, lb / g);
    }
}

template <int R, int SEG, typename ST, int NDIRS>
__global__ void __launch_bounds__(256, sizeof(ST) == 1 && NDIRS == 4 ? 4 : 1) kb_wta(const WtaArgs* __restrict__ args, const int* __restrict__ pairs,
                                              const int* __restrict__ prefix, const int* __restrict__ gx, int n, int total) {
    __shared__ WtaArgs sa;
    int cur = -1;
    for (int v = blockIdx.x; v < total; v += gridDim.x) {
        const int i = batch_find(prefix, n, v);
        const int p = __ldg(pairs + i);
        if (p != cur) {
            if (threadIdx.x == 0) sa = args[p];
            cur = p;
        }
        __syncthreads();  // the arguments are staged; the previous row's shared memory is free again
        wta_body<R, SEG, ST, NDIRS>(sa, v - __ldg(prefix + i));
        __syncthreads();
    }
}

template <int R, int SEG, typename CW>
__global__ void __launch_bounds__(256) kb_costs(const CostArgs* __restrict__ args, const int* __restrict__ pairs,
                                                const int* __restrict__ prefix, const int* __restrict__ gx, int n, int total) {
    __shared__ CostArgs sa;
    int cur = -1;
    for (int v = blockIdx.x; v < total; v += gridDim.x) {
        const int i = batch_find(prefix, n, v);
        const int p = __ldg(pairs + i);
        if (p != cur) {
            __syncthreads();
            if (threadIdx.x == 0) sa = args[p];
            __syncthreads();
            cur = p;
        }
        costs_body<R, SEG, CW>(sa, v - __ldg(prefix + i));
    }
}

}  // namespace dsk

namespace ds {

template <int R, int SEG, typename CW, typename ST, bool MAT>
cudaError_t bpaths_t(const KernelCfg& cfg, const dsk::PathArgs* args, const BatchGroupDev& g, cudaStream_t st) {
    auto k = cfg.prefetch == 8 ? dsk::kb_paths<R, SEG, CW, ST, MAT, 8> : dsk::kb_paths<R, SEG, CW, ST, MAT, 4>;
    const int threads = cfg.paths_warps * 32;
    // One block per virtual block: scanline groups of different pairs differ in length, and the block
    // scheduler balances them better than a fixed share per resident block.
    k<<<g.total, threads, 0, st>>>(args, g.pairs, g.prefix, g.gx, g.n, g.total);
    return cudaGetLastError();
}

template <int R, int SEG>
cudaError_t bpaths_seg(const KernelCfg& cfg, bool c64, bool wide, const dsk::PathArgs* args, const BatchGroupDev& g,
                       cudaStream_t st) {
    if (cfg.materialize)
        return wide ? bpaths_t<R, SEG, uint32_t, uint16_t, true>(cfg, args, g, st) : bpaths_t<R, SEG, uint32_t, uint8_t, true>(cfg, args, g, st);
    if (c64)
        return wide ? bpaths_t<R, SEG, uint64_t, uint16_t, false>(cfg, args, g, st) : bpaths_t<R, SEG, uint64_t, uint8_t, false>(cfg, args, g, st);
    return wide ? bpaths_t<R, SEG, uint32_t, uint16_t, false>(cfg, args, g, st) : bpaths_t<R, SEG, uint32_t, uint8_t, false>(cfg, args, g, st);
}

template <int R, int SEG, typename ST>
cudaError_t bwta_t(const KernelCfg& cfg, int ndirs, const dsk::WtaArgs* args, const BatchGroupDev& g, size_t smem, cudaStream_t st) {
    auto k = ndirs == 8 ? dsk::kb_wta<R, SEG, ST, 8> : dsk::kb_wta<R, SEG, ST, 4>;
    if (smem > 48 * 1024) {
        const cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, static_cast<int>(smem));
        if (e != cudaSuccess) return e;
    }
    // One block per row: rows are few (about 2-3 per resident block), so a fixed share leaves a tail.
    k<<<g.total, cfg.wta_threads, smem, st>>>(args, g.pairs, g.prefix, g.gx, g.n, g.total);
    return cudaGetLastError();
}

template <int R, int SEG, typename CW>
cudaError_t bcosts_t(const dsk::CostArgs* args, const BatchGroupDev& g, cudaStream_t st) {
    auto k = dsk::kb_costs<R, SEG, CW>;
    k<<<persistent_grid(k, 256, 0, g.total), 256, 0, st>>>(args, g.pairs, g.prefix, g.gx, g.n, g.total);
    return cudaGetLastError();
}

}  // namespace ds

#define DS_DEFINE_BATCH_R(R)                                                                                         \
    namespace ds {                                                                                                   \
    cudaError_t launch_paths_batch_r##R(const KernelCfg& cfg, bool c64, bool wide, const dsk::PathArgs* args,        \
                                        const BatchGroupDev& g, cudaStream_t st) {                                   \
        if (cfg.seg == 8) {                                                                                          \
            if constexpr (R == 4 || R == 6 || R == 8) return bpaths_seg<R, 8>(cfg, c64, wide, args, g, st);          \
            return cudaErrorInvalidValue;                                                                            \
        }                                                                                                            \
        DS_SEG_SWITCH(R, (bpaths_seg<R, (R <= 4 ? 16 : 32)>(cfg, c64, wide, args, g, st)),                           \
                      (bpaths_seg<R, 32>(cfg, c64, wide, args, g, st)))                                              \
    }                                                                                                                \
    cudaError_t launch_wta_batch_r##R(const KernelCfg& cfg, bool wide, int ndirs, const dsk::WtaArgs* args,          \
                                      const BatchGroupDev& g, size_t smem, cudaStream_t st) {                        \
        if (cfg.seg == 8)                                                                                            \
            return wide ? bwta_t<R, 8, uint16_t>(cfg, ndirs, args, g, smem, st)                                      \
                        : bwta_t<R, 8, uint8_t>(cfg, ndirs, args, g, smem, st);                                      \
        if (cfg.seg == 16)                                                                                           \
            return wide ? bwta_t<R, 16, uint16_t>(cfg, ndirs, args, g, smem, st)                                     \
                        : bwta_t<R, 16, uint8_t>(cfg, ndirs, args, g, smem, st);                                     \
        return wide ? bwta_t<R, 32, uint16_t>(cfg, ndirs, args, g, smem, st)                                         \
                    : bwta_t<R, 32, uint8_t>(cfg, ndirs, args, g, smem, st);                                         \
    }                                                                                                                \
    cudaError_t launch_costs_batch_r##R(const KernelCfg& cfg, bool c64, const dsk::CostArgs* args,                   \
                                        const BatchGroupDev& g, cudaStream_t st) {                                   \
        DS_SEG_SWITCH(R,                                                                                             \
                      (c64 ? bcosts_t<R, (R <= 4 ? 16 : 32), uint64_t>(args, g, st)                                  \
                           : bcosts_t<R, (R <= 4 ? 16 : 32), uint32_t>(args, g, st)),                                \
                      (c64 ? bcosts_t<R, 32, uint64_t>(args, g, st) : bcosts_t<R, 32, uint32_t>(args, g, st)))       \
    }                                                                                                                \
    }
