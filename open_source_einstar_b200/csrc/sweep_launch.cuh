// Launch helpers of the sweep kernels (sweep_kernels.cuh); sweep_cols.cu and sweep_rows.cu instantiate them.
// Batches launch the same kernels once per pair (arguments by value, captured into the batch's graph).
#pragma once

#include "dispatch.h"
#include "sweep_kernels.cuh"

namespace ds {

constexpr int kSweepPF = 2;

// Blocks of one frame: columns / rows per block.
inline int sweep_col_blocks(int w, int seg) { return (w + dsk::kSweepColWarps * (32 / seg) - 1) / (dsk::kSweepColWarps * (32 / seg)); }
inline int sweep_row_blocks(int h, int seg) { return (h + dsk::kSweepRowWarps * (32 / seg) - 1) / (dsk::kSweepRowWarps * (32 / seg)); }

// Expands CALL(R, SEG, SLANT, PAD) for the configuration's kernel shape and flags (shapes of sweep_shape_ok).
#define DS_SWEEP_DISPATCH(cfg, slant, pad, CALL)                                              \
    do {                                                                                      \
        const int r_ = (cfg).R, s_ = (cfg).seg;                                               \
        const bool sl_ = (slant), pd_ = (pad);                                                \
        if (r_ == 6 && s_ == 4) return sl_ ? (pd_ ? CALL(6, 4, true, true) : CALL(6, 4, true, false))   \
                                           : (pd_ ? CALL(6, 4, false, true) : CALL(6, 4, false, false)); \
        if (r_ == 6 && s_ == 8) return sl_ ? (pd_ ? CALL(6, 8, true, true) : CALL(6, 8, true, false))   \
                                           : (pd_ ? CALL(6, 8, false, true) : CALL(6, 8, false, false)); \
        if (r_ == 8 && s_ == 4) return sl_ ? (pd_ ? CALL(8, 4, true, true) : CALL(8, 4, true, false))   \
                                           : (pd_ ? CALL(8, 4, false, true) : CALL(8, 4, false, false)); \
        if (r_ == 8 && s_ == 8) return sl_ ? (pd_ ? CALL(8, 8, true, true) : CALL(8, 8, true, false))   \
                                           : (pd_ ? CALL(8, 8, false, true) : CALL(8, 8, false, false)); \
        return cudaErrorInvalidValue;                                                         \
    } while (0)

}  // namespace ds
