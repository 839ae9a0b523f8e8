// Winner-takes-all and L-R check over the per-direction path values (stereo.cpp:411-461) as row sweeps
// (sm_100a): the WTA of the cost / path / WTA pipeline for 4 paths with byte path values, 2 (window + P2) <=
// 255 and lane slabs of 48, 64, 96 or 128 disparities. It replaces the per-pixel WTA there (k_wta) and keeps
// its results.
//
// A row is cut into nchunks chunks of `chunk` columns (the last one runs past the row end over virtual
// columns that hold no candidates); a segment of SEG lanes sweeps one chunk left to right, lane sl holding
// disparities k0 = sl*NV .. k0+NV-1 as R registers of (k, k+1) 16-bit pairs. Per column:
//   sums       the four direction slabs added in pairs as bytes (no carry: a pair is at most 2 * 127), then
//              in 16-bit lanes (the reference's u16 sums, at most 508 here)
//   left WTA   keys (sum << 7) | k, the segment's smallest key (first strict minimum), the best
//              non-adjacent cost (sums within one of the best raised to >= 0xFFFD), and the sums either side of
//              the best (parabola) read by the segment's first lane from shared memory
//   right WTA  candidate (x, k) belongs to right pixel xr = x - min - k: per slot a running minimum key of
//              the right pixel the slot feeds, moved one slot on after every column; the chain leaving slot
//              Dp-1 is complete within the chunk and is stored, the rest when the chunk ends. A right pixel's
//              candidates (Dp columns) touch at most `sets` consecutive chunks, so chunk c stores into key set
//              c % sets and the epilogue takes the smallest key over the chunks that hold its candidates.
// The path values of column s + PF are loaded into registers while column s is reduced. The epilogue of a
// block (its rows, every chunk) finishes the float part (uniqueness, parabola) and the L-R check, as the sweep
// kernels do. No shared-memory atomics and no per-element range tests inside the row.
#pragma once

#include <cstdint>

#include "stereo_kernels.cuh"

namespace dsk {

constexpr int kWtaRowKeyBits = 7;
constexpr uint32_t kWtaRowNoKey = 0xFF00u;
constexpr int kWtaRowWarps = 4;       // warps per block
constexpr int kWtaRowMinBlocks = 8;   // blocks per SM the registers are sized for (32 warps)
constexpr int kWtaRowMaxSets = 5;     // right-WTA key sets (chunks of at least Dp / 4 columns)

constexpr int kWtaRowSmemWords = 2 * 32 * 8;  // per warp: two buffers (column parity) of 32 lanes x 8 words

struct WtaRowArgs {
    const uint8_t* values;  // [dir][y][x][dp] u8 path values, disparity k at byte k of a pixel
    size_t dir_stride;      // bytes per direction slab
    uint2* rec;             // [y][x] (key | second << 16, cost(k-1) | cost(k+1) << 16)
    uint16_t* rk;           // [sets][y][x] right-WTA keys, chunk c in set c % sets
    float* disp;            // L-R checked
    int w, h, nd, dp, min_disp;
    float uniqueness;
    int subpixel, lr_max_diff;
    int chunk;              // columns per chunk; chunk * nchunks >= w > (nchunks - 1) * chunk
    int lg_chunks;          // log2(nchunks); nchunks divides the block's segments (kWtaRowWarps * 32 / SEG)
    int sets;               // ceil((dp - 1) / chunk) + 1 (1 with one chunk), at most kWtaRowMaxSets
};

template <int N>
__device__ __forceinline__ uint32_t wr_tree_min(uint32_t (&v)[N]) {
#pragma unroll
    for (int n = N; n > 1; n = (n + 1) / 2)
#pragma unroll
        for (int r = 0; r < n / 2; ++r) v[r] = vmin2(v[r], v[r + (n + 1) / 2]);
    return v[0];
}

// Minimum of both 16-bit halves over the segment's lanes (a butterfly of shuffles; a redux.sync per segment
// mask measured slower here).
template <int SEG>
__device__ __forceinline__ uint32_t wr_seg_min2(uint32_t m, int seg) {
    return seg_min<SEG>(vmin2(m, prmt(m, m, 0x1032)), seg);
}

// One segment's chunk [xs, xs + chunk) of row y into key set `set`. PAD: nd < Dp (padding slots).
template <int R, int SEG, int PF, bool PAD>
__device__ __forceinline__ void wta_row_chunk(const WtaRowArgs& a, uint32_t* __restrict__ wsm, int y, bool live, int xs,
                                              int set, int seg, int sl) {
    constexpr int NV = 2 * R, CW = NV / 4, Dp = SEG * NV;
    // Shared-memory sums: store i of every lane side by side (QH 16-bit sums a store), no bank conflicts.
    constexpr int QH = R % 4 == 0 ? 8 : 4;
    const int yc = live ? y : a.h - 1;
    const int k0 = sl * NV;
    const int lane = threadIdx.x & 31;
    const long prow = static_cast<long>(yc) * a.w;
    // disparities of register r: kbase2 + 2r * 0x10001 = (k0 + 2r, k0 + 2r + 1)
    const uint32_t kbase2 = static_cast<uint32_t>(k0) | (static_cast<uint32_t>(k0 + 1) << 16);
    // Columns inside the row whose every slot's right pixel lies inside the row.
    const int x_in_lo = a.min_disp + Dp - 1, x_in_hi = min(a.w - 1 + a.min_disp, a.w - 1);
    const uint8_t* v0 = a.values + prow * Dp + k0;
    const size_t ds = a.dir_stride;
    uint32_t ring[PF][4][CW];
    auto fetch = [&](int u, int i) {  // ring slot u <- column xs + i (the row's last column past its end)
        const uint8_t* p = v0 + static_cast<long>(min(xs + i, a.w - 1)) * Dp;
#pragma unroll
        for (int d = 0; d < 4; ++d) ld_chunk<NV, LD_CS>(p + d * ds, ring[u][d]);
    };
    uint16_t* rk = a.rk + static_cast<size_t>(set) * a.w * a.h + prow;
    uint2* rec = a.rec + prow;
    uint32_t acc[R];
#pragma unroll
    for (int r = 0; r < R; ++r) acc[r] = 0xFFFFFFFFu;
    const int n = a.chunk;
#pragma unroll
    for (int u = 0; u < PF; ++u)
        if (u < n) fetch(u, u);
    for (int base = 0; base < n; base += PF) {
#pragma unroll
        for (int u = 0; u < PF; ++u) {
            const int s = base + u;
            if (s >= n) break;
            const int x = xs + s;
            // sums: pairs as bytes, then the two pairs in 16-bit lanes
            uint32_t tot[R];
#pragma unroll
            for (int i = 0; i < CW; ++i) {
                const uint32_t p01 = ring[u][0][i] + ring[u][1][i], p23 = ring[u][2][i] + ring[u][3][i];
                tot[2 * i] = prmt(p01, 0u, 0x4140) + prmt(p23, 0u, 0x4140);
                tot[2 * i + 1] = prmt(p01, 0u, 0x4342) + prmt(p23, 0u, 0x4342);
            }
            if (s + PF < n) fetch(u, s + PF);
            uint32_t key[R];
#pragma unroll
            for (int r = 0; r < R; ++r)
                key[r] = tot[r] * (1u << kWtaRowKeyBits) + (kbase2 + static_cast<uint32_t>(2 * r) * 0x00010001u);
            if constexpr (PAD) {  // padding slots: sums and keys all ones
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    const uint32_t m = (k0 + 2 * r >= a.nd ? 0x0000FFFFu : 0u) | (k0 + 2 * r + 1 >= a.nd ? 0xFFFF0000u : 0u);
                    key[r] |= m;
                    tot[r] |= m;
                }
            }
            if (x < x_in_lo || x > x_in_hi) {  // right pixels outside the row, or a virtual column: no candidates
                const bool in = x < a.w;
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    const int xa = x - a.min_disp - k0 - 2 * r, xb = xa - 1;
                    const uint32_t vm = (in && static_cast<unsigned>(xa) < static_cast<unsigned>(a.w) ? 0x0000FFFFu : 0u) |
                                        (in && static_cast<unsigned>(xb) < static_cast<unsigned>(a.w) ? 0xFFFF0000u : 0u);
                    key[r] |= ~vm;
                    tot[r] |= ~vm;
                }
            }
            // right WTA chains: add, store the chain leaving slot Dp-1, move on by one slot
#pragma unroll
            for (int r = 0; r < R; ++r) acc[r] = vmin2(acc[r], key[r]);
            {
                const int xr = x - a.min_disp - (Dp - 1);
                if (live && sl == SEG - 1 && static_cast<unsigned>(xr) < static_cast<unsigned>(a.w))
                    rk[xr] = static_cast<uint16_t>(acc[R - 1] >> 16);
                uint32_t t = __shfl_up_sync(kFull, acc[R - 1], 1, SEG);
                t = sl == 0 ? 0xFFFFFFFFu : t;
#pragma unroll
                for (int r = R - 1; r > 0; --r) acc[r] = mid2(acc[r - 1], acc[r]);
                acc[0] = mid2(t, acc[0]);
            }
            // left WTA
            const uint32_t kmin = wr_seg_min2<SEG>(wr_tree_min<R>(key), seg) & 0xFFFFu;
            const int bk = static_cast<int>(kmin & ((1u << kWtaRowKeyBits) - 1));
            uint32_t* buf = wsm + (s & 1) * (32 * 8);
            if constexpr (QH == 8) {
#pragma unroll
                for (int i = 0; i < R / 4; ++i)
                    reinterpret_cast<uint4*>(buf)[i * 32 + lane] = make_uint4(tot[4 * i], tot[4 * i + 1], tot[4 * i + 2], tot[4 * i + 3]);
            } else {
#pragma unroll
                for (int i = 0; i < R / 2; ++i) reinterpret_cast<uint2*>(buf)[i * 32 + lane] = make_uint2(tot[2 * i], tot[2 * i + 1]);
            }
            const uint32_t kc = vadd2(kbase2, splat2((1u - static_cast<uint32_t>(bk)) & 0xFFFFu));
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const uint32_t t = __viaddmin_u16x2(kc, static_cast<uint32_t>(2 * r) * 0x00010001u, 0x00030003u);
                tot[r] = __viaddmax_u16x2(t, 0xFFFDFFFDu, tot[r]);
            }
            const uint32_t second = wr_seg_min2<SEG>(wr_tree_min<R>(tot), seg) & 0xFFFFu;
            __syncwarp();
            if (live && sl == 0 && x < a.w) {
                // the sums of disparities bk -+ 1 (clamped into [0, nd): without candidates bk is not a disparity)
                const uint16_t* hb = reinterpret_cast<const uint16_t*>(buf);
                auto at = [&](int k) {
                    const int lk = k / NV, j = k - lk * NV;
                    return static_cast<uint32_t>(hb[((j / QH) * 32 + seg * SEG + lk) * QH + j % QH]);
                };
                const uint32_t cm = at(min(max(bk - 1, 0), a.nd - 1)), cp = at(min(bk + 1, a.nd - 1));
                rec[x] = make_uint2(kmin | (second << 16), cm | (cp << 16));
            }
        }
    }
    // flush: the chains were moved on after the last column, so slot k holds the right pixel of slot k - 1 there
    if (live) {
        const int xl = xs + n - 1;
#pragma unroll
        for (int r = 0; r < R; ++r) {
#pragma unroll
            for (int hf = 0; hf < 2; ++hf) {
                const int k = k0 + 2 * r + hf;
                if (k == 0) continue;  // moved in empty
                const int xr = xl - a.min_disp - (k - 1);
                if (static_cast<unsigned>(xr) < static_cast<unsigned>(a.w))
                    rk[xr] = static_cast<uint16_t>(hf ? (acc[r] >> 16) : acc[r]);
            }
        }
    }
}

// Float part of the WTA and the L-R check of rows [y_first, y_first + rows).
__device__ __forceinline__ void wta_row_epilogue(const WtaRowArgs& a, int y_first, int rows, int Dp) {
    const size_t plane = static_cast<size_t>(a.w) * a.h;
    const int n = rows * a.w;
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
        const int y = y_first + i / a.w, x = i % a.w;
        if (y >= a.h) break;
        const size_t p = static_cast<size_t>(y) * a.w + x;
        const uint2 r = __ldcg(a.rec + p);
        const int lo = max(0, x - a.min_disp - (a.w - 1));
        const int hi = min(a.nd, x - a.min_disp + 1);
        float d = kInvalid;
        if (hi > lo) {
            const uint32_t key = r.x & 0xFFFFu, sec = r.x >> 16;
            const int bk = static_cast<int>(key & ((1u << kWtaRowKeyBits) - 1));
            const uint32_t sb = key >> kWtaRowKeyBits;
            const uint32_t second = sec >= kWtaRowNoKey ? 0xFFFFu : sec;
            const bool unique =
                !(second != 0xFFFFu && static_cast<float>(sb) >= __fmul_rn(a.uniqueness, static_cast<float>(second)));
            if (unique) {
                d = static_cast<float>(a.min_disp + bk);
                if (a.subpixel && bk > lo && bk + 1 < hi)
                    d = __fadd_rn(d, parabola(static_cast<float>(r.y & 0xFFFFu), static_cast<float>(sb),
                                              static_cast<float>(r.y >> 16)));
            }
        }
        if (valid_disparity(d)) {
            const long xr = lroundf(__fsub_rn(static_cast<float>(x), d));
            if (xr < 0 || xr >= a.w) {
                d = kInvalid;
            } else {
                // chunks whose columns hold candidates of xr: [xr + min, xr + min + Dp - 1] within the row
                const int xa = max(static_cast<int>(xr) + a.min_disp, 0);
                const int xb = min(static_cast<int>(xr) + a.min_disp + Dp - 1, a.w - 1);
                uint32_t k = 0xFFFFu;
                if (xa <= xb) {
                    const size_t q = static_cast<size_t>(y) * a.w + xr;
                    const int ca = xa / a.chunk, cb = xb / a.chunk;
                    int set = ca % a.sets;
                    for (int c = ca; c <= cb; ++c) {
                        k = min(k, static_cast<uint32_t>(__ldcg(a.rk + set * plane + q)));
                        set = set + 1 == a.sets ? 0 : set + 1;
                    }
                }
                if (k >= kWtaRowNoKey) {
                    d = kInvalid;
                } else {
                    const int rd = a.min_disp + static_cast<int>(k & ((1u << kWtaRowKeyBits) - 1));
                    if (fabsf(__fsub_rn(static_cast<float>(rd), d)) > static_cast<float>(a.lr_max_diff)) d = kInvalid;
                }
            }
        }
        a.disp[p] = d;
    }
}

// Block: kWtaRowWarps warps, 32 / SEG segments each; segment u of the block sweeps chunk u % nchunks of row
// u / nchunks of the block's rows.
template <int R, int SEG, int PF, bool PAD>
__device__ __forceinline__ void wta_rows_body(const WtaRowArgs& a, uint32_t* __restrict__ smem, int bx) {
    constexpr int SPW = 32 / SEG, U = kWtaRowWarps * SPW;
    const int lane = threadIdx.x & 31, seg = lane / SEG, sl = lane % SEG;
    const int warp = threadIdx.x >> 5;
    const int u = warp * SPW + seg;
    const int rows = U >> a.lg_chunks;
    const int y = bx * rows + (u >> a.lg_chunks), c = u & ((1 << a.lg_chunks) - 1);
    wta_row_chunk<R, SEG, PF, PAD>(a, smem + warp * kWtaRowSmemWords, y, y < a.h, c * a.chunk, c % a.sets, seg, sl);
    __syncthreads();  // every chunk's records and right-WTA keys of the block's rows are stored
    wta_row_epilogue(a, bx * rows, rows, SEG * 2 * R);
}

template <int R, int SEG, int PF, bool PAD>
__global__ void __launch_bounds__(32 * kWtaRowWarps, kWtaRowMinBlocks) k_wta_rows(WtaRowArgs a) {
    __shared__ __align__(16) uint32_t smem[kWtaRowSmemWords * kWtaRowWarps];
    wta_rows_body<R, SEG, PF, PAD>(a, smem, blockIdx.x);
}

// Batch form: one block per virtual block (the rows of one block) of any pair of the group.
template <int R, int SEG, int PF, bool PAD>
__global__ void __launch_bounds__(32 * kWtaRowWarps, kWtaRowMinBlocks) kb_wta_rows(const WtaRowArgs* __restrict__ args,
                                                                                 const int* __restrict__ pairs,
                                                                                 const int* __restrict__ prefix, int n,
                                                                                 int total) {
    __shared__ __align__(16) uint32_t smem[kWtaRowSmemWords * kWtaRowWarps];
    __shared__ WtaRowArgs sa;
    int cur = -1;
    for (int v = blockIdx.x; v < total; v += gridDim.x) {
        int lo = 0, hi = n;
        while (hi - lo > 1) {
            const int m = (lo + hi) >> 1;
            if (__ldg(prefix + m) <= v) lo = m;
            else hi = m;
        }
        const int p = __ldg(pairs + lo);
        if (p != cur) {
            __syncthreads();
            if (threadIdx.x == 0) sa = args[p];
            __syncthreads();
            cur = p;
        }
        wta_rows_body<R, SEG, PF, PAD>(sa, smem, v - __ldg(prefix + lo));
        __syncthreads();  // the epilogue's reads are done before the next virtual block's writes
    }
}

}  // namespace dsk
