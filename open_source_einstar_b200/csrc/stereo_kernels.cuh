// SGM kernels of the stereo hot path (sm_100a): cost volume, path aggregation, WTA + L-R check.
//
// Layout in HBM (per frame, W x H, D disparities, P path directions):
//   rectified left/right    u8  [y][x]
//   census left/right       u32 or u64 [y][x] (u32 when the window has <= 32 neighbours)
//   matching costs          u8 [y][x][Dp] (only when materialised)
//   path values             u8 (or u16) [dir][y][x][Dp], Dp = SEG * 2R >= D; one slab per direction
//   L-R checked disparity   f32 [y][x]
// Outputs (f32 disparity, f32 confidence, u16 disparity, f32 depth) are written by the last kernel.
//
// Bit-exactness: integer stages reproduce libs/depth/src/stereo.cpp exactly; float stages use
// explicitly rounded intrinsics (__fadd_rn, __fmul_rn, __fdiv_rn, ...) so that nvcc cannot contract
// them into FMAs, which the reference's separately rounded x86 arithmetic does not do.
#pragma once

#include <type_traits>

#include <cstdint>
#include <climits>

#include "simd.cuh"

namespace dsk {

constexpr float kInvalid = -1.0e9f;  // depth::kInvalidDisparity (stereo.hpp:23)
constexpr int kNoMatch = INT_MIN;    // sgm_disparity's kNoMatch (stereo.cpp:413)
constexpr int kMaxDisparities = 512;
// Guard rows above and below the census, guide and sweep buffers (>= the deepest prefetch ring), so that
// prefetches past a scanline's end stay inside the allocation.
constexpr int kGuardRows = 8;
constexpr unsigned kFull = 0xFFFFFFFFu;

__host__ __device__ inline bool valid_disparity(float d) { return d > -1.0e8f; }  // stereo.hpp:24

// The median of the valid values of a 3x3 neighbourhood as median3 / the spike filter take it
// (stereo.cpp:129-147, 305-325): element n/2 of the n valid values in ascending order. Invalid values become
// +inf and sink to the end of a 25-comparator sorting network over the nine values, all in registers (an
// insertion sort into an array indexed at run time lives in local memory). Returns n through `count`.
__device__ __forceinline__ float median_of_valid9(float (&v)[9], int& count) {
    int n = 0;
#pragma unroll
    for (int k = 0; k < 9; ++k) {
        const bool ok = valid_disparity(v[k]);
        n += ok;
        v[k] = ok ? v[k] : __int_as_float(0x7F800000);
    }
#define DSK_CE(i, j)                                                 \
    {                                                                \
        const float lo_ = fminf(v[i], v[j]), hi_ = fmaxf(v[i], v[j]); \
        v[i] = lo_;                                                  \
        v[j] = hi_;                                                  \
    }
    DSK_CE(0, 1) DSK_CE(3, 4) DSK_CE(6, 7) DSK_CE(1, 2) DSK_CE(4, 5) DSK_CE(7, 8) DSK_CE(0, 1) DSK_CE(3, 4) DSK_CE(6, 7)
    DSK_CE(0, 3) DSK_CE(3, 6) DSK_CE(0, 3) DSK_CE(1, 4) DSK_CE(4, 7) DSK_CE(1, 4) DSK_CE(2, 5) DSK_CE(5, 8) DSK_CE(2, 5)
    DSK_CE(1, 3) DSK_CE(5, 7) DSK_CE(2, 6) DSK_CE(4, 6) DSK_CE(2, 4) DSK_CE(2, 3) DSK_CE(5, 6)
#undef DSK_CE
    const int m = n / 2;
    float r = v[0];
#pragma unroll
    for (int k = 1; k < 9; ++k) r = m == k ? v[k] : r;
    count = n;
    return r;
}

// Path directions in the reference's order (stereo.cpp:387-388).
static __constant__ int c_dir_dx[8] = {1, -1, 0, 0, 1, -1, 1, -1};
static __constant__ int c_dir_dy[8] = {0, 0, 1, -1, 1, -1, -1, 1};

template <typename W>
__device__ __forceinline__ int popcount_word(W v);
template <>
__device__ __forceinline__ int popcount_word<uint32_t>(uint32_t v) { return __popc(v); }
template <>
__device__ __forceinline__ int popcount_word<uint64_t>(uint64_t v) { return __popcll(v); }

// ------------------------------------------------------------------------------------------------
// Matching costs materialised once per frame (optional; the path kernel can recompute them from the
// census instead): u8 [y][x][dp] in the same per-lane chunks as the path values.

struct CostArgs {
    const void* census_l;  // (y, x) at y * cpitch + x
    const void* census_r;
    uint8_t* costs;
    int w, h, nd, dp, min_disp, invalid_cost, cpitch;
};

template <int R, int SEG, typename CW>
__device__ __forceinline__ void costs_body(const CostArgs& a, int bx) {
    constexpr int NV = 2 * R;
    const int lane = threadIdx.x & 31, seg = lane / SEG, sl = lane % SEG;
    const long px = (static_cast<long>(bx) * (blockDim.x >> 5) + (threadIdx.x >> 5)) * (32 / SEG) + seg;
    if (px >= static_cast<long>(a.w) * a.h) return;
    const int y = static_cast<int>(px / a.w), x = static_cast<int>(px % a.w);
    const CW* cl = static_cast<const CW*>(a.census_l) + static_cast<size_t>(y) * a.cpitch;
    const CW* cr = static_cast<const CW*>(a.census_r) + static_cast<size_t>(y) * a.cpitch;
    const CW vl = __ldg(cl + x);
    const int k0 = sl * NV;
    uint32_t c[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int xa = x - a.min_disp - (k0 + 2 * r), xb = xa - 1;
        const uint32_t ca = (xa >= 0 && xa < a.w) ? popcount_word<CW>(vl ^ __ldg(cr + xa)) : a.invalid_cost;
        const uint32_t cb = (xb >= 0 && xb < a.w) ? popcount_word<CW>(vl ^ __ldg(cr + xb)) : a.invalid_cost;
        c[r] = ca | (cb << 16);
    }
    uint32_t w[chunk_words<NV>()];
    pack<uint8_t, NV>(c, w);
    st_chunk<NV, false>(a.costs + static_cast<size_t>(px) * a.dp + k0, w);
}

template <int R, int SEG, typename CW>
__global__ void __launch_bounds__(256) k_costs(CostArgs a) {
    costs_body<R, SEG, CW>(a, blockIdx.x);
}

// Row-tiled cost volume: one block per tile of kCostTile pixels of a row. The right census words the
// tile needs (kCostTile + dp - 1 of them) are staged in shared memory, four times with shifts of 0..3
// words, so that every thread reads the four words of its four consecutive disparities with one
// aligned 128-bit load (u32 census). Thread t of a pixel writes the bytes of disparities 4t..4t+3, so
// a warp stores whole 128-byte lines. Columns outside the right row give invalid_cost
// (stereo.cpp:366-377).
constexpr int kCostTile = 256;

// Words per shifted copy (a multiple of 4, so that every copy starts 16-byte aligned).
__host__ __device__ constexpr int cost_tile_copy_words(int dp) { return (kCostTile + dp + 3 + 3) / 4 * 4; }

template <typename CW>
__host__ __device__ constexpr size_t cost_tile_smem(int dp) {
    return sizeof(CW) * (static_cast<size_t>(sizeof(CW) == 4 ? 4 : 1) * cost_tile_copy_words(dp) + kCostTile);
}

template <typename CW>
__device__ __forceinline__ void cost_tile_body(const CostArgs& a, int b, CW* sm) {
    constexpr int NC = sizeof(CW) == 4 ? 4 : 1;  // shifted copies
    const int tiles = (a.w + kCostTile - 1) / kCostTile;
    const int y = b / tiles, x0 = (b % tiles) * kCostTile;
    const int nx = min(kCostTile, a.w - x0);
    const int r0 = x0 - a.min_disp - (a.dp - 1);  // right column of window slot 0
    const int nr = nx + a.dp - 1;
    const int cpy = cost_tile_copy_words(a.dp);
    CW* sl = sm + NC * cpy;
    const CW* cl = static_cast<const CW*>(a.census_l) + static_cast<size_t>(y) * a.cpitch;
    const CW* cr = static_cast<const CW*>(a.census_r) + static_cast<size_t>(y) * a.cpitch;
    __syncthreads();  // the previous tile's readers are done
    for (int i = threadIdx.x; i < nr; i += blockDim.x) {
        const int xr = r0 + i;
        const CW v = static_cast<unsigned>(xr) < static_cast<unsigned>(a.w) ? __ldg(cr + xr) : CW(0);
#pragma unroll
        for (int c = 0; c < NC; ++c)
            if (i - c >= 0) sm[c * cpy + i - c] = v;  // copy c holds word i at i - c
    }
    for (int i = threadIdx.x; i < nx; i += blockDim.x) sl[i] = __ldg(cl + x0 + i);
    __syncthreads();
    const uint32_t inv = static_cast<uint32_t>(a.invalid_cost);
    // Interior tiles: every right column of the window inside the row, no per-cost range test.
    const bool interior = r0 >= 0 && r0 + nr <= a.w;
    if constexpr (NC == 4) {
        if ((a.dp & 15) == 0) {
            // Sixteen costs a thread: thread t of a pixel takes the cost words t + j * tq (j < 4, tq = dp / 16
            // threads per pixel), so the threads of a pixel read consecutive 16-byte chunks of one shifted copy
            // and store consecutive words; four popcounts are packed by multiply-adds (FMA pipe).
            const int tq = a.dp >> 4;
            const int ppp = static_cast<int>(blockDim.x) / tq;
            const int t = threadIdx.x % tq, pi = threadIdx.x / tq;
            if (pi >= ppp) return;
            for (int px = pi; px < nx; px += ppp) {
                const CW vl = sl[px];
                uint32_t* dst = reinterpret_cast<uint32_t*>(a.costs + (static_cast<size_t>(y) * a.w + x0 + px) * a.dp);
#pragma unroll
                for (int j = 0; j < 4; ++j) {
                    const int w = t + j * tq;
                    const int g = px + a.dp - 4 - 4 * w;  // window slot of disparity 4w + 3
                    const int c = g & 3;
                    const uint4 q = *reinterpret_cast<const uint4*>(sm + c * cpy + g - c);
                    uint32_t b0 = popcount_word<CW>(vl ^ q.w), b1 = popcount_word<CW>(vl ^ q.z);
                    uint32_t b2 = popcount_word<CW>(vl ^ q.y), b3 = popcount_word<CW>(vl ^ q.x);
                    if (!interior) {  // byte jj: right column r0 + g + 3 - jj
                        const int xr = r0 + g + 3;
                        b0 = static_cast<unsigned>(xr) < static_cast<unsigned>(a.w) ? b0 : inv;
                        b1 = static_cast<unsigned>(xr - 1) < static_cast<unsigned>(a.w) ? b1 : inv;
                        b2 = static_cast<unsigned>(xr - 2) < static_cast<unsigned>(a.w) ? b2 : inv;
                        b3 = static_cast<unsigned>(xr - 3) < static_cast<unsigned>(a.w) ? b3 : inv;
                    }
                    dst[w] = (b3 * 256u + b2) * 65536u + (b1 * 256u + b0);
                }
            }
            return;
        }
    }
    const int tp = a.dp >> 2;  // threads per pixel
    const int ppp = static_cast<int>(blockDim.x) / tp;
    const int t = threadIdx.x % tp, pi = threadIdx.x / tp;
    if (pi >= ppp) return;
    for (int px = pi; px < nx; px += ppp) {
        const CW vl = sl[px];
        const int g = px + a.dp - 4 - 4 * t;  // window slot of disparity 4t + 3; slot g + 3 - j is disparity 4t + j
        CW wv[4];
        if constexpr (NC == 4) {
            const int c = g & 3;
            const uint4 q = *reinterpret_cast<const uint4*>(sm + c * cpy + g - c);
            wv[0] = q.x, wv[1] = q.y, wv[2] = q.z, wv[3] = q.w;
        } else {
#pragma unroll
            for (int j = 0; j < 4; ++j) wv[j] = sm[g + j];
        }
        uint32_t word = 0;
        if (interior) {
#pragma unroll
            for (int j = 0; j < 4; ++j) word |= static_cast<uint32_t>(popcount_word<CW>(vl ^ wv[3 - j])) << (8 * j);
        } else {
#pragma unroll
            for (int j = 0; j < 4; ++j) {  // byte j: disparity 4t + j, right column r0 + g + 3 - j
                const int xr = r0 + g + 3 - j;
                const uint32_t cst = static_cast<unsigned>(xr) < static_cast<unsigned>(a.w)
                                         ? static_cast<uint32_t>(popcount_word<CW>(vl ^ wv[3 - j])) : inv;
                word |= cst << (8 * j);
            }
        }
        *reinterpret_cast<uint32_t*>(a.costs + (static_cast<size_t>(y) * a.w + x0 + px) * a.dp + 4 * t) = word;
    }
}

template <typename CW>
__global__ void __launch_bounds__(256) k_cost_tiles(CostArgs a) {
    extern __shared__ __align__(16) unsigned char cost_smem[];
    cost_tile_body<CW>(a, blockIdx.x, reinterpret_cast<CW*>(cost_smem));
}

// ------------------------------------------------------------------------------------------------
// Path aggregation (stereo.cpp:44-89, directions and start pixels :382-409).
//
// A segment of SEG lanes (8, 16 or 32) runs one scanline; each lane holds NV = 2R consecutive
// disparities as R registers of two 16-bit lanes (k = sl*NV + 2r, +1). Per step and register:
//   k-1 / k+1 neighbours   byte-permutes of adjacent registers (across lanes: one shuffle up, one down)
//   k-2 / k+2 neighbours   the adjacent registers themselves (slant steps)
//   best = min(prev, min(prev) + P2', min(neighbours) + P1)      min.u16x2 / add.u16x2
//   L    = best + cost - min(prev)                                 modular 16-bit lanes (exact)
// min(prev) of the next step is a segment min-reduction (redux.sync). Costs come from the census
// (popcount of XOR) or from the materialised volume. Neighbours outside [0, nd) read INF = 0xFFFF - P1,
// which stays above every path value after + P1 (window + P2 <= 0xFFFF - 2 P1 is validated).
// Every value is exact in 16 bits; u8 storage is used when window + P2 <= 255 (values never exceed it).
// The directions of a frame run concurrently into separate slabs, summed by the WTA kernel.

struct PathArgs {
    const void* census_l;  // (y, x) at y * cpitch + x
    const void* census_r;
    int cpitch;
    const uint8_t* guide;
    const uint8_t* costs;  // materialised costs or nullptr
    void* values;          // [dir][y][x][dp]
    size_t dir_stride;     // elements per direction slab
    int w, h, nd, dp, min_disp, p1, invalid_cost, slant;
    int dir_base;
    int p2_table[32];
};

__device__ __forceinline__ void line_start(int dx, int dy, int line, int w, int h, int& x, int& y) {
    if (dy == 0) {
        x = dx > 0 ? 0 : w - 1;
        y = line;
    } else if (dx == 0) {
        x = line;
        y = dy > 0 ? 0 : h - 1;
    } else if (line < h) {
        x = dx > 0 ? 0 : w - 1;
        y = line;
    } else {
        const int j = line - h;  // entry-row starts, the shared corner excluded
        x = dx > 0 ? j + 1 : j;
        y = dy > 0 ? 0 : h - 1;
    }
}

__host__ __device__ __forceinline__ int lines_of(int dx, int dy, int w, int h) { return dy == 0 ? h : (dx == 0 ? w : h + w - 1); }

__device__ __forceinline__ int line_length(int dx, int dy, int x, int y, int w, int h) {
    int n = 0x7FFFFFFF;
    if (dx > 0) n = min(n, w - x);
    if (dx < 0) n = min(n, x + 1);
    if (dy > 0) n = min(n, h - y);
    if (dy < 0) n = min(n, y + 1);
    return n;
}

// Minimum over the lanes of this lane's segment.
template <int SEG>
__device__ __forceinline__ uint32_t seg_min(uint32_t v, int seg) {
    if constexpr (SEG == 32) {
        return __reduce_min_sync(kFull, v);
    } else if constexpr (SEG <= 8) {  // 4 or 8 segments per warp: one butterfly serves all of them
#pragma unroll
        for (int off = SEG / 2; off >= 1; off /= 2) v = min(v, __shfl_xor_sync(kFull, v, off));
        return v;
    } else {
        static_assert(SEG == 16, "segments of 4, 8, 16 or 32 lanes");
        const uint32_t r0 = __reduce_min_sync(kFull, seg == 0 ? v : 0xFFFFFFFFu);
        const uint32_t r1 = __reduce_min_sync(kFull, seg == 1 ? v : 0xFFFFFFFFu);
        return seg == 0 ? r0 : r1;
    }
}

// PF: depth of the register prefetch ring (the inputs of step s + PF are loaded while step s runs).
// p2: the adaptive-P2 table of `a` in shared memory (it is indexed by the intensity step every step).
template <int R, int SEG, typename CW, typename ST, bool MAT, int PF>
__device__ __forceinline__ void paths_body(const PathArgs& a, const int* p2, int bx, int by) {
    constexpr int NV = 2 * R;
    constexpr int LPW = 32 / SEG;  // lines per warp
    constexpr int CWN = chunk_words<NV>();
    constexpr int VB = NV * static_cast<int>(sizeof(ST));
    const int lane = threadIdx.x & 31, seg = lane / SEG, sl = lane % SEG;
    const int di = a.dir_base + by;
    const int dx = c_dir_dx[di], dy = c_dir_dy[di];
    const int nlines = lines_of(dx, dy, a.w, a.h);
    const int first = (bx * (blockDim.x >> 5) + (threadIdx.x >> 5)) * LPW;
    if (first >= nlines) return;  // warp-uniform
    const int line = first + seg;
    const bool live = line < nlines;
    int x0, y0;
    line_start(dx, dy, live ? line : first, a.w, a.h, x0, y0);
    const int len = live ? line_length(dx, dy, x0, y0, a.w, a.h) : 0;
    int nsteps = len;
    if constexpr (LPW == 2) nsteps = max(nsteps, __shfl_xor_sync(kFull, len, 16));
    if constexpr (LPW == 4) nsteps = static_cast<int>(__reduce_max_sync(kFull, static_cast<unsigned>(len)));

    const CW* __restrict__ cl = static_cast<const CW*>(a.census_l);
    const CW* __restrict__ cr = static_cast<const CW*>(a.census_r);
    ST* __restrict__ out = static_cast<ST*>(a.values) + static_cast<size_t>(di) * a.dir_stride;
    const int k0 = sl * NV;
    const uint32_t INF2 = splat2(0xFFFFu - static_cast<uint32_t>(a.p1)), P12 = splat2(a.p1);
    // 16-bit lanes beyond nd hold INF (so they are neither a minimum nor a neighbour).
    uint32_t pad[R];
    bool any_pad = false;
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int k = k0 + 2 * r;
        pad[r] = (k >= a.nd ? 0x0000FFFFu : 0u) | (k + 1 >= a.nd ? 0xFFFF0000u : 0u);
        any_pad |= pad[r] != 0u;
    }

    // Pixel index of step s: idx0 + s * dstep. Steps past the line's end (the shorter line of a warp's
    // pair, or a lane without a line) read the line's last pixel; their values are never stored.
    const int idx0 = y0 * a.w + x0, dstep = dy * a.w + dx, smax = max(len - 1, 0);
    // Prefetch ring: guide intensity and census words (or the cost chunk) of upcoming steps.
    int pI[PF];
    CW pvl[PF];
    CW pvr[PF][MAT ? 1 : NV];
    uint32_t pcw[PF][MAT ? CWN : 1];
    auto fetch = [&](int s, int u) {
        const int sc = min(s, smax);
        const int idx = idx0 + sc * dstep;
        pI[u] = __ldg(a.guide + idx);
        if constexpr (MAT) {
            ld_chunk<NV, LD_NC>(a.costs + static_cast<size_t>(idx) * a.dp + k0, pcw[u]);
        } else {
            const int cx = x0 + sc * dx, cy = y0 + sc * dy;
            const size_t crow = static_cast<size_t>(cy) * a.cpitch;
            pvl[u] = __ldg(cl + crow + cx);
#pragma unroll
            for (int j = 0; j < NV; ++j) {
                const int xr = cx - a.min_disp - (k0 + j);
                pvr[u][j] = (xr >= 0 && xr < a.w) ? __ldg(cr + crow + xr) : CW(0);
            }
        }
    };
    // Costs of the step at column x from slot u.
    auto costs = [&](int x, int u, uint32_t (&c)[R]) {
        if constexpr (MAT) {
            unpack<uint8_t, NV>(pcw[u], c);
        } else {
            const int cx = min(max(x, 0), a.w - 1);
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const int xa = cx - a.min_disp - (k0 + 2 * r), xb = xa - 1;
                const uint32_t ca = (xa >= 0 && xa < a.w) ? popcount_word<CW>(pvl[u] ^ pvr[u][2 * r]) : a.invalid_cost;
                const uint32_t cb = (xb >= 0 && xb < a.w) ? popcount_word<CW>(pvl[u] ^ pvr[u][2 * r + 1]) : a.invalid_cost;
                c[r] = prmt(ca, cb, 0x5410);
            }
        }
    };
    auto store = [&](int s, const uint32_t (&v)[R]) {
        uint32_t w[chunk_words<VB>()];
        pack<ST, NV>(v, w);
        st_chunk<VB, true>(out + static_cast<size_t>(idx0 + s * dstep) * a.dp + k0, w);
    };

    uint32_t prev[R], c[R];
    fetch(0, 0);
    costs(x0, 0, c);
    int last_i = pI[0];
#pragma unroll
    for (int u = 0; u < PF; ++u)
        if (1 + u < nsteps) fetch(1 + u, u);
    uint32_t lmin = 0xFFFFFFFFu;
#pragma unroll
    for (int r = 0; r < R; ++r) {
        prev[r] = any_pad ? ((c[r] & ~pad[r]) | (INF2 & pad[r])) : c[r];
        lmin = vmin2(lmin, prev[r]);
    }
    uint32_t pm = seg_min<SEG>(hmin2(lmin), seg);
    if (len > 0) store(0, prev);

    int x = x0, y = y0;
    // The step loop twice: with the padding masks, and without them for warps none of whose lanes has
    // padding (predicated-off instructions would still take issue slots on every step).
    auto steps = [&](auto pad_tag) {
    constexpr bool PAD = decltype(pad_tag)::value;
    for (int base = 1; base < nsteps; base += PF) {
#pragma unroll
        for (int u = 0; u < PF; ++u) {
            const int s = base + u;
            if (s >= nsteps) break;  // warp-uniform
            x += dx;
            y += dy;
            const int I = pI[u];
            costs(x, u, c);
            if (s + PF < nsteps) fetch(s + PF, u);
            const int dI = I > last_i ? I - last_i : last_i - I;
            last_i = I;
            const uint32_t jump2 = splat2(pm + static_cast<uint32_t>(p2[dI >> 3]));
            const uint32_t negpm = splat2(0x10000u - pm);
            uint32_t up = __shfl_up_sync(kFull, prev[R - 1], 1, SEG);
            uint32_t dn = __shfl_down_sync(kFull, prev[0], 1, SEG);
            if (sl == 0) up = INF2;
            if (sl == SEG - 1) dn = INF2;
            uint32_t cur[R];
            lmin = 0xFFFFFFFFu;
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const uint32_t lower = r == 0 ? up : prev[r - 1];      // (k-2, k-1)
                const uint32_t upper = r == R - 1 ? dn : prev[r + 1];  // (k+2, k+3)
                uint32_t m = vmin2(mid2(lower, prev[r]), mid2(prev[r], upper));  // k-1, k+1
                if (a.slant) m = vmin2(m, vmin2(lower, upper));
                const uint32_t best = vmin2(vmin2(vadd2(m, P12), prev[r]), jump2);
                uint32_t L = vadd2(vadd2(best, c[r]), negpm);
                if constexpr (PAD) L = (L & ~pad[r]) | (INF2 & pad[r]);
                cur[r] = L;
                lmin = vmin2(lmin, L);
            }
            pm = seg_min<SEG>(hmin2(lmin), seg);
#pragma unroll
            for (int r = 0; r < R; ++r) prev[r] = cur[r];
            if (s < len) store(s, cur);
        }
    }
    };
    if (__any_sync(kFull, any_pad)) steps(std::integral_constant<bool, true>{});
    else steps(std::integral_constant<bool, false>{});
}

template <int R, int SEG, typename CW, typename ST, bool MAT, int PF>
__global__ void __launch_bounds__(256) k_paths(PathArgs a) {
    __shared__ int p2[32];
    if (threadIdx.x < 32) p2[threadIdx.x] = a.p2_table[threadIdx.x];
    __syncthreads();
    paths_body<R, SEG, CW, ST, MAT, PF>(a, p2, blockIdx.x, blockIdx.y);
}

// ------------------------------------------------------------------------------------------------
// Winner-takes-all left + right and the L-R check (stereo.cpp:411-461), one CTA per row.
// A segment of SEG lanes takes one pixel: the direction slabs are summed as 16-bit lanes (the
// reference's u16 sums, wrap included); left WTA = segment min of (cost << 16 | k) keys (first strict
// minimum), best non-adjacent cost by a second reduction, uniqueness as a float compare, parabola from
// the neighbours' costs. Right WTA: every candidate (x, k) offers its key to right pixel x - min - k by
// a shared-memory atomicMin, which leaves the first strict minimum along that diagonal. Warps whose
// pixels are interior (every disparity has a right column) skip the per-element range tests.

struct WtaArgs {
    const void* values;
    size_t dir_stride;
    int ndirs;
    int w, h, nd, dp, min_disp;
    float uniqueness;
    int subpixel;
    int lr_max_diff;
    float* disp;  // L-R checked
    // u8 path values with 2 (window + P2) <= 255: two directions add as whole 32-bit words (no carry
    // crosses a byte), halving the unpacking work. 0 for the general path.
    int pair_sums;
};

__device__ __forceinline__ float parabola(float cm, float c0, float cp) {  // stereo.cpp:92-96
    const float denom = __fadd_rn(__fsub_rn(cm, __fmul_rn(2.0f, c0)), cp);
    if (denom <= 0.0f) return 0.0f;
    const float t = __fdiv_rn(__fmul_rn(0.5f, __fsub_rn(cm, cp)), denom);
    return fminf(fmaxf(t, -0.5f), 0.5f);
}

template <int R>
__device__ __forceinline__ uint32_t pick16(const uint32_t (&v)[R], int j) {  // 16-bit value j of the lane's chunk
    uint32_t w = 0;
#pragma unroll
    for (int i = 0; i < R; ++i)
        if (i == (j >> 1)) w = v[i];
    return (j & 1) ? (w >> 16) : (w & 0xFFFFu);
}

template <int R, int SEG, typename ST, int NDIRS>
__device__ __forceinline__ void wta_body(const WtaArgs& a, int bx) {
    constexpr int NV = 2 * R;
    constexpr int VB = NV * static_cast<int>(sizeof(ST));
    constexpr int VW = chunk_words<VB>();
    constexpr uint32_t kEmpty = 0xFFFFFFFFu;
    extern __shared__ uint32_t smem[];
    uint32_t* rkey = smem;                                // [w]
    float* dleft = reinterpret_cast<float*>(smem + a.w);  // [w]
    const int y = bx;
    const int lane = threadIdx.x & 31, seg = lane / SEG, sl = lane % SEG;
    const int warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    for (int i = threadIdx.x; i < a.w; i += blockDim.x) rkey[i] = kEmpty;
    __syncthreads();

    const ST* __restrict__ vals = static_cast<const ST*>(a.values);
    const int k0 = sl * NV;
    const int per_warp = 32 / SEG;
    const int stride = nwarps * per_warp;
    // Per register r: the (k, k + 1) index pair of the keys, and masks of the disparities >= nd (padding
    // of the lane slabs): full keys and 16-bit halves.
    uint32_t kk[R], pada[R], padb[R], padh[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int ka = k0 + 2 * r;
        kk[r] = static_cast<uint32_t>(ka) | (static_cast<uint32_t>(ka + 1) << 16);
        pada[r] = ka >= a.nd ? kEmpty : 0u;
        padb[r] = ka + 1 >= a.nd ? kEmpty : 0u;
        padh[r] = (pada[r] & 0xFFFFu) | (padb[r] & 0xFFFF0000u);
    }
    const bool unpadded = a.nd == SEG * NV;  // every lane slot is a real disparity
    // Double buffer: the next pixel's chunks are in flight while this one is reduced.
    uint32_t nxt[NDIRS][VW];
    auto fetch = [&](int xb) {
        const int xc = min(xb + seg, a.w - 1);
        const size_t base = (static_cast<size_t>(y) * a.w + xc) * a.dp + k0;
#pragma unroll
        for (int d = 0; d < NDIRS; ++d) ld_chunk<VB, LD_CS>(vals + static_cast<size_t>(d) * a.dir_stride + base, nxt[d]);
    };
    int xb = warp * per_warp;
    if (xb < a.w) fetch(xb);
    for (; xb < a.w; xb += stride) {
        const int x = xb + seg;
        const bool live = x < a.w;
        const int xc = live ? x : a.w - 1;
        uint32_t tot[R];
        bool paired = false;
        if constexpr (sizeof(ST) == 1) {
            if (a.pair_sums) {
                uint32_t ps[VW];
#pragma unroll
                for (int d = 0; d < NDIRS; d += 2) {
#pragma unroll
                    for (int w = 0; w < VW; ++w) ps[w] = nxt[d][w] + nxt[d + 1][w];
                    uint32_t v[R];
                    unpack<uint8_t, NV>(ps, v);
#pragma unroll
                    for (int r = 0; r < R; ++r) tot[r] = d == 0 ? v[r] : vadd2(tot[r], v[r]);
                }
                paired = true;
            }
        }
        if (!paired) {
#pragma unroll
            for (int d = 0; d < NDIRS; ++d) {
                uint32_t v[R];
                unpack<ST, NV>(nxt[d], v);
#pragma unroll
                for (int r = 0; r < R; ++r) tot[r] = d == 0 ? v[r] : vadd2(tot[r], v[r]);
            }
        }
        if (xb + stride < a.w) fetch(xb + stride);
        const int lo = max(0, xc - a.min_disp - (a.w - 1));
        const int hi = min(a.nd, xc - a.min_disp + 1);
        const int rbase = xc - a.min_disp - k0;  // right column of the lane's first disparity
        uint32_t key, second;
        if (__all_sync(kFull, live && lo == 0 && hi == a.nd)) {
            // Interior pixels (every disparity < nd matches a column of the right row): no per-element
            // range tests; padding keys are all ones and take part in nothing. Without padding (nd fills
            // the lane slabs) the padding masks and tests drop out.
            uint32_t kmin = kEmpty;
            if (unpadded) {
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    const uint32_t key_a = prmt(kk[r], tot[r], 0x5410);  // (cost_a << 16) | ka
                    const uint32_t key_b = prmt(kk[r], tot[r], 0x7632);  // (cost_b << 16) | ka + 1
                    kmin = min(kmin, min(key_a, key_b));
                    atomicMin(&rkey[rbase - 2 * r], key_a);
                    atomicMin(&rkey[rbase - 2 * r - 1], key_b);
                }
            } else {
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    const uint32_t key_a = prmt(kk[r], tot[r], 0x5410) | pada[r];
                    const uint32_t key_b = prmt(kk[r], tot[r], 0x7632) | padb[r];
                    kmin = min(kmin, min(key_a, key_b));
                    if (key_a != kEmpty) atomicMin(&rkey[rbase - 2 * r], key_a);
                    if (key_b != kEmpty) atomicMin(&rkey[rbase - 2 * r - 1], key_b);
                }
            }
            key = seg_min<SEG>(kmin, seg);
            const int bk = static_cast<int>(key & 0xFFFFu);
            uint32_t m2 = kEmpty;
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const int ka = k0 + 2 * r;
                // disparities within one of bk are not the second minimum (stereo.cpp:420-424)
                const uint32_t ex = (static_cast<unsigned>(ka - bk + 1) <= 2u ? 0x0000FFFFu : 0u) |
                                    (static_cast<unsigned>(ka - bk + 2) <= 2u ? 0xFFFF0000u : 0u);
                m2 = vmin2(m2, tot[r] | (unpadded ? 0u : padh[r]) | ex);
            }
            second = seg_min<SEG>(hmin2(m2), seg);
        } else {
            uint32_t kmin = kEmpty;
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const int ka = k0 + 2 * r;
                const uint32_t key_a = prmt(kk[r], tot[r], 0x5410);
                const uint32_t key_b = prmt(kk[r], tot[r], 0x7632);
                if (live && ka >= lo && ka < hi) {
                    kmin = min(kmin, key_a);
                    atomicMin(&rkey[rbase - 2 * r], key_a);
                }
                if (live && ka + 1 >= lo && ka + 1 < hi) {
                    kmin = min(kmin, key_b);
                    atomicMin(&rkey[rbase - 2 * r - 1], key_b);
                }
            }
            key = seg_min<SEG>(kmin, seg);
            const int bk = static_cast<int>(key & 0xFFFFu);
            uint32_t sec = 0xFFFFu;
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const int ka = k0 + 2 * r;
                if (ka >= lo && ka < hi && (ka - bk > 1 || bk - ka > 1)) sec = min(sec, tot[r] & 0xFFFFu);
                if (ka + 1 >= lo && ka + 1 < hi && (ka + 1 - bk > 1 || bk - ka - 1 > 1)) sec = min(sec, tot[r] >> 16);
            }
            second = seg_min<SEG>(sec, seg);
        }
        const int bk = static_cast<int>(key & 0xFFFFu);
        const int km = max(bk - 1, 0), kp = min(bk + 1, a.nd - 1);
        const uint32_t vm = __shfl_sync(kFull, pick16<R>(tot, km % NV), km / NV, SEG);
        const uint32_t vp = __shfl_sync(kFull, pick16<R>(tot, kp % NV), kp / NV, SEG);
        if (live && sl == 0) {
            float d = kInvalid;
            if (hi > lo) {
                const uint32_t sb = key >> 16;
                const bool unique = !(second != 0xFFFFu && static_cast<float>(sb) >= __fmul_rn(a.uniqueness, static_cast<float>(second)));
                if (unique) {
                    d = static_cast<float>(a.min_disp + bk);
                    if (a.subpixel && bk > lo && bk + 1 < hi)
                        d = __fadd_rn(d, parabola(static_cast<float>(vm), static_cast<float>(sb), static_cast<float>(vp)));
                }
            }
            dleft[x] = d;
        }
    }
    __syncthreads();

    for (int x = threadIdx.x; x < a.w; x += blockDim.x) {
        float d = dleft[x];
        if (valid_disparity(d)) {
            const long xr = lroundf(__fsub_rn(static_cast<float>(x), d));
            if (xr < 0 || xr >= a.w) {
                d = kInvalid;
            } else {
                const uint32_t k = rkey[xr];
                if (k >= 0xFFFF0000u) {
                    d = kInvalid;
                } else {
                    const int rd = a.min_disp + static_cast<int>(k & 0xFFFFu);
                    if (fabsf(__fsub_rn(static_cast<float>(rd), d)) > static_cast<float>(a.lr_max_diff)) d = kInvalid;
                }
            }
        }
        a.disp[static_cast<size_t>(y) * a.w + x] = d;
    }
}

template <int R, int SEG, typename ST, int NDIRS>
__global__ void __launch_bounds__(256, sizeof(ST) == 1 && NDIRS == 4 ? 4 : 1) k_wta(WtaArgs a) {
    wta_body<R, SEG, ST, NDIRS>(a, blockIdx.x);
}

}  // namespace dsk
