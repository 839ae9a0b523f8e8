// Four-path SGM in two sweep kernels per frame (sm_100a), the throughput form of stereo.cpp:44-89 and
// :364-461 for frames whose summed path costs fit 16-bit WTA keys.
//
//   k_sweep_cols  the down (0,+1) and up (0,-1) directions of a group of columns, as two sets of warps that
//                 meet in the middle: each writes its path values for its first half of the column into S,
//                 then, after a block barrier, adds its own values over the other half. S = L_down + L_up.
//   k_sweep_rows  the left-to-right and right-to-left directions of a group of rows, meeting in the middle
//                 the same way through T. Over its second half each sweep holds the reference's 4-direction
//                 sum S + T + L of a pixel in registers and runs the winner-takes-all there: left WTA and
//                 the best non-adjacent cost (stereo.cpp:414-433), and its part of the right WTA along the
//                 diagonals (:434-447). An epilogue over the block's rows finishes the float part (uniqueness,
//                 parabola) and the L-R check (:450-461).
//
// Costs are computed from the census words: once per pixel in the column kernel (each direction computes the
// rows of its first half and stores them as bytes in C; its second half reads the other direction's), and
// again in each direction of the row kernel, where the right census words come through a sliding window
// in registers (popcount runs on its own pipe). Per-disparity traffic: S written twice and read twice, C
// written and read once, T written and read once: 8 bytes per pixel and disparity, instead of the cost
// volume plus four direction slabs.
//
// Lane layout. SEG lanes run one scanline; lane sl holds NV = 2R disparities k0 = sl*NV .. k0+NV-1 in R
// registers of two 16-bit lanes, register r holding slots (r, r + R). The k-1 / k+1 / k-2 / k+2 neighbours of
// register r are then whole registers (r-1, r+1, r-2, r+2) except at the slab edges, where one byte-permute
// joins this lane's register with the neighbouring lane's (one shuffle each way). Path values are at most
// window + P2 <= 127 here (S must fit a byte), so the recurrence's adds are plain 32-bit adds: no 16-bit lane
// ever carries (INF = 0xFFFF - P1 stays below 0xFFFF after + P1, and best >= min(prev) never borrows).
// In memory a lane's NV bytes are its registers packed pairwise: word i = (reg 2i lo, reg 2i+1 lo, reg 2i hi,
// reg 2i+1 hi), the layout both kernels (and nothing else) read.
//
// WTA keys are (sum << 7) | k in 16 bits: sums are at most 4 * 127 = 508 and k < 128, so a 16-bit min orders
// candidates by cost, then by the lower disparity (the reference's first strict minimum). Keys of candidates
// outside the image row or beyond nd are 0xFFFF; excluded neighbours of the best are raised to >= 0xFFFD.
#pragma once

#include <cstdint>

#include "stereo_kernels.cuh"

namespace dsk {

constexpr int kSweepKeyBits = 7;
constexpr uint32_t kSweepNoKey = 0xFF00u;  // keys at or above this mark no candidate
constexpr int kSweepColWarps = 4;          // warps per direction of a column-kernel block (columns by residue mod 4)
constexpr int kSweepRowWarps = 2;          // warps per direction of a row-kernel block

struct SweepArgs {
    const uint32_t* census_l;  // 32-bit census words, (y, x) at y * cpitch + x; guard rows and columns readable
    const uint32_t* census_r;
    int cpitch;
    const uint8_t* guide;      // left rectified image, (y, x) at y * w + x; guard rows readable
    uint8_t* S;                // [y][x][dp] vertical pair sums (guard rows)
    uint8_t* T;                // [y][x][dp] first-half values of the horizontal sweeps (guard rows)
    uint8_t* C;                // [y][x][dp] matching costs of the column kernel's first halves (guard rows)
    uint2* rec;                // [y][x] left WTA of the row kernel: (key | second << 16, cost(k-1) | cost(k+1) << 16)
    uint16_t* rk;              // [2][y][x] right-WTA keys of the left-to-right and right-to-left sweeps
    float* disp;               // L-R checked disparity [y][x]
    int w, h, nd, dp, min_disp, p1, invalid_cost;
    float uniqueness;
    int subpixel, lr_max_diff;
    uint32_t p2_table2[32];    // P2' per |dI| / 8 in both 16-bit lanes
};

// Sweep kernels exist for these shapes: 2R disparities per lane in R in {6, 8}, SEG lanes per line in {4, 8}
// (D up to 128), and frames with 4 paths, census windows of at most 32 neighbours and 2 (window + P2) <= 255.
__host__ __device__ constexpr bool sweep_shape_ok(int R, int seg) { return (R == 6 || R == 8) && (seg == 4 || seg == 8); }

__device__ __forceinline__ uint32_t sw_min3(uint32_t a, uint32_t b, uint32_t c) { return vmin2(vmin2(a, b), c); }

// Block barrier for warps that reach it from different code (the two sweep directions are separate template
// instances): the non-aligned form of the CTA barrier, with the memory ordering of __syncthreads.
__device__ __forceinline__ void sw_block_barrier() { asm volatile("barrier.sync 0;" ::: "memory"); }

// Minimum over the segment's lanes of a value held in both 16-bit lanes (the result likewise).
template <int SEG>
__device__ __forceinline__ uint32_t sw_seg_min2(uint32_t lmin2, int seg) {
    return seg_min<SEG>(vmin2(lmin2, prmt(lmin2, lmin2, 0x1032)), seg);
}

// Minimum of v[0..N) into v[0] by a tree (a short dependency chain); v is overwritten.
template <int N>
__device__ __forceinline__ uint32_t sw_tree_min(uint32_t (&v)[N]) {
#pragma unroll
    for (int n = N; n > 1; n = (n + 1) / 2)
#pragma unroll
        for (int r = 0; r < n / 2; ++r) v[r] = vmin2(v[r], v[r + (n + 1) / 2]);
    return v[0];
}

template <int R>
__device__ __forceinline__ void sw_unpack(const uint32_t (&w)[R / 2], uint32_t (&v)[R]) {
#pragma unroll
    for (int i = 0; i < R / 2; ++i) {
        v[2 * i] = w[i] & 0x00FF00FFu;
        v[2 * i + 1] = (w[i] >> 8) & 0x00FF00FFu;
    }
}

template <int R>
__device__ __forceinline__ void sw_pack(const uint32_t (&v)[R], uint32_t (&w)[R / 2]) {
#pragma unroll
    for (int i = 0; i < R / 2; ++i) w[i] = v[2 * i] | (v[2 * i + 1] << 8);
}

// One step of the path recurrence (stereo.cpp:64-83) for a lane: v = previous values (updated in place),
// pm2 = their minimum over the scanline in both lanes (updated), c = costs of this pixel, jump2 = pm + P2'.
template <int R, int SEG, bool SLANT, bool PAD>
__device__ __forceinline__ void sw_step(uint32_t (&v)[R], uint32_t& pm2, const uint32_t (&c)[R], uint32_t jump2,
                                        uint32_t INF2, uint32_t P12, const uint32_t (&pad)[R], int sl, int seg) {
    uint32_t up1 = __shfl_up_sync(kFull, v[R - 1], 1, SEG);
    uint32_t dn1 = __shfl_down_sync(kFull, v[0], 1, SEG);
    up1 = sl == 0 ? INF2 : up1;
    dn1 = sl == SEG - 1 ? INF2 : dn1;
    const uint32_t km1_0 = prmt(up1, v[R - 1], 0x5432);  // slots (-1, R-1)
    const uint32_t kp1_e = prmt(v[0], dn1, 0x5432);      // slots (R, 2R)
    uint32_t km2_0 = 0, kp2_e = 0;
    if constexpr (SLANT) {
        uint32_t up2 = __shfl_up_sync(kFull, v[R - 2], 1, SEG);
        uint32_t dn2 = __shfl_down_sync(kFull, v[1], 1, SEG);
        up2 = sl == 0 ? INF2 : up2;
        dn2 = sl == SEG - 1 ? INF2 : dn2;
        km2_0 = prmt(up2, v[R - 2], 0x5432);  // slots (-2, R-2)
        kp2_e = prmt(v[1], dn2, 0x5432);      // slots (R+1, 2R+1)
    }
    uint32_t out[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const uint32_t km1 = r == 0 ? km1_0 : v[r - 1];
        const uint32_t kp1 = r == R - 1 ? kp1_e : v[r + 1];
        uint32_t m;
        if constexpr (SLANT) {
            const uint32_t km2 = r == 0 ? km2_0 : (r == 1 ? km1_0 : v[r - 2]);
            const uint32_t kp2 = r == R - 1 ? kp2_e : (r == R - 2 ? kp1_e : v[r + 2]);
            m = vmin2(vmin2(km1, kp1), vmin2(km2, kp2));
        } else {
            m = vmin2(km1, kp1);
        }
        const uint32_t best = sw_min3(m + P12, v[r], jump2);
        uint32_t L = best + c[r] - pm2;
        if constexpr (PAD) L = (L & ~pad[r]) | (INF2 & pad[r]);
        out[r] = L;
    }
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = out[r];
    pm2 = sw_seg_min2<SEG>(sw_tree_min<R>(out), seg);
}

// The first pixel of a scanline: L = C (padding slots INF).
template <int R, int SEG, bool PAD>
__device__ __forceinline__ void sw_first(uint32_t (&v)[R], uint32_t& pm2, const uint32_t (&c)[R], uint32_t INF2,
                                         const uint32_t (&pad)[R], int seg) {
    uint32_t lmin = 0xFFFFFFFFu;
#pragma unroll
    for (int r = 0; r < R; ++r) {
        v[r] = PAD ? ((c[r] & ~pad[r]) | (INF2 & pad[r])) : c[r];
        lmin = vmin2(lmin, v[r]);
    }
    pm2 = sw_seg_min2<SEG>(lmin, seg);
}

__device__ __forceinline__ uint32_t sw_p2(const uint32_t* __restrict__ p2t, int I, int& last) {
    const int d = I > last ? I - last : last - I;
    last = I;
    return p2t[d >> 3];
}

// Costs of a lane's slots at one pixel from 4*NQ right census words loaded from a 16-byte aligned start:
// slot j's word (right column x - min - k0 - j) is q[AL + NV - 1 - j].
template <int R, int AL, int NW>
__device__ __forceinline__ void sw_costs_aligned(uint32_t lw, const uint32_t (&q)[NW], uint32_t (&c)[R]) {
    constexpr int NV = 2 * R;
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const uint32_t ca = static_cast<uint32_t>(__popc(lw ^ q[AL + NV - 1 - r]));
        const uint32_t cb = static_cast<uint32_t>(__popc(lw ^ q[AL + NV - 1 - r - R]));
        c[r] = ca | (cb << 16);
    }
}

// ------------------------------------------------------------------------------------------------
// Column kernel. Block: kSweepColWarps warps sweep down, as many sweep up. Warp wi takes columns
// base + wi + 4 * seg (one per segment), so that all its columns have the same residue mod 4: the right
// census words of every lane then start at the same offset within a 16-byte line, and each lane loads its
// NV words with NQ aligned 128-bit loads. A block covers 4 * (32 / SEG) columns.
// First half of a column: costs from the census (stored to C), path values to S. Second half: costs from
// C (the other direction's first half), S += own path values.

template <int R, int SEG, bool SLANT, bool PAD, int PF>
__device__ __forceinline__ void sweep_cols_body(const SweepArgs& a, const uint32_t* __restrict__ p2t, int bx) {
    constexpr int NV = 2 * R, LPW = 32 / SEG, NQ = (NV + 6) / 4, NW = 4 * NQ, CW = R / 2;
    const int lane = threadIdx.x & 31, seg = lane / SEG, sl = lane % SEG;
    const int warp = threadIdx.x >> 5;
    const bool down = warp < kSweepColWarps;
    const int wi = down ? warp : warp - kSweepColWarps;
    const int x = bx * (kSweepColWarps * LPW) + wi + kSweepColWarps * seg;  // may lie past the row (dead lane)
    const bool live = x < a.w;
    // A lane past the row keeps its column for the right census words (so that the warp's loads stay on one
    // alignment; the census guard columns cover them) and reads everything else at the row's last column.
    const int xs = live ? x : a.w - 1;
    const int k0 = sl * NV;
    const int wb = x - a.min_disp - k0 - (NV - 1);  // right column of slot NV-1 (the lowest address)
    const int al = wb & 3;                          // the same for every lane of the warp
    const int qb = wb - al;
    const uint32_t INF2 = splat2(0xFFFFu - static_cast<uint32_t>(a.p1)), P12 = splat2(static_cast<uint32_t>(a.p1));
    const uint32_t inv2 = splat2(static_cast<uint32_t>(a.invalid_cost));
    uint32_t vm[R], pad[R];
    bool inside = true;
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int xa = x - a.min_disp - k0 - r, xb = xa - R;
        vm[r] = (static_cast<unsigned>(xa) < static_cast<unsigned>(a.w) ? 0x0000FFFFu : 0u) |
                (static_cast<unsigned>(xb) < static_cast<unsigned>(a.w) ? 0xFFFF0000u : 0u);
        pad[r] = (k0 + r >= a.nd ? 0x0000FFFFu : 0u) | (k0 + r + R >= a.nd ? 0xFFFF0000u : 0u);
        inside &= (vm[r] | pad[r]) == kFull;
    }
    const bool border = !__all_sync(kFull, inside || !live);

    const int mid = a.h / 2;
    const int dy = down ? 1 : -1;
    const int y0 = down ? 0 : a.h - 1;
    const int n1 = down ? mid : a.h - mid, n2 = a.h - n1;
    const long cst = static_cast<long>(dy) * a.cpitch, gst = static_cast<long>(dy) * a.w;
    const long sst = static_cast<long>(dy) * a.w * a.dp;
    const long pix0 = (static_cast<long>(y0) * a.w + xs) * a.dp + k0;  // S / C offset at the first row

    uint32_t v[R], pm2 = 0, c[R], w[CW];
    int last = 0;
    // ---- first half: costs from the census words
    {
        const uint32_t* fl = a.census_l + static_cast<long>(y0) * a.cpitch + xs;
        const uint32_t* fq = a.census_r + static_cast<long>(y0) * a.cpitch + qb;
        const uint8_t* fg = a.guide + static_cast<long>(y0) * a.w + xs;
        int rI[PF];
        uint32_t rl[PF], rq[PF][NW];
        auto fetch = [&](int u) {
            rI[u] = __ldg(fg);
            rl[u] = __ldg(fl);
#pragma unroll
            for (int i = 0; i < NQ; ++i) {
                const uint4 t = __ldg(reinterpret_cast<const uint4*>(fq) + i);
                rq[u][4 * i] = t.x, rq[u][4 * i + 1] = t.y, rq[u][4 * i + 2] = t.z, rq[u][4 * i + 3] = t.w;
            }
            fl += cst;
            fq += cst;
            fg += gst;
        };
        uint8_t* ps = a.S + pix0;
        uint8_t* pc = a.C + pix0;
#pragma unroll
        for (int u = 0; u < PF; ++u)
            if (u < n1) fetch(u);
        for (int base = 0; base < n1; base += PF) {
#pragma unroll
            for (int u = 0; u < PF; ++u) {
                const int s = base + u;
                if (s >= n1) break;
                switch (al) {
                    case 0: sw_costs_aligned<R, 0, NW>(rl[u], rq[u], c); break;
                    case 1: sw_costs_aligned<R, 1, NW>(rl[u], rq[u], c); break;
                    case 2: sw_costs_aligned<R, 2, NW>(rl[u], rq[u], c); break;
                    default: sw_costs_aligned<R, 3, NW>(rl[u], rq[u], c); break;
                }
                if (border) {
#pragma unroll
                    for (int r = 0; r < R; ++r) c[r] = (c[r] & vm[r]) | (inv2 & ~vm[r]);
                }
                const uint32_t p2v = sw_p2(p2t, rI[u], last);
                if (s + PF < n1) fetch(u);
                if (live) {
                    sw_pack<R>(c, w);
                    st_chunk<NV, false>(pc, w);
                }
                if (s == 0) sw_first<R, SEG, PAD>(v, pm2, c, INF2, pad, seg);
                else sw_step<R, SEG, SLANT, PAD>(v, pm2, c, pm2 + p2v, INF2, P12, pad, sl, seg);
                if (live) {
                    sw_pack<R>(v, w);
                    st_chunk<NV, false>(ps, w);
                }
                ps += sst;
                pc += sst;
            }
        }
    }
    __syncthreads();  // the other direction's first-half values and costs are in S and C
    // ---- second half: costs from C, S += own values
    {
        const long off = static_cast<long>(n1) * dy;
        const uint8_t* fg = a.guide + (static_cast<long>(y0) + off) * a.w + xs;
        const uint8_t* fc = a.C + pix0 + off * a.w * a.dp;
        uint8_t* ps = a.S + pix0 + off * a.w * a.dp;
        int rI[PF];
        uint32_t rc[PF][CW], rs[PF][CW];
        auto fetch = [&](int u, int i) {  // ring slot u <- step (current + i)
            rI[u] = __ldg(fg + i * gst);
            ld_chunk<NV, LD_CG>(fc + i * sst, rc[u]);
            ld_chunk<NV, LD_CG>(ps + i * sst, rs[u]);
        };
#pragma unroll
        for (int u = 0; u < PF; ++u)
            if (u < n2) fetch(u, u);
        for (int base = 0; base < n2; base += PF) {
#pragma unroll
            for (int u = 0; u < PF; ++u) {
                const int s = base + u;
                if (s >= n2) break;
                uint32_t o[R];
#pragma unroll
                for (int i = 0; i < CW; ++i) {
                    c[2 * i] = prmt(rc[u][i], 0u, 0x4240);
                    c[2 * i + 1] = prmt(rc[u][i], 0u, 0x4341);
                    o[2 * i] = prmt(rs[u][i], 0u, 0x4240);
                    o[2 * i + 1] = prmt(rs[u][i], 0u, 0x4341);
                }
                const uint32_t p2v = sw_p2(p2t, rI[u], last);
                if (s + PF < n2) fetch(u, PF);
                if (n1 == 0 && s == 0) sw_first<R, SEG, PAD>(v, pm2, c, INF2, pad, seg);
                else sw_step<R, SEG, SLANT, PAD>(v, pm2, c, pm2 + p2v, INF2, P12, pad, sl, seg);
#pragma unroll
                for (int r = 0; r < R; ++r) o[r] += PAD ? (v[r] & ~pad[r]) : v[r];
                if (live) {
                    sw_pack<R>(o, w);
                    st_chunk<NV, false>(ps, w);
                }
                ps += sst;
                fc += sst;
                fg += gst;
            }
        }
    }
}

// ------------------------------------------------------------------------------------------------
// Row kernel. Block: kSweepRowWarps warps sweep left to right, as many right to left, over the same
// 32 / SEG * kSweepRowWarps rows (one row per segment).
//
// Right census words come through a sliding window: at column x lane sl holds win[j] = census_r(y,
// x - min - k0 - j). One step along the row shifts every lane's window by one word; the word entering a
// lane is the one leaving its neighbour (one shuffle), and only the lane at the end of the segment loads
// a new word (the same address for the whole segment).
//
// Right WTA: candidate (x, k) belongs to right pixel xr = x - min - k. Each lane keeps, per slot, the
// running minimum key of the right pixel that slot feeds; after every step the chains move by one slot
// (left to right: k + 1; right to left: k - 1), so every step one chain is complete (slot Dp-1, resp.
// slot 0) and is stored, and the rest are stored when the row ends. The left-to-right sweep covers right
// pixels [mid - min - Dp + 1, w - 1 - min], the other one [-min - Dp + 1, mid - 1 - min]; the epilogue takes
// the smaller key where both do.
//
// Best non-adjacent cost: the sums with the three slots around the best raised to >= 0xFFFD (per 16-bit
// lane: t = min(k - bk + 1, 3) through the wrap, then max(t + 0xFFFD, sum)), reduced like the best. The
// neighbours of the best (parabola) are read by the segment's first lane from the sums every lane stores
// to shared memory.
//
// The step loop is unrolled by 2 steps (register pressure and instruction-cache footprint);
// the strides along the row are compile-time, so loads use immediate offsets from pointers that move once
// per unrolled iteration.

constexpr int kSweepSmemWordsPerWarp = 2 * 32 * 8;  // two buffers (step parity) of 32 lanes x R <= 8 words

template <int R, int SEG, bool SLANT, bool PAD, bool FWD>
__device__ __forceinline__ void sweep_rows_dir(const SweepArgs& a, const uint32_t* __restrict__ p2t, uint32_t* __restrict__ wsm,
                                               int y, bool live, int seg, int sl) {
    constexpr int NV = 2 * R, CW = R / 2, Dp = SEG * NV, U = 2, PF = 2;
    constexpr int dx = FWD ? 1 : -1;
    const int yc = live ? y : a.h - 1;
    const int k0 = sl * NV;
    const int mid = a.w / 2;
    const int x0 = FWD ? 0 : a.w - 1;
    const int n1 = FWD ? mid : a.w - mid, n2 = a.w - n1;
    const uint32_t INF2 = splat2(0xFFFFu - static_cast<uint32_t>(a.p1)), P12 = splat2(static_cast<uint32_t>(a.p1));
    const uint32_t inv2 = splat2(static_cast<uint32_t>(a.invalid_cost));
    // Columns where every slot's right pixel lies inside the row (no cost or candidate masks).
    const int x_in_lo = a.min_disp + Dp - 1, x_in_hi = a.w - 1 + a.min_disp;
    uint32_t pad[R];
#pragma unroll
    for (int r = 0; r < R; ++r) pad[r] = (k0 + r >= a.nd ? 0x0000FFFFu : 0u) | (k0 + r + R >= a.nd ? 0xFFFF0000u : 0u);
    // disparities of register r: kbase2 + r * 0x10001 = (k0 + r, k0 + r + R)
    const uint32_t kbase2 = static_cast<uint32_t>(k0) | (static_cast<uint32_t>(k0 + R) << 16);
    const long row = static_cast<long>(yc) * a.cpitch;
    const uint32_t* cl = a.census_l + row;
    const uint32_t* cr = a.census_r + row;
    const long prow = static_cast<long>(yc) * a.w;
    // The word entering the window at column x: lane 0 takes census_r(x - min) (left to right), lane
    // SEG-1 census_r(x - min - Dp + 1) (right to left).
    const int fresh_off = FWD ? -a.min_disp : -a.min_disp - Dp + 1;

    // Stream pointers at the column of step `at`; a fetch of step at + i reads offset i * dx.
    const uint32_t *pl, *pf;
    const uint8_t *pg, *ps, *pt;
    auto seek = [&](int at) {
        const int x = x0 + at * dx;
        pl = cl + x;
        pf = cr + x + fresh_off;
        pg = a.guide + prow + x;
        ps = a.S + (prow + x) * Dp + k0;
        pt = a.T + (prow + x) * Dp + k0;
    };
    auto move = [&](int steps) {
        pl += steps * dx;
        pf += steps * dx;
        pg += steps * dx;
        ps += steps * dx * Dp;
        pt += steps * dx * Dp;
    };
    int rI[PF];
    uint32_t rl[PF], rf[PF], rs[PF][CW], rt[PF][CW];
    auto fetch = [&](int u, int i, bool phase2) {  // ring slot u <- step at + i
        rI[u] = __ldg(pg + i * dx);
        rl[u] = __ldg(pl + i * dx);
        rf[u] = __ldg(pf + i * dx);
        if (phase2) {
            ld_chunk<NV, LD_CS>(ps + i * dx * Dp, rs[u]);
            ld_chunk<NV, LD_CG>(pt + i * dx * Dp, rt[u]);
        }
    };
    uint32_t win[NV];
#pragma unroll
    for (int j = 0; j < NV; ++j) win[j] = __ldg(cr + x0 - a.min_disp - k0 - j);
    auto advance = [&](uint32_t fresh) {
        if constexpr (FWD) {
            const uint32_t t = __shfl_up_sync(kFull, win[NV - 1], 1, SEG);
#pragma unroll
            for (int j = NV - 1; j > 0; --j) win[j] = win[j - 1];
            win[0] = sl == 0 ? fresh : t;
        } else {
            const uint32_t t = __shfl_down_sync(kFull, win[0], 1, SEG);
#pragma unroll
            for (int j = 0; j < NV - 1; ++j) win[j] = win[j + 1];
            win[NV - 1] = sl == SEG - 1 ? fresh : t;
        }
    };
    // Costs of column x; at columns where some slot's right pixel is outside the row, vm marks the valid
    // slots (0xFFFF lanes) and the others take the invalid cost.
    auto costs = [&](uint32_t lw, int x, uint32_t (&c)[R], uint32_t (&vm)[R]) -> bool {
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const uint32_t ca = static_cast<uint32_t>(__popc(lw ^ win[r]));
            const uint32_t cb = static_cast<uint32_t>(__popc(lw ^ win[r + R]));
            c[r] = ca | (cb << 16);
        }
        const bool edge = x < x_in_lo || x > x_in_hi;  // one column per warp: uniform
        if (edge) {
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const int xa = x - a.min_disp - k0 - r, xb = xa - R;
                vm[r] = (static_cast<unsigned>(xa) < static_cast<unsigned>(a.w) ? 0x0000FFFFu : 0u) |
                        (static_cast<unsigned>(xb) < static_cast<unsigned>(a.w) ? 0xFFFF0000u : 0u);
                c[r] = (c[r] & vm[r]) | (inv2 & ~vm[r]);
            }
        }
        return edge;
    };

    uint32_t v[R], pm2 = 0, vm[R];
    int last = 0;
    int x = x0;
    // ---- phase 1: the first half of the row, path values to T
    seek(0);
#pragma unroll
    for (int u = 0; u < PF; ++u)
        if (u < n1) fetch(u, u, false);
    for (int base = 0; base < n1; base += U) {
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int s = base + u;
            if (s >= n1) break;
            if (s > 0) advance(rf[u % PF]);
            uint32_t c[R];
            costs(rl[u % PF], x, c, vm);
            const uint32_t p2v = sw_p2(p2t, rI[u % PF], last);
            if (s + PF < n1) fetch(u % PF, u + PF, false);
            if (s == 0) sw_first<R, SEG, PAD>(v, pm2, c, INF2, pad, seg);
            else sw_step<R, SEG, SLANT, PAD>(v, pm2, c, pm2 + p2v, INF2, P12, pad, sl, seg);
            if (live) {
                uint32_t w[CW];
                sw_pack<R>(v, w);
                st_chunk<NV, false>(a.T + (prow + x) * Dp + k0, w);
            }
            x += dx;
        }
        move(U);
    }
    sw_block_barrier();  // the other direction's first half is in T

    // ---- phase 2: the second half, with the 4-direction sums and the WTA
    uint16_t* rk = a.rk + (FWD ? 0 : static_cast<size_t>(a.w) * a.h) + prow;
    uint2* rec = a.rec + prow;
    uint32_t acc[R];  // running right-WTA keys of the right pixels x - min - (k0 + slot)
#pragma unroll
    for (int r = 0; r < R; ++r) acc[r] = 0xFFFFFFFFu;
    const int lane = threadIdx.x & 31;
    uint16_t* hb = reinterpret_cast<uint16_t*>(wsm);
    seek(n1);
#pragma unroll
    for (int u = 0; u < PF; ++u)
        if (u < n2) fetch(u, u, true);
    for (int base = 0; base < n2; base += U) {
#pragma unroll
        for (int u = 0; u < U; ++u) {
            const int s = base + u;
            if (s >= n2) break;
            if (n1 + s > 0) advance(rf[u % PF]);
            uint32_t c[R];
            const bool edge = costs(rl[u % PF], x, c, vm);
            const uint32_t p2v = sw_p2(p2t, rI[u % PF], last);
            if (n1 == 0 && s == 0) sw_first<R, SEG, PAD>(v, pm2, c, INF2, pad, seg);
            else sw_step<R, SEG, SLANT, PAD>(v, pm2, c, pm2 + p2v, INF2, P12, pad, sl, seg);
            // The reference's 4-direction sum S + T + L (S <= 254 and T <= 127 per byte, no overflow) and the
            // keys (sum << 7 | k); candidates outside the row or beyond nd get 0xFFFF.
            uint32_t tot[R], key[R];
#pragma unroll
            for (int i = 0; i < CW; ++i) {
                tot[2 * i] = prmt(rs[u % PF][i], 0u, 0x4240) + prmt(rt[u % PF][i], 0u, 0x4240);
                tot[2 * i + 1] = prmt(rs[u % PF][i], 0u, 0x4341) + prmt(rt[u % PF][i], 0u, 0x4341);
            }
            if (s + PF < n2) fetch(u % PF, u + PF, true);
#pragma unroll
            for (int r = 0; r < R; ++r) {
                tot[r] += PAD ? (v[r] & ~pad[r]) : v[r];
                key[r] = tot[r] * (1u << kSweepKeyBits) + (kbase2 + static_cast<uint32_t>(r) * 0x00010001u);
                if (PAD) {
                    key[r] |= pad[r];
                    tot[r] |= pad[r];
                }
            }
            if (edge) {
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    key[r] |= ~vm[r];
                    tot[r] |= ~vm[r];
                }
            }
            // Right WTA chains: add this column's candidates, store the completed chain, shift.
#pragma unroll
            for (int r = 0; r < R; ++r) acc[r] = vmin2(acc[r], key[r]);
            if constexpr (FWD) {
                const int xr = x - a.min_disp - (Dp - 1);
                if (live && sl == SEG - 1 && static_cast<unsigned>(xr) < static_cast<unsigned>(a.w))
                    rk[xr] = static_cast<uint16_t>(acc[R - 1] >> 16);
                uint32_t t = __shfl_up_sync(kFull, acc[R - 1], 1, SEG);
                t = sl == 0 ? 0xFFFFFFFFu : t;
                const uint32_t a0 = prmt(t, acc[R - 1], 0x5432);
#pragma unroll
                for (int r = R - 1; r > 0; --r) acc[r] = acc[r - 1];
                acc[0] = a0;
            } else {
                const int xr = x - a.min_disp;
                if (live && sl == 0 && static_cast<unsigned>(xr) < static_cast<unsigned>(a.w))
                    rk[xr] = static_cast<uint16_t>(acc[0]);
                uint32_t t = __shfl_down_sync(kFull, acc[0], 1, SEG);
                t = sl == SEG - 1 ? 0xFFFFFFFFu : t;
                const uint32_t ae = prmt(acc[0], t, 0x5432);
#pragma unroll
                for (int r = 0; r < R - 1; ++r) acc[r] = acc[r + 1];
                acc[R - 1] = ae;
            }
            // Left WTA: the segment's smallest key (key[] is reduced in place).
            const uint32_t kmin = sw_seg_min2<SEG>(sw_tree_min<R>(key), seg) & 0xFFFFu;
            const int bk = static_cast<int>(kmin & ((1u << kSweepKeyBits) - 1));
            // The sums to shared memory (lane l's R words at l * R) for the neighbours of the best.
            uint32_t* buf = wsm + (u & 1) * (32 * 8);
            {
                uint32_t* q = buf + lane * R;  // 16-byte aligned when R % 4 == 0, else 8-byte aligned
                if constexpr (R % 4 == 0) {
#pragma unroll
                    for (int i = 0; i < R / 4; ++i)
                        reinterpret_cast<uint4*>(q)[i] = make_uint4(tot[4 * i], tot[4 * i + 1], tot[4 * i + 2], tot[4 * i + 3]);
                } else {
#pragma unroll
                    for (int i = 0; i < R / 2; ++i) reinterpret_cast<uint2*>(q)[i] = make_uint2(tot[2 * i], tot[2 * i + 1]);
                }
            }
            // Best non-adjacent cost: slots within one of bk raised to >= 0xFFFD (tot[] reduced in place).
            const uint32_t kc = vadd2(kbase2, splat2((1u - static_cast<uint32_t>(bk)) & 0xFFFFu));
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const uint32_t t = __viaddmin_u16x2(kc, static_cast<uint32_t>(r) * 0x00010001u, 0x00030003u);
                tot[r] = __viaddmax_u16x2(t, 0xFFFDFFFDu, tot[r]);
            }
            const uint32_t second = sw_seg_min2<SEG>(sw_tree_min<R>(tot), seg) & 0xFFFFu;
            __syncwarp();
            if (live && sl == 0) {
                // u16 index of disparity k within the segment: lane k / NV, register (k % NV) % R, half (k % NV) / R.
                // k is clamped into [0, nd): without any candidate (every key 0xFFFF) bk is not a disparity, and
                // the record is not used.
                auto hidx = [&](int k) {
                    k = min(max(k, 0), a.nd - 1);
                    const int j = k % NV;
                    return (u & 1) * 512 + ((seg * SEG + k / NV) * R + j % R) * 2 + j / R;
                };
                const uint32_t cm = hb[hidx(bk - 1)];
                const uint32_t cp = hb[hidx(bk + 1)];
                rec[x] = make_uint2(kmin | (second << 16), cm | (cp << 16));
            }
            x += dx;
        }
        move(U);
    }
    // Flush: every chain is complete (no later column feeds it). The chains were shifted after the last
    // step, so slot k holds the right pixel of slot k - dx at the last column.
    if (live) {
        const int xl = FWD ? a.w - 1 : 0;  // the last column of the sweep
#pragma unroll
        for (int r = 0; r < R; ++r) {
#pragma unroll
            for (int hf = 0; hf < 2; ++hf) {
                const int k = k0 + r + hf * R;
                if (FWD ? k == 0 : k == Dp - 1) continue;  // shifted in: no chain
                const int xr = xl - a.min_disp - (k - dx);
                if (static_cast<unsigned>(xr) < static_cast<unsigned>(a.w))
                    rk[xr] = static_cast<uint16_t>(hf ? (acc[r] >> 16) : acc[r]);
            }
        }
    }
}

// The float part of the WTA and the L-R check for the block's rows (stereo.cpp:425-433, 450-461).
__device__ __forceinline__ void sweep_rows_epilogue(const SweepArgs& a, int y_first, int rows, int Dp) {
    const int mid = a.w / 2;
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
            const int bk = static_cast<int>(key & ((1u << kSweepKeyBits) - 1));
            const uint32_t sb = key >> kSweepKeyBits;
            const uint32_t second = sec >= kSweepNoKey ? 0xFFFFu : sec;
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
                const size_t q = static_cast<size_t>(y) * a.w + xr;
                uint32_t k = 0xFFFFu;
                if (xr >= mid - a.min_disp - Dp + 1) k = min(k, static_cast<uint32_t>(__ldcg(a.rk + q)));
                if (xr <= mid - 1 - a.min_disp) k = min(k, static_cast<uint32_t>(__ldcg(a.rk + plane + q)));
                if (k >= kSweepNoKey) {
                    d = kInvalid;
                } else {
                    const int rd = a.min_disp + static_cast<int>(k & ((1u << kSweepKeyBits) - 1));
                    if (fabsf(__fsub_rn(static_cast<float>(rd), d)) > static_cast<float>(a.lr_max_diff)) d = kInvalid;
                }
            }
        }
        a.disp[p] = d;
    }
}

template <int R, int SEG, bool SLANT, bool PAD, int PF>
__device__ __forceinline__ void sweep_rows_body(const SweepArgs& a, const uint32_t* __restrict__ p2t, uint32_t* __restrict__ smem,
                                                int bx) {
    constexpr int LPW = 32 / SEG;
    const int lane = threadIdx.x & 31, seg = lane / SEG, sl = lane % SEG;
    const int warp = threadIdx.x >> 5;
    const bool fwd = warp < kSweepRowWarps;
    const int wi = fwd ? warp : warp - kSweepRowWarps;
    const int rows = kSweepRowWarps * LPW;
    const int y = bx * rows + wi * LPW + seg;
    const bool live = y < a.h;
    uint32_t* wsm = smem + warp * kSweepSmemWordsPerWarp;
    if (fwd) sweep_rows_dir<R, SEG, SLANT, PAD, true>(a, p2t, wsm, y, live, seg, sl);
    else sweep_rows_dir<R, SEG, SLANT, PAD, false>(a, p2t, wsm, y, live, seg, sl);
    __syncthreads();  // records and right-WTA keys of the block's rows are stored
    sweep_rows_epilogue(a, bx * rows, rows, SEG * 2 * R);
}

constexpr int kSweepRowThreads = 64 * kSweepRowWarps;
constexpr int kSweepColThreads = 64 * kSweepColWarps;
constexpr size_t kSweepRowSmemBytes = sizeof(uint32_t) * kSweepSmemWordsPerWarp * 2 * kSweepRowWarps;

// Register budgets: two column blocks (16 warps) and four row blocks (16 warps) per SM.
constexpr int kSweepColMinBlocks = 2, kSweepRowMinBlocks = 4;

template <int R, int SEG, bool SLANT, bool PAD, int PF>
__global__ void __launch_bounds__(kSweepColThreads, kSweepColMinBlocks) k_sweep_cols(SweepArgs a) {
    __shared__ uint32_t p2t[32];
    if (threadIdx.x < 32) p2t[threadIdx.x] = a.p2_table2[threadIdx.x];
    __syncthreads();
    sweep_cols_body<R, SEG, SLANT, PAD, PF>(a, p2t, blockIdx.x);
}

template <int R, int SEG, bool SLANT, bool PAD, int PF>
__global__ void __launch_bounds__(kSweepRowThreads, kSweepRowMinBlocks) k_sweep_rows(SweepArgs a) {
    __shared__ uint32_t p2t[32];
    __shared__ __align__(16) uint32_t smem[kSweepSmemWordsPerWarp * 2 * kSweepRowWarps];
    if (threadIdx.x < 32) p2t[threadIdx.x] = a.p2_table2[threadIdx.x];
    __syncthreads();
    sweep_rows_body<R, SEG, SLANT, PAD, PF>(a, p2t, smem, blockIdx.x);
}

}  // namespace dsk
