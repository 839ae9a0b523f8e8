// Fused 4-path SGM (sm_100a): each pair of opposite directions runs as two warps that sweep towards
// each other over the same scanlines and meet in the middle, so that one direction's values are
// stored once and consumed by the other while they are still likely to be in L2.
//
//   k_vert      down (0,+1) and up (0,-1) sweeps of a column group. Phase 1: each direction writes its
//               path values for its first half of the column into S. Barrier. Phase 2: each
//               direction adds its values into S over the other half. S = L_down + L_up.
//   k_horz_wta  left-to-right and right-to-left sweeps of a row group. Phase 1: path values of the
//               first half of the row go to T. Barrier. Phase 2: at each pixel the total
//               S + T + L (the reference's 4-direction sum) is reduced in registers: WTA left and
//               right inline, then the L-R check over the rows (the arithmetic of stereo.cpp:411-461,
//               as k_wta).
// The path recurrence is the one of k_paths (stereo.cpp:44-89); costs are recomputed from the census.
// Sums keep the reference's u16 wrap semantics; S is u8 when 2 (window + P2) <= 255 (values never
// exceed it), else u16.
//
// Every input of a step is loaded PF steps ahead into a register ring through one pointer per stream
// (immediate offsets, one add per step). The streamed buffers carry guard rows (and the census guard
// columns) so that prefetches past a scanline's end stay inside the allocation: census (y, x) is
// readable for y in [-kGuardRows, h + kGuardRows) and x in [-guard, w + guard); guide, S and T rows
// likewise in y.
#pragma once

#include "stereo_kernels.cuh"

namespace dsk {

constexpr int kGuardRows = 8;  // >= the deepest prefetch ring

struct FusedArgs {
    const void* census_l;  // padded census, (y, x) at y * cpitch + x
    const void* census_r;
    int cpitch;
    const uint8_t* guide;  // left rectified image, (y, x) at y * w + x
    void* S;               // [y][x][dp] vertical pair sums (k_vert writes, k_horz_wta reads)
    void* T;               // [y][x][dp] horizontal first-half values (k_horz_wta scratch)
    int w, h, nd, dp, min_disp, p1, invalid_cost, slant;
    uint32_t p2_table2[32];  // P2' per |dI| / 8, both 16-bit lanes
    float uniqueness;
    int subpixel, lr_max_diff;
    float* disp;  // L-R checked disparities (k_horz_wta)
};

// Segment min of a value held in both 16-bit lanes; the result is again in both lanes.
template <int SEG>
__device__ __forceinline__ uint32_t seg_min2(uint32_t lmin2, int seg) {
    const uint32_t both = vmin2(lmin2, prmt(lmin2, lmin2, 0x1032));
    return seg_min<SEG>(both, seg);
}

// One scanline's recurrence for a lane: NV = 2R disparities as R registers of 16-bit lanes.
template <int R, int SEG>
struct Path {
    uint32_t prev[R];
    uint32_t pad[R];  // 16-bit lanes beyond nd (forced to INF)
    bool any_pad;
    uint32_t pm2;     // min(prev) in both lanes

    __device__ __forceinline__ void init(int k0, int nd) {
        any_pad = false;
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const int k = k0 + 2 * r;
            pad[r] = (k >= nd ? 0x0000FFFFu : 0u) | (k + 1 >= nd ? 0xFFFF0000u : 0u);
            any_pad |= pad[r] != 0u;
        }
    }
    __device__ __forceinline__ void first(const uint32_t (&c)[R], uint32_t INF2, int seg, uint32_t (&out)[R]) {
        uint32_t lmin = 0xFFFFFFFFu;
#pragma unroll
        for (int r = 0; r < R; ++r) {
            prev[r] = any_pad ? ((c[r] & ~pad[r]) | (INF2 & pad[r])) : c[r];
            out[r] = prev[r];
            lmin = vmin2(lmin, prev[r]);
        }
        pm2 = seg_min2<SEG>(lmin, seg);
    }
    // p2v2: P2' of this step in both lanes.
    __device__ __forceinline__ void step(const uint32_t (&c)[R], uint32_t p2v2, bool slant, uint32_t INF2, uint32_t P12,
                                         int sl, int seg, uint32_t (&out)[R]) {
        const uint32_t jump2 = vadd2(pm2, p2v2);
        const uint32_t negpm = vadd2(~pm2, 0x00010001u);  // (0x10000 - pm) per lane
        uint32_t up = __shfl_up_sync(kFull, prev[R - 1], 1, SEG);
        uint32_t dn = __shfl_down_sync(kFull, prev[0], 1, SEG);
        if (sl == 0) up = INF2;
        if (sl == SEG - 1) dn = INF2;
        uint32_t lmin = 0xFFFFFFFFu;
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const uint32_t lower = r == 0 ? up : prev[r - 1];      // (k-2, k-1)
            const uint32_t upper = r == R - 1 ? dn : prev[r + 1];  // (k+2, k+3)
            uint32_t m = vmin2(mid2(lower, prev[r]), mid2(prev[r], upper));
            if (slant) m = vmin2(m, vmin2(lower, upper));
            const uint32_t best = vmin2(vmin2(vadd2(m, P12), prev[r]), jump2);
            uint32_t L = vadd2(vadd2(best, c[r]), negpm);
            if (any_pad) L = (L & ~pad[r]) | (INF2 & pad[r]);
            out[r] = L;
            lmin = vmin2(lmin, L);
        }
        pm2 = seg_min2<SEG>(lmin, seg);
#pragma unroll
        for (int r = 0; r < R; ++r) prev[r] = out[r];
    }
};

// Costs of a lane's NV disparities from the census words; vm: 0xFFFF lanes where the right pixel is in
// the image (else the invalid cost).
template <typename CW, int R>
__device__ __forceinline__ void costs_from(CW lw, const CW (&rw)[2 * R], const uint32_t (&vm)[R], uint32_t inv2,
                                           uint32_t (&c)[R]) {
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const uint32_t ca = popcount_word<CW>(lw ^ rw[2 * r]);
        const uint32_t cb = popcount_word<CW>(lw ^ rw[2 * r + 1]);
        c[r] = (prmt(ca, cb, 0x5410) & vm[r]) | (inv2 & ~vm[r]);
    }
}

template <int N>
__device__ __forceinline__ uint32_t pick32(const uint32_t (&v)[N], int j) {
    uint32_t r = v[0];
#pragma unroll
    for (int i = 1; i < N; ++i)
        if (i == j) r = v[i];
    return r;
}

// Validity masks for the lane's disparities at column x.
template <int R>
__device__ __forceinline__ void valid_masks(int x, int k0, int min_disp, int w, uint32_t (&vm)[R]) {
    const int t = x - min_disp - k0;  // right pixel of disparity k0
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const bool va = static_cast<unsigned>(t - 2 * r) < static_cast<unsigned>(w);
        const bool vb = static_cast<unsigned>(t - 2 * r - 1) < static_cast<unsigned>(w);
        vm[r] = (va ? 0x0000FFFFu : 0u) | (vb ? 0xFFFF0000u : 0u);
    }
}

// ------------------------------------------------------------------------------------------------
// Vertical pair. Block = 2 * NWD warps: warps [0, NWD) sweep down, [NWD, 2 NWD) sweep up the same
// columns; each warp covers 32 / SEG columns. blockIdx.x: column group.

template <int R, int SEG, typename CW, typename SV, int PF>
__global__ void __launch_bounds__(256) k_vert(FusedArgs a) {
    constexpr int NV = 2 * R;
    constexpr int LPW = 32 / SEG;
    constexpr int SB = NV * static_cast<int>(sizeof(SV));
    constexpr int SW = chunk_words<SB>();
    const int lane = threadIdx.x & 31, seg = lane / SEG, sl = lane % SEG;
    const int warp = threadIdx.x >> 5, nwd = blockDim.x >> 6;
    const bool down = warp < nwd;
    const int wi = down ? warp : warp - nwd;
    const int x = (blockIdx.x * nwd + wi) * LPW + seg;
    const bool live = x < a.w;
    const int xc = live ? x : a.w - 1;
    const int mid = a.h / 2;
    const int dy = down ? 1 : -1;
    const int y0 = down ? 0 : a.h - 1;
    const int n1 = down ? mid : a.h - mid, n2 = a.h - n1;
    const int k0 = sl * NV;
    const uint32_t INF2 = splat2(0xFFFFu - static_cast<uint32_t>(a.p1)), P12 = splat2(a.p1);
    const uint32_t inv2 = splat2(a.invalid_cost);
    const bool slant = a.slant != 0;
    uint32_t vm[R];
    valid_masks<R>(xc, k0, a.min_disp, a.w, vm);

    const long cstep = static_cast<long>(dy) * a.cpitch, gstep = static_cast<long>(dy) * a.w;
    const long sstep = static_cast<long>(dy) * a.w * a.dp;
    const CW* cl = static_cast<const CW*>(a.census_l);
    const CW* cr = static_cast<const CW*>(a.census_r);
    SV* S = static_cast<SV*>(a.S);

    Path<R, SEG> st;
    st.init(k0, a.nd);
    uint32_t rs[PF][SW];
    int rI[PF];
    CW rl[PF], rr[PF][NV];
    const CW *fl, *fr;
    const uint8_t* fg;
    const SV* fs;
    auto seek = [&](int s) {  // fetch pointers at step s
        const long y = y0 + static_cast<long>(s) * dy;
        fl = cl + y * a.cpitch + xc;
        fr = cr + y * a.cpitch + xc - a.min_disp - k0;
        fg = a.guide + y * a.w + xc;
        fs = S + (y * a.w + xc) * a.dp + k0;
    };
    auto fetch = [&](int u, bool with_s) {
        rI[u] = __ldg(fg);
        rl[u] = __ldg(fl);
#pragma unroll
        for (int j = 0; j < NV; ++j) rr[u][j] = __ldg(fr - j);
        if (with_s) ld_chunk<SB, LD_CG>(fs, rs[u]);
        fl += cstep;
        fr += cstep;
        fg += gstep;
        fs += sstep;
    };

    seek(0);
#pragma unroll
    for (int u = 0; u < PF; ++u) fetch(u, false);
    SV* ps = S + (static_cast<long>(y0) * a.w + xc) * a.dp + k0;
    uint32_t c[R], L[R], wv[SW];
    int lastI = 0;
    auto p2_of = [&](int I) {
        const int d = I > lastI ? I - lastI : lastI - I;
        lastI = I;
        return a.p2_table2[d >> 3];
    };
    for (int base = 0; base < n1; base += PF) {
#pragma unroll
        for (int u = 0; u < PF; ++u) {
            const int s = base + u;
            if (s >= n1) break;
            costs_from<CW, R>(rl[u], rr[u], vm, inv2, c);
            const uint32_t p2v2 = p2_of(rI[u]);
            fetch(u, false);
            if (s == 0) st.first(c, INF2, seg, L);
            else st.step(c, p2v2, slant, INF2, P12, sl, seg, L);
            if (live) {
                pack<SV, NV>(L, wv);
                st_chunk<SB, false>(ps, wv);
            }
            ps += sstep;
        }
    }
    __syncthreads();  // the other direction's phase-1 values are in S
    seek(n1);
#pragma unroll
    for (int u = 0; u < PF; ++u) fetch(u, true);
    for (int base = 0; base < n2; base += PF) {
#pragma unroll
        for (int u = 0; u < PF; ++u) {
            const int s = base + u;
            if (s >= n2) break;
            costs_from<CW, R>(rl[u], rr[u], vm, inv2, c);
            const uint32_t p2v2 = p2_of(rI[u]);
            uint32_t o[R];
            unpack<SV, NV>(rs[u], o);
            fetch(u, true);
            if (n1 == 0 && s == 0) st.first(c, INF2, seg, L);
            else st.step(c, p2v2, slant, INF2, P12, sl, seg, L);
#pragma unroll
            for (int r = 0; r < R; ++r) o[r] = vadd2(o[r], L[r]);
            if (live) {
                pack<SV, NV>(o, wv);
                st_chunk<SB, false>(ps, wv);
            }
            ps += sstep;
        }
    }
}

// ------------------------------------------------------------------------------------------------
// Horizontal pair + WTA + L-R. Block = 2 * NRW warps: warps [0, NRW) sweep left-to-right, the others
// right-to-left over the same rows; each warp covers 32 / SEG rows.
//
// WTA right without atomics: the key (cost << 16 | k) of candidate (x, k) belongs to right pixel
// xr = x - min - k, so along a sweep the candidates of one xr arrive on consecutive steps at
// consecutive k. Each lane keeps, per disparity slot, the running minimum key of the right pixel that
// slot currently feeds; after every step the slots shift by one disparity (within the lane and by one
// shuffle across lanes), and the slot leaving the range holds a complete minimum, written once to
// shared memory. The two sweeps each see part of a diagonal; the L-R phase takes the minimum of both.
// WTA left: per pixel the segment reductions give (best cost, best k) and the best non-adjacent cost;
// lane 0 stores them with the two neighbouring costs, and the float part (uniqueness, parabola) runs
// in the L-R phase.
// Shared memory per row: 5 words per pixel (rows * w * 20 bytes).

constexpr int kHorzWordsPerPixel = 5;

template <int R, int SEG, typename CW, typename SV, int PF>
__global__ void __launch_bounds__(256) k_horz_wta(FusedArgs a) {
    constexpr int NV = 2 * R;
    constexpr int LPW = 32 / SEG;
    constexpr int SB = NV * static_cast<int>(sizeof(SV));
    constexpr int SW = chunk_words<SB>();
    extern __shared__ uint32_t smem[];
    const int lane = threadIdx.x & 31, seg = lane / SEG, sl = lane % SEG;
    const int warp = threadIdx.x >> 5, nrw = blockDim.x >> 6;
    const int rows = nrw * LPW;
    const size_t plane = static_cast<size_t>(rows) * a.w;
    uint32_t* rkf = smem;             // [rows][w] right-WTA keys, left-to-right sweep
    uint32_t* rkb = rkf + plane;      // right-to-left sweep
    uint32_t* pkey = rkb + plane;     // left WTA: (best cost << 16) | best k, or ~0 without candidates
    uint32_t* psec = pkey + plane;    // (best non-adjacent cost << 16) | cost(best - 1)
    uint32_t* pnxt = psec + plane;    // cost(best + 1)
    for (size_t i = threadIdx.x; i < 2 * plane; i += blockDim.x) rkf[i] = 0xFFFFFFFFu;
    __syncthreads();

    const bool fwd = warp < nrw;
    const int wi = fwd ? warp : warp - nrw;
    const int rl = wi * LPW + seg;  // row within the block
    const int y = blockIdx.x * rows + rl;
    const bool live = y < a.h;
    const int yc = live ? y : a.h - 1;
    const int mid = a.w / 2;
    const int dx = fwd ? 1 : -1;
    const int x0 = fwd ? 0 : a.w - 1;
    const int n1 = fwd ? mid : a.w - mid, n2 = a.w - n1;
    const int k0 = sl * NV;
    const uint32_t INF2 = splat2(0xFFFFu - static_cast<uint32_t>(a.p1)), P12 = splat2(a.p1);
    const uint32_t inv2 = splat2(a.invalid_cost);
    const bool slant = a.slant != 0;
    const long vstep = static_cast<long>(dx) * a.dp;
    // Columns where every disparity's right pixel is inside the row (uniform per warp).
    const int x_in_lo = a.min_disp + a.nd - 1, x_in_hi = a.w - 1 + a.min_disp;
    const CW* cl = static_cast<const CW*>(a.census_l) + static_cast<long>(yc) * a.cpitch;
    const CW* cr = static_cast<const CW*>(a.census_r) + static_cast<long>(yc) * a.cpitch;
    const uint8_t* grow = a.guide + static_cast<long>(yc) * a.w;
    const SV* S = static_cast<const SV*>(a.S) + static_cast<long>(yc) * a.w * a.dp + k0;
    SV* T = static_cast<SV*>(a.T) + static_cast<long>(yc) * a.w * a.dp + k0;

    Path<R, SEG> st;
    st.init(k0, a.nd);
    uint32_t rs[PF][SW], rt[PF][SW];
    int rI[PF];
    CW rlw[PF], rr[PF][NV];
    const CW *fl, *fr;
    const uint8_t* fg;
    const SV *fs, *ft;
    auto seek = [&](int s) {
        const int x = x0 + s * dx;
        fl = cl + x;
        fr = cr + x - a.min_disp - k0;
        fg = grow + x;
        fs = S + static_cast<long>(x) * a.dp;
        ft = T + static_cast<long>(x) * a.dp;
    };
    auto fetch = [&](int u, bool phase2) {
        rI[u] = __ldg(fg);
        rlw[u] = __ldg(fl);
#pragma unroll
        for (int j = 0; j < NV; ++j) rr[u][j] = __ldg(fr - j);
        if (phase2) {
            ld_chunk<SB, LD_CS>(fs, rs[u]);
            ld_chunk<SB, LD_CG>(ft, rt[u]);
        }
        fl += dx;
        fr += dx;
        fg += dx;
        fs += vstep;
        ft += vstep;
    };
    auto masks = [&](int x, uint32_t (&vm)[R]) {
        if (x >= x_in_lo && x <= x_in_hi) {
#pragma unroll
            for (int r = 0; r < R; ++r) vm[r] = 0xFFFFFFFFu;
        } else {
            valid_masks<R>(x, k0, a.min_disp, a.w, vm);
        }
    };
    int lastI = 0;
    auto p2_of = [&](int I) {
        const int d = I > lastI ? I - lastI : lastI - I;
        lastI = I;
        return a.p2_table2[d >> 3];
    };

    seek(0);
#pragma unroll
    for (int u = 0; u < PF; ++u) fetch(u, false);
    uint32_t c[R], L[R], vm[R], wv[SW];
    int x = x0;
    for (int base = 0; base < n1; base += PF) {
#pragma unroll
        for (int u = 0; u < PF; ++u) {
            const int s = base + u;
            if (s >= n1) break;
            masks(x, vm);
            costs_from<CW, R>(rlw[u], rr[u], vm, inv2, c);
            const uint32_t p2v2 = p2_of(rI[u]);
            fetch(u, false);
            if (s == 0) st.first(c, INF2, seg, L);
            else st.step(c, p2v2, slant, INF2, P12, sl, seg, L);
            if (live) {
                pack<SV, NV>(L, wv);
                st_chunk<SB, false>(T + static_cast<long>(x) * a.dp, wv);
            }
            x += dx;
        }
    }
    __syncthreads();  // the other direction's first half is in T

    const size_t rowoff = static_cast<size_t>(rl) * a.w;
    uint32_t* rk = (fwd ? rkf : rkb) + rowoff;
    uint32_t acc[NV];  // running right-WTA keys of the right pixels x - min - (k0 + j)
#pragma unroll
    for (int j = 0; j < NV; ++j) acc[j] = 0xFFFFFFFFu;
    const int k_out = fwd ? a.nd - 1 : 0;  // the slot whose right pixel is complete after each step
    const bool owns_out = k_out >= k0 && k_out < k0 + NV;
    seek(n1);
#pragma unroll
    for (int u = 0; u < PF; ++u) fetch(u, true);
    for (int base = 0; base < n2; base += PF) {
#pragma unroll
        for (int u = 0; u < PF; ++u) {
            const int s = base + u;
            if (s >= n2) break;
            masks(x, vm);
            costs_from<CW, R>(rlw[u], rr[u], vm, inv2, c);
            const uint32_t p2v2 = p2_of(rI[u]);
            uint32_t tot[R], tv[R];
            unpack<SV, NV>(rs[u], tot);
            unpack<SV, NV>(rt[u], tv);
            fetch(u, true);
            if (n1 == 0 && s == 0) st.first(c, INF2, seg, L);
            else st.step(c, p2v2, slant, INF2, P12, sl, seg, L);
#pragma unroll
            for (int r = 0; r < R; ++r) tot[r] = vadd2(vadd2(tot[r], tv[r]), L[r]);

            const bool interior = x >= x_in_lo && x <= x_in_hi;  // every k in [0, nd) is a candidate
            const int lo = max(0, x - a.min_disp - (a.w - 1));
            const int hi = min(a.nd, x - a.min_disp + 1);
            uint32_t kmin = 0xFFFFFFFFu;
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const int ka = k0 + 2 * r;
                const uint32_t kk = static_cast<uint32_t>(ka) | (static_cast<uint32_t>(ka + 1) << 16);
                uint32_t key_a = prmt(kk, tot[r], 0x5410);  // (cost_a << 16) | ka
                uint32_t key_b = prmt(kk, tot[r], 0x7632);  // (cost_b << 16) | ka + 1
                if (!(interior ? ka < a.nd : (ka >= lo && ka < hi))) key_a = 0xFFFFFFFFu;
                if (!(interior ? ka + 1 < a.nd : (ka + 1 >= lo && ka + 1 < hi))) key_b = 0xFFFFFFFFu;
                kmin = min(kmin, min(key_a, key_b));
                acc[2 * r] = min(acc[2 * r], key_a);
                acc[2 * r + 1] = min(acc[2 * r + 1], key_b);
            }
            const bool last = s == n2 - 1;
            if (live) {
                if (last) {  // every slot is complete: no later step feeds these right pixels
#pragma unroll
                    for (int j = 0; j < NV; ++j) {
                        const int xr = x - a.min_disp - (k0 + j);
                        if (k0 + j < a.nd && xr >= 0 && xr < a.w) rk[xr] = acc[j];
                    }
                } else if (owns_out) {
                    const int xr = x - a.min_disp - k_out;
                    if (xr >= 0 && xr < a.w) rk[xr] = pick32<NV>(acc, k_out - k0);
                }
            }
            if (fwd) {  // next step: slot k feeds the right pixel slot k - 1 fed now
                uint32_t t = __shfl_up_sync(kFull, acc[NV - 1], 1, SEG);
                if (sl == 0) t = 0xFFFFFFFFu;
#pragma unroll
                for (int j = NV - 1; j > 0; --j) acc[j] = acc[j - 1];
                acc[0] = t;
            } else {
                uint32_t t = __shfl_down_sync(kFull, acc[0], 1, SEG);
                if (sl == SEG - 1) t = 0xFFFFFFFFu;
#pragma unroll
                for (int j = 0; j < NV - 1; ++j) acc[j] = acc[j + 1];
                acc[NV - 1] = t;
            }

            const uint32_t key = seg_min<SEG>(kmin, seg);
            const int bk = static_cast<int>(key & 0xFFFFu);
            uint32_t second = 0xFFFFu;
            if (interior && (k0 > bk + 1 || k0 + NV - 1 < bk - 1) && k0 + NV <= a.nd) {
                uint32_t m2 = tot[0];
#pragma unroll
                for (int r = 1; r < R; ++r) m2 = vmin2(m2, tot[r]);
                second = hmin2(m2);
            } else {
#pragma unroll
                for (int r = 0; r < R; ++r) {
                    const int ka = k0 + 2 * r;
                    if (ka >= lo && ka < hi && (ka - bk > 1 || bk - ka > 1)) second = min(second, tot[r] & 0xFFFFu);
                    if (ka + 1 >= lo && ka + 1 < hi && (ka + 1 - bk > 1 || bk - ka - 1 > 1)) second = min(second, tot[r] >> 16);
                }
            }
            second = seg_min<SEG>(second, seg);
            const int km = max(bk - 1, 0), kp = min(bk + 1, a.nd - 1);
            const uint32_t vmv = __shfl_sync(kFull, pick16<R>(tot, km % NV), km / NV, SEG);
            const uint32_t vpv = __shfl_sync(kFull, pick16<R>(tot, kp % NV), kp / NV, SEG);
            if (live && sl == 0) {
                pkey[rowoff + x] = hi > lo ? key : 0xFFFFFFFFu;
                psec[rowoff + x] = (second << 16) | (vmv & 0xFFFFu);
                pnxt[rowoff + x] = vpv;
            }
            x += dx;
        }
    }
    __syncthreads();

    // Finish the WTA (uniqueness, parabola) and the L-R check of the block's rows.
    for (size_t i = threadIdx.x; i < plane; i += blockDim.x) {
        const int r = static_cast<int>(i / a.w), xx = static_cast<int>(i % a.w);
        const int yy = blockIdx.x * rows + r;
        if (yy >= a.h) continue;
        float d = kInvalid;
        const uint32_t key = pkey[i];
        if (key != 0xFFFFFFFFu) {
            const int lo = max(0, xx - a.min_disp - (a.w - 1));
            const int hi = min(a.nd, xx - a.min_disp + 1);
            const int bk = static_cast<int>(key & 0xFFFFu);
            const uint32_t sb = key >> 16, second = psec[i] >> 16;
            const bool unique =
                !(second != 0xFFFFu && static_cast<float>(sb) >= __fmul_rn(a.uniqueness, static_cast<float>(second)));
            if (unique) {
                d = static_cast<float>(a.min_disp + bk);
                if (a.subpixel && bk > lo && bk + 1 < hi)
                    d = __fadd_rn(d, parabola(static_cast<float>(psec[i] & 0xFFFFu), static_cast<float>(sb),
                                              static_cast<float>(pnxt[i])));
            }
        }
        if (valid_disparity(d)) {
            const long xr = lroundf(__fsub_rn(static_cast<float>(xx), d));
            if (xr < 0 || xr >= a.w) {
                d = kInvalid;
            } else {
                const size_t ri = static_cast<size_t>(r) * a.w + xr;
                const uint32_t k = min(rkf[ri], rkb[ri]);
                if (k >= 0xFFFF0000u) {
                    d = kInvalid;
                } else {
                    const int rd = a.min_disp + static_cast<int>(k & 0xFFFFu);
                    if (fabsf(__fsub_rn(static_cast<float>(rd), d)) > static_cast<float>(a.lr_max_diff)) d = kInvalid;
                }
            }
        }
        a.disp[static_cast<size_t>(yy) * a.w + xx] = d;
    }
}

}  // namespace dsk
