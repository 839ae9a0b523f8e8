// Fused 4-path SGM (sm_100a): each pair of opposite directions runs as two warps that sweep towards
// each other over the same scanlines and meet in the middle, so that one direction's values are
// stored once and consumed by the other while they are still likely to be in L2.
//
//   k_vert      down (0,+1) and up (0,-1) sweeps of a column group. Phase 1: each direction writes its
//               path values for its first half of the column into S. Barrier. Phase 2: each
//               direction adds its values into S over the other half. S = L_down + L_up.
//   k_horz_wta  left-to-right and right-to-left sweeps of a row group. Phase 1: path values of the
//               first half of the row go to T. Barrier. Phase 2: at each pixel the total
//               S + T + L (the reference's 4-direction sum) is reduced in registers: WTA left inline,
//               WTA right by shared-memory atomicMin, then the L-R check over the rows (same
//               arithmetic as k_wta, stereo.cpp:411-461).
// The path recurrence is the one of k_paths (stereo.cpp:44-89); costs are recomputed from the census.
// Sums keep the reference's u16 wrap semantics; S is u8 when 2 (window + P2) <= 255 (values never exceed
// it), else u16.
#pragma once

#include "stereo_kernels.cuh"

namespace dsk {

struct FusedArgs {
    const void* census_l;
    const void* census_r;
    const uint8_t* guide;
    void* S;   // [y][x][dp] vertical pair sums (k_vert writes, k_horz_wta reads)
    void* T;   // [y][x][dp] horizontal first-half values (k_horz_wta scratch)
    int w, h, nd, dp, min_disp, p1, invalid_cost, slant;
    int p2_table[32];
    // WTA / L-R (k_horz_wta)
    float uniqueness;
    int subpixel, lr_max_diff;
    float* disp;
};

// One scanline's recurrence state for a lane: NV = 2R disparities as R registers of 16-bit lanes.
template <int R, int SEG>
struct PathState {
    uint32_t prev[R];
    uint32_t pad[R];
    bool any_pad;
    uint32_t pm;
    int last_i;

    __device__ __forceinline__ void init(int k0, int nd) {
        any_pad = false;
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const int k = k0 + 2 * r;
            pad[r] = (k >= nd ? 0x0000FFFFu : 0u) | (k + 1 >= nd ? 0xFFFF0000u : 0u);
            any_pad |= pad[r] != 0u;
        }
    }
    // First pixel of the line: L = C.
    __device__ __forceinline__ void first(const uint32_t (&c)[R], uint32_t INF2, int I, int seg, uint32_t (&out)[R]) {
        uint32_t lmin = 0xFFFFFFFFu;
#pragma unroll
        for (int r = 0; r < R; ++r) {
            prev[r] = any_pad ? ((c[r] & ~pad[r]) | (INF2 & pad[r])) : c[r];
            out[r] = prev[r];
            lmin = vmin2(lmin, prev[r]);
        }
        pm = seg_min<SEG>(hmin2(lmin), seg);
        last_i = I;
    }
    // Following pixels.
    __device__ __forceinline__ void step(const uint32_t (&c)[R], int I, const FusedArgs& a, uint32_t INF2, uint32_t P12,
                                         int sl, int seg, uint32_t (&out)[R]) {
        const int dI = I > last_i ? I - last_i : last_i - I;
        last_i = I;
        const uint32_t jump2 = splat2(pm + static_cast<uint32_t>(a.p2_table[dI >> 3]));
        const uint32_t negpm = splat2(0x10000u - pm);
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
            if (a.slant) m = vmin2(m, vmin2(lower, upper));
            const uint32_t best = vmin2(vmin2(vadd2(m, P12), prev[r]), jump2);
            uint32_t L = vadd2(vadd2(best, c[r]), negpm);
            if (any_pad) L = (L & ~pad[r]) | (INF2 & pad[r]);
            out[r] = L;
            lmin = vmin2(lmin, L);
        }
        pm = seg_min<SEG>(hmin2(lmin), seg);
#pragma unroll
        for (int r = 0; r < R; ++r) prev[r] = out[r];
    }
};

// Census inputs of one pixel for a lane: the left word and the NV right words it compares with.
template <typename CW, int NV>
struct CensusSlot {
    CW l;
    CW r[NV];
    int I;
};

template <typename CW, int NV>
__device__ __forceinline__ void fetch_census(const FusedArgs& a, int x, int y, int k0, CensusSlot<CW, NV>& s) {
    const int cx = min(max(x, 0), a.w - 1), cy = min(max(y, 0), a.h - 1);
    const size_t row = static_cast<size_t>(cy) * a.w;
    s.I = __ldg(a.guide + row + cx);
    s.l = __ldg(static_cast<const CW*>(a.census_l) + row + cx);
    const CW* cr = static_cast<const CW*>(a.census_r) + row;
#pragma unroll
    for (int j = 0; j < NV; ++j) {
        const int xr = cx - a.min_disp - (k0 + j);
        s.r[j] = (xr >= 0 && xr < a.w) ? __ldg(cr + xr) : CW(0);
    }
}

template <typename CW, int R>
__device__ __forceinline__ void census_costs(const FusedArgs& a, int x, int k0, const CensusSlot<CW, 2 * R>& s,
                                             uint32_t (&c)[R]) {
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int xa = x - a.min_disp - (k0 + 2 * r), xb = xa - 1;
        const uint32_t ca = (xa >= 0 && xa < a.w) ? popcount_word<CW>(s.l ^ s.r[2 * r]) : a.invalid_cost;
        const uint32_t cb = (xb >= 0 && xb < a.w) ? popcount_word<CW>(s.l ^ s.r[2 * r + 1]) : a.invalid_cost;
        c[r] = prmt(ca, cb, 0x5410);
    }
}

// ------------------------------------------------------------------------------------------------
// Vertical pair. Block = 2 * NWD warps: warps [0, NWD) sweep down, [NWD, 2 NWD) sweep up the same
// columns. Each warp covers 32 / SEG columns. blockIdx.x: column group.

template <int R, int SEG, typename CW, typename SV, int PF>
__global__ void __launch_bounds__(256) k_vert(FusedArgs a) {
    constexpr int NV = 2 * R;
    constexpr int LPW = 32 / SEG;
    constexpr int SB = NV * static_cast<int>(sizeof(SV));
    const int lane = threadIdx.x & 31, seg = lane / SEG, sl = lane % SEG;
    const int warp = threadIdx.x >> 5, nwd = blockDim.x >> 6;
    const bool down = warp < nwd;
    const int wi = down ? warp : warp - nwd;
    const int x = (blockIdx.x * nwd + wi) * LPW + seg;
    const bool live = x < a.w;
    const int xc = live ? x : a.w - 1;
    const int mid = a.h / 2;
    // down: rows 0..h-1 (phase 1 rows [0, mid)); up: rows h-1..0 (phase 1 rows [mid, h)).
    const int dy = down ? 1 : -1;
    const int y0 = down ? 0 : a.h - 1;
    const int n1 = down ? mid : a.h - mid;
    const int k0 = sl * NV;
    SV* __restrict__ S = static_cast<SV*>(a.S);
    const uint32_t INF2 = splat2(0xFFFFu - static_cast<uint32_t>(a.p1)), P12 = splat2(a.p1);

    PathState<R, SEG> st;
    st.init(k0, a.nd);
    CensusSlot<CW, NV> ring[PF];
#pragma unroll
    for (int u = 0; u < PF; ++u) fetch_census<CW, NV>(a, xc, y0 + u * dy, k0, ring[u]);

    auto put = [&](int y, const uint32_t (&v)[R]) {
        uint32_t wv[chunk_words<SB>()];
        pack<SV, NV>(v, wv);
        st_chunk<SB, false>(S + (static_cast<size_t>(y) * a.w + xc) * a.dp + k0, wv);
    };

    uint32_t c[R], L[R];
    int y = y0;
    // Phase 1: steps [0, n1).
    for (int base = 0; base < n1; base += PF) {
#pragma unroll
        for (int u = 0; u < PF; ++u) {
            const int s = base + u;
            if (s >= n1) break;
            census_costs<CW, R>(a, xc, k0, ring[u], c);
            const int I = ring[u].I;
            fetch_census<CW, NV>(a, xc, y + PF * dy, k0, ring[u]);
            if (s == 0) st.first(c, INF2, I, seg, L);
            else st.step(c, I, a, INF2, P12, sl, seg, L);
            if (live) put(y, L);
            y += dy;
        }
    }
    // The ring holds steps n1 .. n1+PF-1 in slots (n1 % PF) ...; rotate by re-fetching in order.
#pragma unroll
    for (int u = 0; u < PF; ++u) fetch_census<CW, NV>(a, xc, y + u * dy, k0, ring[u]);
    __syncthreads();  // the other direction's phase-1 values are in S
    // Phase 2: the remaining rows, S += L.
    const int n2 = a.h - n1;
    for (int base = 0; base < n2; base += PF) {
#pragma unroll
        for (int u = 0; u < PF; ++u) {
            const int s = base + u;
            if (s >= n2) break;
            census_costs<CW, R>(a, xc, k0, ring[u], c);
            const int I = ring[u].I;
            fetch_census<CW, NV>(a, xc, y + PF * dy, k0, ring[u]);
            uint32_t wv[chunk_words<SB>()], o[R];
            SV* p = S + (static_cast<size_t>(y) * a.w + xc) * a.dp + k0;
            ld_chunk<SB, LD_CG>(p, wv);
            unpack<SV, NV>(wv, o);
            if (n1 == 0 && s == 0) st.first(c, INF2, I, seg, L);
            else st.step(c, I, a, INF2, P12, sl, seg, L);
#pragma unroll
            for (int r = 0; r < R; ++r) o[r] = vadd2(o[r], L[r]);
            if (live) {
                pack<SV, NV>(o, wv);
                st_chunk<SB, false>(p, wv);
            }
            y += dy;
        }
    }
}

// ------------------------------------------------------------------------------------------------
// Horizontal pair + WTA + L-R. Block = 2 * NRW warps: warps [0, NRW) sweep left-to-right, the others
// right-to-left over the same rows; each warp covers 32 / SEG rows. Shared memory: right-WTA keys and
// left disparities of the block's rows (rows * w * 8 bytes).

template <int R, int SEG, typename CW, typename SV, int PF>
__global__ void __launch_bounds__(256) k_horz_wta(FusedArgs a) {
    constexpr int NV = 2 * R;
    constexpr int LPW = 32 / SEG;
    constexpr int SB = NV * static_cast<int>(sizeof(SV));
    constexpr int TB = NV;  // T holds single-direction values: u8 (window + P2 <= 255) or u16 -> use SV's width
    extern __shared__ uint32_t smem[];
    const int lane = threadIdx.x & 31, seg = lane / SEG, sl = lane % SEG;
    const int warp = threadIdx.x >> 5, nrw = blockDim.x >> 6;
    const int rows = nrw * LPW;
    uint32_t* rkey = smem;                                           // [rows][w]
    float* dleft = reinterpret_cast<float*>(smem + static_cast<size_t>(rows) * a.w);  // [rows][w]
    for (int i = threadIdx.x; i < rows * a.w; i += blockDim.x) rkey[i] = 0xFFFFFFFFu;
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
    const int n1 = fwd ? mid : a.w - mid;
    const int k0 = sl * NV;
    const SV* __restrict__ S = static_cast<const SV*>(a.S);
    SV* __restrict__ T = static_cast<SV*>(a.T);
    const uint32_t INF2 = splat2(0xFFFFu - static_cast<uint32_t>(a.p1)), P12 = splat2(a.p1);
    (void)TB;

    PathState<R, SEG> st;
    st.init(k0, a.nd);
    CensusSlot<CW, NV> ring[PF];
#pragma unroll
    for (int u = 0; u < PF; ++u) fetch_census<CW, NV>(a, x0 + u * dx, yc, k0, ring[u]);

    uint32_t c[R], L[R];
    int x = x0;
    for (int base = 0; base < n1; base += PF) {
#pragma unroll
        for (int u = 0; u < PF; ++u) {
            const int s = base + u;
            if (s >= n1) break;
            census_costs<CW, R>(a, x, k0, ring[u], c);
            const int I = ring[u].I;
            fetch_census<CW, NV>(a, x + PF * dx, yc, k0, ring[u]);
            if (s == 0) st.first(c, INF2, I, seg, L);
            else st.step(c, I, a, INF2, P12, sl, seg, L);
            if (live) {
                uint32_t wv[chunk_words<SB>()];
                pack<SV, NV>(L, wv);
                st_chunk<SB, false>(T + (static_cast<size_t>(yc) * a.w + x) * a.dp + k0, wv);
            }
            x += dx;
        }
    }
#pragma unroll
    for (int u = 0; u < PF; ++u) fetch_census<CW, NV>(a, x + u * dx, yc, k0, ring[u]);
    __syncthreads();  // the other direction's first half is in T

    uint32_t* rk = rkey + static_cast<size_t>(rl) * a.w;
    float* dl = dleft + static_cast<size_t>(rl) * a.w;
    const int n2 = a.w - n1;
    for (int base = 0; base < n2; base += PF) {
#pragma unroll
        for (int u = 0; u < PF; ++u) {
            const int s = base + u;
            if (s >= n2) break;
            census_costs<CW, R>(a, x, k0, ring[u], c);
            const int I = ring[u].I;
            fetch_census<CW, NV>(a, x + PF * dx, yc, k0, ring[u]);
            const size_t off = (static_cast<size_t>(yc) * a.w + x) * a.dp + k0;
            uint32_t ws[chunk_words<SB>()], wt[chunk_words<SB>()], tot[R], tv[R];
            ld_chunk<SB, LD_CS>(S + off, ws);
            ld_chunk<SB, LD_CG>(T + off, wt);
            if (n1 == 0 && s == 0) st.first(c, INF2, I, seg, L);
            else st.step(c, I, a, INF2, P12, sl, seg, L);
            unpack<SV, NV>(ws, tot);
            unpack<SV, NV>(wt, tv);
#pragma unroll
            for (int r = 0; r < R; ++r) tot[r] = vadd2(vadd2(tot[r], tv[r]), L[r]);
            // WTA for pixel x (same reductions as k_wta).
            const int lo = max(0, x - a.min_disp - (a.w - 1));
            const int hi = min(a.nd, x - a.min_disp + 1);
            uint32_t kmin = 0xFFFFFFFFu;
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const int ka = k0 + 2 * r;
                const uint32_t kk = static_cast<uint32_t>(ka) | (static_cast<uint32_t>(ka + 1) << 16);
                const uint32_t key_a = prmt(kk, tot[r], 0x5410);
                const uint32_t key_b = prmt(kk, tot[r], 0x7632);
                if (live && ka >= lo && ka < hi) {
                    kmin = min(kmin, key_a);
                    atomicMin(&rk[x - a.min_disp - ka], key_a);
                }
                if (live && ka + 1 >= lo && ka + 1 < hi) {
                    kmin = min(kmin, key_b);
                    atomicMin(&rk[x - a.min_disp - ka - 1], key_b);
                }
            }
            const uint32_t key = seg_min<SEG>(kmin, seg);
            const int bk = static_cast<int>(key & 0xFFFFu);
            uint32_t second = 0xFFFFu;
#pragma unroll
            for (int r = 0; r < R; ++r) {
                const int ka = k0 + 2 * r;
                if (ka >= lo && ka < hi && (ka - bk > 1 || bk - ka > 1)) second = min(second, tot[r] & 0xFFFFu);
                if (ka + 1 >= lo && ka + 1 < hi && (ka + 1 - bk > 1 || bk - ka - 1 > 1)) second = min(second, tot[r] >> 16);
            }
            second = seg_min<SEG>(second, seg);
            const int km = max(bk - 1, 0), kp = min(bk + 1, a.nd - 1);
            const uint32_t vm = __shfl_sync(kFull, pick16<R>(tot, km % NV), km / NV, SEG);
            const uint32_t vp = __shfl_sync(kFull, pick16<R>(tot, kp % NV), kp / NV, SEG);
            if (live && sl == 0) {
                float d = kInvalid;
                if (hi > lo) {
                    const uint32_t sb = key >> 16;
                    const bool unique =
                        !(second != 0xFFFFu && static_cast<float>(sb) >= __fmul_rn(a.uniqueness, static_cast<float>(second)));
                    if (unique) {
                        d = static_cast<float>(a.min_disp + bk);
                        if (a.subpixel && bk > lo && bk + 1 < hi)
                            d = __fadd_rn(d, parabola(static_cast<float>(vm), static_cast<float>(sb), static_cast<float>(vp)));
                    }
                }
                dl[x] = d;
            }
            x += dx;
        }
    }
    __syncthreads();

    // L-R check of the block's rows.
    for (int i = threadIdx.x; i < rows * a.w; i += blockDim.x) {
        const int r = i / a.w, xx = i % a.w;
        const int yy = blockIdx.x * rows + r;
        if (yy >= a.h) continue;
        float d = dleft[i];
        if (valid_disparity(d)) {
            const long xr = lroundf(__fsub_rn(static_cast<float>(xx), d));
            if (xr < 0 || xr >= a.w) {
                d = kInvalid;
            } else {
                const uint32_t k = rkey[static_cast<size_t>(r) * a.w + xr];
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
