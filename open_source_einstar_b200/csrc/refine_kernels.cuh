// The stages of depth::compute_disparity after SGM (libs/depth/src/stereo.cpp:151-326, 465-536): image
// pyramid, slanted-window ZNCC refinement per level, detail refinement on the full-resolution images,
// occlusion and spike filters, speckle removal. All float and double arithmetic follows the reference's
// evaluation order with explicitly rounded intrinsics (no fused multiply-adds), so results are the
// reference's bit for bit.
#pragma once

#include <cstdint>

#include "stereo_kernels.cuh"
#include "union_find.cuh"

namespace dsk {

constexpr float kZnccNoWindow = -2.0f;  // the window leaves the right image
constexpr int kMaxRefineCandidates = 127;
constexpr int kMaxDetailCandidates = 33;

// depth::downsample2 (stereo.cpp:348-359): 2x2 box, (sum + 2) / 4; out is (w/2) x (h/2).
static __global__ void k_downsample2(const uint8_t* __restrict__ in, int w, int h, uint8_t* __restrict__ out) {
    const int ow = w / 2, oh = h / 2;
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= ow || y >= oh) return;
    const uint8_t* r0 = in + static_cast<size_t>(2 * y) * w + 2 * x;
    const uint8_t* r1 = r0 + w;
    out[static_cast<size_t>(y) * ow + x] = static_cast<uint8_t>((r0[0] + r0[1] + r1[0] + r1[1] + 2) / 4);
}

// (anonymous) median3 (stereo.cpp:129-147): valid neighbours of a valid pixel, element n/2 in order.
static __global__ void k_median3(const float* __restrict__ in, int w, int h, float* __restrict__ out) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= w || y >= h) return;
    const size_t i = static_cast<size_t>(y) * w + x;
    float d = in[i];
    if (valid_disparity(d)) {
        float v[9];
#pragma unroll
        for (int dy = -1; dy <= 1; ++dy)
#pragma unroll
            for (int dx = -1; dx <= 1; ++dx) {
                const int xx = x + dx, yy = y + dy;
                const bool inside = xx >= 0 && yy >= 0 && xx < w && yy < h;
                v[(dy + 1) * 3 + dx + 1] = inside ? in[static_cast<size_t>(yy) * w + xx] : kInvalid;
            }
        int n;
        d = median_of_valid9(v, n);
    } else {
        d = kInvalid;
    }
    out[i] = d;
}

// The window sums of a ZNCC score. The reference accumulates all five in double, sample by sample. Sums over
// the left window (sa, saa) are sums of integers below 2^53, exact in any order, so they are summed once per
// pixel in integers; the three sums that involve the bilinear right samples (sb, sbb, sab) keep the
// reference's order and rounding.
struct ZnccSums {
    double sb = 0, sbb = 0, sab = 0;
    __device__ __forceinline__ void add(double ia, double ib) {
        sb = __dadd_rn(sb, ib);
        sbb = __dadd_rn(sbb, __dmul_rn(ib, ib));
        sab = __dadd_rn(sab, __dmul_rn(ia, ib));
    }
    __device__ __forceinline__ float score(double sa, double saa, double n) const {
        const double va = __dsub_rn(saa, __ddiv_rn(__dmul_rn(sa, sa), n));
        const double vb = __dsub_rn(sbb, __ddiv_rn(__dmul_rn(sb, sb), n));
        if (va < 1e-6 || vb < 1e-6) return -1.0f;
        return __double2float_rn(__ddiv_rn(__dsub_rn(sab, __ddiv_rn(__dmul_rn(sa, sb), n)), __dsqrt_rn(__dmul_rn(va, vb))));
    }
};

// Sum and sum of squares of an n x m byte window (rows `stride` apart), as exact doubles.
__device__ __forceinline__ void window_moments(const uint8_t* a, size_t stride, int n, int m, double& sa, double& saa) {
    int s1 = 0, s2 = 0;
    for (int j = 0; j < m; ++j) {
        const uint8_t* row = a + static_cast<size_t>(j) * stride;
        for (int i = 0; i < n; ++i) {
            const int v = row[i];
            s1 += v;
            s2 += v * v;
        }
    }
    sa = static_cast<double>(s1);
    saa = static_cast<double>(s2);
}

// Integer-to-float conversions and floor() run on the SM's conversion unit, a quarter of the FMA rate, and
// would bound the ZNCC loops (several per sample). The samples below convert on the FMA and ALU pipes
// instead, with the same values:
// - a byte v as a float: the float with bits 0x4B000000 | v is 2^23 + v, exactly; subtract 2^23;
// - a byte as a double: likewise with 2^52;
// - floor(xb) for |xb| < 2^22: xb + 1.5 * 2^23 lies in [2^23, 2^24), where the float spacing is 1, so the
//   sum is xb rounded to an integer (then one less where that rounded up), and its low mantissa bits
//   hold that integer. A larger |xb| puts the sample outside any image row (at most 16384 wide), which
//   the reference also rejects.
__device__ __forceinline__ float byte_to_float(uint32_t v) { return __fsub_rn(__uint_as_float(0x4B000000u | v), 8388608.0f); }
__device__ __forceinline__ double byte_to_double(uint32_t v) {
    return __dsub_rn(__hiloint2double(0x43300000, static_cast<int>(v)), 4503599627370496.0);
}

// One bilinear sample of the right row at xb, float(rb[x0] (1 - f) + rb[x0 + 1] f) with x0 = floor(xb) and
// f = xb - x0, as a double; false when x0 or x0 + 1 leave the row (stereo.cpp:110-114).
__device__ __forceinline__ bool sample_row(const uint8_t* rb, int bw, float xb, double& ib) {
    if (!(fabsf(xb) < 4194304.0f)) return false;
    const float t = __fadd_rn(xb, 12582912.0f);
    float fl = __fsub_rn(t, 12582912.0f);
    int x0 = __float_as_int(t) - 0x4B400000;
    if (fl > xb) {
        fl = __fsub_rn(fl, 1.0f);
        --x0;
    }
    if (x0 < 0 || x0 + 1 >= bw) return false;
    const float f = __fsub_rn(xb, fl);
    ib = static_cast<double>(__fadd_rn(__fmul_rn(byte_to_float(rb[x0]), __fsub_rn(1.0f, f)),
                                       __fmul_rn(byte_to_float(rb[x0 + 1]), f)));
    return true;
}

// zncc_slanted (stereo.cpp:102-126). Loop counters are carried as floats too (small integers, exact).
__device__ float zncc_slanted(const uint8_t* a, const uint8_t* b, int w, int x, int y, float d, float gx, float gy, int r,
                              double sa, double saa) {
    ZnccSums s;
    const int n = (2 * r + 1) * (2 * r + 1);
    const float fr = static_cast<float>(r), fx = static_cast<float>(x);
    float fv = -fr;
    for (int v = -r; v <= r; ++v, fv = __fadd_rn(fv, 1.0f)) {
        const uint8_t* ra = a + static_cast<size_t>(y + v) * w + x;
        const uint8_t* rb = b + static_cast<size_t>(y + v) * w;
        const float gyv = __fmul_rn(gy, fv);
        float fu = -fr;
        for (int u = -r; u <= r; ++u, fu = __fadd_rn(fu, 1.0f)) {
            const float shift = __fadd_rn(__fadd_rn(d, __fmul_rn(gx, fu)), gyv);
            const float xb = __fsub_rn(__fadd_rn(fx, fu), shift);
            double ib;
            if (!sample_row(rb, w, xb, ib)) return kZnccNoWindow;
            s.add(byte_to_double(ra[u]), ib);
        }
    }
    return s.score(sa, saa, static_cast<double>(n));
}

// ---- two candidates at once on the f32x2 pipe --------------------------------------------------------------
// Blackwell executes a pair of float adds as one instruction (__fadd2_rn), each component rounded as the
// scalar add. The ZNCC loops below evaluate two candidate disparities per sample that way and share the left
// sample and its conversion. Products stay scalar (__fmul_rn): a pair multiply followed by a pair add was
// measured to come out fused (one rounding, the last bit off the reference's) in some kernels despite
// explicit rounding, while scalar products into pair adds matched the scalar path on every sample tried.
// The pair loops take no range checks: callers use them only where a bound on the whole window
// (window_inside) puts every sample inside the right row. floor() is one round-down add: xb + 1.5 * 2^23
// rounded down is floor(xb) + 1.5 * 2^23 for |xb| < 2^22.
__device__ __forceinline__ float2 f2(float a, float b) { return make_float2(a, b); }
__device__ __forceinline__ float2 neg2(float2 a) { return make_float2(-a.x, -a.y); }
__device__ __forceinline__ float2 add2_rn(float2 a, float2 b) { return __fadd2_rn(a, b); }
__device__ __forceinline__ float2 add2_rm(float2 a, float2 b) { return __fadd2_rd(a, b); }
__device__ __forceinline__ float2 mul2_scalar(float2 a, float2 b) { return f2(__fmul_rn(a.x, b.x), __fmul_rn(a.y, b.y)); }

__device__ __forceinline__ float2 bilinear_pair(const uint8_t* rb, float2 xb) {
    const float2 t = add2_rm(xb, f2(12582912.0f, 12582912.0f));
    const float2 fl = add2_rn(t, f2(-12582912.0f, -12582912.0f));
    const float2 f = add2_rn(xb, neg2(fl));
    const int xa = __float_as_int(t.x) - 0x4B400000, xc = __float_as_int(t.y) - 0x4B400000;
    const float2 b0 = add2_rn(f2(__uint_as_float(0x4B000000u | rb[xa]), __uint_as_float(0x4B000000u | rb[xc])),
                                 f2(-8388608.0f, -8388608.0f));
    const float2 b1 = add2_rn(f2(__uint_as_float(0x4B000000u | rb[xa + 1]), __uint_as_float(0x4B000000u | rb[xc + 1])),
                                 f2(-8388608.0f, -8388608.0f));
    return add2_rn(mul2_scalar(b0, add2_rn(f2(1.0f, 1.0f), neg2(f))), mul2_scalar(b1, f));
}

// zncc_slanted for the disparities d.x and d.y.
__device__ float2 zncc_slanted_pair(const uint8_t* a, const uint8_t* b, int w, int x, int y, float2 d, float gx, float gy, int r,
                                    double sa, double saa) {
    ZnccSums s0, s1;
    const float fr = static_cast<float>(r), fx = static_cast<float>(x);
    float fv = -fr;
    for (int v = -r; v <= r; ++v, fv = __fadd_rn(fv, 1.0f)) {
        const uint8_t* ra = a + static_cast<size_t>(y + v) * w + x;
        const uint8_t* rb = b + static_cast<size_t>(y + v) * w;
        const float gyv = __fmul_rn(gy, fv);
        float fu = -fr;
        for (int u = -r; u <= r; ++u, fu = __fadd_rn(fu, 1.0f)) {
            const float gxu = __fmul_rn(gx, fu), xu = __fadd_rn(fx, fu);
            const float2 shift = add2_rn(add2_rn(d, f2(gxu, gxu)), f2(gyv, gyv));
            const float2 ib = bilinear_pair(rb, add2_rn(f2(xu, xu), neg2(shift)));
            const double ia = byte_to_double(ra[u]);
            s0.add(ia, static_cast<double>(ib.x));
            s1.add(ia, static_cast<double>(ib.y));
        }
    }
    const double n = static_cast<double>((2 * r + 1) * (2 * r + 1));
    return f2(s0.score(sa, saa, n), s1.score(sa, saa, n));
}

// True when every sample x0 = floor(xb) of a window has 0 <= x0 and x0 + 1 < width, for xb between lo and
// hi in exact arithmetic: the float evaluation of xb is within a few ulp (< 0.01 px here) of it, and the
// bound keeps half a pixel to spare.
__device__ __forceinline__ bool window_inside(float lo, float hi, int width) {
    return lo >= 0.5f && hi <= static_cast<float>(width) - 1.5f;
}

// The best score of a candidate sequence and its two neighbours, as the reference reads them from its
// score array (stereo.cpp:181-199, 263-278): strict improvements only; the first best wins ties.
struct PeakTracker {
    float best = -2.0f, prev = -2.0f, before = -2.0f, after = -2.0f;
    int best_k = -1;
    __device__ __forceinline__ void push(int k, float sc) {
        if (k == best_k + 1) after = sc;  // the score right after the current best
        if (sc > best) {
            best = sc;
            best_k = k;
            before = prev;
            after = -3.0f;  // not yet known
        }
        prev = sc;
    }
};

struct RefineArgs {
    const uint8_t* left;   // this level, w x h
    const uint8_t* right;
    const float* coarse;   // median3 of the coarser level's disparity, cw x ch
    int w, h, cw, ch;
    int search_radius, zncc_radius;
    float min_zncc;
    int reject_edge_winners, subpixel;
    float* disp;  // w x h
    float* conf;
};

// refine_level (stereo.cpp:151-207): per pixel, ZNCC of slanted windows at 2x the coarse disparity +/-
// search_radius in half-pixel steps; the best above min_zncc, with a parabola between its neighbours.
static __global__ void __launch_bounds__(128, 6) k_refine_level(RefineArgs a) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= a.w || y >= a.h) return;
    const size_t i = static_cast<size_t>(y) * a.w + x;
    float out_d = kInvalid, out_c = 0.0f;
    const int r = a.zncc_radius;
    if (y >= r && y < a.h - r && x >= r && x < a.w - r) {
        const int cy = min(y / 2, a.ch - 1), cx = min(x / 2, a.cw - 1);
        const float d0 = a.coarse[static_cast<size_t>(cy) * a.cw + cx];
        if (valid_disparity(d0)) {
            // slope (stereo.cpp:161-173)
            auto C = [&](int xx, int yy) { return a.coarse[static_cast<size_t>(yy) * a.cw + xx]; };
            float gx = 0.0f, gy = 0.0f;
            if (cx > 0 && cx + 1 < a.cw && valid_disparity(C(cx - 1, cy)) && valid_disparity(C(cx + 1, cy))) {
                const float g = __fmul_rn(0.5f, __fsub_rn(C(cx + 1, cy), C(cx - 1, cy)));
                if (fabsf(__fsub_rn(C(cx + 1, cy), d0)) < 2.0f && fabsf(__fsub_rn(d0, C(cx - 1, cy))) < 2.0f) gx = g;
            }
            if (cy > 0 && cy + 1 < a.ch && valid_disparity(C(cx, cy - 1)) && valid_disparity(C(cx, cy + 1))) {
                const float g = __fmul_rn(0.5f, __fsub_rn(C(cx, cy + 1), C(cx, cy - 1)));
                if (fabsf(__fsub_rn(C(cx, cy + 1), d0)) < 2.0f && fabsf(__fsub_rn(d0, C(cx, cy - 1))) < 2.0f) gy = g;
            }
            gx = fminf(fmaxf(gx, -0.9f), 0.9f);
            gy = fminf(fmaxf(gy, -0.9f), 0.9f);
            constexpr float kStep = 0.5f;
            const float center = __fmul_rn(2.0f, d0);
            const int nd = min(kMaxRefineCandidates, static_cast<int>(__fdiv_rn(static_cast<float>(2 * a.search_radius), kStep)) + 1);
            const float lo = __fsub_rn(center, static_cast<float>(a.search_radius));
            double sa, saa;
            window_moments(a.left + static_cast<size_t>(y - r) * a.w + (x - r), a.w, 2 * r + 1, 2 * r + 1, sa, saa);
            PeakTracker pk;
            // Exact xb over the window and all candidates: x - d + u (1 - gx) - gy v, |u|, |v| <= r.
            const float reach = __fadd_rn(__fmul_rn(static_cast<float>(r), __fsub_rn(1.0f, gx)),
                                          __fmul_rn(static_cast<float>(r), fabsf(gy)));
            const float fx = static_cast<float>(x), hi_d = __fadd_rn(lo, __fmul_rn(kStep, static_cast<float>(nd - 1)));
            if (window_inside(__fsub_rn(__fsub_rn(fx, hi_d), reach), __fadd_rn(__fsub_rn(fx, lo), reach), a.w)) {
                int k = 0;
                for (; k + 1 < nd; k += 2) {
                    const float2 d = f2(__fadd_rn(lo, __fmul_rn(kStep, static_cast<float>(k))),
                                        __fadd_rn(lo, __fmul_rn(kStep, static_cast<float>(k + 1))));
                    const float2 sc = zncc_slanted_pair(a.left, a.right, a.w, x, y, d, gx, gy, r, sa, saa);
                    pk.push(k, sc.x);
                    pk.push(k + 1, sc.y);
                }
                if (k < nd)
                    pk.push(k, zncc_slanted(a.left, a.right, a.w, x, y, __fadd_rn(lo, __fmul_rn(kStep, static_cast<float>(k))), gx,
                                            gy, r, sa, saa));
            } else {
                for (int k = 0; k < nd; ++k) {
                    const float d = __fadd_rn(lo, __fmul_rn(kStep, static_cast<float>(k)));
                    pk.push(k, zncc_slanted(a.left, a.right, a.w, x, y, d, gx, gy, r, sa, saa));
                }
            }
            const float best = pk.best, before_best = pk.before, after_best = pk.after;
            const int best_k = pk.best_k;
            bool keep = !(best_k < 0 || best < a.min_zncc);
            if (keep && a.reject_edge_winners && (best_k == 0 || best_k == nd - 1)) keep = false;
            if (keep) {
                float d = __fadd_rn(lo, __fmul_rn(kStep, static_cast<float>(best_k)));
                if (a.subpixel && best_k > 0 && best_k + 1 < nd && before_best > -2.0f && after_best > -2.0f)
                    d = __fadd_rn(d, __fmul_rn(kStep, parabola(__fsub_rn(1.0f, before_best), __fsub_rn(1.0f, best),
                                                               __fsub_rn(1.0f, after_best))));
                out_d = d;
                out_c = best;
            }
        }
    }
    a.disp[i] = out_d;
    a.conf[i] = out_c;
}

// zncc_window (stereo.cpp:211-238).
__device__ float zncc_window(const uint8_t* a, const uint8_t* b, int bw, int x0, int y0, int n, float cx, float cy, float D,
                             float gx, float gy, double sa, double saa) {
    ZnccSums s;
    float fY = static_cast<float>(y0);
    for (int j = 0; j < n; ++j, fY = __fadd_rn(fY, 1.0f)) {
        const int Y = y0 + j;
        const uint8_t* ra = a + static_cast<size_t>(Y) * bw + x0;
        const uint8_t* rb = b + static_cast<size_t>(Y) * bw;
        const float dy = __fmul_rn(gy, __fsub_rn(fY, cy));
        float fX = static_cast<float>(x0);
        for (int i = 0; i < n; ++i, fX = __fadd_rn(fX, 1.0f)) {
            const float shift = __fadd_rn(__fadd_rn(D, __fmul_rn(gx, __fsub_rn(fX, cx))), dy);
            const float xb = __fsub_rn(fX, shift);
            double ib;
            if (!sample_row(rb, bw, xb, ib)) return kZnccNoWindow;
            s.add(byte_to_double(ra[i]), ib);
        }
    }
    return s.score(sa, saa, __dmul_rn(static_cast<double>(n), static_cast<double>(n)));
}

// zncc_window for the disparities D.x and D.y (no range checks: see window_inside).
__device__ float2 zncc_window_pair(const uint8_t* a, const uint8_t* b, int bw, int x0, int y0, int n, float cx, float cy, float2 D,
                                   float gx, float gy, double sa, double saa) {
    ZnccSums s0, s1;
    float fY = static_cast<float>(y0);
    for (int j = 0; j < n; ++j, fY = __fadd_rn(fY, 1.0f)) {
        const int Y = y0 + j;
        const uint8_t* ra = a + static_cast<size_t>(Y) * bw + x0;
        const uint8_t* rb = b + static_cast<size_t>(Y) * bw;
        const float dy = __fmul_rn(gy, __fsub_rn(fY, cy));
        float fX = static_cast<float>(x0);
        for (int i = 0; i < n; ++i, fX = __fadd_rn(fX, 1.0f)) {
            const float gxx = __fmul_rn(gx, __fsub_rn(fX, cx));
            const float2 shift = add2_rn(add2_rn(D, f2(gxx, gxx)), f2(dy, dy));
            const float2 ib = bilinear_pair(rb, add2_rn(f2(fX, fX), neg2(shift)));
            const double ia = byte_to_double(ra[i]);
            s0.add(ia, static_cast<double>(ib.x));
            s1.add(ia, static_cast<double>(ib.y));
        }
    }
    const double m = __dmul_rn(static_cast<double>(n), static_cast<double>(n));
    return f2(s0.score(sa, saa, m), s1.score(sa, saa, m));
}

struct DetailArgs {
    const uint8_t* full_left;  // W x H
    const uint8_t* full_right;
    int W, H;
    const float* first;        // the disparity before this stage, w x h
    float* disp;               // output (starts as a copy of first)
    int w, h;
    int radius, K;
    float step, min_zncc;
    int subpixel;
};

__device__ __forceinline__ float detail_grad(float l, float c, float r) {
    if (!valid_disparity(l) || !valid_disparity(r) || fabsf(__fsub_rn(r, c)) >= 1.0f || fabsf(__fsub_rn(c, l)) >= 1.0f)
        return 0.0f;
    return fminf(fmaxf(__fmul_rn(0.5f, __fsub_rn(r, l)), -0.9f), 0.9f);
}

// refine_detail (stereo.cpp:243-284): re-match each half-resolution disparity with a small full-resolution
// window; keep the first estimate unless a clear peak lies inside the search.
static __global__ void __launch_bounds__(128, 6) k_refine_detail(DetailArgs a) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= a.w || y >= a.h) return;
    const int n = 2 * a.radius, nc = 2 * a.K + 1;
    const int y0 = 2 * y - a.radius + 1, x0 = 2 * x - a.radius + 1;
    if (y < 1 || y + 1 >= a.h || y0 < 0 || y0 + n > a.H) return;
    if (x < 1 || x + 1 >= a.w || x0 < 0 || x0 + n > a.W) return;
    auto F = [&](int xx, int yy) { return a.first[static_cast<size_t>(yy) * a.w + xx]; };
    const float d = F(x, y);
    if (!valid_disparity(d)) return;
    const float gx = detail_grad(F(x - 1, y), d, F(x + 1, y)), gy = detail_grad(F(x, y - 1), d, F(x, y + 1));
    const float cx = __fadd_rn(__fmul_rn(2.0f, static_cast<float>(x)), 0.5f), cy = __fadd_rn(__fmul_rn(2.0f, static_cast<float>(y)), 0.5f);
    const float D0 = __fmul_rn(2.0f, d);
    double sa, saa;
    window_moments(a.full_left + static_cast<size_t>(y0) * a.W + x0, a.W, n, n, sa, saa);
    PeakTracker pk;
    // Exact xb over the window and all candidates: X (1 - gx) + gx cx - D - gy (Y - cy), X in [x0, x0 + n),
    // Y in [y0, y0 + n), D within step * K of D0.
    const float ax = __fmul_rn(fmaxf(fabsf(__fsub_rn(static_cast<float>(y0), cy)), fabsf(__fsub_rn(static_cast<float>(y0 + n - 1), cy))),
                               fabsf(gy));
    const float span = __fmul_rn(a.step, static_cast<float>(a.K));
    const float base = __fmul_rn(gx, cx);
    const float lo_x = __fsub_rn(__fsub_rn(__fadd_rn(__fmul_rn(static_cast<float>(x0), __fsub_rn(1.0f, gx)), base), __fadd_rn(D0, span)), ax);
    const float hi_x = __fadd_rn(__fsub_rn(__fadd_rn(__fmul_rn(static_cast<float>(x0 + n - 1), __fsub_rn(1.0f, gx)), base),
                                           __fsub_rn(D0, span)), ax);
    if (window_inside(lo_x, hi_x, a.W)) {
        int k = 0;
        for (; k + 1 < nc; k += 2) {
            const float2 D = f2(__fadd_rn(D0, __fmul_rn(a.step, static_cast<float>(k - a.K))),
                                __fadd_rn(D0, __fmul_rn(a.step, static_cast<float>(k + 1 - a.K))));
            const float2 sc = zncc_window_pair(a.full_left, a.full_right, a.W, x0, y0, n, cx, cy, D, gx, gy, sa, saa);
            pk.push(k, sc.x);
            pk.push(k + 1, sc.y);
        }
        if (k < nc)
            pk.push(k, zncc_window(a.full_left, a.full_right, a.W, x0, y0, n, cx, cy,
                                   __fadd_rn(D0, __fmul_rn(a.step, static_cast<float>(k - a.K))), gx, gy, sa, saa));
    } else {
        for (int k = 0; k < nc; ++k) {
            const float D = __fadd_rn(D0, __fmul_rn(a.step, static_cast<float>(k - a.K)));
            pk.push(k, zncc_window(a.full_left, a.full_right, a.W, x0, y0, n, cx, cy, D, gx, gy, sa, saa));
        }
    }
    const float best = pk.best, before_best = pk.before, after_best = pk.after;
    const int best_k = pk.best_k;
    if (best_k <= 0 || best_k + 1 >= nc || best < a.min_zncc || before_best <= -2.0f || after_best <= -2.0f) return;
    float D = __fadd_rn(D0, __fmul_rn(a.step, static_cast<float>(best_k - a.K)));
    if (a.subpixel)
        D = __fadd_rn(D, __fmul_rn(a.step, parabola(__fsub_rn(1.0f, before_best), __fsub_rn(1.0f, best), __fsub_rn(1.0f, after_best))));
    a.disp[static_cast<size_t>(y) * a.w + x] = __fmul_rn(0.5f, D);
}

// Order-preserving int image of a float (for atomicMax on disparities of either sign).
__device__ __forceinline__ int float_order(float f) {
    const int i = __float_as_int(f);
    return i >= 0 ? i : i ^ 0x7FFFFFFF;
}
__device__ __forceinline__ float order_float(int k) { return __int_as_float(k >= 0 ? k : k ^ 0x7FFFFFFF); }

// filter_disparity, occlusion part (stereo.cpp:288-304): one block per row; the nearest claimant (largest
// disparity) of each right pixel, then every farther claimant beyond the tolerance is invalid.
static __global__ void k_filter_occlusion(float* __restrict__ disp, int w, float tolerance) {
    extern __shared__ int nearest[];
    const int y = blockIdx.x;
    float* row = disp + static_cast<size_t>(y) * w;
    for (int x = threadIdx.x; x < w; x += blockDim.x) nearest[x] = float_order(kInvalid);
    __syncthreads();
    for (int x = threadIdx.x; x < w; x += blockDim.x) {
        const float d = row[x];
        if (!valid_disparity(d)) continue;
        const long xr = lroundf(__fsub_rn(static_cast<float>(x), d));
        if (xr >= 0 && xr < w) atomicMax(&nearest[xr], float_order(d));
    }
    __syncthreads();
    for (int x = threadIdx.x; x < w; x += blockDim.x) {
        const float d = row[x];
        if (!valid_disparity(d)) continue;
        const long xr = lroundf(__fsub_rn(static_cast<float>(x), d));
        if (xr >= 0 && xr < w && d < __fsub_rn(order_float(nearest[xr]), tolerance)) row[x] = kInvalid;
    }
}

// filter_disparity, spike part (stereo.cpp:305-325): `in` is the disparity before this pass.
static __global__ void k_filter_spikes(const float* __restrict__ in, int w, int h, float threshold, float* __restrict__ out) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= w || y >= h) return;
    const size_t i = static_cast<size_t>(y) * w + x;
    const float d = in[i];
    float res = d;
    if (valid_disparity(d)) {
        float v[9];
#pragma unroll
        for (int dy = -1; dy <= 1; ++dy)
#pragma unroll
            for (int dx = -1; dx <= 1; ++dx) {
                const int xx = x + dx, yy = y + dy;
                const bool inside = xx >= 0 && yy >= 0 && xx < w && yy < h;
                v[(dy + 1) * 3 + dx + 1] = inside ? in[static_cast<size_t>(yy) * w + xx] : kInvalid;
            }
        int n;
        const float med = median_of_valid9(v, n);
        if (n >= 3 && fabsf(__fsub_rn(d, med)) > threshold) res = kInvalid;
    }
    out[i] = res;
}

// ---- speckle removal (stereo.cpp:465-494) as connected components by union-find -------------------------
// Regions are connected under |d_a - d_b| <= max_diff between 4-neighbours, which is symmetric, so the
// components (and therefore the removed pixels) do not depend on the order the reference visits them.
// Speckle regions: valid pixels, linked when their disparities differ by at most max_diff.
struct SpeckleConn {
    const float* disp;
    int w;
    float max_diff;
    __device__ __forceinline__ bool active(int x, int y) const { return valid_disparity(disp[static_cast<size_t>(y) * w + x]); }
    __device__ __forceinline__ bool link(int x, int y, int x2, int y2) const {
        const float d = disp[static_cast<size_t>(y) * w + x], dj = disp[static_cast<size_t>(y2) * w + x2];
        return valid_disparity(dj) && !(fabsf(__fsub_rn(dj, d)) > max_diff);
    }
};

// Component sizes once every union has landed. A find returns the true root however other threads halve
// paths meanwhile, so the root is found again where it is used rather than stored in parent[]. Lanes of a
// warp with the same root add their count in one atomic (large regions would otherwise serialise on one
// address).
static __global__ void k_speckle_count(const float* __restrict__ disp, int n, int* parent, int* size, int* err) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool act = i < n && valid_disparity(disp[i]);
    const int r = act ? uf_find<false>(parent, i, err) : -1;
    const unsigned same = __match_any_sync(0xFFFFFFFFu, r);
    if (act && (__ffs(same) - 1) == static_cast<int>(threadIdx.x & 31)) atomicAdd(&size[r], __popc(same));
}

static __global__ void k_speckle_apply(float* __restrict__ disp, int n, int* parent, const int* __restrict__ size,
                                       int max_region_size, int* err) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || !valid_disparity(disp[i])) return;
    if (size[uf_find<false>(parent, i, err)] < max_region_size) disp[i] = kInvalid;
}

// The result's confidence is 0 wherever the disparity is invalid (stereo.cpp:531-533).
static __global__ void k_zero_invalid_conf(const float* __restrict__ disp, int n, float* __restrict__ conf) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (!valid_disparity(disp[i])) conf[i] = 0.0f;
}

}  // namespace dsk
