// The stages of depth::compute_disparity after SGM (libs/depth/src/stereo.cpp:151-326, 465-536): image
// pyramid, slanted-window ZNCC refinement per level, detail refinement on the full-resolution images,
// occlusion and spike filters, speckle removal. All float and double arithmetic follows the reference's
// evaluation order with explicitly rounded intrinsics (no fused multiply-adds), so results are the
// reference's bit for bit.
#pragma once

#include <cstdint>

#include "stereo_kernels.cuh"

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
        int n = 0;
        for (int dy = -1; dy <= 1; ++dy)
            for (int dx = -1; dx <= 1; ++dx) {
                const int xx = x + dx, yy = y + dy;
                if (xx < 0 || yy < 0 || xx >= w || yy >= h) continue;
                const float q = in[static_cast<size_t>(yy) * w + xx];
                if (!valid_disparity(q)) continue;
                int p = n++;
                while (p > 0 && v[p - 1] > q) {
                    v[p] = v[p - 1];
                    --p;
                }
                v[p] = q;
            }
        d = v[n / 2];
    } else {
        d = kInvalid;
    }
    out[i] = d;
}

struct ZnccSums {
    double sa = 0, sb = 0, saa = 0, sbb = 0, sab = 0;
    __device__ __forceinline__ void add(double ia, double ib) {
        sa = __dadd_rn(sa, ia);
        sb = __dadd_rn(sb, ib);
        saa = __dadd_rn(saa, __dmul_rn(ia, ia));
        sbb = __dadd_rn(sbb, __dmul_rn(ib, ib));
        sab = __dadd_rn(sab, __dmul_rn(ia, ib));
    }
    __device__ __forceinline__ float score(double n) const {
        const double va = __dsub_rn(saa, __ddiv_rn(__dmul_rn(sa, sa), n));
        const double vb = __dsub_rn(sbb, __ddiv_rn(__dmul_rn(sb, sb), n));
        if (va < 1e-6 || vb < 1e-6) return -1.0f;
        return __double2float_rn(__ddiv_rn(__dsub_rn(sab, __ddiv_rn(__dmul_rn(sa, sb), n)), __dsqrt_rn(__dmul_rn(va, vb))));
    }
};

// One bilinear sample of the right row at xb: rb[x0] (1 - f) + rb[x0 + 1] f in float, as a double; false
// when x0 or x0 + 1 leave the row.
__device__ __forceinline__ bool sample_row(const uint8_t* rb, int bw, float xb, double& ib) {
    const int x0 = static_cast<int>(floorf(xb));
    if (x0 < 0 || x0 + 1 >= bw) return false;
    const float f = __fsub_rn(xb, static_cast<float>(x0));
    ib = static_cast<double>(__fadd_rn(__fmul_rn(static_cast<float>(rb[x0]), __fsub_rn(1.0f, f)),
                                       __fmul_rn(static_cast<float>(rb[x0 + 1]), f)));
    return true;
}

// zncc_slanted (stereo.cpp:102-126).
__device__ float zncc_slanted(const uint8_t* a, const uint8_t* b, int w, int x, int y, float d, float gx, float gy, int r) {
    ZnccSums s;
    const int n = (2 * r + 1) * (2 * r + 1);
    for (int v = -r; v <= r; ++v) {
        const uint8_t* ra = a + static_cast<size_t>(y + v) * w;
        const uint8_t* rb = b + static_cast<size_t>(y + v) * w;
        for (int u = -r; u <= r; ++u) {
            const float shift = __fadd_rn(__fadd_rn(d, __fmul_rn(gx, static_cast<float>(u))), __fmul_rn(gy, static_cast<float>(v)));
            const float xb = __fsub_rn(static_cast<float>(x + u), shift);
            double ib;
            if (!sample_row(rb, w, xb, ib)) return kZnccNoWindow;
            s.add(static_cast<double>(ra[x + u]), ib);
        }
    }
    return s.score(static_cast<double>(n));
}

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
static __global__ void __launch_bounds__(128) k_refine_level(RefineArgs a) {
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
            float best = -2.0f, prev = -2.0f, before_best = -2.0f, after_best = -2.0f;
            int best_k = -1;
            for (int k = 0; k < nd; ++k) {
                const float d = __fadd_rn(lo, __fmul_rn(kStep, static_cast<float>(k)));
                const float sc = zncc_slanted(a.left, a.right, a.w, x, y, d, gx, gy, r);
                if (k == best_k + 1) after_best = sc;  // the score right after the current best
                if (sc > best) {
                    best = sc;
                    best_k = k;
                    before_best = prev;
                    after_best = -3.0f;  // not yet known
                }
                prev = sc;
            }
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
                             float gx, float gy) {
    ZnccSums s;
    for (int j = 0; j < n; ++j) {
        const int Y = y0 + j;
        const uint8_t* ra = a + static_cast<size_t>(Y) * bw;
        const uint8_t* rb = b + static_cast<size_t>(Y) * bw;
        const float dy = __fmul_rn(gy, __fsub_rn(static_cast<float>(Y), cy));
        for (int i = 0; i < n; ++i) {
            const int X = x0 + i;
            const float shift = __fadd_rn(__fadd_rn(D, __fmul_rn(gx, __fsub_rn(static_cast<float>(X), cx))), dy);
            const float xb = __fsub_rn(static_cast<float>(X), shift);
            double ib;
            if (!sample_row(rb, bw, xb, ib)) return kZnccNoWindow;
            s.add(static_cast<double>(ra[X]), ib);
        }
    }
    return s.score(__dmul_rn(static_cast<double>(n), static_cast<double>(n)));
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
static __global__ void __launch_bounds__(128) k_refine_detail(DetailArgs a) {
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
    float best = -2.0f, prev = -2.0f, before_best = -2.0f, after_best = -2.0f;
    int best_k = -1;
    for (int k = 0; k < nc; ++k) {
        const float D = __fadd_rn(D0, __fmul_rn(a.step, static_cast<float>(k - a.K)));
        const float sc = zncc_window(a.full_left, a.full_right, a.W, x0, y0, n, cx, cy, D, gx, gy);
        if (k == best_k + 1) after_best = sc;
        if (sc > best) {
            best = sc;
            best_k = k;
            before_best = prev;
            after_best = -3.0f;
        }
        prev = sc;
    }
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
        int n = 0;
        for (int dy = -1; dy <= 1; ++dy)
            for (int dx = -1; dx <= 1; ++dx) {
                const int xx = x + dx, yy = y + dy;
                if (xx < 0 || yy < 0 || xx >= w || yy >= h) continue;
                const float q = in[static_cast<size_t>(yy) * w + xx];
                if (!valid_disparity(q)) continue;
                int p = n++;
                while (p > 0 && v[p - 1] > q) {
                    v[p] = v[p - 1];
                    --p;
                }
                v[p] = q;
            }
        if (n >= 3 && fabsf(__fsub_rn(d, v[n / 2])) > threshold) res = kInvalid;
    }
    out[i] = res;
}

// ---- speckle removal (stereo.cpp:465-494) as connected components by union-find -------------------------
// Regions are connected under |d_a - d_b| <= max_diff between 4-neighbours, which is symmetric, so the
// components (and therefore the removed pixels) do not depend on the order the reference visits them.
// Every loop here is bounded; a bound that runs out sets *err.
constexpr int kFindLimit = 1 << 22;

// Root of x with path halving. Every parent index is at most its child's (roots are only ever hung under a
// smaller root), so a halving store written concurrently with other finds or unions still names an
// ancestor. Reads bypass L1 so that roots linked by other blocks are seen.
__device__ __forceinline__ int uf_find(int* parent, int x, int* err) {
    for (int it = 0; it < kFindLimit; ++it) {
        const int p = __ldcg(parent + x);
        if (p == x) return x;
        const int gp = __ldcg(parent + p);
        if (gp != p) parent[x] = gp;
        x = gp;
    }
    *err = 1;
    return x;
}

static __global__ void k_speckle_init(const float* __restrict__ disp, int n, int* __restrict__ parent, int* __restrict__ size) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    parent[i] = i;
    size[i] = 0;
}

// Union of each pixel with its right and lower neighbours: the larger root is hung under the smaller.
static __global__ void k_speckle_union(const float* __restrict__ disp, int w, int h, float max_diff, int* parent, int* err) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= w || y >= h) return;
    const int i = y * w + x;
    const float d = disp[i];
    if (!valid_disparity(d)) return;
    const int nb[2] = {x + 1 < w ? i + 1 : -1, y + 1 < h ? i + w : -1};
    for (int q = 0; q < 2; ++q) {
        const int j = nb[q];
        if (j < 0) continue;
        const float dj = disp[j];
        if (!valid_disparity(dj) || fabsf(__fsub_rn(dj, d)) > max_diff) continue;
        int a = i, b = j;
        for (int it = 0; it < kFindLimit; ++it) {
            a = uf_find(parent, a, err);
            b = uf_find(parent, b, err);
            if (a == b) break;
            if (a < b) {
                const int t = a;
                a = b;
                b = t;
            }
            // a > b: hang root a under b unless another thread changed a's parent first
            const int old = atomicCAS(&parent[a], a, b);
            if (old == a) break;
            a = old;
            if (it + 1 == kFindLimit) *err = 1;
        }
    }
}

// Component sizes once every union has landed. A find returns the true root however other threads halve
// paths meanwhile, so the root is found again where it is used rather than stored in parent[].
static __global__ void k_speckle_count(const float* __restrict__ disp, int n, int* parent, int* size, int* err) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || !valid_disparity(disp[i])) return;
    atomicAdd(&size[uf_find(parent, i, err)], 1);
}

static __global__ void k_speckle_apply(float* __restrict__ disp, int n, int* parent, const int* __restrict__ size,
                                       int max_region_size, int* err) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || !valid_disparity(disp[i])) return;
    if (size[uf_find(parent, i, err)] < max_region_size) disp[i] = kInvalid;
}

// The result's confidence is 0 wherever the disparity is invalid (stereo.cpp:531-533).
static __global__ void k_zero_invalid_conf(const float* __restrict__ disp, int n, float* __restrict__ conf) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (!valid_disparity(disp[i])) conf[i] = 0.0f;
}

}  // namespace dsk
