// Marker blob search on a raw IR image: the per-pixel part of markers::detect_markers (connected pixels
// above a grey threshold, libs/markers/src/detect.cpp:14-45) with the candidate gates of the reference's GPU
// search (depth_metal blob_select, libs/depth_metal/src/stereo_kernels.metal.inc:770-901): box size,
// aspect, fill and border as in the CPU detector, then a dark-ring pre-check on the blob's moment ellipse.
//
// Components are found by union-find (union_find.cuh): each blob's root is its first pixel in raster
// order, the pixel the CPU flood fill starts from. Per-root statistics (pixels, box, peak, second moments
// relative to the root) are exact integer atomics. The candidate test is float arithmetic written with
// explicitly rounded operations and no transcendental function: the moment ellipse's orientation enters
// only through cos and sin of its angle, which follow from the moments by half-angle formulas (IEEE
// square roots), and the 16 ring directions are a table of cos / sin (2 pi k / 16). The candidates are
// therefore reproducible bit for bit by a CPU restatement.
#pragma once

#include <cstdint>

#include "union_find.cuh"

namespace dsk {

struct BlobCand {
    uint32_t x0, y0, x1, y1, pixels, peak;
    uint32_t root;  // first pixel of the blob in raster order (orders the candidates)
    uint32_t pad;
};

struct BlobArgs {
    const uint8_t* img;  // w x h, rows w bytes apart
    int w, h;
    uint32_t threshold, min_diameter, max_diameter, border, max_out;
    float max_aspect, min_fill, max_axis_ratio, ring_scale, ring_contrast, ring_max_bright;
    int* parent;         // w*h labels (-1: background)
    uint32_t* count;     // per root: pixels
    uint32_t* box;       // per root: x0, y0, x1, y1, peak (5 words)
    int* mom;            // per root: sum dx, dy, dx^2, dx dy, dy^2 relative to the root (5 words)
    BlobCand* out;
    uint32_t* n_out;     // candidates found (may exceed max_out; only max_out are written)
    int* err;
};

// cos and sin of 2 pi k / 16, k = 0..15, rounded to float.
__constant__ float c_ring_cos[16] = {1.0f, 0.923879533f, 0.707106781f, 0.382683432f, 0.0f, -0.382683432f, -0.707106781f, -0.923879533f,
                                     -1.0f, -0.923879533f, -0.707106781f, -0.382683432f, 0.0f, 0.382683432f, 0.707106781f, 0.923879533f};
__constant__ float c_ring_sin[16] = {0.0f, 0.382683432f, 0.707106781f, 0.923879533f, 1.0f, 0.923879533f, 0.707106781f, 0.382683432f,
                                     0.0f, -0.382683432f, -0.707106781f, -0.923879533f, -1.0f, -0.923879533f, -0.707106781f, -0.382683432f};

static __global__ void k_blob_init(BlobArgs a) {
    const int n = a.w * a.h;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const bool fg = a.img[i] > a.threshold;
    a.parent[i] = fg ? i : -1;
    if (!fg) return;  // only foreground pixels become roots, and statistics are read at roots only
    a.count[i] = 0u;
    uint32_t* b = a.box + 5 * static_cast<size_t>(i);
    b[0] = b[1] = 0xFFFFFFFFu;
    b[2] = b[3] = b[4] = 0u;
    int* m = a.mom + 5 * static_cast<size_t>(i);
    m[0] = m[1] = m[2] = m[3] = m[4] = 0;
}

// Blobs: pixels above the threshold, 4-neighbours linked.
struct BlobConn {
    const uint8_t* img;
    int w;
    uint32_t threshold;
    __device__ __forceinline__ bool active(int x, int y) const { return img[static_cast<size_t>(y) * w + x] > threshold; }
    __device__ __forceinline__ bool link(int, int, int x2, int y2) const { return active(x2, y2); }
};

// Per-root statistics. Lanes of a warp with the same root reduce first (one set of atomics per root and
// warp): a bright surface under the ring light is one large component.
static __global__ void k_blob_stats(BlobArgs a) {
    const int n = a.w * a.h;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    const bool act = i < n && a.img[i] > a.threshold;
    const int r = act ? uf_find<false>(a.parent, i, a.err) : -1;
    const unsigned grp = __match_any_sync(0xFFFFFFFFu, r);
    if (!act) return;
    const int x = i % a.w, y = i / a.w, rx = r % a.w, ry = r / a.w;
    const int dx = x - rx, dy = y - ry;
    const uint32_t cnt = __popc(grp);
    const uint32_t x0 = __reduce_min_sync(grp, static_cast<uint32_t>(x)), y0 = __reduce_min_sync(grp, static_cast<uint32_t>(y));
    const uint32_t x1 = __reduce_max_sync(grp, static_cast<uint32_t>(x)), y1 = __reduce_max_sync(grp, static_cast<uint32_t>(y));
    const uint32_t pk = __reduce_max_sync(grp, static_cast<uint32_t>(a.img[i]));
    // Moment sums in 32-bit two's complement (wrapping for blobs far beyond the size gates, which reject
    // them by their box first).
    const uint32_t m0 = __reduce_add_sync(grp, static_cast<uint32_t>(dx)), m1 = __reduce_add_sync(grp, static_cast<uint32_t>(dy));
    const uint32_t m2 = __reduce_add_sync(grp, static_cast<uint32_t>(dx * dx)), m3 = __reduce_add_sync(grp, static_cast<uint32_t>(dx * dy));
    const uint32_t m4 = __reduce_add_sync(grp, static_cast<uint32_t>(dy * dy));
    if (static_cast<int>(threadIdx.x & 31) != __ffs(grp) - 1) return;
    atomicAdd(a.count + r, cnt);
    uint32_t* b = a.box + 5 * static_cast<size_t>(r);
    atomicMin(b + 0, x0);
    atomicMin(b + 1, y0);
    atomicMax(b + 2, x1);
    atomicMax(b + 3, y1);
    atomicMax(b + 4, pk);
    unsigned* m = reinterpret_cast<unsigned*>(a.mom + 5 * static_cast<size_t>(r));
    atomicAdd(m + 0, m0);
    atomicAdd(m + 1, m1);
    atomicAdd(m + 2, m2);
    atomicAdd(m + 3, m3);
    atomicAdd(m + 4, m4);
}

// Grey level at the nearest pixel of (x, y), clamped to the image (round half away from zero). The
// coordinates are clamped before the conversion to int, so that any float (also from the wrapped moments of
// a huge blob) converts the same way everywhere.
__device__ __forceinline__ float blob_sample(const BlobArgs& a, float x, float y) {
    x = fminf(fmaxf(x, -1.0f), static_cast<float>(a.w));
    y = fminf(fmaxf(y, -1.0f), static_cast<float>(a.h));
    const int sx = min(max(static_cast<int>(roundf(x)), 0), a.w - 1), sy = min(max(static_cast<int>(roundf(y)), 0), a.h - 1);
    return static_cast<float>(a.img[static_cast<size_t>(sy) * a.w + sx]);
}

// Point k of the ellipse with semi-axes (su, sv) along directions (ct, st) / (-st, ct), centred at (cx, cy).
__device__ __forceinline__ float blob_ring(const BlobArgs& a, int k, float su, float sv, float ct, float st, float cx, float cy) {
    const float u = __fmul_rn(su, c_ring_cos[k]), v = __fmul_rn(sv, c_ring_sin[k]);
    const float px = __fsub_rn(__fadd_rn(cx, __fmul_rn(ct, u)), __fmul_rn(st, v));
    const float py = __fadd_rn(__fadd_rn(cy, __fmul_rn(st, u)), __fmul_rn(ct, v));
    return blob_sample(a, px, py);
}

// Gates and the dark-ring pre-check at every root; candidates go to a compact list.
static __global__ void k_blob_select(BlobArgs a) {
    const int n = a.w * a.h;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || a.img[i] <= a.threshold || a.parent[i] != i) return;
    const uint32_t* b = a.box + 5 * static_cast<size_t>(i);
    const uint32_t x0 = b[0], y0 = b[1], x1 = b[2], y1 = b[3], pk = b[4], px = a.count[i];
    const float bw = static_cast<float>(x1 - x0 + 1), bh = static_cast<float>(y1 - y0 + 1);
    const float dmin = static_cast<float>(a.min_diameter), dmax = static_cast<float>(a.max_diameter);
    if (bw < dmin || bh < dmin || bw > dmax || bh > dmax) return;
    if (fmaxf(bw, bh) > __fmul_rn(a.max_aspect, fminf(bw, bh))) return;
    constexpr float kPi = 3.14159265358979f;
    if (static_cast<float>(px) < __fdiv_rn(__fmul_rn(__fmul_rn(__fmul_rn(a.min_fill, bw), bh), kPi), 4.0f)) return;
    const int m = max(3, static_cast<int>(fmaxf(bw, bh)) / 2);
    const int bd = static_cast<int>(a.border);
    if (static_cast<int>(x0) - m < bd || static_cast<int>(y0) - m < bd || static_cast<int>(x1) + m >= a.w - bd ||
        static_cast<int>(y1) + m >= a.h - bd)
        return;
    // Semi-axes from the eigenvalues of the central moment matrix: spread uniformly over an ellipse, the pixels
    // have variance s^2 / 4 along a semi-axis of length s, so s = 2 sqrt(lambda).
    const int* mo = a.mom + 5 * static_cast<size_t>(i);
    const float fn = static_cast<float>(px);
    const float mx = __fdiv_rn(static_cast<float>(mo[0]), fn), my = __fdiv_rn(static_cast<float>(mo[1]), fn);
    const float cxx = __fsub_rn(__fdiv_rn(static_cast<float>(mo[2]), fn), __fmul_rn(mx, mx));
    const float cxy = __fsub_rn(__fdiv_rn(static_cast<float>(mo[3]), fn), __fmul_rn(mx, my));
    const float cyy = __fsub_rn(__fdiv_rn(static_cast<float>(mo[4]), fn), __fmul_rn(my, my));
    const float dxy = __fsub_rn(cxx, cyy);
    const float tr = __fmul_rn(0.5f, __fadd_rn(cxx, cyy));
    const float det = __fsqrt_rn(fmaxf(0.0f, __fadd_rn(__fmul_rn(__fmul_rn(0.25f, dxy), dxy), __fmul_rn(cxy, cxy))));
    const float l1 = __fadd_rn(tr, det), l2 = fmaxf(__fsub_rn(tr, det), 0.0625f);
    // + 0.5: the pixels above the threshold stop about half a pixel short of the blob's true outline
    const float ea = __fadd_rn(__fmul_rn(2.0f, __fsqrt_rn(fmaxf(l1, 0.0f))), 0.5f), eb = __fadd_rn(__fmul_rn(2.0f, __fsqrt_rn(l2)), 0.5f);
    if (__fdiv_rn(ea, eb) > __fmul_rn(a.max_axis_ratio, 1.2f)) return;
    // Major-axis direction (angle th = atan2(2 cxy, cxx - cyy) / 2): cos th = sqrt((1 + cos 2th) / 2),
    // sin th = sign(sin 2th) sqrt((1 - cos 2th) / 2). The ring samples are symmetric under th -> th + pi.
    const float s2 = __fmul_rn(2.0f, cxy);
    const float r2 = __fsqrt_rn(__fadd_rn(__fmul_rn(dxy, dxy), __fmul_rn(s2, s2)));
    float ct = 1.0f, st = 0.0f;
    if (r2 > 0.0f) {
        const float c2 = fminf(fmaxf(__fdiv_rn(dxy, r2), -1.0f), 1.0f);
        ct = __fsqrt_rn(__fmul_rn(0.5f, __fadd_rn(1.0f, c2)));
        st = __fsqrt_rn(__fmul_rn(0.5f, __fsub_rn(1.0f, c2)));
        if (s2 < 0.0f) st = -st;
    }
    const float cx = __fadd_rn(static_cast<float>(i % a.w), mx), cy = __fadd_rn(static_cast<float>(i / a.w), my);
    // Local background level: the 4th smallest grey value among 16 points of an ellipse 2.2 times the blob's.
    float bg[16];
    const float bu = __fmul_rn(2.2f, ea), bv = __fmul_rn(2.2f, eb);
#pragma unroll
    for (int k = 0; k < 16; ++k) bg[k] = blob_ring(a, k, bu, bv, ct, st, cx, cy);
#pragma unroll
    for (int p = 0; p < 4; ++p)
#pragma unroll
        for (int q = p + 1; q < 16; ++q)
            if (bg[q] < bg[p]) {
                const float t = bg[p];
                bg[p] = bg[q];
                bg[q] = t;
            }
    const float level = __fadd_rn(bg[3], __fmul_rn(a.ring_contrast, __fsub_rn(static_cast<float>(pk), bg[3])));
    // A retro-reflective marker is framed by a dark annulus; a projected speckle dot has bright dots around it.
    // Reject the blob when too many points of the ring_scale ellipse are brighter than the level.
    const float ru = __fmul_rn(a.ring_scale, ea), rv = __fmul_rn(a.ring_scale, eb);
    int bright = 0;
#pragma unroll
    for (int k = 0; k < 16; ++k) bright += blob_ring(a, k, ru, rv, ct, st, cx, cy) > level ? 1 : 0;
    if (static_cast<float>(bright) > __fmul_rn(a.ring_max_bright, 16.0f)) return;
    const uint32_t slot = atomicAdd(a.n_out, 1u);
    if (slot < a.max_out) a.out[slot] = BlobCand{x0, y0, x1, y1, px, pk, static_cast<uint32_t>(i), 0u};
}

}  // namespace dsk
