// Per-frame CUDA kernels of the stereo hot path (sm_100a).
//
// Layout in HBM (per frame, W x H, D disparities, P path directions):
//   rectified left/right    u8  [y][x]
//   census left/right       u32 or u64 [y][x] (u32 when the window has <= 32 neighbours)
//   path values             u8 (or u16) [dir][y][x][Dp], Dp = 32 * VPL >= D; one slab per direction
//   L-R checked disparity   f32 [y][x]
// Outputs (f32 disparity, f32 confidence, u16 disparity, f32 depth) are written by the last kernel.
//
// Bit-exactness: integer stages reproduce libs/depth/src/stereo.cpp exactly; float stages use
// explicitly rounded intrinsics (__fadd_rn, __fmul_rn, __fdiv_rn, ...) so that nvcc cannot contract
// them into FMAs, which the reference's separately rounded x86 arithmetic does not do.
#pragma once

#include <cstdint>
#include <climits>

namespace dsk {

constexpr float kInvalid = -1.0e9f;  // depth::kInvalidDisparity (stereo.hpp:23)
constexpr int kNoMatch = INT_MIN;    // sgm_disparity's kNoMatch (stereo.cpp:413)
constexpr int kMaxDisparities = 512;
constexpr int kInf = 0x3FFFFFFF;     // "no such neighbour" in the path recurrence (above every path value)
constexpr unsigned kFull = 0xFFFFFFFFu;

__host__ __device__ inline bool valid_disparity(float d) { return d > -1.0e8f; }  // stereo.hpp:24

// Path directions in the reference's order (stereo.cpp:387-388).
__constant__ int c_dir_dx[8] = {1, -1, 0, 0, 1, -1, 1, -1};
__constant__ int c_dir_dy[8] = {0, 0, 1, -1, 1, -1, -1, 1};

template <typename W>
__device__ __forceinline__ int popcount_word(W v);
template <>
__device__ __forceinline__ int popcount_word<uint32_t>(uint32_t v) { return __popc(v); }
template <>
__device__ __forceinline__ int popcount_word<uint64_t>(uint64_t v) { return __popcll(v); }

// ------------------------------------------------------------------------------------------------
// Rectification: bilinear remap (libs/calib/src/rectify.cpp:133-148), optionally followed by the
// 2x2 box downsample of depth::downsample2 (stereo.cpp:348-359) when the tables are twice the size.

struct RectifyArgs {
    const uint8_t* raw[2];
    const float* map_x[2];
    const float* map_y[2];
    uint8_t* out[2];
    int raw_w, raw_h;
    int map_w;
    int out_w, out_h;
    int half;
};

__device__ __forceinline__ uint32_t remap_sample(const uint8_t* __restrict__ src, int sw, int sh, float sx, float sy) {
    const int x0 = static_cast<int>(floorf(sx)), y0 = static_cast<int>(floorf(sy));
    if (x0 < 0 || y0 < 0 || x0 + 1 >= sw || y0 + 1 >= sh) return 0u;
    const float fx = __fsub_rn(sx, static_cast<float>(x0));
    const float fy = __fsub_rn(sy, static_cast<float>(y0));
    const float gx = __fsub_rn(1.0f, fx), gy = __fsub_rn(1.0f, fy);
    const uint8_t* r0 = src + static_cast<size_t>(y0) * sw + x0;
    const uint8_t* r1 = r0 + sw;
    const float a = __ldg(r0), b = __ldg(r0 + 1), c = __ldg(r1), d = __ldg(r1 + 1);
    const float top = __fadd_rn(__fmul_rn(a, gx), __fmul_rn(b, fx));
    const float bot = __fadd_rn(__fmul_rn(c, gx), __fmul_rn(d, fx));
    float v = __fadd_rn(__fmul_rn(top, gy), __fmul_rn(bot, fy));
    v = fminf(fmaxf(__fadd_rn(v, 0.5f), 0.0f), 255.0f);
    return static_cast<uint32_t>(__float2uint_rz(v));
}

__global__ void k_rectify(RectifyArgs a) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int side = blockIdx.z;
    if (x >= a.out_w || y >= a.out_h) return;
    const uint8_t* src = a.raw[side];
    const float* mx = a.map_x[side];
    const float* my = a.map_y[side];
    uint32_t v;
    if (!a.half) {
        const size_t i = static_cast<size_t>(y) * a.map_w + x;
        v = remap_sample(src, a.raw_w, a.raw_h, __ldg(mx + i), __ldg(my + i));
    } else {
        uint32_t acc = 0;
        for (int j = 0; j < 2; ++j)
            for (int i = 0; i < 2; ++i) {
                const size_t m = static_cast<size_t>(2 * y + j) * a.map_w + (2 * x + i);
                acc += remap_sample(src, a.raw_w, a.raw_h, __ldg(mx + m), __ldg(my + m));
            }
        v = (acc + 2u) / 4u;
    }
    a.out[side][static_cast<size_t>(y) * a.out_w + x] = static_cast<uint8_t>(v);
}

// ------------------------------------------------------------------------------------------------
// Census (stereo.cpp:328-346): bit per window neighbour, row-major, centre skipped, MSB first,
// set when neighbour < centre; 0 within (rx, ry) of the border.

struct CensusArgs {
    const uint8_t* img[2];
    void* out[2];
    int w, h, rx, ry;
};

template <typename W>
__global__ void k_census(CensusArgs a) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int side = blockIdx.z;
    if (x >= a.w || y >= a.h) return;
    const uint8_t* img = a.img[side];
    W word = 0;
    if (y >= a.ry && y < a.h - a.ry && x >= a.rx && x < a.w - a.rx) {
        const uint8_t c = __ldg(img + static_cast<size_t>(y) * a.w + x);
        for (int v = -a.ry; v <= a.ry; ++v) {
            const uint8_t* row = img + static_cast<size_t>(y + v) * a.w + x;
            for (int u = -a.rx; u <= a.rx; ++u) {
                if (u == 0 && v == 0) continue;
                word = static_cast<W>((word << 1) | static_cast<W>(__ldg(row + u) < c));
            }
        }
    }
    static_cast<W*>(a.out[side])[static_cast<size_t>(y) * a.w + x] = word;
}

// ------------------------------------------------------------------------------------------------
// Path aggregation (stereo.cpp:44-89, directions and start pixels :382-409).
// One warp per scanline; lane l holds disparities k = l*VPL + j (j < VPL). Each step:
//   cost c[k]  = popcount(census_l(x) ^ census_r(x - min - k)) or the window area when outside,
//   P2'        = table[|I - I_prev| / 8] (adaptive) from the left image,
//   best[k]    = min(prev[k], min(prev) + P2', prev[k+-1] + P1 [, prev[k+-2] + P1]),
//   L[k]       = c[k] + best[k] - min(prev),
// neighbours across lanes come from warp shuffles, min(prev) from a warp min-reduction. L goes to the
// direction's slab; the directions are summed by the WTA kernel (u16 wrap, same as the reference's
// sequential u16 accumulation).

struct PathArgs {
    const void* census_l;
    const void* census_r;
    const uint8_t* guide;
    void* values;        // [dir][y][x][dp]
    size_t dir_stride;   // elements per direction slab
    int w, h, nd, dp, min_disp, p1, invalid_cost, slant;
    int dir_base;
    int p2_table[32];
};

__device__ __forceinline__ void line_start(int dx, int dy, int line, int w, int h, int& x, int& y, int& nlines) {
    nlines = dy == 0 ? h : (dx == 0 ? w : h + w - 1);
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

template <int VPL, typename CW, typename ST>
__global__ void __launch_bounds__(128) k_paths(PathArgs a) {
    const int lane = threadIdx.x & 31;
    const int line = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int di = a.dir_base + blockIdx.y;
    const int dx = c_dir_dx[di], dy = c_dir_dy[di];
    int x, y, nlines;
    line_start(dx, dy, line, a.w, a.h, x, y, nlines);
    if (line >= nlines) return;  // whole warp leaves together

    const CW* __restrict__ cl = static_cast<const CW*>(a.census_l);
    const CW* __restrict__ cr = static_cast<const CW*>(a.census_r);
    ST* __restrict__ out = static_cast<ST*>(a.values) + static_cast<size_t>(di) * a.dir_stride;
    const int k0 = lane * VPL;

    int prev[VPL];
    int pmin;
    int last_i = __ldg(a.guide + static_cast<size_t>(y) * a.w + x);

    auto costs = [&](int cx, int cy, int* c) {
        const size_t row = static_cast<size_t>(cy) * a.w;
        const CW vl = __ldg(cl + row + cx);
#pragma unroll
        for (int j = 0; j < VPL; ++j) {
            const int k = k0 + j;
            const int xr = cx - a.min_disp - k;
            c[j] = (k < a.nd && xr >= 0 && xr < a.w) ? popcount_word<CW>(vl ^ __ldg(cr + row + xr)) : a.invalid_cost;
        }
    };
    auto store = [&](int sx, int sy, const int* v) {
        ST* o = out + (static_cast<size_t>(sy) * a.w + sx) * a.dp + k0;
#pragma unroll
        for (int j = 0; j < VPL; ++j)
            if (k0 + j < a.nd) o[j] = static_cast<ST>(v[j]);
    };

    {
        int c[VPL];
        costs(x, y, c);
        int m = kInf;
#pragma unroll
        for (int j = 0; j < VPL; ++j) {
            prev[j] = (k0 + j < a.nd) ? c[j] : kInf;
            m = min(m, prev[j]);
        }
        pmin = static_cast<int>(__reduce_min_sync(kFull, static_cast<unsigned>(m)));
        store(x, y, prev);
    }

    for (x += dx, y += dy; x >= 0 && y >= 0 && x < a.w && y < a.h; x += dx, y += dy) {
        const int I = __ldg(a.guide + static_cast<size_t>(y) * a.w + x);
        const int d_i = I > last_i ? I - last_i : last_i - I;
        const int jump = pmin + a.p2_table[d_i >> 3];
        last_i = I;

        // prev[k-2 .. k+VPL+1] of this lane's window, INF outside [0, nd).
        int ext[VPL + 4];
#pragma unroll
        for (int j = 0; j < VPL; ++j) ext[j + 2] = prev[j];
        const int up1 = __shfl_up_sync(kFull, prev[VPL - 1], 1);
        const int up2 = VPL >= 2 ? __shfl_up_sync(kFull, prev[VPL >= 2 ? VPL - 2 : 0], 1) : __shfl_up_sync(kFull, prev[0], 2);
        const int dn1 = __shfl_down_sync(kFull, prev[0], 1);
        const int dn2 = VPL >= 2 ? __shfl_down_sync(kFull, prev[VPL >= 2 ? 1 : 0], 1) : __shfl_down_sync(kFull, prev[0], 2);
        ext[1] = k0 - 1 >= 0 ? up1 : kInf;
        ext[0] = k0 - 2 >= 0 ? up2 : kInf;
        ext[VPL + 2] = k0 + VPL < a.nd ? dn1 : kInf;
        ext[VPL + 3] = k0 + VPL + 1 < a.nd ? dn2 : kInf;

        int c[VPL];
        costs(x, y, c);
        int cur[VPL];
        int m = kInf;
#pragma unroll
        for (int j = 0; j < VPL; ++j) {
            int b = min(ext[j + 2], jump);
            b = min(b, min(ext[j + 1], ext[j + 3]) + a.p1);
            if (a.slant) b = min(b, min(ext[j], ext[j + 4]) + a.p1);
            const int v = (k0 + j < a.nd) ? c[j] + b - pmin : kInf;
            cur[j] = v;
            m = min(m, v);
        }
        pmin = static_cast<int>(__reduce_min_sync(kFull, static_cast<unsigned>(m)));
#pragma unroll
        for (int j = 0; j < VPL; ++j) prev[j] = cur[j];
        store(x, y, cur);
    }
}

// ------------------------------------------------------------------------------------------------
// Winner-takes-all left + right and the L-R check (stereo.cpp:411-461), one CTA per row.
// Left: warp per pixel over the summed path values; first strict minimum via a min-reduction of
// (cost << 16 | k) keys; the best non-adjacent cost; uniqueness as a float compare; parabola.
// Right: each candidate (x, k) offers its key to right pixel xr = x - min - k with a shared-memory
// atomicMin, which yields the first strict minimum along the diagonal.

struct WtaArgs {
    const void* values;
    size_t dir_stride;
    int ndirs;
    int w, h, nd, dp, min_disp;
    float uniqueness;
    int subpixel;
    int lr_max_diff;
    float* disp;  // L-R checked
};

__device__ __forceinline__ float parabola(float cm, float c0, float cp) {  // stereo.cpp:92-96
    const float denom = __fadd_rn(__fsub_rn(cm, __fmul_rn(2.0f, c0)), cp);
    if (denom <= 0.0f) return 0.0f;
    const float t = __fdiv_rn(__fmul_rn(0.5f, __fsub_rn(cm, cp)), denom);
    return fminf(fmaxf(t, -0.5f), 0.5f);
}

template <int VPL>
__device__ __forceinline__ uint32_t pick(const uint32_t (&v)[VPL], int j) {
    uint32_t r = 0;
#pragma unroll
    for (int i = 0; i < VPL; ++i)
        if (i == j) r = v[i];
    return r;
}

template <int VPL, typename ST>
__global__ void __launch_bounds__(256) k_wta(WtaArgs a) {
    extern __shared__ uint32_t smem[];
    uint32_t* rkey = smem;                                  // [w]
    float* dleft = reinterpret_cast<float*>(smem + a.w);    // [w]
    const int y = blockIdx.x;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    for (int i = threadIdx.x; i < a.w; i += blockDim.x) rkey[i] = 0xFFFFFFFFu;
    __syncthreads();

    const ST* __restrict__ vals = static_cast<const ST*>(a.values);
    const int k0 = lane * VPL;
    for (int x = warp; x < a.w; x += nwarps) {
        uint32_t tot[VPL];
#pragma unroll
        for (int j = 0; j < VPL; ++j) tot[j] = 0;
        const size_t base = (static_cast<size_t>(y) * a.w + x) * a.dp + k0;
        for (int d = 0; d < a.ndirs; ++d) {
            const ST* p = vals + static_cast<size_t>(d) * a.dir_stride + base;
#pragma unroll
            for (int j = 0; j < VPL; ++j)
                if (k0 + j < a.nd) tot[j] += p[j];
        }
        const int lo = max(0, x - a.min_disp - (a.w - 1));
        const int hi = min(a.nd, x - a.min_disp + 1);
        uint32_t key = 0xFFFFFFFFu;
#pragma unroll
        for (int j = 0; j < VPL; ++j) {
            tot[j] &= 0xFFFFu;
            const int k = k0 + j;
            if (k >= lo && k < hi) {
                const uint32_t kk = (tot[j] << 16) | static_cast<uint32_t>(k);
                key = min(key, kk);
                atomicMin(&rkey[x - a.min_disp - k], kk);
            }
        }
        key = __reduce_min_sync(kFull, key);
        float d = kInvalid;
        if (hi > lo) {
            const int bk = static_cast<int>(key & 0xFFFFu);
            const uint32_t sb = key >> 16;
            uint32_t second = 0xFFFFu;
#pragma unroll
            for (int j = 0; j < VPL; ++j) {
                const int k = k0 + j;
                if (k >= lo && k < hi && (k - bk > 1 || bk - k > 1)) second = min(second, tot[j]);
            }
            second = __reduce_min_sync(kFull, second);
            const bool unique = !(second != 0xFFFFu &&
                                  static_cast<float>(sb) >= __fmul_rn(a.uniqueness, static_cast<float>(second)));
            // The neighbours' costs (all lanes join the shuffles).
            const int km = max(bk - 1, 0), kp = min(bk + 1, a.nd - 1);
            const uint32_t vm = __shfl_sync(kFull, pick<VPL>(tot, km % VPL), km / VPL);
            const uint32_t vp = __shfl_sync(kFull, pick<VPL>(tot, kp % VPL), kp / VPL);
            if (unique) {
                d = static_cast<float>(a.min_disp + bk);
                if (a.subpixel && bk > lo && bk + 1 < hi)
                    d = __fadd_rn(d, parabola(static_cast<float>(vm), static_cast<float>(sb), static_cast<float>(vp)));
            }
        }
        if (lane == 0) dleft[x] = d;
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

// ------------------------------------------------------------------------------------------------
// 3x3 median (stereo.cpp:129-147) + outputs: f32 disparity, confidence (stereo.cpp:515-519), u16
// disparity, depth z = f B / (d + cx_offset) in double with the gates of point_image.cpp:18-20.

struct PostArgs {
    const float* disp;
    int w, h, median, min_disp;
    float* out_disp;
    float* out_conf;
    uint16_t* out_u16;
    float* out_depth;
    double f, baseline, cx_offset;
    float min_depth, max_depth;
};

__global__ void k_post(PostArgs a) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= a.w || y >= a.h) return;
    const size_t i = static_cast<size_t>(y) * a.w + x;
    float d = __ldg(a.disp + i);
    if (a.median && valid_disparity(d)) {
        float v[9];
        int n = 0;
        for (int dy = -1; dy <= 1; ++dy)
            for (int dx = -1; dx <= 1; ++dx) {
                const int xx = x + dx, yy = y + dy;
                if (xx < 0 || yy < 0 || xx >= a.w || yy >= a.h) continue;
                const float q = __ldg(a.disp + static_cast<size_t>(yy) * a.w + xx);
                if (!valid_disparity(q)) continue;
                int p = n++;
                while (p > 0 && v[p - 1] > q) {
                    v[p] = v[p - 1];
                    --p;
                }
                v[p] = q;
            }
        d = v[n / 2];
    }
    const bool ok = valid_disparity(d);
    if (a.out_disp) a.out_disp[i] = d;
    if (a.out_conf) a.out_conf[i] = ok ? 1.0f : 0.0f;
    if (a.out_u16) {
        uint16_t u = 0xFFFFu;
        if (ok) {
            const float q = __fmul_rn(__fsub_rn(d, static_cast<float>(a.min_disp)), 64.0f);
            const int r = min(max(__float2int_rn(q), 0), 0xFFFE);
            u = static_cast<uint16_t>(r);
        }
        a.out_u16[i] = u;
    }
    if (a.out_depth) {
        float z = 0.0f;
        if (ok) {
            const double dd = __dadd_rn(static_cast<double>(d), a.cx_offset);
            if (dd > 0.0) {
                const double zz = __ddiv_rn(__dmul_rn(a.f, a.baseline), dd);
                if (!(zz < static_cast<double>(a.min_depth) || zz > static_cast<double>(a.max_depth)))
                    z = __double2float_rn(zz);
            }
        }
        a.out_depth[i] = z;
    }
}

// Debug: summed path values as u16 [y][x][nd] (the reference's `sum` volume).
struct SumArgs {
    const void* values;
    size_t dir_stride;
    int ndirs, w, h, nd, dp;
    uint16_t* out;
};

template <typename ST>
__global__ void k_debug_sums(SumArgs a) {
    const size_t n = static_cast<size_t>(a.w) * a.h * a.nd;
    const ST* v = static_cast<const ST*>(a.values);
    for (size_t i = blockIdx.x * static_cast<size_t>(blockDim.x) + threadIdx.x; i < n; i += static_cast<size_t>(gridDim.x) * blockDim.x) {
        const size_t px = i / a.nd;
        const int k = static_cast<int>(i % a.nd);
        uint32_t s = 0;
        for (int d = 0; d < a.ndirs; ++d) s += v[static_cast<size_t>(d) * a.dir_stride + px * a.dp + k];
        a.out[i] = static_cast<uint16_t>(s);
    }
}

}  // namespace dsk
