// Per-frame kernels around the SGM core (sm_100a): rectification remap, census, median + outputs.
// The non-template kernels have internal linkage, so that several translation units may include this.
#pragma once

#include "stereo_kernels.cuh"

namespace dsk {

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

// Four horizontally adjacent output pixels per thread (a block covers 128 x 8): the map entries come as
// one 128-bit load per table and the four bytes leave as one 32-bit store when rows are 4-aligned.
constexpr int kRectifyPixelsPerThread = 4;

__device__ __forceinline__ void rectify_body(const RectifyArgs& a, int bx, int by, int bz) {
    const int x4 = (bx * blockDim.x + threadIdx.x) * kRectifyPixelsPerThread;
    const int y = by * blockDim.y + threadIdx.y;
    const int side = bz;
    if (x4 >= a.out_w || y >= a.out_h) return;
    // (selected, not indexed: a run-time index into the argument's arrays would copy them to local memory)
    const uint8_t* src = side ? a.raw[1] : a.raw[0];
    const float* mx = side ? a.map_x[1] : a.map_x[0];
    const float* my = side ? a.map_y[1] : a.map_y[0];
    const bool full = x4 + 4 <= a.out_w;
    uint32_t v[4] = {0u, 0u, 0u, 0u};
    if (!a.half) {
        const size_t i = static_cast<size_t>(y) * a.map_w + x4;
        if (full && (a.map_w & 3) == 0) {
            const float4 fx = __ldg(reinterpret_cast<const float4*>(mx + i));
            const float4 fy = __ldg(reinterpret_cast<const float4*>(my + i));
            v[0] = remap_sample(src, a.raw_w, a.raw_h, fx.x, fy.x);
            v[1] = remap_sample(src, a.raw_w, a.raw_h, fx.y, fy.y);
            v[2] = remap_sample(src, a.raw_w, a.raw_h, fx.z, fy.z);
            v[3] = remap_sample(src, a.raw_w, a.raw_h, fx.w, fy.w);
        } else {
            for (int j = 0; j < 4 && x4 + j < a.out_w; ++j)
                v[j] = remap_sample(src, a.raw_w, a.raw_h, __ldg(mx + i + j), __ldg(my + i + j));
        }
    } else {
        for (int j = 0; j < 4 && x4 + j < a.out_w; ++j) {
            const int x = x4 + j;
            uint32_t acc = 0;
            for (int jj = 0; jj < 2; ++jj)
                for (int ii = 0; ii < 2; ++ii) {
                    const size_t m = static_cast<size_t>(2 * y + jj) * a.map_w + (2 * x + ii);
                    acc += remap_sample(src, a.raw_w, a.raw_h, __ldg(mx + m), __ldg(my + m));
                }
            v[j] = (acc + 2u) / 4u;
        }
    }
    uint8_t* out = (side ? a.out[1] : a.out[0]) + static_cast<size_t>(y) * a.out_w + x4;
    if (full && (a.out_w & 3) == 0) {
        *reinterpret_cast<uint32_t*>(out) = v[0] | (v[1] << 8) | (v[2] << 16) | (v[3] << 24);
    } else {
        for (int j = 0; j < 4 && x4 + j < a.out_w; ++j) out[j] = static_cast<uint8_t>(v[j]);
    }
}

static __global__ void k_rectify(RectifyArgs a) { rectify_body(a, blockIdx.x, blockIdx.y, blockIdx.z); }

// ------------------------------------------------------------------------------------------------
// Census (stereo.cpp:328-346): bit per window neighbour, row-major, centre skipped, MSB first,
// set when neighbour < centre; 0 within (rx, ry) of the border.

struct CensusArgs {
    const uint8_t* img[2];
    void* out[2];  // (y, x) at y * pitch + x
    int w, h, rx, ry, pitch;
    uint8_t* left_copy;  // optional: the left image is also copied here (the sweep kernels' guide in batches)
};

// One 32 x 8 block of pixels per (bx, by): the block's image tile with its window halo is staged in
// shared memory, then each thread builds its pixel's word from the tile. Every thread of the block
// takes part in the staging (the persistent batch kernel calls this once per virtual block).
constexpr int kCensusMaxRx = 4, kCensusMaxRy = 3;  // windows up to 9 x 7 (64-bit words)

template <typename W>
__device__ __forceinline__ void census_body(const CensusArgs& a, int bx, int by, int bz) {
    __shared__ uint8_t tile[8 + 2 * kCensusMaxRy][32 + 2 * kCensusMaxRx];
    const int x0 = bx * 32, y0 = by * 8;
    const uint8_t* img = bz ? a.img[1] : a.img[0];  // selected, not indexed (see rectify_body)
    const int tw = 32 + 2 * a.rx, th = 8 + 2 * a.ry;
    __syncthreads();  // the previous virtual block's readers are done
    for (int ty = threadIdx.y; ty < th; ty += 8) {  // block (32, 8)
        const int gy = y0 - a.ry + ty;
        const bool row_in = gy >= 0 && gy < a.h;
        for (int tx = threadIdx.x; tx < tw; tx += 32) {
            const int gx = x0 - a.rx + tx;
            tile[ty][tx] = (row_in && gx >= 0 && gx < a.w) ? __ldg(img + static_cast<size_t>(gy) * a.w + gx) : 0;
        }
    }
    __syncthreads();
    const int x = x0 + threadIdx.x, y = y0 + threadIdx.y;
    if (x >= a.w || y >= a.h) return;
    if (bz == 0 && a.left_copy) a.left_copy[static_cast<size_t>(y) * a.w + x] = tile[threadIdx.y + a.ry][threadIdx.x + a.rx];
    W word = 0;
    if (y >= a.ry && y < a.h - a.ry && x >= a.rx && x < a.w - a.rx) {
        const int cx = threadIdx.x + a.rx, cy = threadIdx.y + a.ry;
        const uint8_t c = tile[cy][cx];
        if (a.rx == 2 && a.ry == 2) {  // the reference's default 5 x 5 window, unrolled
#pragma unroll
            for (int v = -2; v <= 2; ++v)
#pragma unroll
                for (int u = -2; u <= 2; ++u)
                    if (u != 0 || v != 0) word = static_cast<W>((word << 1) | static_cast<W>(tile[cy + v][cx + u] < c));
        } else {
            for (int v = -a.ry; v <= a.ry; ++v)
                for (int u = -a.rx; u <= a.rx; ++u) {
                    if (u == 0 && v == 0) continue;
                    word = static_cast<W>((word << 1) | static_cast<W>(tile[cy + v][cx + u] < c));
                }
        }
    }
    static_cast<W*>(bz ? a.out[1] : a.out[0])[static_cast<size_t>(y) * a.pitch + x] = word;
}

template <typename W>
__global__ void k_census(CensusArgs a) {
    census_body<W>(a, blockIdx.x, blockIdx.y, blockIdx.z);
}

// ------------------------------------------------------------------------------------------------
// 3x3 median (stereo.cpp:129-147) + outputs: f32 disparity, confidence (stereo.cpp:515-519), u16
// disparity, depth z = f B / (d + cx_offset) in double with the gates of point_image.cpp:18-20.

struct PostArgs {
    const float* disp;
    const float* conf_in;  // confidence of valid pixels (refinement: the ZNCC score); null: 1
    int w, h, median, min_disp;
    float* out_disp;
    float* out_conf;
    uint16_t* out_u16;
    float* out_depth;
    double f, baseline, cx_offset;
    float min_depth, max_depth;
};

__device__ __forceinline__ void post_body(const PostArgs& a, int bx, int by) {
    const int x = bx * blockDim.x + threadIdx.x;
    const int y = by * blockDim.y + threadIdx.y;
    if (x >= a.w || y >= a.h) return;
    const size_t i = static_cast<size_t>(y) * a.w + x;
    float d = __ldg(a.disp + i);
    if (a.median && valid_disparity(d)) {
        float v[9];
#pragma unroll
        for (int dy = -1; dy <= 1; ++dy)
#pragma unroll
            for (int dx = -1; dx <= 1; ++dx) {
                const int xx = x + dx, yy = y + dy;
                const bool in = xx >= 0 && yy >= 0 && xx < a.w && yy < a.h;
                v[(dy + 1) * 3 + dx + 1] = in ? __ldg(a.disp + static_cast<size_t>(yy) * a.w + xx) : kInvalid;
            }
        int n;
        d = median_of_valid9(v, n);
    }
    const bool ok = valid_disparity(d);
    if (a.out_disp) a.out_disp[i] = d;
    if (a.out_conf) a.out_conf[i] = ok ? (a.conf_in ? a.conf_in[i] : 1.0f) : 0.0f;
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

static __global__ void k_post(PostArgs a) { post_body(a, blockIdx.x, blockIdx.y); }

// Debug: summed path values as u16 [y][x][nd] (the reference's `sum` volume).
struct SumArgs {
    const void* values;
    size_t dir_stride;
    int ndirs, w, h, nd, dp;
    uint16_t* out;
};

template <typename ST>
static __global__ void k_debug_sums(SumArgs a) {
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
