// Organised points, normals and weights from a disparity map (depth::disparity_to_points,
// libs/depth/src/point_image.cpp:10-54), and the recording layout of a depth frame
// (depth_metal::DepthPacker, libs/depth_metal/src/depth_packer.cpp:10-21), on device buffers.
//
// Float and double operations are written with explicitly rounded intrinsics in the order the reference
// evaluates them (Eigen's 3-vector dot products as (x x' + y y') + z z', cross products component by
// component), so that nvcc contracts nothing into a fused multiply-add and the results are the
// reference's bit for bit.
#include <cuda_runtime.h>

#include "../../include/depth_cuda.h"
#include "dispatch.h"

namespace {

struct PointsArgs {
    const float* disp;
    const float* conf;  // may be null: weight 1
    int w, h;
    double f, cx, cy, baseline, cx_offset;
    float min_depth, max_depth, max_jump, edge_weight, weight_reference_depth;
    float4* points;
    float4* normals;
    float* weights;
};

__device__ __forceinline__ float dot3(float ax, float ay, float az, float bx, float by, float bz) {
    return __fadd_rn(__fadd_rn(__fmul_rn(ax, bx), __fmul_rn(ay, by)), __fmul_rn(az, bz));
}

// point_image.cpp:15-25
__global__ void k_points(PointsArgs a) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= a.w || y >= a.h) return;
    const size_t i = static_cast<size_t>(y) * a.w + x;
    float4 p = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    float wt = 0.0f;
    const float d = __ldg(a.disp + i);
    const double dd = __dadd_rn(static_cast<double>(d), a.cx_offset);
    if (d > -1.0e8f && dd > 0.0) {
        const double z = __ddiv_rn(__dmul_rn(a.f, a.baseline), dd);
        if (!(z < static_cast<double>(a.min_depth) || z > static_cast<double>(a.max_depth))) {
            p.x = __double2float_rn(__ddiv_rn(__dmul_rn(__dsub_rn(static_cast<double>(x), a.cx), z), a.f));
            p.y = __double2float_rn(__ddiv_rn(__dmul_rn(__dsub_rn(static_cast<double>(y), a.cy), z), a.f));
            p.z = __double2float_rn(z);
            p.w = 1.0f;
            wt = a.conf ? __ldg(a.conf + i) : 1.0f;
        }
    }
    a.points[i] = p;
    a.weights[i] = wt;
}

// point_image.cpp:27-51: normals from central differences where the four neighbours exist and the
// depth jumps stay within max_jump; the view term is the worse of the two cameras' incidence.
__global__ void k_normals(PointsArgs a) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= a.w || y >= a.h) return;
    const size_t i = static_cast<size_t>(y) * a.w + x;
    const float4 p = a.points[i];
    float4 n = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    if (p.z != 0.0f) {
        float view = a.edge_weight;
        if (x > 0 && y > 0 && x + 1 < a.w && y + 1 < a.h) {
            const float4 l = a.points[i - 1], r = a.points[i + 1];
            const float4 u = a.points[i - a.w], dn = a.points[i + a.w];
            if (l.z != 0.0f && r.z != 0.0f && u.z != 0.0f && dn.z != 0.0f && fabsf(__fsub_rn(l.z, r.z)) <= a.max_jump &&
                fabsf(__fsub_rn(u.z, dn.z)) <= a.max_jump) {
                const float ax = __fsub_rn(r.x, l.x), ay = __fsub_rn(r.y, l.y), az = __fsub_rn(r.z, l.z);
                const float bx = __fsub_rn(dn.x, u.x), by = __fsub_rn(dn.y, u.y), bz = __fsub_rn(dn.z, u.z);
                float nx = __fsub_rn(__fmul_rn(ay, bz), __fmul_rn(az, by));
                float ny = __fsub_rn(__fmul_rn(az, bx), __fmul_rn(ax, bz));
                float nz = __fsub_rn(__fmul_rn(ax, by), __fmul_rn(ay, bx));
                const float len = __fsqrt_rn(dot3(nx, ny, nz, nx, ny, nz));
                if (len >= 1e-9f) {
                    nx = __fdiv_rn(nx, len), ny = __fdiv_rn(ny, len), nz = __fdiv_rn(nz, len);
                    if (dot3(nx, ny, nz, p.x, p.y, p.z) > 0.0f) nx = -nx, ny = -ny, nz = -nz;
                    n = make_float4(nx, ny, nz, 0.0f);
                    const float pl = __fsqrt_rn(dot3(p.x, p.y, p.z, p.x, p.y, p.z));
                    const float qx = __fsub_rn(p.x, static_cast<float>(a.baseline)), qy = __fsub_rn(p.y, 0.0f),
                                qz = __fsub_rn(p.z, 0.0f);
                    const float ql = __fsqrt_rn(dot3(qx, qy, qz, qx, qy, qz));
                    const float v1 = -dot3(nx, ny, nz, __fdiv_rn(p.x, pl), __fdiv_rn(p.y, pl), __fdiv_rn(p.z, pl));
                    const float v2 = -dot3(nx, ny, nz, __fdiv_rn(qx, ql), __fdiv_rn(qy, ql), __fdiv_rn(qz, ql));
                    const float m = v1 < v2 ? v1 : v2;
                    view = 0.0f > m ? 0.0f : m;
                }
            }
        }
        float dw = 1.0f;  // depth_noise_weight (point_image.hpp:56-60)
        if (a.weight_reference_depth > 0.0f) {
            const float rr = __fdiv_rn(a.weight_reference_depth, p.z);
            const float r2 = __fmul_rn(rr, rr);
            dw = r2 > 1.0f ? 1.0f : (r2 < 0.1f ? 0.1f : r2);
        }
        a.weights[i] = __fmul_rn(a.weights[i], __fmul_rn(view, dw));
    }
    a.normals[i] = n;
}

__device__ __forceinline__ uint32_t quantize_mm50(float z) {
    if (!(z > 0.0f)) return 0u;
    const float q = fminf(fmaxf(roundf(__fmul_rn(z, 50.0f)), 1.0f), 65535.0f);
    return static_cast<uint32_t>(q);
}

// depth_packer.cpp:10-21: u16 depth (1/50 mm) minus its left neighbour's, then u8 confidence.
__global__ void k_pack_depth(const float4* __restrict__ pts, const float* __restrict__ wts, int w, int h,
                             uint8_t* __restrict__ out) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y;
    if (x >= w || y >= h) return;
    const size_t i = static_cast<size_t>(y) * w + x, n = static_cast<size_t>(w) * h;
    const uint32_t q = quantize_mm50(pts[i].z);
    const uint32_t left = x > 0 ? quantize_mm50(pts[i - 1].z) : 0u;
    reinterpret_cast<uint16_t*>(out)[i] = static_cast<uint16_t>((q - left) & 0xFFFFu);
    out[2 * n + i] = static_cast<uint8_t>(fminf(fmaxf(roundf(__fmul_rn(wts[i], 255.0f)), 0.0f), 255.0f));
}

bool aligned(const void* p, size_t a) { return (reinterpret_cast<uintptr_t>(p) & (a - 1)) == 0; }

}  // namespace

extern "C" {

DS_API void ds_default_point_params(ds_point_params* p) {
    if (!p) return;
    p->min_depth_mm = 150.0f;  // depth::PointImageParams defaults (point_image.hpp:41-47)
    p->max_depth_mm = 700.0f;
    p->max_depth_jump_mm = 4.0f;
    p->edge_weight = 0.25f;
    p->weight_reference_depth_mm = 0.0f;
}

DS_API int ds_disparity_to_points(const float* disparity, const float* confidence, int width, int height,
                                  const ds_geometry* geometry, const ds_point_params* params, float* points_xyzw,
                                  float* normals_xyzw, float* weights, void* stream) {
    if (!disparity || !geometry || !params || !points_xyzw || !normals_xyzw || !weights) {
        ds::set_global_error("null argument");
        return DS_INVALID_ARGUMENT;
    }
    if (width < 1 || height < 1 || width > 16384 || height > 16384) {
        ds::set_global_error("image size must be 1..16384 in each dimension");
        return DS_INVALID_ARGUMENT;
    }
    if (!aligned(points_xyzw, 16) || !aligned(normals_xyzw, 16)) {
        ds::set_global_error("points and normals must be 16-byte aligned (float4 per pixel)");
        return DS_INVALID_ARGUMENT;
    }
    PointsArgs a{};
    a.disp = disparity;
    a.conf = confidence;
    a.w = width;
    a.h = height;
    a.f = geometry->f;
    a.cx = geometry->cx;
    a.cy = geometry->cy;
    a.baseline = geometry->baseline;
    a.cx_offset = geometry->cx_offset;
    a.min_depth = params->min_depth_mm;
    a.max_depth = params->max_depth_mm;
    a.max_jump = params->max_depth_jump_mm;
    a.edge_weight = params->edge_weight;
    a.weight_reference_depth = params->weight_reference_depth_mm;
    a.points = reinterpret_cast<float4*>(points_xyzw);
    a.normals = reinterpret_cast<float4*>(normals_xyzw);
    a.weights = weights;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    const dim3 b(32, 8), g((width + 31) / 32, (height + 7) / 8);
    k_points<<<g, b, 0, st>>>(a);
    k_normals<<<g, b, 0, st>>>(a);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        ds::set_global_error(cudaGetErrorString(e));
        return DS_IO;
    }
    ds::count_launches(2);
    return DS_OK;
}

DS_API int ds_pack_depth(const float* points_xyzw, const float* weights, int width, int height, uint8_t* packed,
                         void* stream) {
    if (!points_xyzw || !weights || !packed) {
        ds::set_global_error("null argument");
        return DS_INVALID_ARGUMENT;
    }
    if (width < 1 || height < 1 || width > 16384 || height > 16384) {
        ds::set_global_error("image size must be 1..16384 in each dimension");
        return DS_INVALID_ARGUMENT;
    }
    if (!aligned(points_xyzw, 16) || !aligned(packed, 2)) {
        ds::set_global_error("points must be 16-byte aligned and the packed buffer 2-byte aligned");
        return DS_INVALID_ARGUMENT;
    }
    const dim3 b(32, 8), g((width + 31) / 32, (height + 7) / 8);
    k_pack_depth<<<g, b, 0, static_cast<cudaStream_t>(stream)>>>(reinterpret_cast<const float4*>(points_xyzw), weights, width,
                                                                 height, packed);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        ds::set_global_error(cudaGetErrorString(e));
        return DS_IO;
    }
    ds::count_launches(1);
    return DS_OK;
}

}  // extern "C"
