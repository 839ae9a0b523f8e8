// SGM disparity without any device allocation (ds_sgm_disparity_noalloc in include/depth_cuda.h).
//
// Some callers cannot allocate device memory at the time they need a disparity map: a process that
// reserves a fixed device-memory budget at start-up and forbids allocations afterwards, a real-time loop
// where cudaMalloc/cudaFree may block on the device or fail under memory pressure, or a host framework
// whose own allocator owns all device memory. For them this entry point computes the same result as the
// SGM core of ds_compute_device (census, path aggregation, WTA and left/right check; no median, no depth)
// on buffers the caller passes in, with every intermediate (census words, path values) in one
// statically allocated device array. The array exists on every GPU that loads the library, for the
// life of the process.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "../../include/depth_cuda.h"
#include "dispatch.h"
#include "frame_kernels.cuh"

namespace {

constexpr size_t kScratchBytes = size_t{16} << 20;  // 16 MiB, the limit of one call's intermediates
constexpr int kMaxDevices = 64;

// The device scratch. Host code must not use this name as an address (it is a host-side stand-in);
// its device address comes from cudaGetSymbolAddress, once per device.
static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

std::mutex g_mutex;
void* g_scratch_addr[kMaxDevices] = {};

size_t align256(size_t v) { return (v + 255) / 256 * 256; }

}  // namespace

extern "C" DS_API int ds_sgm_disparity_noalloc(const uint8_t* left, const uint8_t* right, int width, int height,
                                               const ds_sgm_params* sgm, int subpixel, float* disparity, void* stream) {
    if (!left || !right || !disparity || !sgm) {
        ds::set_global_error("null argument");
        return DS_INVALID_ARGUMENT;
    }
    const ds_sgm_params& p = *sgm;
    if (width < 1 || height < 1 || width > 16384 || height > 16384) {
        ds::set_global_error("image size must be 1..16384 in each dimension");
        return DS_INVALID_ARGUMENT;
    }
    if (p.num_disparities < 1 || p.num_disparities > 512 || p.census_radius_x < 0 || p.census_radius_y < 0 ||
        p.census_radius_x * 2 + 1 > 9 || p.census_radius_y * 2 + 1 > 7 || p.p1 < 0 || p.p2 < 0) {
        ds::set_global_error("invalid SGM parameters (1..512 disparities, census window <= 9x7, penalties >= 0)");
        return DS_INVALID_ARGUMENT;
    }
    const int window = (2 * p.census_radius_x + 1) * (2 * p.census_radius_y + 1);
    if (window + p.p2 > 0xFFFF - 2 * p.p1) {
        ds::set_global_error("census window + P2 exceed the 16-bit SGM costs");
        return DS_INVALID_ARGUMENT;
    }
    // Kernel configuration: as the library's default for this D, with costs recomputed from the census
    // (no cost volume) so that the intermediates stay small.
    ds::KernelCfg cfg;
    const int nd = p.num_disparities;
    if (nd <= 32) cfg.R = 1, cfg.seg = 16;
    else if (nd <= 64) cfg.R = 2, cfg.seg = 16;
    else if (nd <= 96) cfg.R = 3, cfg.seg = 16;
    else if (nd <= 128) cfg.R = 4, cfg.seg = 16;
    else if (nd <= 192) cfg.R = 3, cfg.seg = 32;
    else if (nd <= 256) cfg.R = 4, cfg.seg = 32;
    else if (nd <= 384) cfg.R = 6, cfg.seg = 32;
    else cfg.R = 8, cfg.seg = 32;
    cfg.materialize = false;
    cfg.fused = false;
    cfg.prefetch = 4;
    const bool c64 = window - 1 > 32;
    const bool wide = window + p.p2 > 255;
    const int ndirs = p.eight_paths ? 8 : 4;
    const size_t n = static_cast<size_t>(width) * height;
    const size_t dp = static_cast<size_t>(cfg.dp());
    const size_t census_bytes = align256(n * (c64 ? 8 : 4));
    const size_t values_bytes = align256(n * dp * ndirs * (wide ? 2 : 1));
    const size_t need = 2 * census_bytes + values_bytes;
    if (need > kScratchBytes) {
        const std::string m = "the no-allocation entry point needs " + std::to_string(need) + " bytes of scratch for " +
                              std::to_string(width) + "x" + std::to_string(height) + " with " + std::to_string(nd) +
                              " disparities; its static scratch holds " + std::to_string(kScratchBytes) + " bytes";
        ds::set_global_error(m.c_str());
        return DS_INVALID_ARGUMENT;
    }

    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
        ds::set_global_error("no usable CUDA device");
        return DS_IO;
    }
    unsigned char* scratch = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_mutex);
        if (!g_scratch_addr[dev]) {  // first call on this device (with it current): its scratch address
            void* a = nullptr;
            const cudaError_t e = cudaGetSymbolAddress(&a, g_scratch);
            if (e != cudaSuccess || !a) {
                ds::set_global_error((std::string("cudaGetSymbolAddress of the no-allocation scratch failed: ") +
                                      cudaGetErrorString(e)).c_str());
                return DS_IO;
            }
            g_scratch_addr[dev] = a;
        }
        scratch = static_cast<unsigned char*>(g_scratch_addr[dev]);
    }
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    void* census[2] = {scratch, scratch + census_bytes};
    void* values = scratch + 2 * census_bytes;

    // Every scratch byte a kernel reads was written earlier in the same call, so nothing is cleared.
    dsk::CensusArgs c{};
    c.img[0] = left;
    c.img[1] = right;
    c.out[0] = census[0];
    c.out[1] = census[1];
    c.w = width;
    c.h = height;
    c.rx = p.census_radius_x;
    c.ry = p.census_radius_y;
    c.pitch = width;
    const dim3 b(32, 8), g((width + 31) / 32, (height + 7) / 8, 2);
    if (c64) dsk::k_census<uint64_t><<<g, b, 0, st>>>(c);
    else dsk::k_census<uint32_t><<<g, b, 0, st>>>(c);
    cudaError_t e = cudaGetLastError();

    dsk::PathArgs pa{};
    pa.census_l = census[0];
    pa.census_r = census[1];
    pa.cpitch = width;
    pa.guide = left;
    pa.costs = nullptr;
    pa.values = values;
    pa.dir_stride = n * dp;
    pa.w = width;
    pa.h = height;
    pa.nd = nd;
    pa.dp = static_cast<int>(dp);
    pa.min_disp = p.min_disparity;
    pa.p1 = p.p1;
    pa.invalid_cost = window;
    pa.slant = p.slant_steps ? 1 : 0;
    pa.dir_base = 0;
    for (int q = 0; q < 32; ++q) pa.p2_table[q] = p.adaptive_p2 ? std::max(p.p1 + 1, p.p2 / (q + 1)) : p.p2;
    if (e == cudaSuccess) {
        const int max_lines = ndirs == 8 ? width + height - 1 : std::max(width, height);
        e = ds::launch_paths(cfg, c64, wide, pa, ndirs, max_lines, st);
    }
    dsk::WtaArgs wa{};
    wa.values = values;
    wa.dir_stride = n * dp;
    wa.ndirs = ndirs;
    wa.w = width;
    wa.h = height;
    wa.nd = nd;
    wa.dp = static_cast<int>(dp);
    wa.min_disp = p.min_disparity;
    wa.uniqueness = p.uniqueness;
    wa.subpixel = subpixel ? 1 : 0;
    wa.lr_max_diff = p.lr_max_diff;
    wa.disp = disparity;
    if (e == cudaSuccess) e = ds::launch_wta(cfg, wide, wa, height, static_cast<size_t>(width) * 8, st);
    if (e != cudaSuccess) {
        ds::set_global_error((std::string("CUDA stereo failed: ") + cudaGetErrorString(e)).c_str());
        return DS_IO;
    }
    ds::count_launches(3);
    return DS_OK;
}
