// C-ABI of the per-frame stereo hot path (include/depth_cuda.h): handle life cycle, validation with
// the reference's error codes, resident rectification tables, host and device entry points.
#include <cuda_runtime.h>

#include <atomic>
#include <algorithm>
#include <chrono>
#include <functional>
#include <type_traits>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/depth_cuda.h"
#include "batch_common.cuh"
#include "dispatch.h"
#include "frame_kernels.cuh"
#include "sweep_kernels.cuh"
#include "wta_kernels.cuh"
#include "internal.h"
#include "refine_kernels.cuh"
#include "blob_kernels.cuh"

namespace {

thread_local std::string g_error;
std::atomic<uint64_t> g_launches{0};

constexpr int kProfileRing = 4096;  // frames whose stage events can be pending at once

struct CudaFailure {
    cudaError_t err;
    const char* what;
};

#define DS_CUDA(call)                                           \
    do {                                                        \
        const cudaError_t e_ = (call);                          \
        if (e_ != cudaSuccess) throw CudaFailure{e_, #call};    \
    } while (0)

double now_ms() {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// Default kernel configuration for D disparities: the fewest padded lanes, two scanlines per warp
// (SEG 16) while D <= 96. ds_set_kernel_config overrides it (the autotuner does).
ds::KernelCfg default_cfg(int nd) {
    ds::KernelCfg c;
    c.materialize = true;  // fastest measured on B200 for 1280x1024, D=128 (cost volume read by each direction)
    c.prefetch = 8;
    if (nd <= 32) c.R = 1, c.seg = 16;
    else if (nd <= 64) c.R = 2, c.seg = 16;
    else if (nd <= 96) c.R = 3, c.seg = 16;
    else if (nd <= 128) c.R = 4, c.seg = 16;
    else if (nd <= 192) c.R = 3, c.seg = 32;
    else if (nd <= 256) c.R = 4, c.seg = 32;
    else if (nd <= 384) c.R = 6, c.seg = 32;
    else c.R = 8, c.seg = 32;
    return c;
}

}  // namespace

struct ds_handle {
    ds_stereo_params p{};
    int w = 0, h = 0;
    int nd = 0, dp = 0, ndirs = 4;
    ds::KernelCfg cfg{};
    bool wide = false;      // u16 path values
    bool census64 = false;  // u64 census words
    bool s16 = false;       // vertical pair sums need 16 bits (2 (window + P2) > 255 or wide): no sweep kernels
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;

    uint8_t* d_rect[2] = {nullptr, nullptr};   // inside rect_raw, after kGuardRows guard rows
    uint8_t* rect_raw[2] = {nullptr, nullptr};
    uint8_t* d_raw[2] = {nullptr, nullptr};
    float* d_map[4] = {nullptr, nullptr, nullptr, nullptr};  // lx, ly, rx, ry
    int map_w = 0, map_h = 0, raw_w = 0, raw_h = 0;
    bool have_rect = false;
    bool maps_external = false;  // d_map bound by an owner (the request server's resident calibrations)
    void* d_census[2] = {nullptr, nullptr};    // padded census: (y, x) at y * cpitch + x, inside census_raw
    void* census_raw[2] = {nullptr, nullptr};
    int cpitch = 0, cguard = 0;
    size_t census_bytes = 0;                   // per image, guards included (capacity)
    // Sweep kernels (cfg.fused), all inside d_values: vertical pair sums S, horizontal first-half values T and
    // the column kernel's costs C (u8 slabs with guard rows), the row kernel's per-pixel WTA records and its
    // right-WTA keys.
    void* d_S = nullptr;
    void* d_T = nullptr;
    void* d_C = nullptr;
    uint2* d_rec = nullptr;
    uint16_t* d_rk = nullptr;
    void* d_values = nullptr;
    size_t dir_stride = 0;
    size_t values_bytes = 0;
    uint8_t* d_costs = nullptr;  // materialised costs (cfg.materialize)
    size_t costs_bytes = 0;
    // Volumes (d_values, d_costs) owned by a batch that shares them between pairs run one after another;
    // the handle only sizes them.
    bool external_volumes = false;
    // Frames of this handle may change min_disparity (set_frame_params): census buffers sized for any.
    bool any_min_disparity = false;
    float* d_disp_lr = nullptr;
    float* d_out_disp = nullptr;
    float* d_out_conf = nullptr;
    uint16_t* d_out_u16 = nullptr;
    float* d_out_depth = nullptr;

    // depth::compute_disparity beyond the hot path (pyramid, refinements, filters, speckles): SGM at the
    // pyramid's coarsest level runs in `sgm`, a hot-path handle of that size; this handle keeps the
    // rectified pair, the pyramid, the refinement buffers and the outputs.
    bool refine = false;
    ds_handle* sgm = nullptr;
    std::vector<int> lw, lh;                 // level sizes, 0 = the stereo resolution
    std::vector<uint8_t*> pyr[2];            // levels 1..pyramid_levels (entry 0 unused)
    float* d_ra = nullptr;                   // disparity ping-pong and confidence, W*H
    float* d_rb = nullptr;
    float* d_rconf = nullptr;
    float* d_rmed = nullptr;                 // median3 of the coarser level
    uint8_t* d_full[2] = {nullptr, nullptr}; // full-resolution rectified pair (detail refinement)
    int* d_parent = nullptr;                 // speckle union-find
    int* d_size = nullptr;
    int* d_err = nullptr;

    // Marker blob search (ds_set_blob_params), one set of buffers per side, sized for blob_px pixels.
    bool have_blobs = false;
    ds_blob_params blob_p{};
    size_t blob_px = 0;
    struct BlobBufs {
        int* parent = nullptr;
        uint32_t* count = nullptr;
        uint32_t* box = nullptr;
        int* mom = nullptr;
        dsk::BlobCand* out = nullptr;
        uint32_t* n_out = nullptr;  // [0] candidates found, [1] error flag
        uint8_t* img = nullptr;     // a host image's upload (ds_find_blobs)
    } blob[2];
    uint32_t blob_cap = 0;
    cudaStream_t blob_stream = nullptr;
    cudaEvent_t blob_ev = nullptr;

    ds_geometry geom{};
    float min_depth = 150.0f, max_depth = 700.0f, max_jump = 4.0f;
    bool have_points = false;

    ds_timings timings{};
    std::string err;
    size_t bytes = 0;

    // Stage profiling: a ring of (DS_STAGES + 1) events per frame.
    bool profile = false;
    std::vector<cudaEvent_t> prof_events;
    int prof_head = 0, prof_pending = 0;

    int fail(int code, std::string msg) {
        err = std::move(msg);
        return code;
    }
    template <typename T>
    T* alloc(size_t n) {
        void* p = nullptr;
        DS_CUDA(cudaMalloc(&p, n * sizeof(T)));
        bytes += n * sizeof(T);
        return static_cast<T*>(p);
    }
};

namespace {

void release(ds_handle* h) {
    if (!h) return;
    auto f = [](void* p) {
        if (p) cudaFree(p);
    };
    for (auto* p : h->rect_raw) f(p);
    for (auto* p : h->d_raw) f(p);
    if (!h->maps_external)
        for (auto* p : h->d_map) f(p);
    for (auto* p : h->census_raw) f(p);
    if (!h->external_volumes) {
        f(h->d_values);
        f(h->d_costs);
    }
    f(h->d_disp_lr);
    for (int s = 0; s < 2; ++s) {
        for (auto* p : h->pyr[s]) f(p);
        f(h->d_full[s]);
    }
    f(h->d_ra);
    f(h->d_rb);
    f(h->d_rconf);
    f(h->d_rmed);
    f(h->d_parent);
    f(h->d_size);
    f(h->d_err);
    for (auto& b : h->blob) {
        f(b.parent);
        f(b.count);
        f(b.box);
        f(b.mom);
        f(b.out);
        f(b.n_out);
        f(b.img);
    }
    if (h->blob_ev) cudaEventDestroy(h->blob_ev);
    if (h->blob_stream) cudaStreamDestroy(h->blob_stream);
    if (h->sgm) {
        release(h->sgm);
        delete h->sgm;
    }
    f(h->d_out_disp);
    f(h->d_out_conf);
    f(h->d_out_u16);
    f(h->d_out_depth);
    for (auto e : h->prof_events) cudaEventDestroy(e);
    if (h->ev0) cudaEventDestroy(h->ev0);
    if (h->ev1) cudaEventDestroy(h->ev1);
    if (h->stream) cudaStreamDestroy(h->stream);
}

// Validation of metal_stereo.cpp:115-120, plus the limits of this implementation.
int validate(const ds_stereo_params& p, int w, int h, std::string& msg) {
    const auto& s = p.sgm;
    if (w < 1 || h < 1 || w > 16384 || h > 16384) {
        msg = "image size must be 1..16384 in each dimension";
        return DS_INVALID_ARGUMENT;
    }
    if (s.num_disparities < 1 || s.num_disparities > dsk::kMaxDisparities) {
        msg = "CUDA SGM supports 1..512 disparities";
        return DS_INVALID_ARGUMENT;
    }
    if (s.census_radius_x < 0 || s.census_radius_y < 0 || s.census_radius_x * 2 + 1 > 9 || s.census_radius_y * 2 + 1 > 7) {
        msg = "census window too large for 64 bits";
        return DS_INVALID_ARGUMENT;
    }
    if (s.p1 < 0 || s.p2 < 0) {
        msg = "SGM penalties must be non-negative";
        return DS_INVALID_ARGUMENT;
    }
    const int window = (2 * s.census_radius_x + 1) * (2 * s.census_radius_y + 1);
    if (window + s.p2 > 0xFFFF - 2 * s.p1) {
        msg = "census window + P2 exceed the 16-bit SGM costs";
        return DS_INVALID_ARGUMENT;
    }
    if (p.pyramid_levels < 0 || p.pyramid_levels > 4 || (w >> p.pyramid_levels) < 1 || (h >> p.pyramid_levels) < 1) {
        msg = "pyramid_levels must be 0..4 with at least one pixel at the coarsest level";
        return DS_INVALID_ARGUMENT;
    }
    if (p.pyramid_levels > 0 &&
        (p.refine_zncc_radius < 1 || p.refine_zncc_radius > 15 || p.refine_search_radius < 1 || p.refine_search_radius > 31)) {
        msg = "refinement: zncc_radius 1..15, search_radius 1..31";
        return DS_INVALID_ARGUMENT;
    }
    if (p.detail_enabled && (p.detail_radius < 1 || p.detail_radius > 32 || !(p.detail_step > 0.0f) || !(p.detail_search >= 0.0f))) {
        msg = "detail refinement: radius 1..32, step > 0, search >= 0";
        return DS_INVALID_ARGUMENT;
    }
    if (p.speckle_max_region_size < 0 || !(p.speckle_max_diff >= 0.0f)) {
        msg = "speckle removal: max_region_size and max_diff must be non-negative";
        return DS_INVALID_ARGUMENT;
    }
    return DS_OK;
}

// Whether a frame runs depth::compute_disparity's later stages (not only the hot path).
bool refines(const ds_stereo_params& p) {
    return p.pyramid_levels > 0 || p.detail_enabled || p.filter_occlusion || p.filter_spikes || p.speckle_max_region_size > 1;
}

dsk::SweepArgs sweep_args(const ds_handle* h) {
    const auto& sg = h->p.sgm;
    dsk::SweepArgs a{};
    a.census_l = static_cast<const uint32_t*>(h->d_census[0]);
    a.census_r = static_cast<const uint32_t*>(h->d_census[1]);
    a.cpitch = h->cpitch;
    a.guide = h->d_rect[0];
    a.S = static_cast<uint8_t*>(h->d_S);
    a.T = static_cast<uint8_t*>(h->d_T);
    a.C = static_cast<uint8_t*>(h->d_C);
    a.rec = h->d_rec;
    a.rk = h->d_rk;
    a.disp = h->d_disp_lr;
    a.w = h->w;
    a.h = h->h;
    a.nd = h->nd;
    a.dp = h->dp;
    a.min_disp = sg.min_disparity;
    a.p1 = sg.p1;
    a.invalid_cost = (2 * sg.census_radius_x + 1) * (2 * sg.census_radius_y + 1);
    a.uniqueness = sg.uniqueness;
    a.subpixel = h->p.subpixel ? 1 : 0;
    a.lr_max_diff = sg.lr_max_diff;
    for (int q = 0; q < 32; ++q) {
        const int p2 = sg.adaptive_p2 ? std::max(sg.p1 + 1, sg.p2 / (q + 1)) : sg.p2;
        a.p2_table2[q] = static_cast<uint32_t>(p2) * 0x00010001u;
    }
    return a;
}

bool sweep_slant(const ds_handle* h) { return h->p.sgm.slant_steps != 0; }
bool sweep_pad(const ds_handle* h) { return h->nd < h->dp; }

// Why the sweep kernels cannot run this handle's frames ("" when they can).
const char* sweep_unfit(const ds_handle* h, int R, int seg) {
    if (h->ndirs != 4) return "the sweep kernels need 4 paths";
    if (h->census64) return "the sweep kernels need census windows of at most 32 neighbours";
    if (h->s16) return "the sweep kernels need 2 (window + P2) <= 255 (byte pair sums)";
    if (!dsk::sweep_shape_ok(R, seg)) return "the sweep kernels need 6 or 8 registers per lane and 4 or 8 lanes per line";
    return "";
}

// The materialised cost volume (nothing when the path kernels recompute costs from the census).
void launch_costs(ds_handle* h, cudaStream_t st) {
    if (h->cfg.fused || !h->cfg.materialize) return;
    const auto& sg = h->p.sgm;
    const int window = (2 * sg.census_radius_x + 1) * (2 * sg.census_radius_y + 1);
    dsk::CostArgs c{h->d_census[0], h->d_census[1], h->d_costs, h->w, h->h, h->nd, h->dp, sg.min_disparity, window,
                    h->cpitch};
    const int tiles = (h->w + dsk::kCostTile - 1) / dsk::kCostTile;
    if (h->census64)
        dsk::k_cost_tiles<uint64_t><<<h->h * tiles, 256, dsk::cost_tile_smem<uint64_t>(h->dp), st>>>(c);
    else
        dsk::k_cost_tiles<uint32_t><<<h->h * tiles, 256, dsk::cost_tile_smem<uint32_t>(h->dp), st>>>(c);
    DS_CUDA(cudaGetLastError());
    ++g_launches;
}

void launch_paths(ds_handle* h, cudaStream_t st) {
    if (h->cfg.fused) {
        DS_CUDA(ds::launch_sweep_cols(h->cfg, sweep_slant(h), sweep_pad(h), sweep_args(h), st));
        ++g_launches;
        return;
    }
    const auto& sg = h->p.sgm;
    const int window = (2 * sg.census_radius_x + 1) * (2 * sg.census_radius_y + 1);
    dsk::PathArgs a{};
    a.census_l = h->d_census[0];
    a.census_r = h->d_census[1];
    a.cpitch = h->cpitch;
    a.guide = h->d_rect[0];
    a.costs = h->cfg.materialize ? h->d_costs : nullptr;
    a.values = h->d_values;
    a.dir_stride = h->dir_stride;
    a.w = h->w;
    a.h = h->h;
    a.nd = h->nd;
    a.dp = h->dp;
    a.min_disp = sg.min_disparity;
    a.p1 = sg.p1;
    a.invalid_cost = window;
    a.slant = sg.slant_steps ? 1 : 0;
    a.dir_base = 0;
    for (int q = 0; q < 32; ++q) a.p2_table[q] = sg.adaptive_p2 ? std::max(sg.p1 + 1, sg.p2 / (q + 1)) : sg.p2;
    const int max_lines = h->ndirs == 8 ? h->w + h->h - 1 : std::max(h->w, h->h);
    DS_CUDA(ds::launch_paths(h->cfg, h->census64, h->wide, a, h->ndirs, max_lines, st));
    ++g_launches;
}

// Whether the WTA of the per-direction path runs as row sweeps (wta_kernels.cuh): 4 paths with byte path
// values whose pairs fit a byte, and lane slabs of 48, 64, 96 or 128 disparities.
bool wta_rows_fit(const ds_handle* h) {
    int chunk = 0, lg = 0, sets = 0;
    return !h->cfg.fused && h->ndirs == 4 && !h->wide && !h->s16 && ds::wta_rows_layout(h->w, h->dp, chunk, lg, sets);
}

dsk::WtaRowArgs wta_row_args(const ds_handle* h) {
    dsk::WtaRowArgs a{};
    a.values = static_cast<const uint8_t*>(h->d_values);
    a.dir_stride = h->dir_stride;
    a.rec = h->d_rec;
    a.rk = h->d_rk;
    a.disp = h->d_disp_lr;
    a.w = h->w;
    a.h = h->h;
    a.nd = h->nd;
    a.dp = h->dp;
    a.min_disp = h->p.sgm.min_disparity;
    a.uniqueness = h->p.sgm.uniqueness;
    a.subpixel = h->p.subpixel ? 1 : 0;
    a.lr_max_diff = h->p.sgm.lr_max_diff;
    ds::wta_rows_layout(h->w, h->dp, a.chunk, a.lg_chunks, a.sets);
    return a;
}

void launch_wta(ds_handle* h, cudaStream_t st) {
    if (h->cfg.fused) {
        DS_CUDA(ds::launch_sweep_rows(h->cfg, sweep_slant(h), sweep_pad(h), sweep_args(h), st));
        ++g_launches;
        return;
    }
    if (wta_rows_fit(h)) {
        DS_CUDA(ds::launch_wta_rows(wta_row_args(h), st));
        ++g_launches;
        return;
    }
    dsk::WtaArgs a{};
    a.values = h->d_values;
    a.dir_stride = h->dir_stride;
    a.ndirs = h->ndirs;
    a.w = h->w;
    a.h = h->h;
    a.nd = h->nd;
    a.dp = h->dp;
    a.min_disp = h->p.sgm.min_disparity;
    a.uniqueness = h->p.sgm.uniqueness;
    a.subpixel = h->p.subpixel ? 1 : 0;
    a.lr_max_diff = h->p.sgm.lr_max_diff;
    a.disp = h->d_disp_lr;
    a.pair_sums = h->s16 ? 0 : 1;
    DS_CUDA(ds::launch_wta(h->cfg, h->wide, a, h->h, static_cast<size_t>(h->w) * 8, st));
    ++g_launches;
}

void free_counted(ds_handle* h, void*& p, size_t bytes) {
    if (p) {
        cudaFree(p);
        h->bytes -= bytes;
        p = nullptr;
    }
}

// WTA records (8 bytes per pixel) and right-WTA keys (2 bytes per pixel and key set: 2 sets for the sweep
// kernels, up to kWtaRowMaxSets for the row-sweep WTA), after the path values in the volume.
size_t aux_bytes(const ds_handle* h) {
    const size_t n = static_cast<size_t>(h->w) * h->h;
    return (n * 8 + 255) / 256 * 256 + n * 2 * (h->cfg.fused ? 2 : dsk::kWtaRowMaxSets);
}
// The sweep kernels' buffers inside the path-value volume: S, T and C slabs (u8 [y][x][dp] with kGuardRows
// guard rows above and below), then the WTA records and the right-WTA keys.
size_t sweep_slab_bytes(const ds_handle* h) {
    return (static_cast<size_t>(h->h + 2 * dsk::kGuardRows) * h->w * h->dp + 255) / 256 * 256;
}
size_t sweep_volume_bytes(const ds_handle* h) { return 3 * sweep_slab_bytes(h) + aux_bytes(h); }
size_t direction_slab_bytes(const ds_handle* h) {  // the per-direction path's values
    return (h->dir_stride * h->ndirs * (h->wide ? 2 : 1) + 255) / 256 * 256;
}
void bind_sweep_buffers(ds_handle* h) {
    h->d_S = h->d_T = h->d_C = nullptr;
    h->d_rec = nullptr;
    h->d_rk = nullptr;
    if (!h->d_values) return;
    const size_t n = static_cast<size_t>(h->w) * h->h;
    uint8_t* base = static_cast<uint8_t*>(h->d_values);
    size_t at = 0;
    if (h->cfg.fused) {
        const size_t slab = sweep_slab_bytes(h), lead = static_cast<size_t>(dsk::kGuardRows) * h->w * h->dp;
        h->d_S = base + lead;
        h->d_T = base + slab + lead;
        h->d_C = base + 2 * slab + lead;
        at = 3 * slab;
    } else if (wta_rows_fit(h)) {
        at = direction_slab_bytes(h);
    } else {
        return;
    }
    h->d_rec = reinterpret_cast<uint2*>(base + at);
    h->d_rk = reinterpret_cast<uint16_t*>(base + at + (n * 8 + 255) / 256 * 256);
}

constexpr int kCensusSlack = 40;

// (Re)allocates the buffers whose size depends on the kernel configuration. The census and the fused
// slabs carry kGuardRows guard rows above and below (and the census guard columns) for the prefetches.
void size_config_buffers(ds_handle* h) {
    if (h->refine) return;  // its SGM buffers belong to h->sgm
    constexpr int g = dsk::kGuardRows;
    h->dp = h->cfg.dp();
    const size_t n = static_cast<size_t>(h->w) * h->h;
    h->dir_stride = n * static_cast<size_t>(h->dp);
    {
        const int mind = h->p.sgm.min_disparity;
        // + kCensusSlack: the column sweep kernel's lanes past the row end (a column group is up to 32 columns)
        // and its 16-byte aligned loads read up to 36 words beyond the last real column's window.
        const int guard = (std::max(mind + h->dp, 0) + std::max(-mind, 0) + g + kCensusSlack + 3) / 4 * 4;
        const int pitch = (h->w + 2 * guard + 3) / 4 * 4;
        const size_t cw = h->census64 ? 8 : 4;
        const size_t cb = static_cast<size_t>(h->h + 2 * g) * pitch * cw;
        if (cb > h->census_bytes) {  // capacity: a smaller layout reuses the buffers
            size_t cap = cb;
            if (h->any_min_disparity) {  // room for the guards of every min_disparity in [-512, 512]
                const int gmax = (dsk::kMaxDisparities + h->dp + g + kCensusSlack + 3) / 4 * 4;
                cap = std::max(cap, static_cast<size_t>(h->h + 2 * g) * ((h->w + 2 * gmax + 3) / 4 * 4) * cw);
            }
            for (auto*& p : h->census_raw) free_counted(h, p, h->census_bytes);
            h->census_bytes = 0;
            for (auto*& p : h->census_raw) p = h->alloc<uint8_t>(cap);
            h->census_bytes = cap;
        }
        h->cguard = guard;
        h->cpitch = pitch;
        for (int s = 0; s < 2; ++s)
            h->d_census[s] = static_cast<uint8_t*>(h->census_raw[s]) + (static_cast<size_t>(g) * pitch + guard) * cw;
    }
    const size_t vb = h->cfg.fused ? sweep_volume_bytes(h)
                                   : direction_slab_bytes(h) + (wta_rows_fit(h) ? aux_bytes(h) : 0);
    const size_t cb = h->cfg.materialize && !h->cfg.fused ? n * static_cast<size_t>(h->dp) : 0;
    if (h->external_volumes) {  // a batch or the request server binds shared volumes later
        h->values_bytes = vb;
        h->costs_bytes = cb;
        h->d_values = nullptr;
        h->d_costs = nullptr;
        bind_sweep_buffers(h);
        return;
    }
    if (vb != h->values_bytes) {
        if (h->d_values) {
            cudaFree(h->d_values);
            h->bytes -= h->values_bytes;
            h->d_values = nullptr;
            h->values_bytes = 0;
        }
        h->d_values = h->alloc<uint8_t>(vb);
        h->values_bytes = vb;
    }
    bind_sweep_buffers(h);
    if (cb != h->costs_bytes) {
        if (h->d_costs) {
            cudaFree(h->d_costs);
            h->bytes -= h->costs_bytes;
            h->d_costs = nullptr;
            h->costs_bytes = 0;
        }
        if (cb) h->d_costs = h->alloc<uint8_t>(cb);
        h->costs_bytes = cb;
    }
}

struct StageMarks {
    ds_handle* h;
    cudaStream_t st;
    int slot = -1;
    void mark(int i) {
        if (slot >= 0) DS_CUDA(cudaEventRecord(h->prof_events[static_cast<size_t>(slot) * (DS_STAGES + 1) + i], st));
    }
};

StageMarks begin_marks(ds_handle* h, cudaStream_t st) {
    StageMarks marks{h, st};
    if (h->profile) {
        if (h->prof_pending == kProfileRing) throw CudaFailure{cudaErrorNotReady, "profile ring full: call ds_profile_collect"};
        marks.slot = (h->prof_head + h->prof_pending) % kProfileRing;
        ++h->prof_pending;
    }
    return marks;
}

// Raw pair -> rectified (out_w x out_h) with the handle's tables; `half`: tables at twice the size.
void enqueue_rectify(ds_handle* h, const uint8_t* const raw[2], uint8_t* const out[2], int out_w, int out_h, int half,
                     cudaStream_t st) {
    dsk::RectifyArgs r{};
    for (int s = 0; s < 2; ++s) {
        r.raw[s] = raw[s];
        r.map_x[s] = h->d_map[2 * s];
        r.map_y[s] = h->d_map[2 * s + 1];
        r.out[s] = out[s];
    }
    r.raw_w = h->raw_w;
    r.raw_h = h->raw_h;
    r.map_w = h->map_w;
    r.out_w = out_w;
    r.out_h = out_h;
    r.half = half;
    dim3 b(32, 8), g((out_w + 32 * dsk::kRectifyPixelsPerThread - 1) / (32 * dsk::kRectifyPixelsPerThread), (out_h + 7) / 8, 2);
    dsk::k_rectify<<<g, b, 0, st>>>(r);
    ++g_launches;
}

// The frame's input pair in h->d_rect: rectified from raw, or copied from the caller's device images.
void enqueue_inputs(ds_handle* h, const uint8_t* left, const uint8_t* right, bool raw, cudaStream_t st) {
    const uint8_t* img[2] = {left, right};
    if (raw) {
        enqueue_rectify(h, img, h->d_rect, h->w, h->h, h->map_w == 2 * h->w ? 1 : 0, st);
    } else if (left != h->d_rect[0]) {
        // Device inputs of the caller: the path kernel reads the left image as its guide.
        DS_CUDA(cudaMemcpyAsync(h->d_rect[0], left, static_cast<size_t>(h->w) * h->h, cudaMemcpyDeviceToDevice, st));
        DS_CUDA(cudaMemcpyAsync(h->d_rect[1], right, static_cast<size_t>(h->w) * h->h, cudaMemcpyDeviceToDevice, st));
    }
}

// census -> [costs] -> paths -> WTA + L-R on h->d_rect into h->d_disp_lr; stage marks 2..5.
void enqueue_sgm(ds_handle* h, StageMarks& marks, cudaStream_t st) {
    {
        dsk::CensusArgs c{};
        c.img[0] = h->d_rect[0];
        c.img[1] = h->d_rect[1];
        c.out[0] = h->d_census[0];
        c.out[1] = h->d_census[1];
        c.w = h->w;
        c.h = h->h;
        c.rx = h->p.sgm.census_radius_x;
        c.ry = h->p.sgm.census_radius_y;
        c.pitch = h->cpitch;
        dim3 b(32, 8), g((h->w + 31) / 32, (h->h + 7) / 8, 2);
        if (h->census64) dsk::k_census<uint64_t><<<g, b, 0, st>>>(c);
        else dsk::k_census<uint32_t><<<g, b, 0, st>>>(c);
        ++g_launches;
    }
    marks.mark(2);
    launch_costs(h, st);
    marks.mark(3);
    launch_paths(h, st);
    marks.mark(4);
    launch_wta(h, st);
    marks.mark(5);
}

// Median (optional) and the outputs of disparity `disp` (W x H); confidence from `conf` (else 1 where valid).
void enqueue_post(ds_handle* h, const float* disp, const float* conf, int median, const ds_outputs& out, cudaStream_t st) {
    dsk::PostArgs q{};
    q.disp = disp;
    q.conf_in = conf;
    q.w = h->w;
    q.h = h->h;
    q.median = median;
    q.min_disp = h->p.sgm.min_disparity;
    q.out_disp = out.disparity;
    q.out_conf = out.confidence;
    q.out_u16 = out.disparity_u16;
    q.out_depth = h->have_points ? out.depth : nullptr;
    q.f = h->geom.f;
    q.baseline = h->geom.baseline;
    q.cx_offset = h->geom.cx_offset;
    q.min_depth = h->min_depth;
    q.max_depth = h->max_depth;
    dim3 b(32, 8), g((h->w + 31) / 32, (h->h + 7) / 8);
    dsk::k_post<<<g, b, 0, st>>>(q);
    ++g_launches;
}

// depth::compute_disparity (stereo.cpp:501-536): pyramid, SGM at the coarsest level, refine_level up to the
// stereo resolution, detail refinement (raw frames with tables at twice the size), filters, speckles. Raw
// frames with tables at twice the size are rectified at full resolution and box-downsampled, as the CPU
// frontend prepares them (stereo_frontend.cpp:331-335).
void enqueue_refine(ds_handle* h, const uint8_t* left, const uint8_t* right, bool raw, const ds_outputs& out,
                    StageMarks& marks, cudaStream_t st) {
    const auto& p = h->p;
    const int L = p.pyramid_levels;
    ds_handle* sg = h->sgm;
    const int w = h->w, ht = h->h;
    const size_t n = static_cast<size_t>(w) * ht;
    const dim3 b2(32, 8);
    auto grid2 = [](int gw, int gh) { return dim3((gw + 31) / 32, (gh + 7) / 8); };
    marks.mark(0);
    const bool full = raw && h->d_full[0] && h->map_w == 2 * w;
    if (full) {  // the full-resolution pair for the detail refinement, box-downsampled to the stereo resolution
        const uint8_t* img[2] = {left, right};
        enqueue_rectify(h, img, h->d_full, 2 * w, 2 * ht, 0, st);
        for (int s = 0; s < 2; ++s) dsk::k_downsample2<<<grid2(w, ht), b2, 0, st>>>(h->d_full[s], 2 * w, 2 * ht, h->d_rect[s]);
        g_launches += 2;
    } else {
        enqueue_inputs(h, left, right, raw, st);
    }
    for (int l = 1; l <= L; ++l)
        for (int s = 0; s < 2; ++s) {
            const uint8_t* src = l == 1 ? h->d_rect[s] : h->pyr[s][l - 1];
            uint8_t* dst = l == L ? sg->d_rect[s] : h->pyr[s][l];
            dsk::k_downsample2<<<grid2(h->lw[l], h->lh[l]), b2, 0, st>>>(src, h->lw[l - 1], h->lh[l - 1], dst);
            ++g_launches;
        }
    if (L == 0)
        for (int s = 0; s < 2; ++s) DS_CUDA(cudaMemcpyAsync(sg->d_rect[s], h->d_rect[s], n, cudaMemcpyDeviceToDevice, st));
    marks.mark(1);
    enqueue_sgm(sg, marks, st);
    auto other = [&](const float* c) { return c == h->d_ra ? h->d_rb : h->d_ra; };
    const float* cur = sg->d_disp_lr;
    for (int l = L - 1; l >= 0; --l) {
        dsk::k_median3<<<grid2(h->lw[l + 1], h->lh[l + 1]), b2, 0, st>>>(cur, h->lw[l + 1], h->lh[l + 1], h->d_rmed);
        dsk::RefineArgs ra{};
        ra.left = l == 0 ? h->d_rect[0] : h->pyr[0][l];
        ra.right = l == 0 ? h->d_rect[1] : h->pyr[1][l];
        ra.coarse = h->d_rmed;
        ra.w = h->lw[l];
        ra.h = h->lh[l];
        ra.cw = h->lw[l + 1];
        ra.ch = h->lh[l + 1];
        ra.search_radius = p.refine_search_radius;
        ra.zncc_radius = p.refine_zncc_radius;
        ra.min_zncc = p.refine_min_zncc;
        ra.reject_edge_winners = p.refine_reject_edge_winners ? 1 : 0;
        ra.subpixel = p.subpixel ? 1 : 0;
        ra.disp = other(cur);
        ra.conf = h->d_rconf;
        dsk::k_refine_level<<<dim3((ra.w + 31) / 32, (ra.h + 3) / 4), dim3(32, 4), 0, st>>>(ra);
        g_launches += 2;
        cur = ra.disp;
    }
    float* dcur = const_cast<float*>(cur);  // the later stages work in place or ping-pong through d_ra / d_rb
    if (p.detail_enabled && full) {
        float* nxt = other(dcur);
        DS_CUDA(cudaMemcpyAsync(nxt, dcur, n * sizeof(float), cudaMemcpyDeviceToDevice, st));
        dsk::DetailArgs da{};
        da.full_left = h->d_full[0];
        da.full_right = h->d_full[1];
        da.W = 2 * w;
        da.H = 2 * ht;
        da.first = dcur;
        da.disp = nxt;
        da.w = w;
        da.h = ht;
        da.radius = p.detail_radius;
        da.K = std::min(16, static_cast<int>(lroundf(p.detail_search / p.detail_step)));
        da.step = p.detail_step;
        da.min_zncc = p.detail_min_zncc;
        da.subpixel = p.subpixel ? 1 : 0;
        dsk::k_refine_detail<<<dim3((w + 31) / 32, (ht + 3) / 4), dim3(32, 4), 0, st>>>(da);
        ++g_launches;
        dcur = nxt;
    }
    if (p.filter_occlusion) {
        dsk::k_filter_occlusion<<<ht, 256, static_cast<size_t>(w) * sizeof(int), st>>>(dcur, w, p.occlusion_tolerance);
        ++g_launches;
    }
    if (p.filter_spikes) {
        float* nxt = other(dcur);
        dsk::k_filter_spikes<<<grid2(w, ht), b2, 0, st>>>(dcur, w, ht, p.spike_threshold, nxt);
        ++g_launches;
        dcur = nxt;
    }
    if (p.speckle_max_region_size > 1) {
        const int nn = static_cast<int>(n), bl = (nn + 255) / 256;
        DS_CUDA(cudaMemsetAsync(h->d_err, 0, sizeof(int), st));
        DS_CUDA(cudaMemsetAsync(h->d_size, 0, n * sizeof(int), st));
        const dsk::SpeckleConn conn{dcur, w, p.speckle_max_diff};
        g_launches += dsk::launch_ccl(conn, w, ht, h->d_parent, h->d_err, st);
        dsk::k_speckle_count<<<bl, 256, 0, st>>>(dcur, nn, h->d_parent, h->d_size, h->d_err);
        dsk::k_speckle_apply<<<bl, 256, 0, st>>>(dcur, nn, h->d_parent, h->d_size, p.speckle_max_region_size, h->d_err);
        g_launches += 2;
    }
    enqueue_post(h, dcur, L > 0 ? h->d_rconf : nullptr, 0, out, st);
    marks.mark(6);
    DS_CUDA(cudaGetLastError());
}

// The whole frame on `st`: [rectify] -> census -> [costs] -> paths -> WTA + L-R -> median + outputs, or
// depth::compute_disparity's stages when the handle refines.
void enqueue_frame(ds_handle* h, const uint8_t* left, const uint8_t* right, bool raw, const ds_outputs& out,
                   cudaStream_t st) {
    StageMarks marks = begin_marks(h, st);
    if (h->refine) {
        enqueue_refine(h, left, right, raw, out, marks, st);
        return;
    }
    marks.mark(0);
    enqueue_inputs(h, left, right, raw, st);
    marks.mark(1);
    enqueue_sgm(h, marks, st);
    enqueue_post(h, h->d_disp_lr, nullptr, h->p.median ? 1 : 0, out, st);
    marks.mark(6);
    DS_CUDA(cudaGetLastError());
}

ds_outputs internal_outputs(ds_handle* h) {
    ds_outputs o{};
    o.disparity = h->d_out_disp;
    o.confidence = h->d_out_conf;
    o.disparity_u16 = h->d_out_u16;
    o.depth = h->d_out_depth;
    return o;
}

// ---- marker blob search -------------------------------------------------------------------------------------
void ensure_blob_buffers(ds_handle* h, size_t npx) {
    const uint32_t cap = h->blob_p.max_blobs;
    if (npx <= h->blob_px && cap == h->blob_cap) return;
    npx = std::max(npx, h->blob_px);
    for (auto& b : h->blob) {
        for (void* q : {static_cast<void*>(b.parent), static_cast<void*>(b.count), static_cast<void*>(b.box), static_cast<void*>(b.mom),
                        static_cast<void*>(b.out), static_cast<void*>(b.n_out), static_cast<void*>(b.img)})
            if (q) cudaFree(q);
        b = ds_handle::BlobBufs{};
        b.parent = h->alloc<int>(npx);
        b.count = h->alloc<uint32_t>(npx);
        b.box = h->alloc<uint32_t>(5 * npx);
        b.mom = h->alloc<int>(5 * npx);
        b.out = h->alloc<dsk::BlobCand>(cap);
        b.n_out = h->alloc<uint32_t>(2);
        b.img = h->alloc<uint8_t>(npx);
    }
    h->blob_px = npx;
    h->blob_cap = cap;
    if (!h->blob_stream) {
        DS_CUDA(cudaStreamCreateWithFlags(&h->blob_stream, cudaStreamNonBlocking));
        DS_CUDA(cudaEventCreateWithFlags(&h->blob_ev, cudaEventDisableTiming));
    }
}

// The blob search of one image (w x h, tightly packed, on the device) into side `side`'s candidate list.
void enqueue_blob_search(ds_handle* h, int side, const uint8_t* img, int w, int ht, cudaStream_t st) {
    auto& b = h->blob[side];
    const auto& bp = h->blob_p;
    dsk::BlobArgs a{};
    a.img = img;
    a.w = w;
    a.h = ht;
    a.threshold = bp.threshold;
    a.min_diameter = bp.min_diameter;
    a.max_diameter = bp.max_diameter;
    a.border = bp.border;
    a.max_out = h->blob_cap;
    a.max_aspect = bp.max_aspect;
    a.min_fill = bp.min_fill;
    a.max_axis_ratio = bp.max_axis_ratio;
    a.ring_scale = bp.ring_scale;
    a.ring_contrast = bp.ring_contrast;
    a.ring_max_bright = bp.ring_max_bright;
    a.parent = b.parent;
    a.count = b.count;
    a.box = b.box;
    a.mom = b.mom;
    a.out = b.out;
    a.n_out = b.n_out;
    a.err = reinterpret_cast<int*>(b.n_out + 1);
    DS_CUDA(cudaMemsetAsync(b.n_out, 0, 2 * sizeof(uint32_t), st));
    const int n = w * ht, bl = (n + 255) / 256;
    dsk::k_blob_init<<<bl, 256, 0, st>>>(a);
    const dsk::BlobConn conn{img, w, bp.threshold};
    g_launches += dsk::launch_ccl(conn, w, ht, a.parent, a.err, st);
    dsk::k_blob_stats<<<bl, 256, 0, st>>>(a);
    dsk::k_blob_select<<<bl, 256, 0, st>>>(a);
    g_launches += 3;
    DS_CUDA(cudaGetLastError());
}

// Host side of a search: the found count, the error flag and the candidate list, read back on `st`.
struct BlobHost {
    std::vector<dsk::BlobCand> cand;
    uint32_t head[2] = {0, 0};
};

void blob_readback(ds_handle* h, int side, BlobHost& hb, cudaStream_t st) {
    hb.cand.resize(h->blob_cap);
    DS_CUDA(cudaMemcpyAsync(hb.head, h->blob[side].n_out, sizeof(hb.head), cudaMemcpyDeviceToHost, st));
    DS_CUDA(cudaMemcpyAsync(hb.cand.data(), h->blob[side].out, h->blob_cap * sizeof(dsk::BlobCand), cudaMemcpyDeviceToHost, st));
}

// After the stream has finished: candidates ordered by first pixel, at most `capacity` written.
int blob_finish(ds_handle* h, const BlobHost& hb, ds_blob_box* out, uint32_t capacity, uint32_t* found, uint32_t* kept) {
    if (hb.head[1]) return h->fail(DS_IO, "blob search: union-find exceeded its iteration bound");
    const uint32_t n = std::min(hb.head[0], h->blob_cap);
    std::vector<dsk::BlobCand> c(hb.cand.begin(), hb.cand.begin() + n);
    std::sort(c.begin(), c.end(), [](const dsk::BlobCand& p, const dsk::BlobCand& q) { return p.root < q.root; });
    const uint32_t k = std::min(n, capacity);
    for (uint32_t i = 0; i < k; ++i) out[i] = ds_blob_box{c[i].x0, c[i].y0, c[i].x1, c[i].y1, c[i].pixels, c[i].peak};
    if (found) *found = hb.head[0];
    if (kept) *kept = k;
    return DS_OK;
}

// What a ds_compute_frame call adds to a host frame: blob search outputs and their callback, device points.
struct FrameExtras {
    ds_blob_boxes* blobs = nullptr;
    ds_blob_callback on_blobs = nullptr;
    void* user = nullptr;
    float* points = nullptr;   // device, W*H float4 each (points, normals), W*H weights
    float* normals = nullptr;
    float* weights = nullptr;
};

int run_host(ds_handle* h, const uint8_t* left, const uint8_t* right, ptrdiff_t stride, const ds_outputs* out, bool raw,
             const FrameExtras* fx = nullptr) {
    ds_blob_boxes* blobs = fx ? fx->blobs : nullptr;
    const double t0 = now_ms();
    const int iw = raw ? h->raw_w : h->w, ih = raw ? h->raw_h : h->h;
    if (!left || !right) return h->fail(DS_INVALID_ARGUMENT, "null image");
    if (stride < iw) return h->fail(DS_INVALID_ARGUMENT, "stride smaller than the image width");
    if (out && out->depth && !h->have_points) return h->fail(DS_INVALID_ARGUMENT, "set_point_params() not called");
    uint8_t* dst[2] = {raw ? h->d_raw[0] : h->d_rect[0], raw ? h->d_raw[1] : h->d_rect[1]};
    const uint8_t* src[2] = {left, right};
    for (int s = 0; s < 2; ++s)
        DS_CUDA(cudaMemcpy2DAsync(dst[s], iw, src[s], stride, iw, ih, cudaMemcpyHostToDevice, h->stream));
    DS_CUDA(cudaEventRecord(h->ev0, h->stream));
    BlobHost bh[2];
    if (blobs) {  // on the raw images, concurrently with the stereo
        ensure_blob_buffers(h, static_cast<size_t>(iw) * ih);
        DS_CUDA(cudaEventRecord(h->blob_ev, h->stream));
        DS_CUDA(cudaStreamWaitEvent(h->blob_stream, h->blob_ev, 0));
        for (int s = 0; s < 2; ++s) {
            enqueue_blob_search(h, s, dst[s], iw, ih, h->blob_stream);
            blob_readback(h, s, bh[s], h->blob_stream);
        }
    }
    enqueue_frame(h, dst[0], dst[1], raw, internal_outputs(h), h->stream);
    if (fx && fx->points) {  // the frame's points, normals and weights stay on the device
        ds_point_params pp{};
        ds_default_point_params(&pp);
        pp.min_depth_mm = h->min_depth;
        pp.max_depth_mm = h->max_depth;
        pp.max_depth_jump_mm = h->max_jump;
        if (const int rc = ds_disparity_to_points(h->d_out_disp, h->d_out_conf, h->w, h->h, &h->geom, &pp, fx->points, fx->normals,
                                                  fx->weights, h->stream);
            rc != DS_OK)
            return h->fail(rc, ds_last_global_error());
    }
    DS_CUDA(cudaEventRecord(h->ev1, h->stream));
    const size_t n = static_cast<size_t>(h->w) * h->h;
    if (out) {
        if (out->disparity) DS_CUDA(cudaMemcpyAsync(out->disparity, h->d_out_disp, n * 4, cudaMemcpyDeviceToHost, h->stream));
        if (out->confidence) DS_CUDA(cudaMemcpyAsync(out->confidence, h->d_out_conf, n * 4, cudaMemcpyDeviceToHost, h->stream));
        if (out->disparity_u16) DS_CUDA(cudaMemcpyAsync(out->disparity_u16, h->d_out_u16, n * 2, cudaMemcpyDeviceToHost, h->stream));
        if (out->depth) DS_CUDA(cudaMemcpyAsync(out->depth, h->d_out_depth, n * 4, cudaMemcpyDeviceToHost, h->stream));
        if (out->rect_left) DS_CUDA(cudaMemcpyAsync(out->rect_left, h->d_rect[0], n, cudaMemcpyDeviceToHost, h->stream));
        if (out->rect_right) DS_CUDA(cudaMemcpyAsync(out->rect_right, h->d_rect[1], n, cudaMemcpyDeviceToHost, h->stream));
    }
    if (blobs) {  // the candidates are handed over while the stereo may still run
        DS_CUDA(cudaStreamSynchronize(h->blob_stream));
        ds_blob_box* bo[2] = {blobs->left, blobs->right};
        int rc = DS_OK;
        for (int s = 0; s < 2 && rc == DS_OK; ++s) rc = blob_finish(h, bh[s], bo[s], blobs->capacity, &blobs->found[s], &blobs->kept[s]);
        if (rc != DS_OK) {
            DS_CUDA(cudaStreamSynchronize(h->stream));
            return rc;
        }
        if (fx->on_blobs) fx->on_blobs(blobs, fx->user);
    }
    DS_CUDA(cudaStreamSynchronize(h->stream));
    if (h->refine && h->p.speckle_max_region_size > 1) {
        int err = 0;
        DS_CUDA(cudaMemcpy(&err, h->d_err, sizeof(int), cudaMemcpyDeviceToHost));
        if (err) return h->fail(DS_IO, "speckle removal: union-find exceeded its iteration bound");
    }
    float ms = 0.0f;
    DS_CUDA(cudaEventElapsedTime(&ms, h->ev0, h->ev1));
    h->timings.gpu_ms = ms;
    h->timings.speckle_ms = 0.0;
    h->timings.total_ms = now_ms() - t0;
    return DS_OK;
}

template <typename F>
int guarded(ds_handle* h, F&& f) {
    try {
        return f();
    } catch (const CudaFailure& e) {
        std::string m = std::string("CUDA stereo failed: ") + e.what + ": " + cudaGetErrorString(e.err);
        if (h) h->err = m;
        g_error = m;
        return DS_IO;
    } catch (const std::bad_alloc&) {
        if (h) h->err = "host allocation failed";
        g_error = "host allocation failed";
        return DS_IO;
    }
}

}  // namespace

namespace ds {

void set_global_error(const char* message) { g_error = message ? message : ""; }
void count_launches(int n) { g_launches += static_cast<uint64_t>(n); }

bool cfg_supported(int R, int seg) {
    if (seg == 8) return R == 4 || R == 6 || R == 8;
    if (seg == 16) return R == 1 || R == 2 || R == 3 || R == 4;
    if (seg == 32) return R == 1 || R == 2 || R == 3 || R == 4 || R == 6 || R == 8;
    return false;
}

#define DS_BY_R(FN, ...)                        \
    switch (cfg.R) {                            \
        case 1: return FN##_r1(__VA_ARGS__);    \
        case 2: return FN##_r2(__VA_ARGS__);    \
        case 3: return FN##_r3(__VA_ARGS__);    \
        case 4: return FN##_r4(__VA_ARGS__);    \
        case 6: return FN##_r6(__VA_ARGS__);    \
        case 8: return FN##_r8(__VA_ARGS__);    \
        default: return cudaErrorInvalidValue;  \
    }

cudaError_t launch_paths(const KernelCfg& cfg, bool c64, bool wide, const dsk::PathArgs& a, int ndirs, int max_lines,
                         cudaStream_t st) {
    DS_BY_R(launch_paths, cfg, c64, wide, a, ndirs, max_lines, st)
}
// The WTA splits the Dp disparities of a pixel over its own lanes: the fewest lanes (8, 16 or 32) whose
// slab of 2R disparities has an instantiated R, so that more pixels share a warp's per-pixel work.
KernelCfg wta_split(const KernelCfg& cfg) {
    const int dp = cfg.dp();
    for (int seg : {8, 16, 32}) {
        if (dp % (2 * seg)) continue;
        const int r = dp / (2 * seg);
        if (r == 1 || r == 2 || r == 3 || r == 4 || r == 6 || r == 8) {
            KernelCfg c = cfg;
            c.R = r;
            c.seg = seg;
            return c;
        }
    }
    return cfg;
}

cudaError_t launch_wta(const KernelCfg& cfg0, bool wide, const dsk::WtaArgs& a, int rows, size_t smem, cudaStream_t st) {
    const KernelCfg cfg = wta_split(cfg0);
    DS_BY_R(launch_wta, cfg, wide, a, rows, smem, st)
}
cudaError_t launch_costs(const KernelCfg& cfg, bool c64, const dsk::CostArgs& a, cudaStream_t st) {
    DS_BY_R(launch_costs, cfg, c64, a, st)
}
cudaError_t launch_paths_batch(const KernelCfg& cfg, bool c64, bool wide, const dsk::PathArgs* args, const BatchGroupDev& g,
                               cudaStream_t st) {
    DS_BY_R(launch_paths_batch, cfg, c64, wide, args, g, st)
}
cudaError_t launch_wta_batch(const KernelCfg& cfg0, bool wide, int ndirs, const dsk::WtaArgs* args,
                             const BatchGroupDev& g, size_t smem, cudaStream_t st) {
    const KernelCfg cfg = wta_split(cfg0);
    DS_BY_R(launch_wta_batch, cfg, wide, ndirs, args, g, smem, st)
}
cudaError_t launch_costs_batch(const KernelCfg& cfg, bool c64, const dsk::CostArgs* args, const BatchGroupDev& g,
                               cudaStream_t st) {
    DS_BY_R(launch_costs_batch, cfg, c64, args, g, st)
}
#undef DS_BY_R

}  // namespace ds

namespace dsk {

// Persistent batch launches of the per-pixel stages; per group pair i: grid gx[i] x gy[i] x (2 or 1).
// Virtual blocks of the 2D stages cover a run of tiles along x (one decode and argument check per run).
constexpr int kRectifyRun = 2, kTileRun = 4;

__device__ __forceinline__ void decode3(int lb, int gx, int gy, int& bx, int& by, int& bz) {
    bx = lb % gx;
    const int t = lb / gx;
    by = t % gy;
    bz = t / gy;
}

// Block-uniform staging of a pair's arguments in shared memory (all threads call it).
template <typename A>
__device__ __forceinline__ void stage_args(A& sa, const A* args, int p, int& cur) {
    if (p != cur) {
        __syncthreads();
        if (threadIdx.x == 0 && threadIdx.y == 0) sa = args[p];
        __syncthreads();
        cur = p;
    }
}

__global__ void kb_rectify(const RectifyArgs* __restrict__ args, const int* __restrict__ pairs, const int* __restrict__ prefix,
                           const int* __restrict__ gx, const int* __restrict__ gy, int n, int total) {
    __shared__ RectifyArgs sa;
    int cur = -1;
    for (int v = blockIdx.x; v < total; v += gridDim.x) {
        const int i = batch_find(prefix, n, v);
        int bx, by, bz;
        decode3(v - __ldg(prefix + i), __ldg(gx + i), __ldg(gy + i), bx, by, bz);
        stage_args(sa, args, __ldg(pairs + i), cur);
#pragma unroll 1
        for (int j = 0; j < kRectifyRun; ++j) rectify_body(sa, bx * kRectifyRun + j, by, bz);
    }
}

template <typename W>
__global__ void kb_census(const CensusArgs* __restrict__ args, const int* __restrict__ pairs, const int* __restrict__ prefix,
                          const int* __restrict__ gx, const int* __restrict__ gy, int n, int total) {
    __shared__ CensusArgs sa;
    int cur = -1;
    for (int v = blockIdx.x; v < total; v += gridDim.x) {
        const int i = batch_find(prefix, n, v);
        int bx, by, bz;
        decode3(v - __ldg(prefix + i), __ldg(gx + i), __ldg(gy + i), bx, by, bz);
        stage_args(sa, args, __ldg(pairs + i), cur);
#pragma unroll 1
        for (int j = 0; j < kTileRun; ++j) census_body<W>(sa, bx * kTileRun + j, by, bz);
    }
}

// Cost tiles of all pairs of a group: virtual block = (row, tile) of a pair.
template <typename W>
__global__ void __launch_bounds__(256) kb_cost_tiles(const CostArgs* __restrict__ args, const int* __restrict__ pairs,
                                                     const int* __restrict__ prefix, int n, int total) {
    extern __shared__ __align__(16) unsigned char cost_smem[];
    __shared__ CostArgs sa;
    int cur = -1;
    for (int v = blockIdx.x; v < total; v += gridDim.x) {
        const int i = batch_find(prefix, n, v);
        stage_args(sa, args, __ldg(pairs + i), cur);
        cost_tile_body<W>(sa, v - __ldg(prefix + i), reinterpret_cast<W*>(cost_smem));
    }
}

__global__ void kb_post(const PostArgs* __restrict__ args, const int* __restrict__ pairs, const int* __restrict__ prefix,
                        const int* __restrict__ gx, const int* __restrict__ gy, int n, int total) {
    __shared__ PostArgs sa;
    int cur = -1;
    for (int v = blockIdx.x; v < total; v += gridDim.x) {
        const int i = batch_find(prefix, n, v);
        int bx, by, bz;
        decode3(v - __ldg(prefix + i), __ldg(gx + i), __ldg(gy + i), bx, by, bz);
        stage_args(sa, args, __ldg(pairs + i), cur);
#pragma unroll 1
        for (int j = 0; j < kTileRun; ++j) post_body(sa, bx * kTileRun + j, by);
    }
}

}  // namespace dsk

namespace {

int create_handle(const ds_stereo_params* params, int width, int height, bool external_volumes, ds_handle** out,
                  bool any_min_disparity = false) {
    if (!params || !out) {
        g_error = "null argument";
        return DS_INVALID_ARGUMENT;
    }
    *out = nullptr;
    std::string msg;
    if (const int rc = validate(*params, width, height, msg); rc != DS_OK) {
        g_error = msg;
        return rc;
    }
    auto* h = new (std::nothrow) ds_handle();
    if (!h) {
        g_error = "host allocation failed";
        return DS_IO;
    }
    const int rc = guarded(h, [&]() -> int {
        h->p = *params;
        h->w = width;
        h->h = height;
        h->nd = params->sgm.num_disparities;
        h->cfg = default_cfg(h->nd);
        h->ndirs = params->sgm.eight_paths ? 8 : 4;
        const int window = (2 * params->sgm.census_radius_x + 1) * (2 * params->sgm.census_radius_y + 1);
        h->census64 = window - 1 > 32;
        // Path values are at most window + P2 (the recurrence never lets best exceed min(prev) + P2).
        h->wide = params->wide_costs || window + params->sgm.p2 > 255;
        h->s16 = h->wide || 2 * (window + params->sgm.p2) > 255;
        h->cfg.fused = false;  // the sweep kernels are selectable (ds_set_kernel_config / autotuner)
        h->external_volumes = external_volumes;
        h->any_min_disparity = any_min_disparity;
        DS_CUDA(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
        DS_CUDA(cudaEventCreate(&h->ev0));
        DS_CUDA(cudaEventCreate(&h->ev1));
        const size_t n = static_cast<size_t>(width) * height;
        for (int s = 0; s < 2; ++s) {
            h->rect_raw[s] = h->alloc<uint8_t>(n + 2 * static_cast<size_t>(dsk::kGuardRows) * width);
            h->d_rect[s] = h->rect_raw[s] + static_cast<size_t>(dsk::kGuardRows) * width;
        }
        if (refines(*params)) {
            if (external_volumes) return h->fail(DS_UNSUPPORTED, "the refinement stages run per frame (ds_compute*), "
                                                                 "not in batches or the request server");
            h->refine = true;
            const int L = params->pyramid_levels;
            h->lw.assign(1, width);
            h->lh.assign(1, height);
            for (int l = 1; l <= L; ++l) {
                h->lw.push_back(h->lw.back() / 2);
                h->lh.push_back(h->lh.back() / 2);
            }
            for (int s = 0; s < 2; ++s) {
                h->pyr[s].assign(std::max(L, 1), nullptr);
                for (int l = 1; l < L; ++l) h->pyr[s][l] = h->alloc<uint8_t>(static_cast<size_t>(h->lw[l]) * h->lh[l]);
            }
            ds_stereo_params ip = *params;  // the coarsest level: the hot path without the median
            ip.pyramid_levels = 0;
            ip.median = 0;
            ip.detail_enabled = ip.filter_occlusion = ip.filter_spikes = 0;
            ip.speckle_max_region_size = 0;
            const int rc = create_handle(&ip, h->lw[L], h->lh[L], false, &h->sgm);
            if (rc != DS_OK) return h->fail(rc, std::string("SGM level: ") + g_error);
            h->d_ra = h->alloc<float>(n);
            h->d_rb = h->alloc<float>(n);
            h->d_rconf = h->alloc<float>(n);
            h->d_rmed = h->alloc<float>(n);
            h->d_parent = h->alloc<int>(n);
            h->d_size = h->alloc<int>(n);
            h->d_err = h->alloc<int>(1);
        }
        size_config_buffers(h);
        h->d_disp_lr = h->alloc<float>(n);
        h->d_out_disp = h->alloc<float>(n);
        h->d_out_conf = h->alloc<float>(n);
        h->d_out_u16 = h->alloc<uint16_t>(n);
        h->d_out_depth = h->alloc<float>(n);
        return DS_OK;
    });
    if (rc != DS_OK) {
        g_error = h->err;
        release(h);
        delete h;
        return rc;
    }
    *out = h;
    return DS_OK;
}

}  // namespace

namespace ds {

int validate_params(const ds_stereo_params& params, int width, int height, std::string& message) {
    const int rc = validate(params, width, height, message);
    if (rc == DS_OK && refines(params)) {
        message = "the refinement stages run per frame (ds_compute*), not in the request server";
        return DS_UNSUPPORTED;
    }
    return rc;
}

int create_shared_volume_handle(const ds_stereo_params* params, int width, int height, ds_handle** out) {
    return create_handle(params, width, height, true, out, true);
}

size_t volume_bytes(const ds_handle* h) { return (h->values_bytes + 255) / 256 * 256 + h->costs_bytes; }

void bind_volumes(ds_handle* h, void* base) {
    h->d_values = base;
    h->d_costs = h->costs_bytes ? static_cast<uint8_t*>(base) + (h->values_bytes + 255) / 256 * 256 : nullptr;
    bind_sweep_buffers(h);
}

int bind_rectification(ds_handle* h, float* const maps[4], int map_w, int map_h, int raw_w, int raw_h) {
    const bool same = map_w == h->w && map_h == h->h;
    const bool twice = map_w == 2 * h->w && map_h == 2 * h->h;
    if (!same && !twice) return h->fail(DS_INVALID_ARGUMENT, "remap resolution must be the stereo resolution or twice it");
    if (raw_w < 2 || raw_h < 2 || raw_w > 16384 || raw_h > 16384) return h->fail(DS_INVALID_ARGUMENT, "raw size out of range");
    return guarded(h, [&]() -> int {
        if (!h->maps_external) {
            for (auto*& p : h->d_map)
                if (p) cudaFree(p), h->bytes -= static_cast<size_t>(h->map_w) * h->map_h * 4;
        }
        for (int i = 0; i < 4; ++i) h->d_map[i] = maps[i];
        h->maps_external = true;
        if (h->raw_w != raw_w || h->raw_h != raw_h) {
            for (auto*& p : h->d_raw) {
                if (p) {
                    cudaFree(p);
                    h->bytes -= static_cast<size_t>(h->raw_w) * h->raw_h;
                    p = nullptr;
                }
            }
            for (auto*& p : h->d_raw) p = h->alloc<uint8_t>(static_cast<size_t>(raw_w) * raw_h);
        }
        h->map_w = map_w;
        h->map_h = map_h;
        h->raw_w = raw_w;
        h->raw_h = raw_h;
        h->have_rect = true;
        return DS_OK;
    });
}

int set_frame_params(ds_handle* h, const ds_stereo_params& p) {
    ds_stereo_params a = h->p, b = p;
    a.sgm.min_disparity = b.sgm.min_disparity = 0;
    if (std::memcmp(&a, &b, sizeof(a)) != 0) return h->fail(DS_INVALID_ARGUMENT, "frame parameters differ beyond min_disparity");
    if (p.sgm.min_disparity == h->p.sgm.min_disparity) return DS_OK;
    return guarded(h, [&]() -> int {
        h->p.sgm.min_disparity = p.sgm.min_disparity;
        size_config_buffers(h);  // census guards follow min_disparity; buffers are reused when large enough
        return DS_OK;
    });
}

void input_buffers(ds_handle* h, bool raw, uint8_t* out[2]) {
    for (int s = 0; s < 2; ++s) out[s] = raw ? h->d_raw[s] : h->d_rect[s];
}

ds_outputs device_outputs(ds_handle* h) { return internal_outputs(h); }

int input_width(const ds_handle* h, bool raw) { return raw ? h->raw_w : h->w; }
int input_height(const ds_handle* h, bool raw) { return raw ? h->raw_h : h->h; }

}  // namespace ds

extern "C" {

DS_API void ds_default_params(ds_stereo_params* p) {
    if (!p) return;
    *p = ds_stereo_params{};
    p->pyramid_levels = 0;
    p->sgm.min_disparity = 0;
    p->sgm.num_disparities = 64;
    p->sgm.census_radius_x = 2;
    p->sgm.census_radius_y = 2;
    p->sgm.p1 = 8;
    p->sgm.p2 = 96;
    p->sgm.adaptive_p2 = 1;
    p->sgm.eight_paths = 0;
    p->sgm.slant_steps = 1;
    p->sgm.uniqueness = 0.9f;
    p->sgm.lr_max_diff = 1;
    p->subpixel = 1;
    p->median = 1;
    p->refine_search_radius = 2;  // depth::RefineParams, DetailParams, FilterParams, SpeckleParams defaults
    p->refine_zncc_radius = 3;
    p->refine_min_zncc = 0.5f;
    p->refine_reject_edge_winners = 1;
    p->detail_radius = 5;
    p->detail_search = 1.0f;
    p->detail_step = 0.5f;
    p->detail_min_zncc = 0.5f;
    p->occlusion_tolerance = 1.0f;
    p->spike_threshold = 1.0f;
    p->speckle_max_diff = 1.0f;
}

DS_API const char* ds_last_global_error(void) { return g_error.c_str(); }

DS_API int ds_create(const ds_stereo_params* params, int width, int height, ds_handle** out) {
    return create_handle(params, width, height, false, out);
}

DS_API void ds_destroy(ds_handle* h) {
    if (!h) return;
    if (h->stream) cudaStreamSynchronize(h->stream);
    release(h);
    delete h;
}

DS_API int ds_set_rectification(ds_handle* h, const float* lx, const float* ly, const float* rx, const float* ry, int map_w,
                                int map_h, int raw_w, int raw_h) {
    if (!h) return DS_INVALID_ARGUMENT;
    if (!lx || !ly || !rx || !ry) return h->fail(DS_INVALID_ARGUMENT, "null remap table");
    const bool same = map_w == h->w && map_h == h->h;
    const bool twice = map_w == 2 * h->w && map_h == 2 * h->h;
    if (!same && !twice) return h->fail(DS_INVALID_ARGUMENT, "remap resolution must be the stereo resolution or twice it");
    if (raw_w < 2 || raw_h < 2 || raw_w > 16384 || raw_h > 16384) return h->fail(DS_INVALID_ARGUMENT, "raw size out of range");
    return guarded(h, [&]() -> int {
        const size_t n = static_cast<size_t>(map_w) * map_h;
        if (h->maps_external || h->map_w != map_w || h->map_h != map_h) {
            for (auto*& p : h->d_map) {
                if (p && !h->maps_external) {
                    cudaFree(p);
                    h->bytes -= static_cast<size_t>(h->map_w) * h->map_h * 4;
                }
                p = nullptr;
            }
            h->maps_external = false;
            for (auto*& p : h->d_map) p = h->alloc<float>(n);
        }
        if (h->raw_w != raw_w || h->raw_h != raw_h) {
            for (auto*& p : h->d_raw) {
                if (p) {
                    cudaFree(p);
                    h->bytes -= static_cast<size_t>(h->raw_w) * h->raw_h;
                    p = nullptr;
                }
            }
            for (auto*& p : h->d_raw) p = h->alloc<uint8_t>(static_cast<size_t>(raw_w) * raw_h);
        }
        const float* src[4] = {lx, ly, rx, ry};
        for (int i = 0; i < 4; ++i) DS_CUDA(cudaMemcpyAsync(h->d_map[i], src[i], n * 4, cudaMemcpyHostToDevice, h->stream));
        DS_CUDA(cudaStreamSynchronize(h->stream));
        if (h->refine && twice && !h->d_full[0])  // full-resolution rectified pair (downsampled; detail refinement)
            for (auto*& q : h->d_full) q = h->alloc<uint8_t>(static_cast<size_t>(map_w) * map_h);
        h->map_w = map_w;
        h->map_h = map_h;
        h->raw_w = raw_w;
        h->raw_h = raw_h;
        h->have_rect = true;
        return DS_OK;
    });
}

DS_API int ds_set_point_params(ds_handle* h, const ds_geometry* g, float min_depth, float max_depth, float max_jump) {
    if (!h) return DS_INVALID_ARGUMENT;
    if (!g) return h->fail(DS_INVALID_ARGUMENT, "null geometry");
    h->geom = *g;
    h->min_depth = min_depth;
    h->max_depth = max_depth;
    h->max_jump = max_jump;
    h->have_points = true;
    return DS_OK;
}

DS_API int ds_compute(ds_handle* h, const uint8_t* left, const uint8_t* right, ptrdiff_t stride, const ds_outputs* out) {
    if (!h) return DS_INVALID_ARGUMENT;
    return guarded(h, [&] { return run_host(h, left, right, stride, out, false); });
}

DS_API int ds_compute_raw(ds_handle* h, const uint8_t* left, const uint8_t* right, ptrdiff_t stride, const ds_outputs* out) {
    if (!h) return DS_INVALID_ARGUMENT;
    if (!h->have_rect) return h->fail(DS_INVALID_ARGUMENT, "set_rectification() not called");
    return guarded(h, [&] { return run_host(h, left, right, stride, out, true); });
}

DS_API void ds_default_blob_params(ds_blob_params* p) {
    if (!p) return;
    *p = ds_blob_params{150u, 3u, 60u, 4.0f, 0.5f, 4u, 3.0f, 1.4f, 0.5f, 0.3f, 1024u};  // depth_metal::BlobParams
}

DS_API int ds_set_blob_params(ds_handle* h, const ds_blob_params* p) {
    if (!h) return DS_INVALID_ARGUMENT;
    if (!p) return h->fail(DS_INVALID_ARGUMENT, "null blob parameters");
    if (p->max_blobs < 1 || p->max_blobs > 65536) return h->fail(DS_INVALID_ARGUMENT, "max_blobs must be 1..65536");
    if (p->min_diameter > p->max_diameter || p->threshold > 255)
        return h->fail(DS_INVALID_ARGUMENT, "blob parameters: threshold 0..255 and min_diameter <= max_diameter");
    h->blob_p = *p;
    h->have_blobs = true;
    return DS_OK;
}

DS_API int ds_compute_raw_blobs(ds_handle* h, const uint8_t* left, const uint8_t* right, ptrdiff_t stride, const ds_outputs* out,
                                ds_blob_boxes* blobs) {
    if (!h) return DS_INVALID_ARGUMENT;
    if (!h->have_rect) return h->fail(DS_INVALID_ARGUMENT, "set_rectification() not called");
    if (!blobs || !blobs->left || !blobs->right) return h->fail(DS_INVALID_ARGUMENT, "null blob outputs");
    if (!h->have_blobs) return h->fail(DS_INVALID_ARGUMENT, "set_blob_params() not called");
    FrameExtras fx;
    fx.blobs = blobs;
    return guarded(h, [&] { return run_host(h, left, right, stride, out, true, &fx); });
}

DS_API int ds_compute_frame(ds_handle* h, const uint8_t* left, const uint8_t* right, ptrdiff_t stride, const ds_frame_request* req,
                            ds_frame_outputs* out) {
    if (!h) return DS_INVALID_ARGUMENT;
    if (!out) return h->fail(DS_INVALID_ARGUMENT, "null frame outputs");
    if (!h->have_rect) return h->fail(DS_INVALID_ARGUMENT, "set_rectification() not called");
    FrameExtras fx;
    const bool any_points = out->points_xyzw || out->normals_xyzw || out->weights;
    if (any_points) {
        if (!out->points_xyzw || !out->normals_xyzw || !out->weights)
            return h->fail(DS_INVALID_ARGUMENT, "points, normals and weights are produced together");
        if (!h->have_points) return h->fail(DS_INVALID_ARGUMENT, "set_point_params() not called");
        fx.points = out->points_xyzw;
        fx.normals = out->normals_xyzw;
        fx.weights = out->weights;
    }
    if (req && req->marker_blobs) {
        if (!h->have_blobs) return h->fail(DS_INVALID_ARGUMENT, "set_blob_params() not called");
        if (!out->blobs || !out->blobs->left || !out->blobs->right) return h->fail(DS_INVALID_ARGUMENT, "null blob outputs");
        fx.blobs = out->blobs;
        fx.on_blobs = req->on_blobs;
        fx.user = req->user;
    }
    return guarded(h, [&] { return run_host(h, left, right, stride, &out->host, true, &fx); });
}

DS_API int ds_compute_frame_raw(ds_handle* h, const uint8_t* left, const uint8_t* right, ptrdiff_t stride, float* points_xyzw,
                                float* normals_xyzw, float* weights, uint8_t* rect_left, uint8_t* rect_right) {
    if (!h) return DS_INVALID_ARGUMENT;
    if (!h->have_points) return h->fail(DS_INVALID_ARGUMENT, "set_point_params() not called");  // metal_stereo.cpp:254
    if (!points_xyzw || !normals_xyzw || !weights) return h->fail(DS_INVALID_ARGUMENT, "null point outputs");
    ds_frame_outputs out{};
    out.points_xyzw = points_xyzw;
    out.normals_xyzw = normals_xyzw;
    out.weights = weights;
    out.host.rect_left = rect_left;
    out.host.rect_right = rect_right;
    return ds_compute_frame(h, left, right, stride, nullptr, &out);
}

DS_API int ds_find_blobs(ds_handle* h, const uint8_t* image, int width, int height, ptrdiff_t stride, ds_blob_box* out,
                         uint32_t capacity, uint32_t* found, uint32_t* kept) {
    if (!h) return DS_INVALID_ARGUMENT;
    if (!image || (!out && capacity > 0)) return h->fail(DS_INVALID_ARGUMENT, "null image or output");
    if (!h->have_blobs) return h->fail(DS_INVALID_ARGUMENT, "set_blob_params() not called");
    if (width < 1 || height < 1 || width > 16384 || height > 16384) return h->fail(DS_INVALID_ARGUMENT, "image size must be 1..16384");
    if (stride < width) return h->fail(DS_INVALID_ARGUMENT, "stride smaller than the image width");
    return guarded(h, [&]() -> int {
        ensure_blob_buffers(h, static_cast<size_t>(width) * height);
        cudaStream_t st = h->blob_stream;
        DS_CUDA(cudaMemcpy2DAsync(h->blob[0].img, width, image, stride, width, height, cudaMemcpyHostToDevice, st));
        enqueue_blob_search(h, 0, h->blob[0].img, width, height, st);
        BlobHost bh;
        blob_readback(h, 0, bh, st);
        DS_CUDA(cudaStreamSynchronize(st));
        return blob_finish(h, bh, out, capacity, found, kept);
    });
}

static int run_device(ds_handle* h, const uint8_t* left, const uint8_t* right, const ds_outputs* out, void* stream, bool raw) {
    if (!left || !right) return h->fail(DS_INVALID_ARGUMENT, "null image");
    if (raw && !h->have_rect) return h->fail(DS_INVALID_ARGUMENT, "set_rectification() not called");
    if (out && out->depth && !h->have_points) return h->fail(DS_INVALID_ARGUMENT, "set_point_params() not called");
    cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : h->stream;
    return guarded(h, [&]() -> int {
        ds_outputs o = out ? *out : ds_outputs{};
        enqueue_frame(h, left, right, raw, o, st);
        const size_t n = static_cast<size_t>(h->w) * h->h;
        if (raw && o.rect_left) DS_CUDA(cudaMemcpyAsync(o.rect_left, h->d_rect[0], n, cudaMemcpyDeviceToDevice, st));
        if (raw && o.rect_right) DS_CUDA(cudaMemcpyAsync(o.rect_right, h->d_rect[1], n, cudaMemcpyDeviceToDevice, st));
        return DS_OK;
    });
}

DS_API int ds_compute_device(ds_handle* h, const uint8_t* left, const uint8_t* right, const ds_outputs* out, void* stream) {
    if (!h) return DS_INVALID_ARGUMENT;
    return run_device(h, left, right, out, stream, false);
}

DS_API int ds_compute_raw_device(ds_handle* h, const uint8_t* left, const uint8_t* right, const ds_outputs* out, void* stream) {
    if (!h) return DS_INVALID_ARGUMENT;
    return run_device(h, left, right, out, stream, true);
}

DS_API int ds_last_timings(const ds_handle* h, ds_timings* out) {
    if (!h || !out) return DS_INVALID_ARGUMENT;
    *out = h->timings;
    return DS_OK;
}

DS_API const char* ds_last_error(const ds_handle* h) { return h ? h->err.c_str() : g_error.c_str(); }

DS_API int ds_debug_read(ds_handle* h, uint64_t* census_left, uint64_t* census_right, uint16_t* path_sums) {
    if (!h) return DS_INVALID_ARGUMENT;
    if (h->refine) return h->fail(DS_UNSUPPORTED, "intermediate reads cover the hot path only");
    return guarded(h, [&]() -> int {
        const size_t n = static_cast<size_t>(h->w) * h->h;
        DS_CUDA(cudaStreamSynchronize(h->stream));
        uint64_t* dst[2] = {census_left, census_right};
        for (int s = 0; s < 2; ++s) {
            if (!dst[s]) continue;
            const size_t cw = h->census64 ? 8 : 4;
            std::vector<uint8_t> tmp(n * cw);
            DS_CUDA(cudaMemcpy2D(tmp.data(), h->w * cw, h->d_census[s], h->cpitch * cw, h->w * cw, h->h, cudaMemcpyDeviceToHost));
            for (size_t i = 0; i < n; ++i) {
                if (h->census64) std::memcpy(&dst[s][i], &tmp[i * 8], 8);
                else {
                    uint32_t v;
                    std::memcpy(&v, &tmp[i * 4], 4);
                    dst[s][i] = v;
                }
            }
        }
        if (path_sums) {
            const size_t m = n * h->nd;
            uint16_t* d = nullptr;
            DS_CUDA(cudaMalloc(&d, m * 2));
            void* vals = h->d_values;
            void* tmp = nullptr;
            cudaError_t e = cudaSuccess;
            size_t stride = h->dir_stride;
            int dp = h->dp;
            if (h->cfg.fused) {
                // The sweep kernels keep no per-direction values: recompute them with the per-direction kernel
                // in the library's default classic configuration.
                ds::KernelCfg gc = default_cfg(h->nd);
                gc.fused = false;
                gc.materialize = false;
                dp = gc.dp();
                stride = n * static_cast<size_t>(dp);
                e = cudaMalloc(&tmp, stride * h->ndirs * (h->wide ? 2 : 1));
                if (e == cudaSuccess) {
                    const auto& sg = h->p.sgm;
                    dsk::PathArgs pa{};
                    pa.census_l = h->d_census[0];
                    pa.census_r = h->d_census[1];
                    pa.cpitch = h->cpitch;
                    pa.guide = h->d_rect[0];
                    pa.values = tmp;
                    pa.dir_stride = stride;
                    pa.w = h->w;
                    pa.h = h->h;
                    pa.nd = h->nd;
                    pa.dp = dp;
                    pa.min_disp = sg.min_disparity;
                    pa.p1 = sg.p1;
                    pa.invalid_cost = (2 * sg.census_radius_x + 1) * (2 * sg.census_radius_y + 1);
                    pa.slant = sg.slant_steps ? 1 : 0;
                    for (int q = 0; q < 32; ++q) pa.p2_table[q] = sg.adaptive_p2 ? std::max(sg.p1 + 1, sg.p2 / (q + 1)) : sg.p2;
                    e = ds::launch_paths(gc, h->census64, h->wide, pa, h->ndirs, std::max(h->w, h->h), h->stream);
                    vals = tmp;
                }
            }
            dsk::SumArgs a{vals, stride, h->ndirs, h->w, h->h, h->nd, dp, d};
            if (e == cudaSuccess) {
                if (h->wide) dsk::k_debug_sums<uint16_t><<<1024, 256, 0, h->stream>>>(a);
                else dsk::k_debug_sums<uint8_t><<<1024, 256, 0, h->stream>>>(a);
                e = cudaGetLastError();
            }
            if (e == cudaSuccess) e = cudaMemcpyAsync(path_sums, d, m * 2, cudaMemcpyDeviceToHost, h->stream);
            if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
            cudaFree(d);
            if (tmp) cudaFree(tmp);
            if (e != cudaSuccess) throw CudaFailure{e, "debug sums"};
        }
        return DS_OK;
    });
}

DS_API size_t ds_device_bytes(const ds_handle* h) { return h ? h->bytes + (h->sgm ? h->sgm->bytes : 0) : 0; }

DS_API int ds_profile_enable(ds_handle* h, int on) {
    if (!h) return DS_INVALID_ARGUMENT;
    return guarded(h, [&]() -> int {
        if (on && h->prof_events.empty()) {
            h->prof_events.resize(static_cast<size_t>(kProfileRing) * (DS_STAGES + 1));
            for (auto& e : h->prof_events) DS_CUDA(cudaEventCreate(&e));
        }
        h->profile = on != 0;
        return DS_OK;
    });
}

DS_API int ds_profile_collect(ds_handle* h, double* stage_ms, int max_frames, int* frames) {
    if (!h || !frames) return DS_INVALID_ARGUMENT;
    return guarded(h, [&]() -> int {
        int n = 0;
        while (h->prof_pending > 0) {
            cudaEvent_t* ev = &h->prof_events[static_cast<size_t>(h->prof_head) * (DS_STAGES + 1)];
            DS_CUDA(cudaEventSynchronize(ev[DS_STAGES]));
            if (n < max_frames && stage_ms) {
                for (int i = 0; i < DS_STAGES; ++i) {
                    float ms = 0.0f;
                    DS_CUDA(cudaEventElapsedTime(&ms, ev[i], ev[i + 1]));
                    stage_ms[static_cast<size_t>(n) * DS_STAGES + i] = ms;
                }
                ++n;
            }
            h->prof_head = (h->prof_head + 1) % kProfileRing;
            --h->prof_pending;
        }
        *frames = n;
        return DS_OK;
    });
}

DS_API uint64_t ds_kernel_launches(void) { return g_launches.load(); }

DS_API int ds_set_kernel_config(ds_handle* h, const ds_kernel_config* c) {
    if (!h) return DS_INVALID_ARGUMENT;
    if (!c) return h->fail(DS_INVALID_ARGUMENT, "null kernel config");
    if (h->refine) {  // the SGM level's kernels
        const int rc = ds_set_kernel_config(h->sgm, c);
        if (rc != DS_OK) h->err = h->sgm->err;
        return rc;
    }
    if (c->fused_pairs) {
        const char* why = sweep_unfit(h, c->regs_per_lane, c->lanes_per_line);
        if (*why) return h->fail(DS_INVALID_ARGUMENT, why);
    } else if (!ds::cfg_supported(c->regs_per_lane, c->lanes_per_line)) {
        return h->fail(DS_INVALID_ARGUMENT,
                       "unsupported kernel configuration (lanes per line 8: R 4,6,8; 16: R 1-4; 32: R 1,2,3,4,6,8)");
    }
    if (c->lanes_per_line * 2 * c->regs_per_lane < h->nd)
        return h->fail(DS_INVALID_ARGUMENT, "kernel configuration holds fewer disparities than num_disparities");
    if (c->path_warps_per_block < 1 || c->path_warps_per_block > 8 || c->wta_threads < 32 || c->wta_threads > 256 ||
        c->wta_threads % 32 || (c->prefetch_steps != 4 && c->prefetch_steps != 8))
        return h->fail(DS_INVALID_ARGUMENT, "block shape or prefetch depth out of range");
    return guarded(h, [&]() -> int {
        DS_CUDA(cudaStreamSynchronize(h->stream));
        h->cfg.R = c->regs_per_lane;
        h->cfg.seg = c->lanes_per_line;
        h->cfg.materialize = c->materialize_costs != 0;
        h->cfg.paths_warps = c->path_warps_per_block;
        h->cfg.wta_threads = c->wta_threads;
        h->cfg.prefetch = c->prefetch_steps;
        h->cfg.fused = c->fused_pairs != 0;
        h->cfg.horz_warps = c->horz_warps_per_block;
        size_config_buffers(h);
        return DS_OK;
    });
}

DS_API int ds_get_kernel_config(const ds_handle* h, ds_kernel_config* c) {
    if (!h || !c) return DS_INVALID_ARGUMENT;
    if (h->refine) return ds_get_kernel_config(h->sgm, c);  // the SGM level's kernels
    c->regs_per_lane = h->cfg.R;
    c->lanes_per_line = h->cfg.seg;
    c->materialize_costs = h->cfg.materialize ? 1 : 0;
    c->path_warps_per_block = h->cfg.paths_warps;
    c->wta_threads = h->cfg.wta_threads;
    c->prefetch_steps = h->cfg.prefetch;
    c->fused_pairs = h->cfg.fused ? 1 : 0;
    c->horz_warps_per_block = h->cfg.horz_warps;
    return DS_OK;
}

}  // extern "C"

// ================================================================================================
// Batched path: many pairs of uneven size / disparity range in one persistent launch per stage and
// kernel variant, captured once into a CUDA graph and replayed.

namespace {

template <typename T>
T* dev_upload(const std::vector<T>& v) {
    T* d = nullptr;
    if (v.empty()) return nullptr;
    DS_CUDA(cudaMalloc(&d, v.size() * sizeof(T)));
    DS_CUDA(cudaMemcpy(d, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
    return d;
}

struct BatchGroup {
    ds::KernelCfg cfg;
    bool c64 = false, wide = false;
    int ndirs = 4;
    int dp = 0;        // row-sweep WTA groups: lane slab and padding
    bool pad = false;
    size_t smem = 0;
    std::vector<int> pairs, prefix, gx, gy;
    int total = 0;
    int *d_pairs = nullptr, *d_prefix = nullptr, *d_gx = nullptr, *d_gy = nullptr;
    ds::BatchGroupDev dev() const { return {d_pairs, d_prefix, d_gx, static_cast<int>(pairs.size()), total, 0}; }
    void upload() {
        std::vector<int> pre = prefix;
        pre.push_back(total);
        d_pairs = dev_upload(pairs);
        d_prefix = dev_upload(pre);
        d_gx = dev_upload(gx);
        d_gy = dev_upload(gy);
    }
    void release() {
        for (int* p : {d_pairs, d_prefix, d_gx, d_gy})
            if (p) cudaFree(p);
        d_pairs = d_prefix = d_gx = d_gy = nullptr;
    }
};

struct BatchCalib {
    float* map[4] = {nullptr, nullptr, nullptr, nullptr};
    int map_w = 0, map_h = 0, raw_w = 0, raw_h = 0;
};

}  // namespace

struct ds_batch {
    std::vector<ds_pair_desc> desc;
    std::vector<ds_handle*> h;
    std::vector<BatchCalib> calib;
    std::vector<const uint8_t*> in_l, in_r;
    std::vector<ds_outputs> out;
    // per-pair stage arguments (host mirrors and device arrays)
    std::vector<dsk::RectifyArgs> a_rect;
    std::vector<dsk::CensusArgs> a_census;
    std::vector<dsk::CostArgs> a_costs;
    std::vector<dsk::PathArgs> a_paths;
    std::vector<dsk::WtaArgs> a_wta;
    std::vector<dsk::PostArgs> a_post;
    std::vector<dsk::SweepArgs> a_sweep;  // by value into the graph: they name only the pair's own buffers
    std::vector<dsk::WtaRowArgs> a_wrow;
    dsk::RectifyArgs* d_rect = nullptr;
    dsk::CensusArgs* d_census = nullptr;
    dsk::CostArgs* d_costs = nullptr;
    dsk::PathArgs* d_paths = nullptr;
    dsk::WtaArgs* d_wta = nullptr;
    dsk::PostArgs* d_post = nullptr;
    dsk::WtaRowArgs* d_wrow = nullptr;
    struct Micro {
        std::vector<int> pairs;  // heaviest first
        BatchGroup g_rect, g_post;
        std::vector<BatchGroup> g_census, g_costs, g_paths, g_wta, g_wrow;
        std::vector<int> sweep;  // pairs on the sweep kernels: one column and one row launch each
        int launches() const {
            return (g_rect.total > 0 ? 1 : 0) +
                   static_cast<int>(g_census.size() + g_costs.size() + g_paths.size() + g_wta.size() + g_wrow.size()) +
                   2 * static_cast<int>(sweep.size()) + 1;
        }
    };
    std::vector<Micro> micro;  // pairs in micro-batches run through all stages back to back
    std::vector<void*> volumes;  // shared cost / path-value volumes, one per (branch, position) slot
    size_t volume_bytes = 0;
    int micro_batch = 1, branches = 8;  // best measured for 16 pairs of 1280x1024, D=128 on B200
    std::vector<cudaStream_t> branch_st;
    std::vector<cudaEvent_t> fork_join;
    cudaStream_t stream = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    bool args_dirty = true;
    bool profile = false;
    cudaEvent_t ev[DS_BATCH_STAGES + 1] = {};
    std::string err;
    size_t bytes = 0;
    int fail(int code, std::string m) {
        err = std::move(m);
        return code;
    }
};

namespace {

void batch_release(ds_batch* b) {
    if (!b) return;
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    for (auto e : b->ev)
        if (e) cudaEventDestroy(e);
    for (auto* p : b->volumes)
        if (p) cudaFree(p);
    for (auto* h : b->h) {
        if (!h) continue;
        for (auto*& p : h->d_map) p = nullptr;  // the maps belong to the batch's calibrations
        h->d_values = nullptr;                  // and the volumes to its slots
        h->d_costs = nullptr;
        release(h);
        delete h;
    }
    for (auto& c : b->calib)
        for (auto* p : c.map)
            if (p) cudaFree(p);
    for (void* p : {static_cast<void*>(b->d_rect), static_cast<void*>(b->d_census), static_cast<void*>(b->d_costs),
                    static_cast<void*>(b->d_paths), static_cast<void*>(b->d_wta), static_cast<void*>(b->d_post),
                    static_cast<void*>(b->d_wrow)})
        if (p) cudaFree(p);
    for (auto& m : b->micro) {
        m.g_rect.release();
        m.g_post.release();
        for (auto* gs : {&m.g_census, &m.g_costs, &m.g_paths, &m.g_wta, &m.g_wrow})
            for (auto& g : *gs) g.release();
    }
    for (auto s : b->branch_st)
        if (s) cudaStreamDestroy(s);
    for (auto e : b->fork_join)
        if (e) cudaEventDestroy(e);
    if (b->stream) cudaStreamDestroy(b->stream);
}

// Per-pair stage arguments from the pair's handle and current bindings.
void batch_fill_args(ds_batch* b) {
    const int n = static_cast<int>(b->h.size());
    b->a_rect.assign(n, {});
    b->a_census.assign(n, {});
    b->a_costs.assign(n, {});
    b->a_paths.assign(n, {});
    b->a_wta.assign(n, {});
    b->a_post.assign(n, {});
    b->a_sweep.assign(n, {});
    b->a_wrow.assign(n, {});
    for (int i = 0; i < n; ++i) {
        ds_handle* h = b->h[i];
        const ds_pair_desc& d = b->desc[i];
        const auto& sg = h->p.sgm;
        const int window = (2 * sg.census_radius_x + 1) * (2 * sg.census_radius_y + 1);
        const uint8_t* img[2] = {b->in_l[i], b->in_r[i]};
        if (d.raw) {
            const BatchCalib& c = b->calib[d.calib];
            auto& r = b->a_rect[i];
            for (int s = 0; s < 2; ++s) {
                r.raw[s] = img[s];
                r.map_x[s] = c.map[2 * s];
                r.map_y[s] = c.map[2 * s + 1];
                r.out[s] = h->d_rect[s];
            }
            r.raw_w = c.raw_w;
            r.raw_h = c.raw_h;
            r.map_w = c.map_w;
            r.out_w = h->w;
            r.out_h = h->h;
            r.half = c.map_w == 2 * h->w ? 1 : 0;
            img[0] = h->d_rect[0];
            img[1] = h->d_rect[1];
        }
        auto& ce = b->a_census[i];
        ce.img[0] = img[0];
        ce.img[1] = img[1];
        ce.out[0] = h->d_census[0];
        ce.out[1] = h->d_census[1];
        ce.w = h->w;
        ce.h = h->h;
        ce.rx = sg.census_radius_x;
        ce.ry = sg.census_radius_y;
        ce.pitch = h->cpitch;
        if (h->cfg.fused) {
            // The sweep kernels read the left image as their guide from the pair's own buffer (an input of the
            // caller can be re-bound without re-capturing the graph): raw pairs are rectified into it, the
            // census kernel copies rectified inputs there.
            if (!d.raw) ce.left_copy = h->d_rect[0];
            b->a_sweep[i] = sweep_args(h);
        }
        b->a_costs[i] = dsk::CostArgs{h->d_census[0], h->d_census[1], h->d_costs, h->w, h->h, h->nd, h->dp, sg.min_disparity,
                                      window, h->cpitch};
        auto& pa = b->a_paths[i];
        pa.census_l = h->d_census[0];
        pa.census_r = h->d_census[1];
        pa.cpitch = h->cpitch;
        pa.guide = img[0];
        pa.costs = h->cfg.materialize ? h->d_costs : nullptr;
        pa.values = h->d_values;
        pa.dir_stride = h->dir_stride;
        pa.w = h->w;
        pa.h = h->h;
        pa.nd = h->nd;
        pa.dp = h->dp;
        pa.min_disp = sg.min_disparity;
        pa.p1 = sg.p1;
        pa.invalid_cost = window;
        pa.slant = sg.slant_steps ? 1 : 0;
        pa.dir_base = 0;
        for (int q = 0; q < 32; ++q) pa.p2_table[q] = sg.adaptive_p2 ? std::max(sg.p1 + 1, sg.p2 / (q + 1)) : sg.p2;
        auto& wa = b->a_wta[i];
        wa.values = h->d_values;
        wa.dir_stride = h->dir_stride;
        wa.ndirs = h->ndirs;
        wa.w = h->w;
        wa.h = h->h;
        wa.nd = h->nd;
        wa.dp = h->dp;
        wa.min_disp = sg.min_disparity;
        wa.uniqueness = sg.uniqueness;
        wa.subpixel = h->p.subpixel ? 1 : 0;
        wa.lr_max_diff = sg.lr_max_diff;
        wa.disp = h->d_disp_lr;
        wa.pair_sums = h->s16 ? 0 : 1;
        if (wta_rows_fit(h)) b->a_wrow[i] = wta_row_args(h);
        auto& q = b->a_post[i];
        const ds_outputs& o = b->out[i];
        q.disp = h->d_disp_lr;
        q.w = h->w;
        q.h = h->h;
        q.median = h->p.median ? 1 : 0;
        q.min_disp = sg.min_disparity;
        q.out_disp = o.disparity ? o.disparity : h->d_out_disp;
        q.out_conf = o.confidence;
        q.out_u16 = o.disparity_u16 ? o.disparity_u16 : h->d_out_u16;
        q.out_depth = d.have_geometry ? (o.depth ? o.depth : h->d_out_depth) : nullptr;
        q.f = d.geometry.f;
        q.baseline = d.geometry.baseline;
        q.cx_offset = d.geometry.cx_offset;
        q.min_depth = d.min_depth_mm;
        q.max_depth = d.max_depth_mm;
    }
    auto put = [](auto& v, auto*& dst) {
        using T = typename std::remove_reference_t<decltype(v)>::value_type;
        if (!dst) DS_CUDA(cudaMalloc(&dst, v.size() * sizeof(T)));
        DS_CUDA(cudaMemcpy(dst, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
    };
    put(b->a_rect, b->d_rect);
    put(b->a_census, b->d_census);
    put(b->a_costs, b->d_costs);
    put(b->a_paths, b->d_paths);
    put(b->a_wta, b->d_wta);
    put(b->a_post, b->d_post);
    put(b->a_wrow, b->d_wrow);
    b->args_dirty = false;
}

void batch_plan_micro(ds_batch* b, ds_batch::Micro& m, const std::vector<int>& order);

// Splits the pairs (heaviest first) into micro-batches; within each, groups pairs by kernel variant and
// lays out each group's virtual blocks.
void batch_plan(ds_batch* b) {
    const int n = static_cast<int>(b->h.size());
    std::vector<int> all(n);
    for (int i = 0; i < n; ++i) all[i] = i;
    std::stable_sort(all.begin(), all.end(), [&](int x, int y) {
        const ds_handle *a = b->h[x], *c = b->h[y];
        return static_cast<double>(a->w) * a->h * a->nd > static_cast<double>(c->w) * c->h * c->nd;
    });
    const int mb = std::max(1, std::min(b->micro_batch, n));
    for (int first = 0; first < n; first += mb) {
        b->micro.emplace_back();
        std::vector<int> order(all.begin() + first, all.begin() + std::min(n, first + mb));
        b->micro.back().pairs = order;
        batch_plan_micro(b, b->micro.back(), order);
    }
}

// Volumes shared between pairs that never run at the same time: micro-batch i runs on branch i % nb
// after micro-batch i - nb has finished all its stages (stream order), so its j-th pair can reuse the
// cost and path-value volumes of micro-batch i - nb's j-th pair. Slot (branch, j) is sized for the
// largest pair it serves.
void batch_bind_volumes(ds_batch* b) {
    const int nm = static_cast<int>(b->micro.size());
    const int nb = std::max(1, std::min(b->branches, nm));
    std::vector<std::vector<int>> slots;  // pairs per slot
    for (int i = 0; i < nm; ++i) {
        const auto& ps = b->micro[i].pairs;
        for (size_t j = 0; j < ps.size(); ++j) {
            const size_t slot = static_cast<size_t>(i % nb) * static_cast<size_t>(b->micro_batch) + j;
            if (slot >= slots.size()) slots.resize(slot + 1);
            slots[slot].push_back(ps[j]);
        }
    }
    for (const auto& ps : slots) {
        if (ps.empty()) continue;
        size_t vb = 0, cb = 0;
        for (int p : ps) {
            vb = std::max(vb, (b->h[p]->values_bytes + 255) / 256 * 256);
            cb = std::max(cb, b->h[p]->costs_bytes);
        }
        void* mem = nullptr;
        DS_CUDA(cudaMalloc(&mem, vb + cb));
        b->volumes.push_back(mem);
        b->volume_bytes += vb + cb;
        b->bytes += vb + cb;
        for (int p : ps) {
            b->h[p]->d_values = mem;
            b->h[p]->d_costs = b->h[p]->costs_bytes ? static_cast<uint8_t*>(mem) + vb : nullptr;
            bind_sweep_buffers(b->h[p]);
        }
    }
}

void batch_plan_micro(ds_batch* b, ds_batch::Micro& m, const std::vector<int>& order) {
    auto add = [](BatchGroup& g, int pair, int blocks, int gx, int gy) {
        g.pairs.push_back(pair);
        g.prefix.push_back(g.total);
        g.gx.push_back(gx);
        g.gy.push_back(gy);
        g.total += blocks;
    };
    auto find_or_add = [](std::vector<BatchGroup>& gs, auto match) -> BatchGroup& {
        for (auto& g : gs)
            if (match(g)) return g;
        gs.emplace_back();
        return gs.back();
    };
    for (int i : order) {
        ds_handle* h = b->h[i];
        const int tx = (h->w + 31) / 32, ty = (h->h + 7) / 8;
        const int tx4 = (h->w + 32 * dsk::kRectifyPixelsPerThread - 1) / (32 * dsk::kRectifyPixelsPerThread);
        const int rx4 = (tx4 + dsk::kRectifyRun - 1) / dsk::kRectifyRun, rx = (tx + dsk::kTileRun - 1) / dsk::kTileRun;
        if (b->desc[i].raw) add(m.g_rect, i, rx4 * ty * 2, rx4, ty);
        add(m.g_post, i, rx * ty, rx, ty);
        {
            BatchGroup& g = find_or_add(m.g_census, [&](const BatchGroup& x) { return x.c64 == h->census64; });
            g.c64 = h->census64;
            add(g, i, rx * ty * 2, rx, ty);
        }
        const ds::KernelCfg& c = h->cfg;
        if (c.fused) {
            m.sweep.push_back(i);
            continue;
        }
        if (c.materialize) {
            BatchGroup& g = find_or_add(m.g_costs, [&](const BatchGroup& x) {
                return x.cfg.R == c.R && x.cfg.seg == c.seg && x.c64 == h->census64;
            });
            g.cfg = c;
            g.c64 = h->census64;
            add(g, i, h->h * ((h->w + dsk::kCostTile - 1) / dsk::kCostTile), 1, 1);
        }
        {
            BatchGroup& g = find_or_add(m.g_paths, [&](const BatchGroup& x) {
                return x.cfg.R == c.R && x.cfg.seg == c.seg && x.cfg.materialize == c.materialize && x.cfg.prefetch == c.prefetch &&
                       x.cfg.paths_warps == c.paths_warps && x.c64 == h->census64 && x.wide == h->wide;
            });
            g.cfg = c;
            g.c64 = h->census64;
            g.wide = h->wide;
            const int max_lines = h->ndirs == 8 ? h->w + h->h - 1 : std::max(h->w, h->h);
            const int lpb = c.paths_warps * (32 / c.seg);
            const int gx = (max_lines + lpb - 1) / lpb;
            add(g, i, gx * h->ndirs, gx, 1);
        }
        if (wta_rows_fit(h)) {
            const bool pad = h->nd < h->dp;
            BatchGroup& g = find_or_add(m.g_wrow, [&](const BatchGroup& x) { return x.dp == h->dp && x.pad == pad; });
            g.dp = h->dp;
            g.pad = pad;
            int R = 0, seg = 0, chunk = 0, lg = 0, sets = 0;
            ds::wta_rows_shape(h->dp, R, seg);
            ds::wta_rows_layout(h->w, h->dp, chunk, lg, sets);
            const int rows = (dsk::kWtaRowWarps * 32 / seg) >> lg;
            add(g, i, (h->h + rows - 1) / rows, 1, 1);
        } else {
            BatchGroup& g = find_or_add(m.g_wta, [&](const BatchGroup& x) {
                return x.cfg.R == c.R && x.cfg.seg == c.seg && x.cfg.wta_threads == c.wta_threads && x.wide == h->wide &&
                       x.ndirs == h->ndirs;
            });
            g.cfg = c;
            g.wide = h->wide;
            g.ndirs = h->ndirs;
            g.smem = std::max(g.smem, static_cast<size_t>(h->w) * 8);
            add(g, i, h->h, 1, 1);
        }
    }
    m.g_rect.upload();
    m.g_post.upload();
    for (auto* gs : {&m.g_census, &m.g_costs, &m.g_paths, &m.g_wta, &m.g_wrow})
        for (auto& g : *gs) g.upload();
}

void batch_enqueue_micro(ds_batch* b, const ds_batch::Micro& m, cudaStream_t st, bool capturing, bool marks) {
    using namespace dsk;
    auto grid_of = [](auto k, int threads, size_t smem, int total) { return ds::persistent_grid(k, threads, smem, total); };
    auto mark = [&](int i) {
        // Inside a capture, only an external event record becomes a timestamped node of the graph.
        if (marks) DS_CUDA(cudaEventRecordWithFlags(b->ev[i], st, capturing ? cudaEventRecordExternal : cudaEventRecordDefault));
    };
    mark(0);
    if (m.g_rect.total > 0) {
        const auto& g = m.g_rect;
        kb_rectify<<<grid_of(kb_rectify, 256, 0, g.total), dim3(32, 8), 0, st>>>(b->d_rect, g.d_pairs, g.d_prefix, g.d_gx, g.d_gy,
                                                                                 static_cast<int>(g.pairs.size()), g.total);
        ++g_launches;
    }
    mark(1);
    for (const auto& g : m.g_census) {
        if (g.c64)
            kb_census<uint64_t><<<grid_of(kb_census<uint64_t>, 256, 0, g.total), dim3(32, 8), 0, st>>>(
                b->d_census, g.d_pairs, g.d_prefix, g.d_gx, g.d_gy, static_cast<int>(g.pairs.size()), g.total);
        else
            kb_census<uint32_t><<<grid_of(kb_census<uint32_t>, 256, 0, g.total), dim3(32, 8), 0, st>>>(
                b->d_census, g.d_pairs, g.d_prefix, g.d_gx, g.d_gy, static_cast<int>(g.pairs.size()), g.total);
        ++g_launches;
    }
    mark(2);
    for (const auto& g : m.g_costs) {
        const int n = static_cast<int>(g.pairs.size());
        if (g.c64) {
            const size_t sm = cost_tile_smem<uint64_t>(g.cfg.dp());
            kb_cost_tiles<uint64_t><<<grid_of(kb_cost_tiles<uint64_t>, 256, sm, g.total), 256, sm, st>>>(
                b->d_costs, g.d_pairs, g.d_prefix, n, g.total);
        } else {
            const size_t sm = cost_tile_smem<uint32_t>(g.cfg.dp());
            kb_cost_tiles<uint32_t><<<grid_of(kb_cost_tiles<uint32_t>, 256, sm, g.total), 256, sm, st>>>(
                b->d_costs, g.d_pairs, g.d_prefix, n, g.total);
        }
        DS_CUDA(cudaGetLastError());
        ++g_launches;
    }
    mark(3);
    for (int p : m.sweep) {
        DS_CUDA(ds::launch_sweep_cols(b->h[p]->cfg, sweep_slant(b->h[p]), sweep_pad(b->h[p]), b->a_sweep[p], st));
        ++g_launches;
    }
    for (const auto& g : m.g_paths) {
        DS_CUDA(ds::launch_paths_batch(g.cfg, g.c64, g.wide, b->d_paths, g.dev(), st));
        ++g_launches;
    }
    mark(4);
    for (int p : m.sweep) {
        DS_CUDA(ds::launch_sweep_rows(b->h[p]->cfg, sweep_slant(b->h[p]), sweep_pad(b->h[p]), b->a_sweep[p], st));
        ++g_launches;
    }
    for (const auto& g : m.g_wta) {
        DS_CUDA(ds::launch_wta_batch(g.cfg, g.wide, g.ndirs, b->d_wta, g.dev(), g.smem, st));
        ++g_launches;
    }
    for (const auto& g : m.g_wrow) {
        DS_CUDA(ds::launch_wta_rows_batch(g.dp, g.pad, b->d_wrow, g.dev(), st));
        ++g_launches;
    }
    mark(5);
    {
        const auto& g = m.g_post;
        kb_post<<<grid_of(kb_post, 256, 0, g.total), dim3(32, 8), 0, st>>>(b->d_post, g.d_pairs, g.d_prefix, g.d_gx, g.d_gy,
                                                                          static_cast<int>(g.pairs.size()), g.total);
        ++g_launches;
    }
    mark(6);
    DS_CUDA(cudaGetLastError());
}

// All micro-batches: round-robin over `branches` streams forked from `st` and joined back into it.
void batch_enqueue(ds_batch* b, cudaStream_t st, bool capturing) {
    const int nb = std::max(1, std::min(b->branches, static_cast<int>(b->micro.size())));
    if (nb == 1) {
        for (size_t i = 0; i < b->micro.size(); ++i) batch_enqueue_micro(b, b->micro[i], st, capturing, b->profile && i == 0);
        return;
    }
    DS_CUDA(cudaEventRecord(b->fork_join[0], st));
    for (int k = 0; k < nb; ++k) {
        DS_CUDA(cudaStreamWaitEvent(b->branch_st[k], b->fork_join[0], 0));
        for (size_t i = k; i < b->micro.size(); i += nb)
            batch_enqueue_micro(b, b->micro[i], b->branch_st[k], capturing, b->profile && i == 0);
        DS_CUDA(cudaEventRecord(b->fork_join[1 + k], b->branch_st[k]));
    }
    for (int k = 0; k < nb; ++k) DS_CUDA(cudaStreamWaitEvent(st, b->fork_join[1 + k], 0));
}

int batch_guarded(ds_batch* b, const std::function<int()>& f) {
    try {
        return f();
    } catch (const CudaFailure& e) {
        std::string m = std::string("CUDA batch failed: ") + e.what + ": " + cudaGetErrorString(e.err);
        if (b) b->err = m;
        g_error = m;
        return DS_IO;
    } catch (const std::bad_alloc&) {
        if (b) b->err = "host allocation failed";
        g_error = "host allocation failed";
        return DS_IO;
    }
}

}  // namespace

extern "C" {

DS_API int ds_batch_create(const ds_pair_desc* pairs, int n, int n_calib, const ds_batch_options* opt, ds_batch** out) {
    if (!pairs || !out || n < 1 || n > 65536 || n_calib < 0) {
        g_error = "invalid batch description";
        return DS_INVALID_ARGUMENT;
    }
    *out = nullptr;
    auto* b = new (std::nothrow) ds_batch();
    if (!b) {
        g_error = "host allocation failed";
        return DS_IO;
    }
    int rc = DS_OK;
    for (int i = 0; i < n && rc == DS_OK; ++i) {
        const ds_pair_desc& d = pairs[i];
        if (d.raw && (d.calib < 0 || d.calib >= n_calib)) {
            g_error = "pair " + std::to_string(i) + ": calibration index out of range";
            rc = DS_INVALID_ARGUMENT;
            break;
        }
        ds_handle* h = nullptr;
        rc = create_handle(&d.params, d.width, d.height, true, &h);
        if (rc != DS_OK) {
            g_error = "pair " + std::to_string(i) + ": " + g_error;
            break;
        }
        b->h.push_back(h);
        if (d.kernel.regs_per_lane > 0) {
            rc = ds_set_kernel_config(h, &d.kernel);
            if (rc != DS_OK) g_error = "pair " + std::to_string(i) + ": " + h->err;
        }
    }
    if (rc == DS_OK) {
        rc = batch_guarded(b, [&]() -> int {
            b->desc.assign(pairs, pairs + n);
            b->calib.assign(n_calib, BatchCalib{});
            b->in_l.assign(n, nullptr);
            b->in_r.assign(n, nullptr);
            b->out.assign(n, ds_outputs{});
            for (auto* h : b->h) b->bytes += h->bytes;
            if (opt) {
                b->micro_batch = opt->micro_batch > 0 ? opt->micro_batch : b->micro_batch;
                b->branches = opt->branches > 0 ? std::min(opt->branches, 16) : b->branches;
            }
            DS_CUDA(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
            b->branch_st.assign(b->branches, nullptr);
            for (auto& st : b->branch_st) DS_CUDA(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
            b->fork_join.assign(b->branches + 1, nullptr);
            for (auto& e : b->fork_join) DS_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
            batch_plan(b);
            batch_bind_volumes(b);
            return DS_OK;
        });
    }
    if (rc != DS_OK) {
        std::string m = g_error;
        batch_release(b);
        delete b;
        g_error = m;
        return rc;
    }
    *out = b;
    return DS_OK;
}

DS_API void ds_batch_destroy(ds_batch* b) {
    if (!b) return;
    if (b->stream) cudaStreamSynchronize(b->stream);
    batch_release(b);
    delete b;
}

DS_API const char* ds_batch_last_error(const ds_batch* b) { return b ? b->err.c_str() : g_error.c_str(); }

DS_API int ds_batch_set_rectification(ds_batch* b, int calib, const float* lx, const float* ly, const float* rx,
                                      const float* ry, int map_w, int map_h, int raw_w, int raw_h) {
    if (!b) return DS_INVALID_ARGUMENT;
    if (calib < 0 || calib >= static_cast<int>(b->calib.size())) return b->fail(DS_INVALID_ARGUMENT, "calibration index out of range");
    if (!lx || !ly || !rx || !ry) return b->fail(DS_INVALID_ARGUMENT, "null remap table");
    if (raw_w < 2 || raw_h < 2 || raw_w > 16384 || raw_h > 16384) return b->fail(DS_INVALID_ARGUMENT, "raw size out of range");
    for (size_t i = 0; i < b->h.size(); ++i) {
        if (!b->desc[i].raw || b->desc[i].calib != calib) continue;
        const ds_handle* h = b->h[i];
        const bool same = map_w == h->w && map_h == h->h, twice = map_w == 2 * h->w && map_h == 2 * h->h;
        if (!same && !twice) return b->fail(DS_INVALID_ARGUMENT, "remap resolution must be the stereo resolution or twice it");
    }
    return batch_guarded(b, [&]() -> int {
        BatchCalib& c = b->calib[calib];
        const size_t n = static_cast<size_t>(map_w) * map_h;
        if (c.map_w != map_w || c.map_h != map_h) {
            for (auto*& p : c.map) {
                if (p) cudaFree(p), b->bytes -= static_cast<size_t>(c.map_w) * c.map_h * 4;
                p = nullptr;
            }
            for (auto*& p : c.map) {
                DS_CUDA(cudaMalloc(&p, n * 4));
                b->bytes += n * 4;
            }
        }
        const float* src[4] = {lx, ly, rx, ry};
        for (int i = 0; i < 4; ++i) DS_CUDA(cudaMemcpy(c.map[i], src[i], n * 4, cudaMemcpyHostToDevice));
        c.map_w = map_w;
        c.map_h = map_h;
        c.raw_w = raw_w;
        c.raw_h = raw_h;
        b->args_dirty = true;
        return DS_OK;
    });
}

DS_API int ds_batch_bind(ds_batch* b, int pair, const uint8_t* left, const uint8_t* right, const ds_outputs* out) {
    if (!b) return DS_INVALID_ARGUMENT;
    if (pair < 0 || pair >= static_cast<int>(b->h.size())) return b->fail(DS_INVALID_ARGUMENT, "pair index out of range");
    if (!left || !right) return b->fail(DS_INVALID_ARGUMENT, "null image");
    b->in_l[pair] = left;
    b->in_r[pair] = right;
    b->out[pair] = out ? *out : ds_outputs{};
    b->args_dirty = true;
    return DS_OK;
}

DS_API int ds_batch_run(ds_batch* b, void* stream) {
    if (!b) return DS_INVALID_ARGUMENT;
    for (size_t i = 0; i < b->h.size(); ++i) {
        if (!b->in_l[i]) return b->fail(DS_INVALID_ARGUMENT, "pair " + std::to_string(i) + " has no bound input");
        if (b->desc[i].raw && !b->calib[b->desc[i].calib].map[0])
            return b->fail(DS_INVALID_ARGUMENT, "pair " + std::to_string(i) + ": set_rectification() not called");
    }
    cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : b->stream;
    return batch_guarded(b, [&]() -> int {
        if (b->args_dirty) batch_fill_args(b);
        if (!b->exec) {
            // Capture once on the batch's own stream; the graph reads the per-pair argument arrays, so
            // later bindings change what it processes without a new capture.
            DS_CUDA(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
            try {
                batch_enqueue(b, b->stream, true);
            } catch (...) {
                cudaGraph_t g = nullptr;
                cudaStreamEndCapture(b->stream, &g);
                if (g) cudaGraphDestroy(g);
                throw;
            }
            DS_CUDA(cudaStreamEndCapture(b->stream, &b->graph));
            DS_CUDA(cudaGraphInstantiate(&b->exec, b->graph, 0));
        }
        DS_CUDA(cudaGraphLaunch(b->exec, st));
        return DS_OK;
    });
}

DS_API int ds_batch_run_eager(ds_batch* b, void* stream) {
    if (!b) return DS_INVALID_ARGUMENT;
    cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : b->stream;
    return batch_guarded(b, [&]() -> int {
        if (b->args_dirty) batch_fill_args(b);
        batch_enqueue(b, st, false);
        return DS_OK;
    });
}

DS_API size_t ds_batch_device_bytes(const ds_batch* b) { return b ? b->bytes : 0; }

DS_API int ds_batch_profile(ds_batch* b, int on) {
    if (!b) return DS_INVALID_ARGUMENT;
    return batch_guarded(b, [&]() -> int {
        if ((on != 0) == b->profile) return DS_OK;
        if (on && !b->ev[0])
            for (auto& e : b->ev) DS_CUDA(cudaEventCreate(&e));
        b->profile = on != 0;
        if (b->exec) {  // the stage events are part of the captured graph: capture again
            DS_CUDA(cudaStreamSynchronize(b->stream));
            cudaGraphExecDestroy(b->exec);
            cudaGraphDestroy(b->graph);
            b->exec = nullptr;
            b->graph = nullptr;
        }
        return DS_OK;
    });
}

DS_API int ds_batch_stage_ms(ds_batch* b, double* ms) {
    if (!b || !ms) return DS_INVALID_ARGUMENT;
    if (!b->profile) return b->fail(DS_INVALID_ARGUMENT, "ds_batch_profile() not enabled");
    return batch_guarded(b, [&]() -> int {
        DS_CUDA(cudaEventSynchronize(b->ev[DS_BATCH_STAGES]));
        for (int i = 0; i < DS_BATCH_STAGES; ++i) {
            float t = 0.0f;
            DS_CUDA(cudaEventElapsedTime(&t, b->ev[i], b->ev[i + 1]));
            ms[i] = t;
        }
        return DS_OK;
    });
}

DS_API int ds_batch_launches_per_run(const ds_batch* b) {
    if (!b) return 0;
    int n = 0;
    for (const auto& m : b->micro) n += m.launches();
    return n;
}

DS_API int ds_batch_get_options(const ds_batch* b, ds_batch_options* out) {
    if (!b || !out) return DS_INVALID_ARGUMENT;
    out->micro_batch = b->micro_batch;
    out->branches = b->branches;
    return DS_OK;
}

}  // extern "C"
