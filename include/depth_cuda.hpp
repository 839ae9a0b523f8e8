// C++ host side of libdepth_cuda: the reference's GPU stereo-matcher interface
// (depth_metal::MetalStereo, libs/depth_metal/include/einstar/depth_metal/metal_stereo.hpp:67-107) over the
// C ABI in depth_cuda.h. A frontend written against MetalStereo switches to CudaStereo with the same calls:
// create / set_rectification / compute / compute_raw / set_point_params / last_timings, with errors
// carried as the reference's Errc values (libs/core/include/einstar/core/error.hpp:8-19).
//
// Header-only; link with libdepth_cuda.so. Requires C++23 (std::expected, as the reference).
#pragma once

#include <array>
#include <cstddef>
#include <cstdint>
#include <expected>
#include <functional>
#include <memory>
#include <string>
#include <utility>
#include <vector>

#include "depth_cuda.h"

namespace depth_cuda {

// einstar::Errc (same values as ds_status).
enum class Errc {
    ok = DS_OK,
    not_found = DS_NOT_FOUND,
    io = DS_IO,
    timeout = DS_TIMEOUT,
    protocol = DS_PROTOCOL,
    invalid_argument = DS_INVALID_ARGUMENT,
    blocked = DS_BLOCKED,
    unsupported = DS_UNSUPPORTED,
    busy = DS_BUSY,
    disconnected = DS_DISCONNECTED,
};

struct Error {
    Errc code;
    std::string message;
};

template <typename T>
using Result = std::expected<T, Error>;

// depth::SgmParams (libs/depth/include/einstar/depth/stereo.hpp:26-40) with the reference's defaults.
struct SgmParams {
    int min_disparity = 0;
    int num_disparities = 64;
    int census_radius_x = 2;
    int census_radius_y = 2;
    int p1 = 8;
    int p2 = 96;
    bool adaptive_p2 = true;
    bool eight_paths = false;
    bool slant_steps = true;
    float uniqueness = 0.9f;
    int lr_max_diff = 1;
};

// depth::RefineParams, depth::DetailParams (libs/depth/include/einstar/depth/stereo.hpp:42-63).
struct RefineParams {
    int search_radius = 2;
    int zncc_radius = 3;
    float min_zncc = 0.5f;
    bool reject_edge_winners = true;
};

struct DetailParams {
    int radius = 5;
    float search = 1.0f;
    float step = 0.5f;
    float min_zncc = 0.5f;
};

// depth::StereoParams with this library's defaults: the hot path (pyramid 0, the later stages off).
// pyramid_levels > 0, detail_enabled, the filters or speckle_max_region_size > 1 run the whole of
// depth::compute_disparity (refinement, detail, filters, speckles; see ds_stereo_params).
struct StereoParams {
    int pyramid_levels = 0;
    SgmParams sgm;
    bool subpixel = true;
    bool median = true;
    bool detail_enabled = false;
    bool filter_occlusion = false;
    bool filter_spikes = false;
    int speckle_max_region_size = 0;
    bool wide_costs = false;
    RefineParams refine;
    DetailParams detail;
    float occlusion_tolerance = 1.0f;
    float spike_threshold = 1.0f;
    float speckle_max_diff = 1.0f;
};

// depth_metal::BlobParams / BlobBox (libs/depth_metal/include/einstar/depth_metal/metal_stereo.hpp:21-39).
struct BlobParams {
    std::uint32_t threshold = 150;
    std::uint32_t min_diameter = 3, max_diameter = 60;
    float max_aspect = 4.0f;
    float min_fill = 0.5f;
    std::uint32_t border = 4;
    float max_axis_ratio = 3.0f;
    float ring_scale = 1.4f;
    float ring_contrast = 0.5f;
    float ring_max_bright = 0.3f;
    std::uint32_t max_blobs = 1024;
};
using BlobBox = ds_blob_box;

// depth::RectifiedGeometry (libs/depth/include/einstar/depth/point_image.hpp:12-26).
struct RectifiedGeometry {
    double f = 0, cx = 0, cy = 0, baseline = 0, cx_offset = 0;
};

// depth_metal::StereoTimings (metal_stereo.hpp:61-65).
struct StereoTimings {
    double gpu_ms = 0, speckle_ms = 0, total_ms = 0;
};

// An 8-bit image in host memory: rows `stride` bytes apart.
struct ImageViewU8 {
    const std::uint8_t* data = nullptr;
    int width = 0, height = 0;
    std::ptrdiff_t stride = 0;
};

// calib::RemapTable (libs/calib/include/einstar/calib/rectify.hpp:40-44): float32 source coordinates.
struct RemapTable {
    int width = 0, height = 0;
    std::vector<float> map_x, map_y;
};

// depth::StereoResult plus this library's u16 disparity and depth (empty when not requested).
struct StereoResult {
    int width = 0, height = 0;
    std::vector<float> disparity, confidence;
    std::vector<std::uint16_t> disparity_u16;
    std::vector<float> depth;
    // compute_raw with marker blobs: candidates of the left and right raw images and how many passed
    // (depth_metal::FrameOutputs::blobs / blobs_found).
    std::array<std::vector<BlobBox>, 2> blobs;
    std::array<std::uint32_t, 2> blobs_found{};
};

// depth_metal::FrameRequest (metal_stereo.hpp:41-50), the parts a CUDA frame has.
struct FrameRequest {
    bool marker_blobs = false;
    std::function<void(const std::array<std::vector<BlobBox>, 2>&)> on_blobs;
};

// The device buffers a frame's points, normals (float4 per pixel) and weights go to (gpu::MetalFrameData).
struct DeviceFrame {
    float* points_xyzw = nullptr;
    float* normals_xyzw = nullptr;
    float* weights = nullptr;
};

class CudaStereo {
public:
    static Result<std::unique_ptr<CudaStereo>> create(const StereoParams& p, int width, int height) {
        const ds_stereo_params c = to_c(p);
        ds_handle* h = nullptr;
        if (const int rc = ds_create(&c, width, height, &h); rc != DS_OK)
            return std::unexpected(Error{static_cast<Errc>(rc), ds_last_global_error()});
        return std::unique_ptr<CudaStereo>(new CudaStereo(h, width, height));
    }
    ~CudaStereo() { ds_destroy(h_); }
    CudaStereo(const CudaStereo&) = delete;
    CudaStereo& operator=(const CudaStereo&) = delete;

    [[nodiscard]] int width() const { return w_; }
    [[nodiscard]] int height() const { return h_px_; }

    Result<void> set_rectification(const RemapTable& left, const RemapTable& right, int raw_width, int raw_height) {
        if (left.width != right.width || left.height != right.height)
            return std::unexpected(Error{Errc::invalid_argument, "left and right remap tables differ in size"});
        return check(ds_set_rectification(h_, left.map_x.data(), left.map_y.data(), right.map_x.data(), right.map_y.data(),
                                          left.width, left.height, raw_width, raw_height));
    }

    void set_point_params(const RectifiedGeometry& g, float min_depth_mm, float max_depth_mm,
                          float max_depth_jump_mm = 4.0f) {
        const ds_geometry dg{g.f, g.cx, g.cy, g.baseline, g.cx_offset};
        ds_set_point_params(h_, &dg, min_depth_mm, max_depth_mm, max_depth_jump_mm);
        have_points_ = true;
    }

    Result<StereoResult> compute(ImageViewU8 left, ImageViewU8 right) { return run(left, right, false, nullptr, nullptr); }

    Result<StereoResult> compute_raw(ImageViewU8 raw_left, ImageViewU8 raw_right, std::vector<std::uint8_t>* rect_left = nullptr,
                                     std::vector<std::uint8_t>* rect_right = nullptr) {
        return run(raw_left, raw_right, true, rect_left, rect_right);
    }

    // MetalStereo::set_blob_params: enables compute_raw(..., marker_blobs = true) and find_blobs.
    Result<void> set_blob_params(const BlobParams& p) {
        const ds_blob_params c{p.threshold, p.min_diameter, p.max_diameter, p.max_aspect, p.min_fill, p.border,
                               p.max_axis_ratio, p.ring_scale, p.ring_contrast, p.ring_max_bright, p.max_blobs};
        if (auto r = check(ds_set_blob_params(h_, &c)); !r) return r;
        max_blobs_ = p.max_blobs;
        return {};
    }

    // Raw pair -> stereo, with the marker blob search on both raw images (FrameRequest::marker_blobs).
    Result<StereoResult> compute_raw_blobs(ImageViewU8 raw_left, ImageViewU8 raw_right) {
        return run(raw_left, raw_right, true, nullptr, nullptr, true);
    }

    // MetalStereo::compute_frame, the frontend's per-frame call: raw pair in; points, normals (float4 per pixel)
    // and weights written to the caller's device buffers (all three, or none); the host result as compute_raw;
    // with marker_blobs, the candidates in res.blobs, and on_blobs called with them (on this thread) as soon
    // as the blob search has finished, while the stereo may still run.
    Result<StereoResult> compute_frame(ImageViewU8 raw_left, ImageViewU8 raw_right, const FrameRequest& req, DeviceFrame frame = {}) {
        if (!raw_left.data || !raw_right.data || raw_left.stride != raw_right.stride)
            return std::unexpected(Error{Errc::invalid_argument, "null images or different strides"});
        const std::size_t n = static_cast<std::size_t>(w_) * h_px_;
        StereoResult res;
        res.width = w_;
        res.height = h_px_;
        res.disparity.resize(n);
        res.confidence.resize(n);
        res.disparity_u16.resize(n);
        if (have_points_) res.depth.resize(n);
        ds_frame_outputs o{};
        o.points_xyzw = frame.points_xyzw;
        o.normals_xyzw = frame.normals_xyzw;
        o.weights = frame.weights;
        o.host = ds_outputs{res.disparity.data(), res.confidence.data(), res.disparity_u16.data(), have_points_ ? res.depth.data() : nullptr,
                            nullptr, nullptr};
        ds_blob_boxes bb{};
        struct Ctx {
            const FrameRequest* req;
            StereoResult* res;
        } ctx{&req, &res};
        ds_frame_request r{};
        if (req.marker_blobs) {
            res.blobs[0].resize(max_blobs_);
            res.blobs[1].resize(max_blobs_);
            bb = ds_blob_boxes{res.blobs[0].data(), res.blobs[1].data(), max_blobs_, {0, 0}, {0, 0}};
            o.blobs = &bb;
            r.marker_blobs = 1;
            r.user = &ctx;
            r.on_blobs = [](const ds_blob_boxes* b, void* user) {
                auto* c = static_cast<Ctx*>(user);
                c->res->blobs[0].resize(b->kept[0]);
                c->res->blobs[1].resize(b->kept[1]);
                c->res->blobs_found = {b->found[0], b->found[1]};
                if (c->req->on_blobs) c->req->on_blobs(c->res->blobs);
            };
        }
        if (const int rc = ds_compute_frame(h_, raw_left.data, raw_right.data, raw_left.stride, &r, &o); rc != DS_OK)
            return std::unexpected(Error{static_cast<Errc>(rc), ds_last_error(h_)});
        return res;
    }

    // The blob search alone on one image: candidates ordered by first pixel.
    Result<std::vector<BlobBox>> find_blobs(ImageViewU8 img, std::uint32_t* found = nullptr) {
        std::vector<BlobBox> out(max_blobs_);
        std::uint32_t f = 0, k = 0;
        if (auto r = check(ds_find_blobs(h_, img.data, img.width, img.height, img.stride, out.data(), max_blobs_, &f, &k)); !r)
            return std::unexpected(r.error());
        out.resize(k);
        if (found) *found = f;
        return out;
    }

    const StereoTimings& last_timings() {
        ds_timings t{};
        ds_last_timings(h_, &t);
        timings_ = {t.gpu_ms, t.speckle_ms, t.total_ms};
        return timings_;
    }

private:
    CudaStereo(ds_handle* h, int w, int ht) : h_(h), w_(w), h_px_(ht) {}

    static ds_stereo_params to_c(const StereoParams& p) {
        ds_stereo_params c{};
        ds_default_params(&c);
        c.pyramid_levels = p.pyramid_levels;
        c.sgm = {p.sgm.min_disparity, p.sgm.num_disparities, p.sgm.census_radius_x, p.sgm.census_radius_y, p.sgm.p1, p.sgm.p2,
                 p.sgm.adaptive_p2, p.sgm.eight_paths, p.sgm.slant_steps, p.sgm.uniqueness, p.sgm.lr_max_diff};
        c.subpixel = p.subpixel;
        c.median = p.median;
        c.detail_enabled = p.detail_enabled;
        c.filter_occlusion = p.filter_occlusion;
        c.filter_spikes = p.filter_spikes;
        c.speckle_max_region_size = p.speckle_max_region_size;
        c.wide_costs = p.wide_costs;
        c.refine_search_radius = p.refine.search_radius;
        c.refine_zncc_radius = p.refine.zncc_radius;
        c.refine_min_zncc = p.refine.min_zncc;
        c.refine_reject_edge_winners = p.refine.reject_edge_winners;
        c.detail_radius = p.detail.radius;
        c.detail_search = p.detail.search;
        c.detail_step = p.detail.step;
        c.detail_min_zncc = p.detail.min_zncc;
        c.occlusion_tolerance = p.occlusion_tolerance;
        c.spike_threshold = p.spike_threshold;
        c.speckle_max_diff = p.speckle_max_diff;
        return c;
    }

    Result<void> check(int rc) const {
        if (rc == DS_OK) return {};
        return std::unexpected(Error{static_cast<Errc>(rc), ds_last_error(h_)});
    }

    Result<StereoResult> run(ImageViewU8 l, ImageViewU8 r, bool raw, std::vector<std::uint8_t>* rl,
                             std::vector<std::uint8_t>* rr, bool blobs = false) {
        if (!l.data || !r.data) return std::unexpected(Error{Errc::invalid_argument, "null image"});
        if (l.stride != r.stride || l.width != r.width || l.height != r.height)
            return std::unexpected(Error{Errc::invalid_argument, "left and right images differ in size or stride"});
        if (!raw && (l.width != w_ || l.height != h_px_))
            return std::unexpected(Error{Errc::invalid_argument, "image size does not match the configured size"});
        const std::size_t n = static_cast<std::size_t>(w_) * h_px_;
        StereoResult res;
        res.width = w_;
        res.height = h_px_;
        res.disparity.resize(n);
        res.confidence.resize(n);
        res.disparity_u16.resize(n);
        if (have_points_) res.depth.resize(n);
        if (rl) rl->resize(n);
        if (rr) rr->resize(n);
        ds_outputs o{res.disparity.data(), res.confidence.data(), res.disparity_u16.data(),
                     have_points_ ? res.depth.data() : nullptr, rl ? rl->data() : nullptr, rr ? rr->data() : nullptr};
        int rc = DS_OK;
        if (blobs) {
            res.blobs[0].resize(max_blobs_);
            res.blobs[1].resize(max_blobs_);
            ds_blob_boxes bb{res.blobs[0].data(), res.blobs[1].data(), max_blobs_, {0, 0}, {0, 0}};
            rc = ds_compute_raw_blobs(h_, l.data, r.data, l.stride, &o, &bb);
            res.blobs[0].resize(bb.kept[0]);
            res.blobs[1].resize(bb.kept[1]);
            res.blobs_found = {bb.found[0], bb.found[1]};
        } else {
            rc = raw ? ds_compute_raw(h_, l.data, r.data, l.stride, &o) : ds_compute(h_, l.data, r.data, l.stride, &o);
        }
        if (rc != DS_OK) return std::unexpected(Error{static_cast<Errc>(rc), ds_last_error(h_)});
        return res;
    }

    ds_handle* h_;
    int w_, h_px_;
    bool have_points_ = false;
    std::uint32_t max_blobs_ = 1024;
    StereoTimings timings_;
};

}  // namespace depth_cuda
