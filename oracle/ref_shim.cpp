// C entry points over the reference CPU stereo, compiled from the reference's own unmodified
// libs/depth/src/stereo.cpp (included below, so that the anonymous-namespace median3 is reachable).
// Built by oracle/Makefile into oracle/_ref/ only; never shipped. Test infrastructure: the tests,
// the smoke check and the bench's CPU baseline use it as the checker / the timed reference arm.
//
// Entry points:
//   ref_census        -> depth::census_transform      (libs/depth/src/stereo.cpp:328-346)
//   ref_sgm_disparity -> depth::sgm_disparity         (libs/depth/src/stereo.cpp:361-463)
//   ref_median3       -> (anonymous) median3          (libs/depth/src/stereo.cpp:129-147)
//   ref_downsample2   -> depth::downsample2           (libs/depth/src/stereo.cpp:348-359)
//   ref_refine_level  -> (anonymous) refine_level      (libs/depth/src/stereo.cpp:151-207)
//   ref_refine_detail -> depth::refine_detail          (libs/depth/src/stereo.cpp:243-284)
//   ref_filter_disparity -> depth::filter_disparity    (libs/depth/src/stereo.cpp:286-326)
//   ref_remove_speckles  -> depth::remove_speckles     (libs/depth/src/stereo.cpp:465-494)
//   ref_compute_disparity -> depth::compute_disparity  (libs/depth/src/stereo.cpp:501-536)
//   ref_threads       -> worker count of the TBB stand-in pool (oracle/tbb_stub)

#include "stereo.cpp"  // NOLINT: the reference translation unit, from the reference tree

#include <cstdint>
#include <cstring>

extern "C" {

// Plain-C mirror of depth::SgmParams (libs/depth/include/einstar/depth/stereo.hpp:26-40).
struct ref_sgm_params {
    int min_disparity;
    int num_disparities;
    int census_radius_x;
    int census_radius_y;
    int p1;
    int p2;
    int adaptive_p2;
    int eight_paths;
    int slant_steps;
    float uniqueness;
    int lr_max_diff;
};

int ref_census(const std::uint8_t* img, int w, int h, int rx, int ry, std::uint64_t* out) {
    const einstar::ImageView<const std::uint8_t> v(img, w, h);
    const auto c = einstar::depth::census_transform(v, rx, ry);
    std::memcpy(out, c.data(), c.size() * sizeof(std::uint64_t));
    return 0;
}

int ref_sgm_disparity(const std::uint8_t* left, const std::uint8_t* right, int w, int h, const ref_sgm_params* p, int subpixel,
                      float* out) {
    einstar::depth::SgmParams sp;
    sp.min_disparity = p->min_disparity;
    sp.num_disparities = p->num_disparities;
    sp.census_radius_x = p->census_radius_x;
    sp.census_radius_y = p->census_radius_y;
    sp.p1 = p->p1;
    sp.p2 = p->p2;
    sp.adaptive_p2 = p->adaptive_p2 != 0;
    sp.eight_paths = p->eight_paths != 0;
    sp.slant_steps = p->slant_steps != 0;
    sp.uniqueness = p->uniqueness;
    sp.lr_max_diff = p->lr_max_diff;
    const einstar::ImageView<const std::uint8_t> l(left, w, h), r(right, w, h);
    const auto d = einstar::depth::sgm_disparity(l, r, sp, subpixel != 0);
    std::memcpy(out, d.data(), d.size() * sizeof(float));
    return 0;
}

int ref_median3(const float* in, int w, int h, float* out) {
    einstar::ImageF32 img(w, h);
    std::memcpy(img.data(), in, img.size() * sizeof(float));
    const auto m = einstar::depth::median3(img);
    std::memcpy(out, m.data(), m.size() * sizeof(float));
    return 0;
}

// Plain-C mirror of depth::StereoParams (libs/depth/include/einstar/depth/stereo.hpp:41-88).
struct ref_stereo_params {
    int pyramid_levels;
    ref_sgm_params sgm;
    int refine_search_radius, refine_zncc_radius;
    float refine_min_zncc;
    int refine_reject_edge_winners;
    int detail_enabled, detail_radius;
    float detail_search, detail_step, detail_min_zncc;
    int filter_occlusion;
    float filter_occlusion_tolerance;
    int filter_spikes;
    float filter_spike_threshold;
    int speckle_max_region_size;
    float speckle_max_diff;
    int subpixel;
};

static einstar::depth::StereoParams to_params(const ref_stereo_params* p) {
    einstar::depth::StereoParams sp;
    sp.pyramid_levels = p->pyramid_levels;
    const ref_sgm_params& g = p->sgm;
    sp.sgm.min_disparity = g.min_disparity;
    sp.sgm.num_disparities = g.num_disparities;
    sp.sgm.census_radius_x = g.census_radius_x;
    sp.sgm.census_radius_y = g.census_radius_y;
    sp.sgm.p1 = g.p1;
    sp.sgm.p2 = g.p2;
    sp.sgm.adaptive_p2 = g.adaptive_p2 != 0;
    sp.sgm.eight_paths = g.eight_paths != 0;
    sp.sgm.slant_steps = g.slant_steps != 0;
    sp.sgm.uniqueness = g.uniqueness;
    sp.sgm.lr_max_diff = g.lr_max_diff;
    sp.refine.search_radius = p->refine_search_radius;
    sp.refine.zncc_radius = p->refine_zncc_radius;
    sp.refine.min_zncc = p->refine_min_zncc;
    sp.refine.reject_edge_winners = p->refine_reject_edge_winners != 0;
    sp.detail.enabled = p->detail_enabled != 0;
    sp.detail.radius = p->detail_radius;
    sp.detail.search = p->detail_search;
    sp.detail.step = p->detail_step;
    sp.detail.min_zncc = p->detail_min_zncc;
    sp.filter.occlusion = p->filter_occlusion != 0;
    sp.filter.occlusion_tolerance = p->filter_occlusion_tolerance;
    sp.filter.spikes = p->filter_spikes != 0;
    sp.filter.spike_threshold = p->filter_spike_threshold;
    sp.speckle.max_region_size = p->speckle_max_region_size;
    sp.speckle.max_diff = p->speckle_max_diff;
    sp.subpixel = p->subpixel != 0;
    return sp;
}

static einstar::ImageF32 to_image(const float* d, int w, int h) {
    einstar::ImageF32 img(w, h);
    std::memcpy(img.data(), d, img.size() * sizeof(float));
    return img;
}

int ref_downsample2(const std::uint8_t* in, int w, int h, std::uint8_t* out) {
    const auto o = einstar::depth::downsample2(einstar::ImageView<const std::uint8_t>(in, w, h));
    std::memcpy(out, o.data(), o.size());
    return 0;
}

// `coarse` is cw x ch (the next coarser level), left/right and the outputs w x h.
int ref_refine_level(const std::uint8_t* left, const std::uint8_t* right, int w, int h, const float* coarse, int cw, int ch,
                     const ref_stereo_params* p, float* disp, float* conf) {
    const auto sp = to_params(p);
    einstar::ImageF32 d, c;
    einstar::depth::refine_level(einstar::ImageView<const std::uint8_t>(left, w, h),
                                 einstar::ImageView<const std::uint8_t>(right, w, h), to_image(coarse, cw, ch), sp.refine,
                                 sp.subpixel, d, c);
    std::memcpy(disp, d.data(), d.size() * sizeof(float));
    std::memcpy(conf, c.data(), c.size() * sizeof(float));
    return 0;
}

// disparity (w x h) in place; full images W x H.
int ref_refine_detail(const std::uint8_t* full_left, const std::uint8_t* full_right, int W, int H, float* disp, int w, int h,
                      const ref_stereo_params* p) {
    const auto sp = to_params(p);
    auto d = to_image(disp, w, h);
    einstar::depth::refine_detail(einstar::ImageView<const std::uint8_t>(full_left, W, H),
                                  einstar::ImageView<const std::uint8_t>(full_right, W, H), d, sp.detail, sp.subpixel);
    std::memcpy(disp, d.data(), d.size() * sizeof(float));
    return 0;
}

int ref_filter_disparity(float* disp, int w, int h, const ref_stereo_params* p) {
    const auto sp = to_params(p);
    auto d = to_image(disp, w, h);
    einstar::depth::filter_disparity(d, sp.filter);
    std::memcpy(disp, d.data(), d.size() * sizeof(float));
    return 0;
}

int ref_remove_speckles(float* disp, int w, int h, const ref_stereo_params* p) {
    const auto sp = to_params(p);
    auto d = to_image(disp, w, h);
    einstar::depth::remove_speckles(d, sp.speckle);
    std::memcpy(disp, d.data(), d.size() * sizeof(float));
    return 0;
}

// full_left / full_right: NULL, or the 2w x 2h images left / right were box-downsampled from.
int ref_compute_disparity(const std::uint8_t* left, const std::uint8_t* right, int w, int h, const std::uint8_t* full_left,
                          const std::uint8_t* full_right, const ref_stereo_params* p, float* disp, float* conf) {
    const auto sp = to_params(p);
    const einstar::ImageView<const std::uint8_t> l(left, w, h), r(right, w, h);
    einstar::depth::StereoResult res;
    if (full_left && full_right)
        res = einstar::depth::compute_disparity(l, r, einstar::ImageView<const std::uint8_t>(full_left, 2 * w, 2 * h),
                                                einstar::ImageView<const std::uint8_t>(full_right, 2 * w, 2 * h), sp);
    else
        res = einstar::depth::compute_disparity(l, r, sp);
    std::memcpy(disp, res.disparity.data(), res.disparity.size() * sizeof(float));
    std::memcpy(conf, res.confidence.data(), res.confidence.size() * sizeof(float));
    return 0;
}

int ref_threads() { return tbb::stub_detail::Pool::instance().threads(); }

}  // extern "C"
