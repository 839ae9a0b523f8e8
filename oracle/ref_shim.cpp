// C entry points over the reference CPU stereo, compiled from the reference's own unmodified
// libs/depth/src/stereo.cpp (included below, so that the anonymous-namespace median3 is reachable).
// Built by oracle/Makefile into oracle/_ref/ only; never shipped. Test infrastructure: the tests,
// the smoke check and the bench's CPU baseline use it as the checker / the timed reference arm.
//
// Entry points:
//   ref_census        -> depth::census_transform      (libs/depth/src/stereo.cpp:328-346)
//   ref_sgm_disparity -> depth::sgm_disparity         (libs/depth/src/stereo.cpp:361-463)
//   ref_median3       -> (anonymous) median3          (libs/depth/src/stereo.cpp:129-147)
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

int ref_threads() { return tbb::stub_detail::Pool::instance().threads(); }

}  // extern "C"
