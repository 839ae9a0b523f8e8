// The C++ host side (include/depth_cuda.hpp) driven as a frontend would drive MetalStereo: create, compute,
// error codes. Input: a case file written by tests/test_cpp_host.py (int32 w, h, min_disparity,
// num_disparities, subpixel, median; u8 left and right images; f32 expected disparity). Exit 0 when the
// disparity matches bit for bit and the error paths answer the reference's codes.
#include <cstdio>
#include <cstring>
#include <vector>

#include "depth_cuda.hpp"

int main(int argc, char** argv) {
    if (argc != 2) {
        std::fprintf(stderr, "usage: %s CASE_FILE\n", argv[0]);
        return 2;
    }
    std::FILE* f = std::fopen(argv[1], "rb");
    if (!f) return 2;
    int hdr[6];
    if (std::fread(hdr, sizeof(int), 6, f) != 6) return 2;
    const int w = hdr[0], h = hdr[1];
    const std::size_t n = static_cast<std::size_t>(w) * h;
    std::vector<std::uint8_t> left(n), right(n);
    std::vector<float> want(n);
    if (std::fread(left.data(), 1, n, f) != n || std::fread(right.data(), 1, n, f) != n ||
        std::fread(want.data(), sizeof(float), n, f) != n)
        return 2;
    std::fclose(f);

    depth_cuda::StereoParams p;
    p.sgm.min_disparity = hdr[2];
    p.sgm.num_disparities = hdr[3];
    p.subpixel = hdr[4] != 0;
    p.median = hdr[5] != 0;
    auto s = depth_cuda::CudaStereo::create(p, w, h);
    if (!s) {
        std::fprintf(stderr, "create failed: %s\n", s.error().message.c_str());
        return 1;
    }
    const depth_cuda::ImageViewU8 l{left.data(), w, h, w}, r{right.data(), w, h, w};
    int bad = 0;
    for (int rep = 0; rep < 2; ++rep) {  // repeated frames give identical bytes
        auto res = (*s)->compute(l, r);
        if (!res) {
            std::fprintf(stderr, "compute failed: %s\n", res.error().message.c_str());
            return 1;
        }
        if (std::memcmp(res->disparity.data(), want.data(), n * sizeof(float)) != 0) {
            std::fprintf(stderr, "disparity differs from the expected bytes (frame %d)\n", rep);
            bad = 1;
        }
        std::size_t valid = 0;
        for (std::size_t i = 0; i < n; ++i) valid += res->confidence[i] == 1.0f;
        if (valid == 0) bad = 1;
    }
    if ((*s)->last_timings().gpu_ms <= 0.0) bad = 1;
    // wrong image size: invalid_argument (metal_stereo.cpp:235-236)
    if (auto res = (*s)->compute({left.data(), w - 1, h, w}, {right.data(), w - 1, h, w});
        res || res.error().code != depth_cuda::Errc::invalid_argument)
        bad = 1;
    // too many disparities: invalid_argument (metal_stereo.cpp:115)
    depth_cuda::StereoParams big = p;
    big.sgm.num_disparities = 600;
    if (auto c = depth_cuda::CudaStereo::create(big, w, h); c || c.error().code != depth_cuda::Errc::invalid_argument) bad = 1;
    // depth::compute_disparity's refinement: one pyramid level runs; five are out of range
    depth_cuda::StereoParams pyr = p;
    pyr.pyramid_levels = 1;
    pyr.sgm.min_disparity = p.sgm.min_disparity / 2 - 2;
    pyr.sgm.num_disparities = p.sgm.num_disparities / 2 + 4;
    pyr.filter_spikes = true;
    pyr.speckle_max_region_size = 20;
    if (auto c = depth_cuda::CudaStereo::create(pyr, w, h); !c) {
        bad = 1;
    } else if (auto res = (*c)->compute(l, r); !res) {
        bad = 1;
    } else {
        std::size_t valid = 0;
        for (std::size_t i = 0; i < n; ++i) valid += res->disparity[i] > -1.0e8f && res->confidence[i] > 0.0f;
        if (valid == 0) bad = 1;
    }
    pyr.pyramid_levels = 5;
    if (auto c = depth_cuda::CudaStereo::create(pyr, w, h); c || c.error().code != depth_cuda::Errc::invalid_argument) bad = 1;
    // marker blob search: find_blobs before set_blob_params is invalid_argument; afterwards it runs
    if (auto b = (*s)->find_blobs(l); b || b.error().code != depth_cuda::Errc::invalid_argument) bad = 1;
    if (!(*s)->set_blob_params({})) bad = 1;
    std::uint32_t found = 0;
    if (auto b = (*s)->find_blobs(l, &found); !b || b->size() != std::min<std::uint32_t>(found, 1024)) bad = 1;
    // compute_raw before set_rectification: invalid_argument (metal_stereo.cpp:343)
    if (auto res = (*s)->compute_raw(l, r); res || res.error().code != depth_cuda::Errc::invalid_argument) bad = 1;
    // the frontend's call (identity remap tables at the stereo size): compute_frame gives compute_raw's
    // disparity, and its marker candidates are find_blobs' of each raw image
    depth_cuda::RemapTable id{w, h, std::vector<float>(n), std::vector<float>(n)};
    for (int y = 0; y < h; ++y)
        for (int x = 0; x < w; ++x) {
            id.map_x[static_cast<std::size_t>(y) * w + x] = static_cast<float>(x);
            id.map_y[static_cast<std::size_t>(y) * w + x] = static_cast<float>(y);
        }
    if (!(*s)->set_rectification(id, id, w, h)) bad = 1;
    int callbacks = 0;
    depth_cuda::FrameRequest req;
    req.marker_blobs = true;
    req.on_blobs = [&](const std::array<std::vector<depth_cuda::BlobBox>, 2>&) { ++callbacks; };
    auto plain = (*s)->compute_raw(l, r);
    auto frame = (*s)->compute_frame(l, r, req);
    if (!plain || !frame || callbacks != 1) {
        std::fprintf(stderr, "compute_frame failed or on_blobs not called once\n");
        bad = 1;
    } else {
        if (std::memcmp(plain->disparity.data(), frame->disparity.data(), n * sizeof(float)) != 0) {
            std::fprintf(stderr, "compute_frame disparity differs from compute_raw's\n");
            bad = 1;
        }
        auto bl = (*s)->find_blobs(l), br = (*s)->find_blobs(r);
        if (!bl || !br || bl->size() != frame->blobs[0].size() || br->size() != frame->blobs[1].size()) {
            std::fprintf(stderr, "compute_frame blob counts differ from find_blobs'\n");
            bad = 1;
        }
        else
            for (int side = 0; side < 2; ++side) {
                const auto& want = side == 0 ? *bl : *br;
                if (!want.empty() && std::memcmp(want.data(), frame->blobs[side].data(), want.size() * sizeof(depth_cuda::BlobBox)) != 0)
                    bad = 1;
            }
    }
    std::printf(bad ? "FAIL\n" : "OK\n");
    return bad;
}
