// Minimal stand-in for oneTBB's blocked_range, used only to compile the reference CPU stereo
// (libs/depth/src/stereo.cpp) for the oracle and the CPU baseline. oneTBB is not installed on this
// image. Test infrastructure, not product code.
#pragma once

#include <cstddef>

namespace tbb {

template <typename T>
class blocked_range {
public:
    blocked_range(T begin, T end, std::size_t grain = 1) : begin_(begin), end_(end), grain_(grain) {}
    T begin() const { return begin_; }
    T end() const { return end_; }
    std::size_t size() const { return static_cast<std::size_t>(end_ - begin_); }
    std::size_t grainsize() const { return grain_; }
    bool empty() const { return !(begin_ < end_); }

private:
    T begin_, end_;
    std::size_t grain_;
};

}  // namespace tbb
