// Pieces shared by the persistent batch launches (launchers.cuh) and the batch host code.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>

namespace dsk {

__device__ __forceinline__ int batch_find(const int* __restrict__ prefix, int n, int v) {
    int lo = 0, hi = n;
    while (hi - lo > 1) {
        const int m = (lo + hi) >> 1;
        if (__ldg(prefix + m) <= v) lo = m;
        else hi = m;
    }
    return lo;
}

}  // namespace dsk

namespace ds {

struct BatchGroupDev {
    const int* pairs;
    const int* prefix;
    const int* gx;
    int n, total, grid;
};

template <typename K>
int persistent_grid(K k, int threads, size_t smem, int total) {
    int dev = 0, sms = 0, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k, threads, smem) != cudaSuccess || per_sm < 1) per_sm = 1;
    return std::max(1, std::min(total, sms * per_sm));
}

}  // namespace ds
