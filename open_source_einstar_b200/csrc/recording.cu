// Raw IR images of a session recording on the device: the RAWI record stores each image row delta-coded
// from its left neighbour (byte minus the byte before it, mod 256, the first byte as is), then zstd
// (libs/session/src/session.cpp:248-272). After zstd decompression on the host, the rows are undone here:
// every output byte is the running sum of its row's coded bytes, mod 256 (session.cpp:829-833).
//
// One warp per row, 512 bytes per step: each lane sums 16 consecutive bytes, the warp scans the lane sums
// by shuffles, and the carry of the previous step is added to the whole step. Sums are taken in 32-bit
// integers and reduced mod 256 at the store, which is the same as adding bytes with wrap-around.
#include <cuda_runtime.h>

#include "../../include/depth_cuda.h"
#include "dispatch.h"

namespace {

constexpr int kRowsPerBlock = 4;

__global__ void k_undelta_rows(const uint8_t* in, ptrdiff_t in_stride, uint8_t* out, ptrdiff_t out_stride, int w, int h) {
    const int row = blockIdx.x * kRowsPerBlock + static_cast<int>(threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (row >= h) return;  // the whole warp leaves together
    const uint8_t* src = in + row * in_stride;
    uint8_t* dst = out + row * out_stride;
    uint32_t carry = 0;
    for (int base = 0; base < w; base += 32 * 16) {
        const int x0 = base + lane * 16;
        uint32_t v[16];
        uint32_t run = 0;
#pragma unroll
        for (int k = 0; k < 16; ++k) {
            run += x0 + k < w ? src[x0 + k] : 0u;
            v[k] = run;
        }
        uint32_t scan = run;  // inclusive scan of the lanes' sums
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const uint32_t t = __shfl_up_sync(0xFFFFFFFFu, scan, d);
            if (lane >= d) scan += t;
        }
        const uint32_t before = carry + scan - run;
#pragma unroll
        for (int k = 0; k < 16; ++k)
            if (x0 + k < w) dst[x0 + k] = static_cast<uint8_t>((before + v[k]) & 0xFFu);
        carry += __shfl_sync(0xFFFFFFFFu, scan, 31);
    }
}

}  // namespace

extern "C" {

DS_API int ds_undelta_rows(const uint8_t* coded, ptrdiff_t coded_stride, uint8_t* image, ptrdiff_t image_stride, int width, int height,
                           void* stream) {
    if (!coded || !image) {
        ds::set_global_error("null argument");
        return DS_INVALID_ARGUMENT;
    }
    if (width < 1 || height < 1 || width > 65536 || height > 65536 || coded_stride < width || image_stride < width) {
        ds::set_global_error("image size must be 1..65536 and strides at least the width");
        return DS_INVALID_ARGUMENT;
    }
    if (coded == image && coded_stride != image_stride) {
        ds::set_global_error("in place (coded == image) needs equal strides");
        return DS_INVALID_ARGUMENT;
    }
    const int blocks = (height + kRowsPerBlock - 1) / kRowsPerBlock;
    k_undelta_rows<<<blocks, 32 * kRowsPerBlock, 0, static_cast<cudaStream_t>(stream)>>>(coded, coded_stride, image, image_stride,
                                                                                         width, height);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        ds::set_global_error(cudaGetErrorString(e));
        return DS_IO;
    }
    ds::count_launches(1);
    return DS_OK;
}

}  // extern "C"
