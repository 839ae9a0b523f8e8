// Row-sweep WTA (wta_kernels.cuh) launchers: one frame and batches.
#include "batch_common.cuh"
#include "dispatch.h"
#include "wta_kernels.cuh"

namespace ds {

namespace {
constexpr int kWtaRowPF = 1;

int wta_rows_per_block(int seg, int lg_chunks) { return (dsk::kWtaRowWarps * 32 / seg) >> lg_chunks; }

template <int R, int SEG, bool PAD>
cudaError_t frame_t(const dsk::WtaRowArgs& a, cudaStream_t st) {
    const int rows = wta_rows_per_block(SEG, a.lg_chunks);
    dsk::k_wta_rows<R, SEG, kWtaRowPF, PAD><<<(a.h + rows - 1) / rows, 32 * dsk::kWtaRowWarps, 0, st>>>(a);
    return cudaGetLastError();
}

template <int R, int SEG, bool PAD>
cudaError_t batch_t(const dsk::WtaRowArgs* args, const BatchGroupDev& g, cudaStream_t st) {
    dsk::kb_wta_rows<R, SEG, kWtaRowPF, PAD><<<g.total, 32 * dsk::kWtaRowWarps, 0, st>>>(args, g.pairs, g.prefix, g.n, g.total);
    return cudaGetLastError();
}

template <bool PAD>
cudaError_t frame_p(int R, int seg, const dsk::WtaRowArgs& a, cudaStream_t st) {
    if (R == 6) return seg == 4 ? frame_t<6, 4, PAD>(a, st) : frame_t<6, 8, PAD>(a, st);
    return seg == 4 ? frame_t<8, 4, PAD>(a, st) : frame_t<8, 8, PAD>(a, st);
}

template <bool PAD>
cudaError_t batch_p(int R, int seg, const dsk::WtaRowArgs* args, const BatchGroupDev& g, cudaStream_t st) {
    if (R == 6) return seg == 4 ? batch_t<6, 4, PAD>(args, g, st) : batch_t<6, 8, PAD>(args, g, st);
    return seg == 4 ? batch_t<8, 4, PAD>(args, g, st) : batch_t<8, 8, PAD>(args, g, st);
}
}  // namespace

bool wta_rows_shape(int dp, int& R, int& seg) {
    switch (dp) {
        case 48: R = 6, seg = 4; return true;
        case 64: R = 8, seg = 4; return true;
        case 96: R = 6, seg = 8; return true;
        case 128: R = 8, seg = 8; return true;
        default: return false;
    }
}

bool wta_rows_layout(int w, int dp, int& chunk, int& lg_chunks, int& sets) {
    int R = 0, seg = 0;
    if (!wta_rows_shape(dp, R, seg) || w < 1) return false;
    // The most chunks (a power of two up to the block's segments) whose chunks keep at least dp / 4 columns
    // (and 16): a right pixel's dp candidate columns then touch at most 5 chunks.
    const int segs = dsk::kWtaRowWarps * 32 / seg, min_cols = std::max((dp + 3) / 4, 16);
    lg_chunks = 0;
    while ((2 << lg_chunks) <= segs && w / (2 << lg_chunks) >= min_cols) ++lg_chunks;
    const int nch = 1 << lg_chunks;
    chunk = (w + nch - 1) / nch;
    sets = nch == 1 ? 1 : std::min(nch, (dp - 1 + chunk - 1) / chunk + 1);
    return sets <= dsk::kWtaRowMaxSets;
}

cudaError_t launch_wta_rows(const dsk::WtaRowArgs& a, cudaStream_t st) {
    int R = 0, seg = 0;
    if (!wta_rows_shape(a.dp, R, seg) || a.sets < 1 || a.sets > dsk::kWtaRowMaxSets ||
        (1 << a.lg_chunks) > dsk::kWtaRowWarps * 32 / seg)
        return cudaErrorInvalidValue;
    return a.nd < a.dp ? frame_p<true>(R, seg, a, st) : frame_p<false>(R, seg, a, st);
}

cudaError_t launch_wta_rows_batch(int dp, bool pad, const dsk::WtaRowArgs* args, const BatchGroupDev& g, cudaStream_t st) {
    int R = 0, seg = 0;
    if (!wta_rows_shape(dp, R, seg)) return cudaErrorInvalidValue;
    return pad ? batch_p<true>(R, seg, args, g, st) : batch_p<false>(R, seg, args, g, st);
}

}  // namespace ds
