// Connected components by union-find over a pixel grid (speckle regions, marker blobs). Labels are linear
// pixel indexes; a root is only ever hung under a smaller root, so every component ends with its first
// pixel in raster order as root. Every loop is bounded; a bound that runs out sets *err.
#pragma once

namespace dsk {

constexpr int kFindLimit = 1 << 22;

// Root of x with path halving. Every parent index is at most its child's, so a halving store written
// concurrently with other finds or unions still names an ancestor. While unions run (kLinking) reads
// bypass L1 so that roots linked by other blocks are seen; afterwards roots no longer change and cached
// reads find them.
template <bool kLinking>
__device__ __forceinline__ int uf_find(int* parent, int x, int* err) {
    for (int it = 0; it < kFindLimit; ++it) {
        const int p = kLinking ? __ldcg(parent + x) : parent[x];
        if (p == x) return x;
        const int gp = kLinking ? __ldcg(parent + p) : parent[p];
        if (gp != p) parent[x] = gp;
        x = gp;
    }
    *err = 1;
    return x;
}

// Joins the components of pixels i and j: the larger root is hung under the smaller, unless another
// thread changed that root's parent first (then the walk continues from its new parent).
__device__ __forceinline__ void uf_union(int* parent, int i, int j, int* err) {
    int a = i, b = j;
    for (int it = 0; it < kFindLimit; ++it) {
        a = uf_find<true>(parent, a, err);
        b = uf_find<true>(parent, b, err);
        if (a == b) return;
        if (a < b) {
            const int t = a;
            a = b;
            b = t;
        }
        const int old = atomicCAS(&parent[a], a, b);
        if (old == a) return;
        a = old;
    }
    *err = 1;
}

// ---- two-level labelling: tiles in shared memory, then the links across tile borders -----------------------
// k_ccl_tiles labels each row of a 32 x 16 tile by horizontal runs (one warp ballot), unites the runs
// vertically in shared memory (same rule: the larger root under the smaller) and writes every active pixel's parent as the global index of its tile-local root, the first
// pixel of that tile component in raster order (raster order inside a tile is raster order of the image).
// k_ccl_borders then joins components across the right and bottom tile borders with the global union-find.
// Only border pixels touch global atomics. `Conn` says which pixels take part (active) and which
// 4-neighbours are connected (link, symmetric).
constexpr int kTileW = 32, kTileH = 16, kTileLimit = 4 * kTileW * kTileH;

__device__ __forceinline__ int tile_find(volatile int* L, int x, int* err) {
    for (int it = 0; it < kTileLimit; ++it) {
        const int p = L[x];
        if (p == x) return x;
        x = p;
    }
    *err = 1;
    return x;
}

__device__ __forceinline__ void tile_union(int* L, int i, int j, int* err) {
    volatile int* V = L;
    int a = i, b = j;
    for (int it = 0; it < kTileLimit; ++it) {
        a = tile_find(V, a, err);
        b = tile_find(V, b, err);
        if (a == b) return;
        if (a < b) {
            const int t = a;
            a = b;
            b = t;
        }
        const int old = atomicCAS(&L[a], a, b);
        if (old == a) return;
        a = old;
    }
    *err = 1;
}

template <class Conn>
static __global__ void __launch_bounds__(kTileW * kTileH) k_ccl_tiles(Conn c, int w, int h, int* parent, int* err) {
    __shared__ int L[kTileW * kTileH];
    const int tx = threadIdx.x, ty = threadIdx.y, li = ty * kTileW + tx;
    const int x = blockIdx.x * kTileW + tx, y = blockIdx.y * kTileH + ty;
    const bool act = x < w && y < h && c.active(x, y);
    // Each warp is one tile row: a pixel's horizontal run starts after the last lane below it that does not
    // link to its right neighbour, so runs are labelled by their first pixel without any union.
    const bool right = act && tx + 1 < kTileW && x + 1 < w && c.link(x, y, x + 1, y);
    const unsigned links = __ballot_sync(0xFFFFFFFFu, right);
    const unsigned breaks = ~links & ((1u << tx) - 1u);
    const int start = breaks ? 32 - __clz(breaks) : 0;
    L[li] = act ? ty * kTileW + start : -1;
    __syncthreads();
    if (act && ty + 1 < kTileH && y + 1 < h && c.link(x, y, x, y + 1)) tile_union(L, li, li + kTileW, err);
    __syncthreads();
    if (act) {
        const int r = tile_find(L, li, err);
        parent[static_cast<size_t>(y) * w + x] = (blockIdx.y * kTileH + r / kTileW) * w + blockIdx.x * kTileW + r % kTileW;
    }
}

// One thread per tile-border pixel: threads [0, nr * h) take the right border columns x = 32 k + 31 (row-major
// over (y, k)), the rest the bottom border rows y = 16 k + 15. A link is skipped when the pixel before it along
// the border (above for a column, to the left for a row) has the same link and is connected to both of its
// ends by links inside a tile: the two ends are then joined through links that k_ccl_tiles makes and the
// border link before it (made, or itself skipped on the same grounds). Links across a tile corner are never
// skipped on the strength of one another, so no two skips rely on each other.
template <class Conn>
static __global__ void k_ccl_borders(Conn c, int w, int h, int nr, int nb, int* parent, int* err) {
    const long t = static_cast<long>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t < static_cast<long>(nr) * h) {
        const int y = static_cast<int>(t / nr), x = static_cast<int>(t % nr) * kTileW + kTileW - 1;
        if (x + 1 >= w || !c.active(x, y) || !c.link(x, y, x + 1, y)) return;
        if (y % kTileH != 0 && c.active(x, y - 1) && c.link(x, y - 1, x + 1, y - 1) && c.link(x, y - 1, x, y) && c.link(x + 1, y - 1, x + 1, y))
            return;
        uf_union(parent, y * w + x, y * w + x + 1, err);
        return;
    }
    const long u = t - static_cast<long>(nr) * h;
    if (u >= static_cast<long>(nb) * w) return;
    const int y = static_cast<int>(u / w) * kTileH + kTileH - 1, x = static_cast<int>(u % w);
    if (y + 1 >= h || !c.active(x, y) || !c.link(x, y, x, y + 1)) return;
    if (x % kTileW != 0 && c.active(x - 1, y) && c.link(x - 1, y, x - 1, y + 1) && c.link(x - 1, y, x, y) && c.link(x - 1, y + 1, x, y + 1)) return;
    uf_union(parent, y * w + x, (y + 1) * w + x, err);
}

// Launch of both kernels for a w x h grid on `st`; returns the number of kernels launched.
template <class Conn>
inline int launch_ccl(const Conn& c, int w, int h, int* parent, int* err, cudaStream_t st) {
    const dim3 tiles((w + kTileW - 1) / kTileW, (h + kTileH - 1) / kTileH);
    k_ccl_tiles<<<tiles, dim3(kTileW, kTileH), 0, st>>>(c, w, h, parent, err);
    const int nr = (w - 1) / kTileW, nb = (h - 1) / kTileH;  // border columns / rows with a neighbour beyond
    const long n = static_cast<long>(nr) * h + static_cast<long>(nb) * w;
    if (n == 0) return 1;
    k_ccl_borders<<<static_cast<unsigned>((n + 255) / 256), 256, 0, st>>>(c, w, h, nr, nb, parent, err);
    return 2;
}

}  // namespace dsk
