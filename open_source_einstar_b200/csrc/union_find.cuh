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

}  // namespace dsk
