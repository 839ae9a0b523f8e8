// Packed 16-bit lane arithmetic (two path values per 32-bit register) and byte packing helpers.
// add/min/max on .u16x2 are native sm_90+/sm_100a instructions; 16-bit lanes wrap independently,
// so subtracting s is adding (0x10000 - s) to each lane.
#pragma once

#include <cstdint>

namespace dsk {

__device__ __forceinline__ uint32_t vmin2(uint32_t a, uint32_t b) {
    uint32_t r;
    asm("min.u16x2 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(b));
    return r;
}
__device__ __forceinline__ uint32_t vmax2(uint32_t a, uint32_t b) {
    uint32_t r;
    asm("max.u16x2 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(b));
    return r;
}
__device__ __forceinline__ uint32_t vadd2(uint32_t a, uint32_t b) {
    uint32_t r;
    asm("add.u16x2 %0, %1, %2;" : "=r"(r) : "r"(a), "r"(b));
    return r;
}
__device__ __forceinline__ uint32_t splat2(uint32_t v) { return (v & 0xFFFFu) * 0x00010001u; }
__device__ __forceinline__ uint32_t prmt(uint32_t a, uint32_t b, uint32_t sel) { return __byte_perm(a, b, sel); }
// (hi half of a, lo half of b): the pair shifted down by one 16-bit lane across two registers.
__device__ __forceinline__ uint32_t mid2(uint32_t a, uint32_t b) { return __byte_perm(a, b, 0x5432); }
__device__ __forceinline__ uint32_t lo16(uint32_t a) { return a & 0xFFFFu; }
__device__ __forceinline__ uint32_t hi16(uint32_t a) { return a >> 16; }
__device__ __forceinline__ uint32_t hmin2(uint32_t a) { return min(a & 0xFFFFu, a >> 16); }

// ---- per-lane chunks of NV path values (u8 or u16 storage) --------------------------------------
// A chunk is NV * sizeof(ST) bytes at a lane-aligned offset; it is moved as 32-bit words (2-byte units
// when its size is 2 or 6 bytes) and converted to / from R = NV/2 registers of two 16-bit lanes.
// Load modes: LD_NC read-only path (data not written during the kernel), LD_CS streaming (evict-first,
// coherent), LD_CG L2-coherent (data another thread of the block wrote earlier in the same kernel).
// Stores: STREAM selects evict-first.

enum LoadMode { LD_NC = 0, LD_CS = 1, LD_CG = 2 };

template <LoadMode M, typename T>
__device__ __forceinline__ T ld_mode(const T* p) {
    if constexpr (M == LD_NC) return __ldg(p);
    else if constexpr (M == LD_CS) return __ldcs(p);
    else return __ldcg(p);
}

template <int BYTES>
__host__ __device__ constexpr int chunk_words() { return (BYTES + 3) / 4; }

template <int BYTES, int MODE>
__device__ __forceinline__ void ld_chunk(const void* __restrict__ p, uint32_t (&w)[chunk_words<BYTES>()]) {
    constexpr LoadMode M = static_cast<LoadMode>(MODE);
    if constexpr (BYTES == 2 || BYTES == 6) {
        const unsigned short* q = static_cast<const unsigned short*>(p);
        uint32_t h[BYTES / 2];
#pragma unroll
        for (int i = 0; i < BYTES / 2; ++i) h[i] = ld_mode<M>(q + i);
        w[0] = BYTES == 2 ? h[0] : (h[0] | (h[BYTES == 2 ? 0 : 1] << 16));
        if constexpr (BYTES == 6) w[1] = h[2];
    } else if constexpr (BYTES % 16 == 0) {
        const uint4* q = static_cast<const uint4*>(p);
#pragma unroll
        for (int i = 0; i < BYTES / 16; ++i) {
            const uint4 v = ld_mode<M>(q + i);
            w[4 * i] = v.x, w[4 * i + 1] = v.y, w[4 * i + 2] = v.z, w[4 * i + 3] = v.w;
        }
    } else if constexpr (BYTES % 8 == 0) {
        const uint2* q = static_cast<const uint2*>(p);
#pragma unroll
        for (int i = 0; i < BYTES / 8; ++i) {
            const uint2 v = ld_mode<M>(q + i);
            w[2 * i] = v.x, w[2 * i + 1] = v.y;
        }
    } else {
        const unsigned int* q = static_cast<const unsigned int*>(p);
#pragma unroll
        for (int i = 0; i < BYTES / 4; ++i) w[i] = ld_mode<M>(q + i);
    }
}

template <int BYTES, bool STREAM>
__device__ __forceinline__ void st_chunk(void* __restrict__ p, const uint32_t (&w)[chunk_words<BYTES>()]) {
    if constexpr (BYTES == 2 || BYTES == 6) {
        unsigned short* q = static_cast<unsigned short*>(p);
        const unsigned short h[3] = {static_cast<unsigned short>(w[0]), static_cast<unsigned short>(w[0] >> 16),
                                     static_cast<unsigned short>(BYTES == 6 ? w[BYTES == 6 ? 1 : 0] : 0u)};
#pragma unroll
        for (int i = 0; i < BYTES / 2; ++i) {
            if (STREAM) __stcs(q + i, h[i]);
            else q[i] = h[i];
        }
    } else if constexpr (BYTES % 16 == 0) {
        uint4* q = static_cast<uint4*>(p);
#pragma unroll
        for (int i = 0; i < BYTES / 16; ++i) {
            const uint4 v = make_uint4(w[4 * i], w[4 * i + 1], w[4 * i + 2], w[4 * i + 3]);
            if (STREAM) __stcs(q + i, v);
            else q[i] = v;
        }
    } else if constexpr (BYTES % 8 == 0) {
        uint2* q = static_cast<uint2*>(p);
#pragma unroll
        for (int i = 0; i < BYTES / 8; ++i) {
            const uint2 v = make_uint2(w[2 * i], w[2 * i + 1]);
            if (STREAM) __stcs(q + i, v);
            else q[i] = v;
        }
    } else {
        unsigned int* q = static_cast<unsigned int*>(p);
#pragma unroll
        for (int i = 0; i < BYTES / 4; ++i) {
            if (STREAM) __stcs(q + i, w[i]);
            else q[i] = w[i];
        }
    }
}

// words of a (ST, NV) chunk -> R = NV/2 registers of (value k, value k+1) as 16-bit lanes
template <typename ST, int NV>
__device__ __forceinline__ void unpack(const uint32_t (&w)[chunk_words<NV * sizeof(ST)>()], uint32_t (&r)[NV / 2]) {
    if constexpr (sizeof(ST) == 2) {
#pragma unroll
        for (int i = 0; i < NV / 2; ++i) r[i] = w[i];
    } else {
#pragma unroll
        for (int i = 0; i < NV / 2; ++i) r[i] = prmt(w[i / 2], 0u, (i & 1) ? 0x4342 : 0x4140);
    }
}

template <typename ST, int NV>
__device__ __forceinline__ void pack(const uint32_t (&r)[NV / 2], uint32_t (&w)[chunk_words<NV * sizeof(ST)>()]) {
    if constexpr (sizeof(ST) == 2) {
#pragma unroll
        for (int i = 0; i < NV / 2; ++i) w[i] = r[i];
    } else {
#pragma unroll
        for (int i = 0; i < NV / 4; ++i) w[i] = prmt(r[2 * i], r[2 * i + 1], 0x6420);
        if constexpr ((NV / 2) % 2) w[NV / 4] = prmt(r[NV / 2 - 1], 0u, 0x0020);
    }
}

}  // namespace dsk
