// Device-side descent shared by the point, range and forest kernels.
//
// A query is served by a group of G lanes of one warp.  At an internal level
// the group reads the node's 128-byte line with one 16-byte vector load per
// lane (F/G separators each), counts the separators below the query, and
// combines the per-lane counts with one warp ballot and one shuffle: because
// the line is sorted, the lanes whose whole chunk is below the query form a
// prefix, so count = KPL * (#full lanes) + (count of the first non-full
// lane).  The child index is node*F + count.  Each group works on I queries
// at once (independent dependency chains) so that several line loads are in
// flight per group.
//
// The reference walks 80 KB pages by scalar binary search, one thread per
// query, about 13 dependent 8-byte loads per level plus a leafFlag load on
// another page per level (BPTreeExactSearch.cu:39-68).  Here each level costs
// one coalesced line per query and the top levels come from shared memory.
#pragma once

#include "bt_internal.cuh"

namespace bt {

template <int BYTES>
struct VecOf;
template <>
struct VecOf<4> { using T = uint32_t; };
template <>
struct VecOf<8> { using T = uint2; };
template <>
struct VecOf<16> { using T = uint4; };

// Loads NK consecutive keys (NK*sizeof(K) in {4, 8, 16, 32} bytes, aligned).
template <typename K, int NK>
__device__ __forceinline__ void load_keys(const K *p, K (&v)[NK]) {
    constexpr int B = NK * (int)sizeof(K);
    if constexpr (B <= 16) {
        using VT = typename VecOf<B>::T;
        VT x = *reinterpret_cast<const VT *>(p);
        memcpy(v, &x, B);
    } else {
        static_assert(B % 16 == 0, "chunk must be a multiple of 16 bytes");
#pragma unroll
        for (int i = 0; i < B / 16; i++) {
            uint4 x = reinterpret_cast<const uint4 *>(p)[i];
            memcpy(reinterpret_cast<char *>(v) + 16 * i, &x, 16);
        }
    }
}

// Same for data in HBM that is touched once per query: read-only path, no L1
// allocation (keeps L1 for the separator lines).
template <typename T, int NK>
__device__ __forceinline__ void load_stream(const T *p, T (&v)[NK]) {
    constexpr int B = NK * (int)sizeof(T);
    if constexpr (B == 4) {
        uint32_t x;
        asm volatile("ld.global.nc.L1::no_allocate.b32 %0, [%1];" : "=r"(x) : "l"(p));
        memcpy(v, &x, 4);
    } else if constexpr (B == 8) {
        uint2 x;
        asm volatile("ld.global.nc.L1::no_allocate.v2.b32 {%0,%1}, [%2];"
                     : "=r"(x.x), "=r"(x.y) : "l"(p));
        memcpy(v, &x, 8);
    } else {
        static_assert(B % 16 == 0, "chunk must be 4, 8 or a multiple of 16 bytes");
#pragma unroll
        for (int i = 0; i < B / 16; i++) {
            uint4 x;
            asm volatile("ld.global.nc.L1::no_allocate.v4.b32 {%0,%1,%2,%3}, [%4];"
                         : "=r"(x.x), "=r"(x.y), "=r"(x.z), "=r"(x.w)
                         : "l"(reinterpret_cast<const char *>(p) + 16 * i));
            memcpy(reinterpret_cast<char *>(v) + 16 * i, &x, 16);
        }
    }
}

// Number of keys in v below q (upper == false) or not above q (upper == true).
template <typename K, int NK>
__device__ __forceinline__ int count_below(const K (&v)[NK], K q, bool upper) {
    int c = 0;
#pragma unroll
    for (int i = 0; i < NK; i++) c += upper ? (v[i] <= q) : (v[i] < q);
    return c;
}

// Combine per-lane counts of a sorted chunk spread over the first ACT lanes
// of a G-lane group (each lane holds NK keys).  All 32 lanes must call it.
template <int G, int ACT, int NK>
__device__ __forceinline__ int group_count(int cnt, bool active, int grp) {
    if constexpr (G == 1) {
        return cnt;
    } else {
        const unsigned full = __ballot_sync(0xffffffffu, active && cnt == NK);
        const unsigned gmask = (G == 32 ? 0xffffffffu : ((1u << G) - 1u)) << (grp * G);
        const int nfull = __popc(full & gmask);
        const int src = grp * G + (nfull < ACT ? nfull : ACT - 1);
        const int part = __shfl_sync(0xffffffffu, cnt, src);
        return nfull * NK + (nfull < ACT ? part : 0);
    }
}

// Walks the separator levels for I queries per group.  qe[s] must satisfy
// qe[s] <= max_key (lower) or qe[s] < max_key (upper) for the walk to stay on
// real separators.  On return node[s] is the leaf sector index.
template <typename K, int G, int I>
__device__ __forceinline__ void descend(const DevTree &t, const K *__restrict__ s_top,
                                        const K (&qe)[I], const bool (&upper)[I],
                                        uint64_t (&node)[I], int grp, int gl) {
    constexpr int F = kLineBytes / (int)sizeof(K);
    constexpr int KPL = F / G;
    const K *gseps = static_cast<const K *>(t.seps);
#pragma unroll
    for (int s = 0; s < I; s++) node[s] = 0;
    for (int lvl = 0; lvl < t.nlevels; lvl++) {
        const K *lp = (lvl < t.smem_levels ? s_top : gseps) + t.lvl_off[lvl];
        K c[I][KPL];
#pragma unroll
        for (int s = 0; s < I; s++) load_keys<K, KPL>(lp + node[s] * F + gl * KPL, c[s]);
#pragma unroll
        for (int s = 0; s < I; s++) {
            const int cnt = count_below<K, KPL>(c[s], qe[s], upper[s]);
            node[s] = node[s] * F + group_count<G, G, KPL>(cnt, true, grp);
        }
    }
}

// Stages the top separator levels into shared memory (16-byte copies).
template <typename K>
__device__ __forceinline__ void stage_top(K *s_top, const DevTree &t) {
    const uint4 *src = static_cast<const uint4 *>(t.seps);
    uint4 *dst = reinterpret_cast<uint4 *>(s_top);
    const uint32_t n16 = (uint32_t)((t.smem_elems * sizeof(K)) / 16);
    for (uint32_t i = threadIdx.x; i < n16; i += blockDim.x) dst[i] = src[i];
}

}  // namespace bt
