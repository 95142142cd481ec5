// Device-side descent shared by the point, range and forest kernels.
//
// A query is served by a group of G lanes of one warp.  At an internal level
// the group reads the node's 128-byte line with 16-byte vector loads (F/G
// separators per lane), counts the separators below the query, and combines
// the per-lane counts with one warp ballot and one shuffle: because the line
// is sorted, the lanes whose whole chunk is below the query form a prefix,
// so count = KPL * (#full lanes) + (count of the first non-full lane).  The
// child index is node*F + count.  Each group works on I queries at once
// (independent dependency chains), so several line loads are in flight per
// group.  The top levels are read from shared memory, the rest from global
// memory (L2-resident in practice), in two separate loops so each uses its
// native load instruction.
//
// The reference walks 80 KB pages by scalar binary search, one thread per
// query, about 13 dependent 8-byte loads per level plus a leafFlag load on
// another page per level (BPTreeExactSearch.cu:39-68).  Here each level costs
// one coalesced line per query and the top levels come from shared memory.
#pragma once

#include "bt_internal.cuh"

namespace bt {

// Loads NB bytes (4, 8, or a multiple of 16; aligned) from p into v.
template <int NB>
__device__ __forceinline__ void load_bytes(const void *p, uint32_t (&v)[NB / 4]) {
    if constexpr (NB == 4) {
        v[0] = *reinterpret_cast<const uint32_t *>(p);
    } else if constexpr (NB == 8) {
        uint2 x = *reinterpret_cast<const uint2 *>(p);
        v[0] = x.x;
        v[1] = x.y;
    } else {
        static_assert(NB % 16 == 0, "chunk must be 4, 8 or a multiple of 16 bytes");
#pragma unroll
        for (int i = 0; i < NB / 16; i++) {
            uint4 x = reinterpret_cast<const uint4 *>(p)[i];
            v[4 * i] = x.x;
            v[4 * i + 1] = x.y;
            v[4 * i + 2] = x.z;
            v[4 * i + 3] = x.w;
        }
    }
}

// 16-byte load of data touched once per query (leaf blocks): read-only path,
// no L1 allocation, so L1 keeps the separator lines.
__device__ __forceinline__ uint4 load_stream16(const void *p) {
    uint4 x;
    asm volatile("ld.global.nc.L1::no_allocate.v4.b32 {%0,%1,%2,%3}, [%4];"
                 : "=r"(x.x), "=r"(x.y), "=r"(x.z), "=r"(x.w)
                 : "l"(p));
    return x;
}

template <typename K>
__device__ __forceinline__ K key_at(const uint32_t *w, int i) {
    if constexpr (sizeof(K) == 4) {
        return w[i];
    } else {
        return ((uint64_t)w[2 * i + 1] << 32) | w[2 * i];
    }
}

// Keys among the NK packed in w that are below q (or not above q, upper).
template <typename K, int NK>
__device__ __forceinline__ int count_below(const uint32_t *w, K q, bool upper) {
    int c = 0;
#pragma unroll
    for (int i = 0; i < NK; i++) {
        const K k = key_at<K>(w, i);
        c += upper ? (k <= q) : (k < q);
    }
    return c;
}

// Combine per-lane counts of a sorted chunk spread over the first ACT lanes
// of a G-lane group (each lane holds NK keys).  All 32 lanes must call it;
// every lane of the group receives the result.
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

// One level for I queries: node[s] <- node[s]*F + (separators of the node
// below qe[s]).
template <typename K, int G, int I>
__device__ __forceinline__ void level_step(const K *__restrict__ lp, const K (&qe)[I],
                                           const bool (&upper)[I], uint32_t (&node)[I], int grp,
                                           int gl) {
    constexpr int F = kLineBytes / (int)sizeof(K);
    constexpr int KPL = F / G;
    constexpr int NB = KPL * (int)sizeof(K);
    uint32_t c[I][NB / 4];
#pragma unroll
    for (int s = 0; s < I; s++) load_bytes<NB>(lp + (size_t)node[s] * F + gl * KPL, c[s]);
#pragma unroll
    for (int s = 0; s < I; s++) {
        const int cnt = count_below<K, KPL>(c[s], qe[s], upper[s]);
        node[s] = node[s] * F + group_count<G, G, KPL>(cnt, true, grp);
    }
}

// Walks all separator levels.  qe[s] must satisfy qe[s] <= max_key (lower
// bound) or qe[s] < max_key (upper bound) for the walk to stay on real
// separators.  On return node[s] is the leaf block index.
template <typename K, int G, int I>
__device__ __forceinline__ void descend(const DevTree &t, const K *__restrict__ s_top,
                                        const K (&qe)[I], const bool (&upper)[I],
                                        uint32_t (&node)[I], int grp, int gl) {
#pragma unroll
    for (int s = 0; s < I; s++) node[s] = 0;
    int lvl = 0;
    for (; lvl < t.smem_levels; lvl++) level_step<K, G, I>(s_top + t.lvl_off[lvl], qe, upper, node, grp, gl);
    const K *gseps = static_cast<const K *>(t.seps);
    for (; lvl < t.nlevels; lvl++) level_step<K, G, I>(gseps + t.lvl_off[lvl], qe, upper, node, grp, gl);
}

// Stages the top separator levels into shared memory (16-byte copies).
template <typename K>
__device__ __forceinline__ void stage_top(K *s_top, const DevTree &t) {
    const uint4 *src = static_cast<const uint4 *>(t.seps);
    uint4 *dst = reinterpret_cast<uint4 *>(s_top);
    const uint32_t n16 = (uint32_t)((t.smem_elems * sizeof(K)) / 16);
    for (uint32_t i = threadIdx.x; i < n16; i += blockDim.x) dst[i] = src[i];
}

// Leaf stage for one leaf block: the 32-byte key sector is NKC = 2 chunks of
// 16 bytes; the value part is NVC chunks.  Chunk c is held by lane c % G of
// the group (CPL chunks per lane).  Returns the lower/upper-bound position
// inside the block, and (for lower bounds) whether the key there equals q.
template <typename K, typename V, int G>
struct LeafStage {
    using LG = LeafGeom<K, V>;
    static constexpr int KPC = 16 / (int)sizeof(K);      // keys per chunk
    static constexpr int VPC = 16 / (int)sizeof(V);      // values per chunk
    static constexpr int NKC = kSectorBytes / 16;        // key chunks (2)
    static constexpr int NVC = (LG::VB + 15) / 16;       // value chunks
    static constexpr int NC = NKC + NVC;
    static constexpr int CPL = (NC + G - 1) / G;         // chunks per lane (values too)
    static constexpr int KCPL = (NKC + G - 1) / G;       // key chunks per lane
};

}  // namespace bt
