// Device-side descent shared by the point, range and forest kernels.
//
// Two phases per warp tile of 32 queries:
//
//  1. One thread per query.  The CTA stages in shared memory the deepest
//     separator level that fits (for 2^26 u32 keys: the 8,192 maxima of the
//     third level, 32 KB) and each lane runs a branchless binary search over
//     it.  That single search resolves every level above the staged one and
//     yields the node index on the first level below it; the query loads are
//     coalesced and nothing crosses lanes.
//  2. G lanes per query.  The remaining levels live in global memory (L2 in
//     practice).  The group reads a node's 128-byte line with 16-byte vector
//     loads (F/G separators per lane), counts the separators below the query,
//     and combines the per-lane counts with one warp ballot and one shuffle:
//     the line is sorted, so the lanes whose whole chunk is below the query
//     form a prefix, and count = KPL * (#full lanes) + (count of the first
//     non-full lane).  The child is node*F + count.  The warp's 32 queries
//     pass in R rounds, each group keeping G/R queries in flight.
//
// The reference walks 80 KB pages by scalar binary search, one thread per
// query, about 13 dependent 8-byte loads per level plus a leafFlag load on
// another page per level (BPTreeExactSearch.cu:39-68).
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

// L2 policy for data touched once per query: its lines are the first the
// L2 evicts, so the separator levels and the result lines stay resident.
__device__ __forceinline__ uint64_t l2_evict_first() {
    uint64_t pol;
    asm("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
    return pol;
}

// 16-byte load of data touched once per query (leaf blocks): read-only path,
// no L1 allocation (L1 keeps the separator lines), evict-first in L2.
__device__ __forceinline__ uint4 load_stream16(const void *p) {
    uint4 x;
    asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.v4.b32 {%0,%1,%2,%3}, [%4], %5;"
                 : "=r"(x.x), "=r"(x.y), "=r"(x.z), "=r"(x.w)
                 : "l"(p), "l"(l2_evict_first()));
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

// Walks the separator levels below the staged one.  qe[s] must satisfy
// qe[s] <= max_key (lower bound) or qe[s] < max_key (upper bound) for the walk
// to stay on real separators.  On entry node[s] is the node index on level
// smem_level + 1 (phase 1's result); on return it is the leaf block index.
template <typename K, int G, int I>
__device__ __forceinline__ void walk_from(const DevTree &t, int from, const K (&qe)[I],
                                          const bool (&upper)[I], uint32_t (&node)[I], int grp,
                                          int gl) {
    const K *gseps = static_cast<const K *>(t.seps);
    for (int lvl = from; lvl < t.nlevels; lvl++)
        level_step<K, G, I>(gseps + t.lvl_off[lvl], qe, upper, node, grp, gl);
}

template <typename K, int G, int I>
__device__ __forceinline__ void walk_global(const DevTree &t, const K (&qe)[I],
                                            const bool (&upper)[I], uint32_t (&node)[I], int grp,
                                            int gl) {
    walk_from<K, G, I>(t, t.smem_level + 1, qe, upper, node, grp, gl);
}

// Leaf block holding the lower bound of q (q <= max key) by one thread:
// every separator line from the root, scanned whole.
template <typename K>
__device__ __forceinline__ uint32_t block_lower_bound(const DevTree &t, K q) {
    constexpr int F = kLineBytes / (int)sizeof(K);
    const K *seps = static_cast<const K *>(t.seps);
    uint32_t node = 0;
    for (int lvl = 0; lvl < t.nlevels; lvl++) {
        const K *line = seps + t.lvl_off[lvl] + (size_t)node * F;
        uint32_t c = 0;
#pragma unroll
        for (int i = 0; i < F; i++) c += line[i] < q ? 1u : 0u;
        node = node * F + c;
    }
    return node;
}

// Shared-memory slot of sorted element p.  A binary search over 2^k
// elements probes positions that differ by multiples of large powers of two,
// which in a plain array all fall into one bank (a 32-way conflict per
// probe).  XOR-ing the bank bits with two higher bit fields spreads every
// such probe set over distinct banks.  It only permutes elements within each
// row of one bank width, so it is a bijection on [0, n).
template <typename K>
__device__ __forceinline__ uint32_t swz(uint32_t p) {
    constexpr int B = sizeof(K) == 4 ? 5 : 4;  // log2(elements per bank row)
    constexpr uint32_t M = (1u << B) - 1u;
    return p ^ (((p >> B) ^ (p >> (2 * B))) & M);
}

// Branchless lower (upper) bound over n >= 1 sorted keys in shared memory
// (stored swizzled): the first index i with s[i] >= q (s[i] > q), n if none.
template <typename K>
__device__ __forceinline__ uint32_t smem_bound(const K *__restrict__ s, uint32_t n, K q,
                                               bool upper) {
    uint32_t base = 0;
    while (n > 1) {
        const uint32_t half = n >> 1;
        const K v = s[swz<K>(base + half)];
        base = (upper ? v <= q : v < q) ? base + half : base;
        n -= half;
    }
    const K v = s[swz<K>(base)];
    return base + ((upper ? v <= q : v < q) ? 1u : 0u);
}

// Stages the binary-searched separator level into shared memory, swizzled.
// The staged region is padded to whole bank rows with all-ones keys.
template <typename K>
__device__ __forceinline__ void stage_level(K *s_lvl, const DevTree &t) {
    const K *src = static_cast<const K *>(t.seps) + t.lvl_off[t.smem_level];
    const uint32_t n = t.smem_bytes / sizeof(K);
    for (uint32_t i = threadIdx.x; i < n; i += blockDim.x)
        s_lvl[swz<K>(i)] = i < t.smem_entries ? src[i] : key_max<K>();
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

// No found flags (leaf_point's default).
struct NoFound {
    __device__ uint8_t *operator()(int) const { return nullptr; }
};

// Leaf stage of I point queries.  Each query's leaf block (key chunks, then
// value chunks) is loaded by its lane group with 16-byte streaming loads, the
// lower-bound slot and the match are found, and the lane holding the value
// writes it -- or all-ones on a miss -- to dst(s), and 1 or 0 to fdst(s)
// when that is not null; dst returns null to skip a slot.  leaves points at
// leaf block 0 of the tree; node[s] is the block.
template <typename K, typename V, int G, int I, typename Dst, typename FDst = NoFound>
__device__ __forceinline__ void leaf_point(const unsigned char *__restrict__ leaves,
                                           const uint32_t (&node)[I], const K (&qv)[I],
                                           const K (&qe)[I], K tmax, int grp, int gl, Dst dst,
                                           FDst fdst = FDst()) {
    using LG = LeafGeom<K, V>;
    using LS = LeafStage<K, V, G>;
    const unsigned gmask = (G == 32 ? 0xffffffffu : ((1u << G) - 1u)) << (grp * G);
    uint32_t ch[I][LS::CPL][4];
#pragma unroll
    for (int s = 0; s < I; s++) {
        const unsigned char *blk = leaves + (size_t)node[s] * LG::BS;
#pragma unroll
        for (int j = 0; j < LS::CPL; j++) {
            const int c = gl + j * G;
            if (c < LS::NC) {
                const uint4 x =
                    load_stream16(blk + (c < LS::NKC ? c * 16 : kSectorBytes + (c - LS::NKC) * 16));
                ch[s][j][0] = x.x;
                ch[s][j][1] = x.y;
                ch[s][j][2] = x.z;
                ch[s][j][3] = x.w;
            }
        }
    }
#pragma unroll
    for (int s = 0; s < I; s++) {
        int cnt = 0;
        bool eq = false;
#pragma unroll
        for (int j = 0; j < LS::KCPL; j++) {
            if (gl + j * G < LS::NKC) {
                cnt += count_below<K, LS::KPC>(ch[s][j], qe[s], false);
#pragma unroll
                for (int k = 0; k < LS::KPC; k++) eq |= key_at<K>(ch[s][j], k) == qv[s];
            }
        }
        int pos0;
        bool found;
        if constexpr (G == 1) {
            pos0 = cnt;
            found = eq;
        } else {
            pos0 = __shfl_sync(0xffffffffu, cnt, grp * G) + __shfl_sync(0xffffffffu, cnt, grp * G + 1);
            found = (__ballot_sync(0xffffffffu, eq) & gmask) != 0;
        }
        found = found && qv[s] <= tmax;  // padding keys are all-ones
        const int pos = pos0 < LG::S ? pos0 : LG::S - 1;
        const int vc = LS::NKC + pos / LS::VPC;  // chunk holding the value
        if (gl == vc % G) {
            V *d = dst(s);
            if (d) {
                V val = 0;
#pragma unroll
                for (int j = 0; j < LS::CPL; j++) {
                    if (j == vc / G) {
                        const int w = (pos % LS::VPC) * (int)(sizeof(V) / 4);
                        if constexpr (sizeof(V) == 4) {
#pragma unroll
                            for (int k = 0; k < 4; k++)
                                if (k == w) val = ch[s][j][k];
                        } else {
                            val = w == 0 ? (((uint64_t)ch[s][j][1] << 32) | ch[s][j][0])
                                         : (((uint64_t)ch[s][j][3] << 32) | ch[s][j][2]);
                        }
                    }
                }
                *d = found ? val : key_max<V>();
                if (uint8_t *f = fdst(s)) *f = found ? 1 : 0;
            }
        }
    }
}

// Lower (upper, per slot) bound slot inside each query's leaf block, keys
// only; every lane of the group receives pos[s].
template <typename K, typename V, int G, int I>
__device__ __forceinline__ void leaf_bound(const unsigned char *__restrict__ leaves,
                                           const uint32_t (&node)[I], const K (&qe)[I],
                                           const bool (&up)[I], int grp, int gl, int (&pos)[I]) {
    using LG = LeafGeom<K, V>;
    using LS = LeafStage<K, V, G>;
    uint32_t ch[I][LS::KCPL][4];
#pragma unroll
    for (int s = 0; s < I; s++) {
        const unsigned char *blk = leaves + (size_t)node[s] * LG::BS;
#pragma unroll
        for (int j = 0; j < LS::KCPL; j++) {
            const int c = gl + j * G;
            if (c < LS::NKC) {
                const uint4 x = load_stream16(blk + c * 16);
                ch[s][j][0] = x.x;
                ch[s][j][1] = x.y;
                ch[s][j][2] = x.z;
                ch[s][j][3] = x.w;
            }
        }
    }
#pragma unroll
    for (int s = 0; s < I; s++) {
        int cnt = 0;
#pragma unroll
        for (int j = 0; j < LS::KCPL; j++)
            if (gl + j * G < LS::NKC) cnt += count_below<K, LS::KPC>(ch[s][j], qe[s], up[s]);
        if constexpr (G == 1)
            pos[s] = cnt;
        else
            pos[s] = __shfl_sync(0xffffffffu, cnt, grp * G) + __shfl_sync(0xffffffffu, cnt, grp * G + 1);
    }
}

}  // namespace bt
