// Point search and range-bound kernels.
//
// point_kernel replaces kernelSearchingNaiveOneStep
// (BPTreeExactSearch.cu:25-105) and, with PERM, the grouped
// kernelSearchingKeyGroupTwoStep (:207-294): same answer (value at the exact
// match, all-ones otherwise), but the grouped variant compares keys, not
// data[] (:269-276), and writes results back in the caller's order.
//
// bounds_line_kernel replaces the range endpoint + count kernels
// (BtreeRangeSearch.cu:215-374 and :33-211).  With implicit leaf positions
// the count is upper_bound(hi) - lower_bound(lo); no leaf-chain walk.
//
// Both kernels are persistent (grid = SMs x resident CTAs), stage one
// separator level into shared memory once per CTA, then loop over warp tiles
// of 32 queries (see bt_search.cuh for the two-phase descent).
// The leaf stage loads the whole leaf block of the query -- key sector and
// value sector side by side, one 64-byte DRAM access -- with its chunks
// spread over the group's lanes, so a hit costs one HBM round trip.
#include <map>
#include <mutex>

#include "bt_search.cuh"

namespace bt {

// Lanes per query (G) below the staged level and rounds (R) per warp tile of
// 32 queries; each group keeps G/R queries in flight.  Set per tree by
// bt_set_search_config / the autotuner.
struct SearchCfg {
    int g, r;
};
constexpr SearchCfg kSearchCfgs[] = {{8, 1}, {8, 2}, {4, 1}, {4, 2}, {2, 1}};
constexpr int kNumSearchCfgs = sizeof(kSearchCfgs) / sizeof(kSearchCfgs[0]);

int search_cfg_index(int g, int r) {
    for (int k = 0; k < kNumSearchCfgs; k++)
        if (kSearchCfgs[k].g == g && kSearchCfgs[k].r == r) return k;
    return -1;
}

int search_cfg_lanes(int cfg) { return kSearchCfgs[cfg].g; }
int search_cfg_rounds(int cfg) { return kSearchCfgs[cfg].r; }

int default_search_cfg(int key_bytes) {
    (void)key_bytes;
    return search_cfg_index(4, 1);
}

namespace {

constexpr int kThreads = 512;
constexpr int kWarps = kThreads / 32;

// Shared memory of a search CTA: the staged level, then (bounds kernel) 64
// 8-byte results per warp.
__host__ __device__ inline size_t scratch_offset(const DevTree &t) { return ((size_t)t.smem_bytes + 15) / 16 * 16; }

template <typename K, typename V, int G, int R, bool PERM>
__global__ void __launch_bounds__(kThreads)
point_kernel(const __grid_constant__ DevTree t, const K *__restrict__ q,
             const uint32_t *__restrict__ perm, uint64_t nq, V *__restrict__ out,
             uint8_t *__restrict__ found) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    K *s_lvl = reinterpret_cast<K *>(smem_raw);
    stage_level<K>(s_lvl, t);
    __syncthreads();

    constexpr int NG = 32 / G;  // lane groups per warp
    constexpr int I = G / R;    // queries in flight per group and round
    const int lane = threadIdx.x & 31;
    const int grp = lane / G;
    const int gl = lane % G;
    const K tmax = (K)t.max_key;
    const unsigned char *leaves = static_cast<const unsigned char *>(t.leaves);
    // Grouped input (PERM): each CTA takes one contiguous run of warp tiles,
    // so a CTA works one key range and its warps share node lines in L1.
    // Ungrouped input: warp tiles are strided over the whole grid.
    const uint64_t ntiles = (nq + 31) / 32;
    const uint64_t per_cta = PERM ? (ntiles + gridDim.x - 1) / gridDim.x : 0;
    const uint64_t t_begin = PERM ? blockIdx.x * per_cta + (threadIdx.x >> 5)
                                  : (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    const uint64_t t_end = PERM ? min(ntiles, (blockIdx.x + 1) * per_cta) : ntiles;
    const uint64_t t_step = PERM ? (blockDim.x >> 5) : ((uint64_t)gridDim.x * blockDim.x) >> 5;

    for (uint64_t tile = t_begin; tile < t_end; tile += t_step) {
        const uint64_t base = tile * 32;
        // phase 1: one lane per query, binary search of the staged level
        const uint64_t my = base + lane;
        const K myq = my < nq ? q[my] : (K)0;
        const uint32_t myperm = PERM && my < nq ? perm[my] : 0u;  // loaded early
        const uint32_t mynode = smem_bound<K>(s_lvl, t.smem_entries, myq < tmax ? myq : tmax, false);

        // phase 2: G lanes per query through the global levels and the leaf
#pragma unroll
        for (int r = 0; r < R; r++) {
            K qv[I], qe[I];
            bool up[I];
            uint32_t node[I], pv[I];
#pragma unroll
            for (int s = 0; s < I; s++) {
                const int k = r * (NG * I) + s * NG + grp;  // query of the tile
                qv[s] = __shfl_sync(0xffffffffu, myq, k);
                node[s] = __shfl_sync(0xffffffffu, mynode, k);
                pv[s] = PERM ? __shfl_sync(0xffffffffu, myperm, k) : 0u;
                qe[s] = qv[s] < tmax ? qv[s] : tmax;
                up[s] = false;
            }
            walk_global<K, G, I>(t, qe, up, node, grp, gl);
            leaf_point<K, V, G, I>(
                leaves, node, qv, qe, tmax, grp, gl,
                [&](int s) -> V * {
                    const uint64_t qi = base + (uint64_t)(r * (NG * I) + s * NG + grp);
                    if (qi >= nq) return nullptr;
                    return out + (PERM ? (uint64_t)pv[s] : qi);
                },
                [&](int s) -> uint8_t * {
                    const uint64_t qi = base + (uint64_t)(r * (NG * I) + s * NG + grp);
                    return found ? found + (PERM ? (uint64_t)pv[s] : qi) : nullptr;
                });
        }
    }
}

// Point search over radix-grouped input (the queries ordered by their top
// kPointGroupBits bits below the tree's key length, as bt_group_queries
// leaves them).  One CTA per SM
// takes a contiguous run of the grouped batch.  For the group of its current
// queries it stages in shared memory the group's window of the deepest
// separator level whose window fits (for 2^26 u32 keys and 256 groups: the
// 32,768 leaf-block maxima of the bottom level, 128 KB), so that one binary
// search in shared memory takes a query straight to its leaf block: the only
// global access left is the leaf block itself.  The window of a group [lo,
// hi] is the level's entries from the lower bound of lo to the lower bound
// of hi; every query of the group has its lower bound inside it.  Warps whose
// tile holds a query of another group (tiles at group boundaries, or input
// that is not grouped at all) take the full descent from the root instead,
// so results never depend on the order of the input.
// The group of a key as the grouping pass forms it: its bits above `shift`
// (the tree's key length less kPointGroupBits), the last group taking
// everything above.
constexpr uint64_t kLastGroup = (1u << kPointGroupBits) - 1u;
__device__ __forceinline__ uint64_t group_of(uint64_t k, int shift) {
    const uint64_t g = k >> shift;
    return g < kLastGroup ? g : kLastGroup;
}

constexpr int kWinThreads = 1024;
constexpr int kWinWarps = kWinThreads / 32;
constexpr size_t kWinBytes = 192 * 1024;
// Below this batch size a window staged per CTA costs more than it saves.
constexpr uint64_t kWinMinQueries = 1ull << 21;

template <typename K, typename V, int G, int R>
__global__ void __launch_bounds__(kWinThreads, 1)
point_window_kernel(const __grid_constant__ DevTree t, const K *__restrict__ q,
                    const uint32_t *__restrict__ perm, uint64_t nq, V *__restrict__ out,
                    uint8_t *__restrict__ found, int shift) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    K *s_win = reinterpret_cast<K *>(smem_raw);
    __shared__ uint32_t s_blk[2];
    constexpr uint32_t kCap = (uint32_t)(kWinBytes / sizeof(K));
    constexpr int F = kLineBytes / (int)sizeof(K);
    constexpr int LOGF = F == 32 ? 5 : 4;
    constexpr uint32_t ROW = sizeof(K) == 4 ? 32u : 16u;  // swizzle row (elements)
    constexpr int NG = 32 / G;
    constexpr int I = G / R;
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int grp = lane / G;
    const int gl = lane % G;
    const K tmax = (K)t.max_key;
    const unsigned char *leaves = static_cast<const unsigned char *>(t.leaves);
    const K *seps = static_cast<const K *>(t.seps);
    const uint64_t ntiles = (nq + 31) / 32;
    const uint64_t per_cta = (ntiles + gridDim.x - 1) / gridDim.x;
    const uint64_t c_begin = blockIdx.x * per_cta;
    const uint64_t c_end = min(ntiles, c_begin + per_cta);
    uint64_t staged = ~0ull;  // group whose window is staged (same in every thread)
    int wlvl = 0;
    uint32_t w0 = 0, wm = 1;
    for (uint64_t t0 = c_begin; t0 < c_end; t0 += kWinWarps) {
        const uint64_t b = group_of((uint64_t)q[t0 * 32], shift);  // group of this step's first query
        if (b != staged) {
            __syncthreads();  // the old window is no longer read
            if (threadIdx.x < 2) {
                const uint64_t lo = b << shift;
                const uint64_t hi = b == kLastGroup ? ~0ull : lo | ((1ull << shift) - 1ull);
                const uint64_t k = threadIdx.x == 0 ? lo : hi;
                s_blk[threadIdx.x] = block_lower_bound<K>(t, k < (uint64_t)tmax ? (K)k : tmax);
            }
            __syncthreads();
            // deepest level whose window fits (level 0 holds at most F entries)
            const uint32_t blo = s_blk[0], bhi = s_blk[1];
            wlvl = t.nlevels - 1;
            int sh = 0;
            while (wlvl > 0 && (bhi >> sh) - (blo >> sh) + 1u > kCap) {
                wlvl--;
                sh += LOGF;
            }
            w0 = blo >> sh;
            wm = (bhi >> sh) - w0 + 1u;
            const K *src = seps + t.lvl_off[wlvl] + w0;
            const uint32_t staged_n = (wm + ROW - 1) / ROW * ROW;
            for (uint32_t i = threadIdx.x; i < staged_n; i += blockDim.x)
                s_win[swz<K>(i)] = i < wm ? src[i] : key_max<K>();
            __syncthreads();
            staged = b;
        }
        const uint64_t tile = t0 + warp;
        if (tile >= c_end) continue;
        const uint64_t base = tile * 32;
        const uint64_t my = base + lane;
        const K myq = my < nq ? q[my] : (K)0;
        const uint32_t myperm = my < nq ? perm[my] : 0u;  // loaded early, off the critical path
        const K myqe = myq < tmax ? myq : tmax;
        // phase 1: the window, or (whole warp) the descent from the root
        const bool inwin = my >= nq || group_of((uint64_t)myq, shift) == staged;
        const bool win = __all_sync(0xffffffffu, inwin);
        uint32_t mynode = 0;
        if (win) {
            const uint32_t p = smem_bound<K>(s_win, wm, myqe, false);
            mynode = w0 + (p < wm ? p : wm - 1u);
        }
        const int from = win ? wlvl + 1 : 0;
#pragma unroll
        for (int r = 0; r < R; r++) {
            K qv[I], qe[I];
            bool up[I];
            uint32_t node[I], pv[I];
#pragma unroll
            for (int s = 0; s < I; s++) {
                const int k = r * (NG * I) + s * NG + grp;
                qv[s] = __shfl_sync(0xffffffffu, myq, k);
                node[s] = __shfl_sync(0xffffffffu, mynode, k);
                pv[s] = __shfl_sync(0xffffffffu, myperm, k);
                qe[s] = qv[s] < tmax ? qv[s] : tmax;
                up[s] = false;
            }
            walk_from<K, G, I>(t, from, qe, up, node, grp, gl);
            leaf_point<K, V, G, I>(
                leaves, node, qv, qe, tmax, grp, gl,
                [&](int s) -> V * {
                    const uint64_t qi = base + (uint64_t)(r * (NG * I) + s * NG + grp);
                    if (qi >= nq) return nullptr;
                    return out + pv[s];
                },
                [&](int s) -> uint8_t * { return found ? found + pv[s] : nullptr; });
        }
    }
}

// Range bounds with the upper bound taken from the lower bound's path.
// A narrow range usually ends in the same bottom separator line as it
// starts: while the group walks lo down, it counts that line's separators
// <= hi as well (the line is already in its registers), which gives hi's
// leaf block whenever the line's last separator is above hi; both leaf
// blocks are then read together.  Only the queries whose range leaves that
// line take a second descent, compacted per warp into as few rounds as they
// need.  counts[i] = ub - lb (0 if lo > hi); lb_out[i] = lb.
template <typename K, typename V, int G, int R, bool PERM>
__global__ void __launch_bounds__(kThreads, 2)
bounds_line_kernel(const __grid_constant__ DevTree t, const K *__restrict__ lo,
                   const K *__restrict__ hi, const uint32_t *__restrict__ perm, uint64_t nq,
                   uint64_t *__restrict__ counts, uint64_t *__restrict__ lb_out) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    K *s_lvl = reinterpret_cast<K *>(smem_raw);
    stage_level<K>(s_lvl, t);
    __syncthreads();

    using LG = LeafGeom<K, V>;
    constexpr int F = kLineBytes / (int)sizeof(K);
    constexpr int KPL = F / G;
    constexpr int NB = KPL * (int)sizeof(K);
    constexpr int NG = 32 / G;
    constexpr int I = G / R;
    const int lane = threadIdx.x & 31;
    const int grp = lane / G;
    const int gl = lane % G;
    uint64_t *res = reinterpret_cast<uint64_t *>(smem_raw + scratch_offset(t)) + (threadIdx.x >> 5) * 64;
    const K tmax = (K)t.max_key;
    const unsigned char *leaves = static_cast<const unsigned char *>(t.leaves);
    const K *gseps = static_cast<const K *>(t.seps);
    const int bottom = t.nlevels - 1;
    // the staged level is the bottom one for small trees: no line to share
    const bool share = t.smem_level < bottom;
    const uint64_t ntiles = (nq + 31) / 32;
    const uint64_t per_cta = PERM ? (ntiles + gridDim.x - 1) / gridDim.x : 0;
    const uint64_t t_begin = PERM ? blockIdx.x * per_cta + (threadIdx.x >> 5)
                                  : (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    const uint64_t t_end = PERM ? min(ntiles, (blockIdx.x + 1) * per_cta) : ntiles;
    const uint64_t t_step = PERM ? (blockDim.x >> 5) : ((uint64_t)gridDim.x * blockDim.x) >> 5;

    for (uint64_t tile = t_begin; tile < t_end; tile += t_step) {
        const uint64_t base = tile * 32;
        const uint64_t my = base + lane;
        const bool v = my < nq;
        const K a = v ? lo[my] : (K)0;
        const K b = v ? hi[my] : (K)0;
        const K qa = a <= tmax ? a : tmax;
        const K qb = b < tmax ? b : tmax;
        const uint32_t na = smem_bound<K>(s_lvl, t.smem_entries, qa, false);
        // hi >= the largest key: the upper bound is n, no walk
        const bool hi_open = v && b < tmax;
        // ---- lower bounds, and upper bounds that end in the same bottom line
#pragma unroll
        for (int r = 0; r < R; r++) {
            K qe[2 * I];
            bool up[2 * I];
            uint32_t node[2 * I];
            bool hin[I];
#pragma unroll
            for (int s = 0; s < I; s++) {
                const int k = r * (NG * I) + s * NG + grp;
                qe[s] = __shfl_sync(0xffffffffu, qa, k);
                qe[I + s] = __shfl_sync(0xffffffffu, qb, k);
                node[s] = __shfl_sync(0xffffffffu, na, k);
                up[s] = false;
                up[I + s] = true;
                hin[s] = false;
            }
            for (int lvl = t.smem_level + 1; lvl < bottom; lvl++) {
                K qs[I];
                bool us[I];
                uint32_t ns[I];
#pragma unroll
                for (int s = 0; s < I; s++) {
                    qs[s] = qe[s];
                    us[s] = false;
                    ns[s] = node[s];
                }
                level_step<K, G, I>(gseps + t.lvl_off[lvl], qs, us, ns, grp, gl);
#pragma unroll
                for (int s = 0; s < I; s++) node[s] = ns[s];
            }
            if (share) {
                // bottom line: separators < lo and <= hi from the same registers
                uint32_t c[I][NB / 4];
#pragma unroll
                for (int s = 0; s < I; s++)
                    load_bytes<NB>(gseps + t.lvl_off[bottom] + (size_t)node[s] * F + gl * KPL, c[s]);
#pragma unroll
                for (int s = 0; s < I; s++) {
                    const int cl = group_count<G, G, KPL>(count_below<K, KPL>(c[s], qe[s], false), true, grp);
                    const int ch = group_count<G, G, KPL>(count_below<K, KPL>(c[s], qe[I + s], true), true, grp);
                    hin[s] = ch < F;  // the line's last separator is above hi
                    // (otherwise read lo's block again: ch = F may be past the last block)
                    node[I + s] = node[s] * F + (uint32_t)(hin[s] ? ch : cl);
                    node[s] = node[s] * F + (uint32_t)cl;
                }
            } else {
#pragma unroll
                for (int s = 0; s < I; s++) node[I + s] = node[s];
            }
            int pos[2 * I];
            leaf_bound<K, V, G, 2 * I>(leaves, node, qe, up, grp, gl, pos);
#pragma unroll
            for (int s = 0; s < I; s++) {
                const int k = r * (NG * I) + s * NG + grp;
                if (gl == 0) {
                    res[k] = (uint64_t)node[s] * LG::S + pos[s];
                    res[32 + k] = hin[s] ? (uint64_t)node[I + s] * LG::S + pos[I + s] : ~0ull;
                }
            }
        }
        __syncwarp();
        // ---- the remaining upper bounds: full descents, compacted
        const bool need = hi_open && res[32 + lane] == ~0ull;
        const unsigned needm = __ballot_sync(0xffffffffu, need);
        if (needm) {
            const uint32_t nb = need ? smem_bound<K>(s_lvl, t.smem_entries, qb, true) : 0u;
            const int nneed = __popc(needm);
            for (int r0 = 0; r0 < nneed; r0 += NG * I) {
                K qe[I];
                bool up[I];
                uint32_t node[I];
                int who[I];
#pragma unroll
                for (int s = 0; s < I; s++) {
                    const int j = r0 + s * NG + grp;  // j-th query that needs a descent
                    unsigned m = needm;               // its lane (the first one as filler)
                    for (int z = 0; z < (j < nneed ? j : 0); z++) m &= m - 1;
                    const int src = __ffs(m) - 1;
                    who[s] = j < nneed ? src : -1;
                    qe[s] = __shfl_sync(0xffffffffu, qb, src);
                    node[s] = __shfl_sync(0xffffffffu, nb, src);
                    up[s] = true;
                }
                walk_global<K, G, I>(t, qe, up, node, grp, gl);
                int pos[I];
                leaf_bound<K, V, G, I>(leaves, node, qe, up, grp, gl, pos);
#pragma unroll
                for (int s = 0; s < I; s++)
                    if (gl == 0 && who[s] >= 0) res[32 + who[s]] = (uint64_t)node[s] * LG::S + pos[s];
            }
        }
        __syncwarp();
        if (v) {
            const uint64_t lb = a <= tmax ? res[lane] : t.n;
            const uint64_t ub = b < tmax ? res[32 + lane] : t.n;
            const uint64_t dst = PERM ? (uint64_t)perm[my] : my;
            counts[dst] = (a <= b && ub > lb) ? ub - lb : 0;
            if (lb_out) lb_out[dst] = lb;
        }
        __syncwarp();
    }
}

// Empty tree: every point query misses, every range is empty.
template <typename V>
__global__ void fill_kernel(V *out, uint64_t n, V v) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x)
        out[i] = v;
}

std::mutex g_occ_mu;
std::map<std::pair<const void *, size_t>, int> g_occ;

// Resident CTAs per SM for a kernel at a given dynamic shared memory size
// (all devices this library runs on are B200s of one kind).
int occupancy(const void *fn, size_t smem) {
    std::lock_guard<std::mutex> lk(g_occ_mu);
    auto key = std::make_pair(fn, smem);
    auto it = g_occ.find(key);
    if (it != g_occ.end()) return it->second;
    int blocks = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, fn, kThreads, smem) != cudaSuccess ||
        blocks < 1)
        blocks = 1;
    g_occ[key] = blocks;
    return blocks;
}

unsigned persistent_grid(const void *fn, size_t smem, uint64_t work_items, uint64_t items_per_cta) {
    uint64_t want = (work_items + items_per_cta - 1) / items_per_cta;
    uint64_t cap = (uint64_t)sm_count() * occupancy(fn, smem);
    if (want > cap) want = cap;
    return (unsigned)(want < 1 ? 1 : want);
}

// Raises a kernel's dynamic shared-memory limit when needed (function
// attributes are per device; the largest size set so far is remembered).
template <typename Fn>
bt_status set_smem(Fn fn, size_t smem) {
    static std::mutex mu;
    static std::map<std::pair<int, const void *>, size_t> done;
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lk(mu);
    const auto key = std::make_pair(dev, (const void *)fn);
    auto it = done.find(key);
    if (it != done.end() && it->second >= smem) return BT_OK;
    if (smem > 48 * 1024)
        BT_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    done[key] = smem;
    return BT_OK;
}

template <typename K, typename V, int G, int R, bool PERM>
bt_status point_launch(const bt_tree *t, const void *d_q, const uint32_t *d_perm, uint64_t nq,
                       void *d_out, uint8_t *d_found, cudaStream_t s) {
    auto fn = point_kernel<K, V, G, R, PERM>;
    const size_t smem = scratch_offset(t->dev);
    bt_status st = set_smem(fn, smem);
    if (st != BT_OK) return st;
    const unsigned grid = persistent_grid((const void *)fn, smem, nq, kThreads);
    count_launch();
    fn<<<grid, kThreads, smem, s>>>(t->dev, (const K *)d_q, d_perm, nq, (V *)d_out, d_found);
    BT_CUDA(cudaGetLastError());
    return BT_OK;
}

template <typename K, typename V, int G, int R>
bt_status window_launch(const bt_tree *t, const void *d_q, const uint32_t *d_perm, uint64_t nq,
                        void *d_out, uint8_t *d_found, cudaStream_t s) {
    auto fn = point_window_kernel<K, V, G, R>;
    bt_status st = set_smem(fn, kWinBytes);
    if (st != BT_OK) return st;
    const uint64_t ntiles = (nq + 31) / 32;
    const unsigned grid = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(ntiles, sm_count()));
    const int shift = std::max(0, bitlen64(t->max_key) - kPointGroupBits);  // as the grouping pass
    count_launch();
    fn<<<grid, kWinThreads, kWinBytes, s>>>(t->dev, (const K *)d_q, d_perm, nq, (V *)d_out, d_found,
                                            shift);
    BT_CUDA(cudaGetLastError());
    return BT_OK;
}

template <typename K, typename V, bool PERM>
bt_status point_cfg(const bt_tree *t, const void *d_q, const uint32_t *d_perm, uint64_t nq,
                    void *d_out, uint8_t *d_found, cudaStream_t s) {
    if (PERM && nq >= kWinMinQueries) {
        switch (t->search_cfg) {
            case 0: return window_launch<K, V, 8, 1>(t, d_q, d_perm, nq, d_out, d_found, s);
            case 1: return window_launch<K, V, 8, 2>(t, d_q, d_perm, nq, d_out, d_found, s);
            case 2: return window_launch<K, V, 4, 1>(t, d_q, d_perm, nq, d_out, d_found, s);
            case 3: return window_launch<K, V, 4, 2>(t, d_q, d_perm, nq, d_out, d_found, s);
            default: return window_launch<K, V, 2, 1>(t, d_q, d_perm, nq, d_out, d_found, s);
        }
    }
    switch (t->search_cfg) {
        case 0: return point_launch<K, V, 8, 1, PERM>(t, d_q, d_perm, nq, d_out, d_found, s);
        case 1: return point_launch<K, V, 8, 2, PERM>(t, d_q, d_perm, nq, d_out, d_found, s);
        case 2: return point_launch<K, V, 4, 1, PERM>(t, d_q, d_perm, nq, d_out, d_found, s);
        case 3: return point_launch<K, V, 4, 2, PERM>(t, d_q, d_perm, nq, d_out, d_found, s);
        default: return point_launch<K, V, 2, 1, PERM>(t, d_q, d_perm, nq, d_out, d_found, s);
    }
}

template <typename K, typename V, int G, int R, bool PERM>
bt_status bounds_launch(const bt_tree *t, const void *d_lo, const void *d_hi,
                        const uint32_t *d_perm, uint64_t nq, uint64_t *d_counts, uint64_t *d_lb,
                        cudaStream_t s) {
    auto fn = bounds_line_kernel<K, V, G, R, PERM>;
    const size_t smem = scratch_offset(t->dev) + (size_t)kWarps * 64 * sizeof(uint64_t);
    bt_status st = set_smem(fn, smem);
    if (st != BT_OK) return st;
    const unsigned grid = persistent_grid((const void *)fn, smem, nq, kThreads);
    count_launch();
    fn<<<grid, kThreads, smem, s>>>(t->dev, (const K *)d_lo, (const K *)d_hi, d_perm, nq, d_counts,
                                    d_lb);
    BT_CUDA(cudaGetLastError());
    return BT_OK;
}

template <typename K, typename V, bool PERM>
bt_status bounds_cfg(const bt_tree *t, const void *d_lo, const void *d_hi, const uint32_t *d_perm,
                     uint64_t nq, uint64_t *d_counts, uint64_t *d_lb, cudaStream_t s) {
    switch (t->search_cfg) {
        case 0: return bounds_launch<K, V, 8, 1, PERM>(t, d_lo, d_hi, d_perm, nq, d_counts, d_lb, s);
        case 1: return bounds_launch<K, V, 8, 2, PERM>(t, d_lo, d_hi, d_perm, nq, d_counts, d_lb, s);
        case 2: return bounds_launch<K, V, 4, 1, PERM>(t, d_lo, d_hi, d_perm, nq, d_counts, d_lb, s);
        case 3: return bounds_launch<K, V, 4, 2, PERM>(t, d_lo, d_hi, d_perm, nq, d_counts, d_lb, s);
        default: return bounds_launch<K, V, 2, 1, PERM>(t, d_lo, d_hi, d_perm, nq, d_counts, d_lb, s);
    }
}

template <bool PERM>
bt_status point_types(const bt_tree *t, const void *d_q, const uint32_t *d_perm, uint64_t nq,
                      void *d_out, uint8_t *d_found, cudaStream_t s) {
    if (t->key_bytes == 4)
        return t->val_bytes == 4 ? point_cfg<uint32_t, uint32_t, PERM>(t, d_q, d_perm, nq, d_out, d_found, s)
                                 : point_cfg<uint32_t, uint64_t, PERM>(t, d_q, d_perm, nq, d_out, d_found, s);
    return t->val_bytes == 4 ? point_cfg<uint64_t, uint32_t, PERM>(t, d_q, d_perm, nq, d_out, d_found, s)
                             : point_cfg<uint64_t, uint64_t, PERM>(t, d_q, d_perm, nq, d_out, d_found, s);
}

template <bool PERM>
bt_status bounds_types(const bt_tree *t, const void *d_lo, const void *d_hi, const uint32_t *d_perm,
                       uint64_t nq, uint64_t *d_counts, uint64_t *d_lb, cudaStream_t s) {
    if (t->key_bytes == 4)
        return t->val_bytes == 4
                   ? bounds_cfg<uint32_t, uint32_t, PERM>(t, d_lo, d_hi, d_perm, nq, d_counts, d_lb, s)
                   : bounds_cfg<uint32_t, uint64_t, PERM>(t, d_lo, d_hi, d_perm, nq, d_counts, d_lb, s);
    return t->val_bytes == 4
               ? bounds_cfg<uint64_t, uint32_t, PERM>(t, d_lo, d_hi, d_perm, nq, d_counts, d_lb, s)
               : bounds_cfg<uint64_t, uint64_t, PERM>(t, d_lo, d_hi, d_perm, nq, d_counts, d_lb, s);
}

}  // namespace

bt_status launch_point_search(const bt_tree *t, const void *d_q, const uint32_t *d_perm,
                              uint64_t nq, void *d_out, cudaStream_t s, uint8_t *d_found) {
    if (nq == 0) return BT_OK;
    if (t->n == 0) {
        unsigned g = (unsigned)std::min<uint64_t>((nq + 255) / 256, 4096);
        count_launch();
        if (t->val_bytes == 4)
            fill_kernel<uint32_t><<<g, 256, 0, s>>>((uint32_t *)d_out, nq, 0xFFFFFFFFu);
        else
            fill_kernel<uint64_t><<<g, 256, 0, s>>>((uint64_t *)d_out, nq, ~0ull);
        BT_CUDA(cudaGetLastError());
        if (d_found) BT_CUDA(cudaMemsetAsync(d_found, 0, nq, s));
        return BT_OK;
    }
    return d_perm ? point_types<true>(t, d_q, d_perm, nq, d_out, d_found, s)
                  : point_types<false>(t, d_q, d_perm, nq, d_out, d_found, s);
}

bt_status launch_bounds(const bt_tree *t, const void *d_lo, const void *d_hi,
                        const uint32_t *d_perm, uint64_t nq, uint64_t *d_counts, uint64_t *d_lb,
                        cudaStream_t s) {
    if (nq == 0) return BT_OK;
    if (t->n == 0) {
        unsigned g = (unsigned)std::min<uint64_t>((nq + 255) / 256, 4096);
        count_launch();
        fill_kernel<uint64_t><<<g, 256, 0, s>>>(d_counts, nq, 0ull);
        if (d_lb) {
            count_launch();
            fill_kernel<uint64_t><<<g, 256, 0, s>>>(d_lb, nq, 0ull);
        }
        BT_CUDA(cudaGetLastError());
        return BT_OK;
    }
    return d_perm ? bounds_types<true>(t, d_lo, d_hi, d_perm, nq, d_counts, d_lb, s)
                  : bounds_types<false>(t, d_lo, d_hi, d_perm, nq, d_counts, d_lb, s);
}

}  // namespace bt
