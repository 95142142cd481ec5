// Point search and range-bound kernels.
//
// point_kernel replaces kernelSearchingNaiveOneStep
// (BPTreeExactSearch.cu:25-105) and, with PERM, the grouped
// kernelSearchingKeyGroupTwoStep (:207-294): same answer (value at the exact
// match, all-ones otherwise), but the grouped variant compares keys, not
// data[] (:269-276), and writes results back in the caller's order.
//
// bounds_kernel replaces the range endpoint + count kernels
// (BtreeRangeSearch.cu:215-374 and :33-211).  With implicit leaf positions
// the count is upper_bound(hi) - lower_bound(lo); no leaf-chain walk.
//
// Both kernels are persistent (grid = SMs x resident CTAs), stage the top
// separator levels into shared memory once per CTA, then loop over warp tiles.
// The leaf stage loads the query's key sector and, speculatively, the value
// sector of the same positions in parallel (one 32-byte DRAM sector each), so
// a hit costs one dependent HBM round trip instead of two.
#include <map>
#include <mutex>

#include "bt_search.cuh"

namespace bt {
namespace {

constexpr int kThreads = 512;

template <typename K, typename V, int G, int I, bool PERM>
__global__ void __launch_bounds__(kThreads)
point_kernel(const __grid_constant__ DevTree t, const K *__restrict__ q,
             const uint32_t *__restrict__ perm, uint64_t nq, V *__restrict__ out) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    K *s_top = reinterpret_cast<K *>(smem_raw);
    stage_top<K>(s_top, t);
    __syncthreads();

    constexpr int S = kSectorBytes / (int)sizeof(K);
    constexpr int LL = S >= G ? G : S;  // lanes holding part of the leaf sector
    constexpr int LPL = S / LL;         // keys per such lane
    constexpr int QPW = 32 / G;         // queries per warp and slot
    constexpr int TILE = QPW * I;
    const int lane = threadIdx.x & 31;
    const int grp = lane / G;
    const int gl = lane % G;
    const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    const K tmax = (K)t.max_key;
    const K *gk = static_cast<const K *>(t.keys);
    const V *gv = static_cast<const V *>(t.vals);
    const bool act = gl < LL;

    for (uint64_t base = warp * TILE; base < nq; base += nwarps * TILE) {
        K qv[I], qe[I];
        bool up[I];
        uint64_t node[I];
        bool valid[I];
#pragma unroll
        for (int s = 0; s < I; s++) {
            const uint64_t qi = base + (uint64_t)s * QPW + grp;
            valid[s] = qi < nq;
            qv[s] = valid[s] ? q[qi] : (K)0;
            qe[s] = qv[s] < tmax ? qv[s] : tmax;
            up[s] = false;
        }
        descend<K, G, I>(t, s_top, qe, up, node, grp, gl);

        K kk[I][LPL];
        V vv[I][LPL];
#pragma unroll
        for (int s = 0; s < I; s++) {
#pragma unroll
            for (int j = 0; j < LPL; j++) {
                kk[s][j] = 0;
                vv[s][j] = 0;
            }
            if (act) {
                const uint64_t p = node[s] * S + (uint64_t)gl * LPL;
                load_stream<K, LPL>(gk + p, kk[s]);
                load_stream<V, LPL>(gv + p, vv[s]);
            }
        }
#pragma unroll
        for (int s = 0; s < I; s++) {
            const int cnt = act ? count_below<K, LPL>(kk[s], qe[s], false) : 0;
            int pos = group_count<G, LL, LPL>(cnt, act, grp);
            pos = pos < S ? pos : S - 1;
            if (gl == pos / LPL && valid[s]) {
                const int j0 = pos % LPL;
                K key = kk[s][0];
                V val = vv[s][0];
#pragma unroll
                for (int j = 1; j < LPL; j++)
                    if (j == j0) {
                        key = kk[s][j];
                        val = vv[s][j];
                    }
                const bool found = qv[s] <= tmax && key == qv[s];
                const uint64_t qi = base + (uint64_t)s * QPW + grp;
                const uint64_t dst = PERM ? (uint64_t)perm[qi] : qi;
                out[dst] = found ? val : key_max<V>();
            }
        }
    }
}

// Lower bound of lo and upper bound of hi for QG queries per group (2*QG
// descents in flight).  counts[i] = ub - lb (0 if lo > hi); lb_out[i] = lb.
template <typename K, int G, int QG, bool PERM>
__global__ void __launch_bounds__(kThreads)
bounds_kernel(const __grid_constant__ DevTree t, const K *__restrict__ lo,
              const K *__restrict__ hi, const uint32_t *__restrict__ perm, uint64_t nq,
              uint64_t *__restrict__ counts, uint64_t *__restrict__ lb_out) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    K *s_top = reinterpret_cast<K *>(smem_raw);
    stage_top<K>(s_top, t);
    __syncthreads();

    constexpr int I = 2 * QG;
    constexpr int S = kSectorBytes / (int)sizeof(K);
    constexpr int LL = S >= G ? G : S;
    constexpr int LPL = S / LL;
    constexpr int QPW = 32 / G;
    constexpr int TILE = QPW * QG;
    const int lane = threadIdx.x & 31;
    const int grp = lane / G;
    const int gl = lane % G;
    const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    const uint64_t nwarps = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    const K tmax = (K)t.max_key;
    const K *gk = static_cast<const K *>(t.keys);
    const bool act = gl < LL;

    for (uint64_t base = warp * TILE; base < nq; base += nwarps * TILE) {
        K a[QG], b[QG], qe[I];
        bool up[I], valid[QG];
        uint64_t node[I];
#pragma unroll
        for (int j = 0; j < QG; j++) {
            const uint64_t qi = base + (uint64_t)j * QPW + grp;
            valid[j] = qi < nq;
            a[j] = valid[j] ? lo[qi] : (K)0;
            b[j] = valid[j] ? hi[qi] : (K)0;
            // lower bound of a: a > max gives n (walk on max instead)
            qe[2 * j] = a[j] <= tmax ? a[j] : tmax;
            up[2 * j] = false;
            // upper bound of b: b >= max gives n (walk a lower bound of max instead)
            qe[2 * j + 1] = b[j] < tmax ? b[j] : tmax;
            up[2 * j + 1] = b[j] < tmax;
        }
        descend<K, G, I>(t, s_top, qe, up, node, grp, gl);
        K kk[I][LPL];
#pragma unroll
        for (int s = 0; s < I; s++) {
#pragma unroll
            for (int j = 0; j < LPL; j++) kk[s][j] = 0;
            if (act) load_stream<K, LPL>(gk + node[s] * S + (uint64_t)gl * LPL, kk[s]);
        }
#pragma unroll
        for (int j = 0; j < QG; j++) {
            int c0 = act ? count_below<K, LPL>(kk[2 * j], qe[2 * j], false) : 0;
            int c1 = act ? count_below<K, LPL>(kk[2 * j + 1], qe[2 * j + 1], up[2 * j + 1]) : 0;
            const int p0 = group_count<G, LL, LPL>(c0, act, grp);
            const int p1 = group_count<G, LL, LPL>(c1, act, grp);
            if (gl == 0 && valid[j]) {
                const uint64_t lb = a[j] <= tmax ? node[2 * j] * S + (uint64_t)p0 : t.n;
                const uint64_t ub = b[j] < tmax ? node[2 * j + 1] * S + (uint64_t)p1 : t.n;
                const uint64_t qi = base + (uint64_t)j * QPW + grp;
                const uint64_t dst = PERM ? (uint64_t)perm[qi] : qi;
                counts[dst] = (a[j] <= b[j] && ub > lb) ? ub - lb : 0;
                if (lb_out) lb_out[dst] = lb;
            }
        }
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

// Resident CTAs per SM for a kernel at a given dynamic shared memory size.
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

template <typename K, typename V, bool PERM>
bt_status point_dispatch(const bt_tree *t, const void *d_q, const uint32_t *d_perm, uint64_t nq,
                         void *d_out, cudaStream_t s) {
    // Lanes per query and queries in flight per group (see bt_search.cuh).
    constexpr int G = 8;
    constexpr int I = 2;
    auto fn = point_kernel<K, V, G, I, PERM>;
    const size_t smem = (size_t)t->dev.smem_elems * sizeof(K);
    const unsigned grid = persistent_grid((const void *)fn, smem, nq, (kThreads / 32) * (32 / G) * I);
    count_launch();
    fn<<<grid, kThreads, smem, s>>>(t->dev, (const K *)d_q, d_perm, nq, (V *)d_out);
    BT_CUDA(cudaGetLastError());
    return BT_OK;
}

template <typename K, bool PERM>
bt_status bounds_dispatch(const bt_tree *t, const void *d_lo, const void *d_hi,
                          const uint32_t *d_perm, uint64_t nq, uint64_t *d_counts,
                          uint64_t *d_lb, cudaStream_t s) {
    constexpr int G = 8;
    constexpr int QG = 1;
    auto fn = bounds_kernel<K, G, QG, PERM>;
    const size_t smem = (size_t)t->dev.smem_elems * sizeof(K);
    const unsigned grid = persistent_grid((const void *)fn, smem, nq, (kThreads / 32) * (32 / G) * QG);
    count_launch();
    fn<<<grid, kThreads, smem, s>>>(t->dev, (const K *)d_lo, (const K *)d_hi, d_perm, nq, d_counts,
                                    d_lb);
    BT_CUDA(cudaGetLastError());
    return BT_OK;
}

}  // namespace

bt_status launch_point_search(const bt_tree *t, const void *d_q, const uint32_t *d_perm,
                              uint64_t nq, void *d_out, cudaStream_t s) {
    if (nq == 0) return BT_OK;
    if (t->n == 0) {
        unsigned g = (unsigned)std::min<uint64_t>((nq + 255) / 256, 4096);
        count_launch();
        if (t->val_bytes == 4)
            fill_kernel<uint32_t><<<g, 256, 0, s>>>((uint32_t *)d_out, nq, 0xFFFFFFFFu);
        else
            fill_kernel<uint64_t><<<g, 256, 0, s>>>((uint64_t *)d_out, nq, ~0ull);
        BT_CUDA(cudaGetLastError());
        return BT_OK;
    }
    const bool perm = d_perm != nullptr;
    if (t->key_bytes == 4) {
        if (t->val_bytes == 4)
            return perm ? point_dispatch<uint32_t, uint32_t, true>(t, d_q, d_perm, nq, d_out, s)
                        : point_dispatch<uint32_t, uint32_t, false>(t, d_q, d_perm, nq, d_out, s);
        return perm ? point_dispatch<uint32_t, uint64_t, true>(t, d_q, d_perm, nq, d_out, s)
                    : point_dispatch<uint32_t, uint64_t, false>(t, d_q, d_perm, nq, d_out, s);
    }
    if (t->val_bytes == 4)
        return perm ? point_dispatch<uint64_t, uint32_t, true>(t, d_q, d_perm, nq, d_out, s)
                    : point_dispatch<uint64_t, uint32_t, false>(t, d_q, d_perm, nq, d_out, s);
    return perm ? point_dispatch<uint64_t, uint64_t, true>(t, d_q, d_perm, nq, d_out, s)
                : point_dispatch<uint64_t, uint64_t, false>(t, d_q, d_perm, nq, d_out, s);
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
    const bool perm = d_perm != nullptr;
    if (t->key_bytes == 4)
        return perm ? bounds_dispatch<uint32_t, true>(t, d_lo, d_hi, d_perm, nq, d_counts, d_lb, s)
                    : bounds_dispatch<uint32_t, false>(t, d_lo, d_hi, d_perm, nq, d_counts, d_lb, s);
    return perm ? bounds_dispatch<uint64_t, true>(t, d_lo, d_hi, d_perm, nq, d_counts, d_lb, s)
                : bounds_dispatch<uint64_t, false>(t, d_lo, d_hi, d_perm, nq, d_counts, d_lb, s);
}

}  // namespace bt
