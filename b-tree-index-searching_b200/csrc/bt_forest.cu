// Batched forest of uneven trees (declared in include/btree_b200.h).
//
// In the reference every tree is its own genBPlusTree call (a 16 GB page
// pool each, BPTree.cu:163) and every batch its own synchronous search call,
// so thousands of small trees cost thousands of host round trips.  Here:
//   build  all trees go into one leaf array and one separator array (the
//          single-tree layout, tree after tree) with a descriptor per tree,
//          in a few flat kernels: one over every leaf block of every tree,
//          then one per level depth over every tree that has that level;
//   search a plan cuts each tree's point and range queries into work items
//          of `tile` queries; one persistent kernel, whose warps take items
//          from a device queue (so trees of very different sizes balance),
//          answers them all; the plan records that launch once as a CUDA
//          graph and replays it.
#include <algorithm>
#include <cstring>
#include <vector>

#include "bt_search.cuh"

namespace bt {
namespace {

constexpr int kFMaxLevels = 10;

struct FTree {
    uint64_t block0;   // first leaf block of the tree
    uint64_t sep0;     // first separator element of the tree
    uint64_t n;        // keys
    uint64_t max_key;  // largest key (valid when n > 0)
    uint64_t in_off;   // offset of the tree's keys in the build input
    int32_t nlevels;   // 0 for an empty tree
    int32_t pad;
    uint64_t lvl_off[kFMaxLevels];  // level offsets relative to sep0, root first
};

struct FItem {
    uint32_t tree;
    uint32_t kind;  // 0 point, 1 range
    uint64_t begin;
    uint64_t count;
    int32_t slvl;  // separator level staged in shared memory for this item, -1 for none
    uint32_t sm;   // its entries (a whole number of 128-byte nodes)
};

// --------------------------------------------------------------- build ----

template <typename K, typename V>
__global__ void forest_leaf_kernel(const K *__restrict__ keys, const V *__restrict__ vals,
                                   const FTree *__restrict__ desc, uint32_t ntrees,
                                   uint64_t total_blocks, unsigned char *__restrict__ leaves,
                                   unsigned int *__restrict__ flags) {
    using LG = LeafGeom<K, V>;
    unsigned int f = 0;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < total_blocks * LG::S;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t b = i / LG::S;
        const int slot = (int)(i % LG::S);
        // tree of block b: last tree with block0 <= b (empty trees own no block)
        uint32_t lo = 0, len = ntrees;
        while (len > 1) {
            const uint32_t half = len >> 1;
            lo = desc[lo + half].block0 <= b ? lo + half : lo;
            len -= half;
        }
        while (lo + 1 < ntrees && desc[lo + 1].block0 == desc[lo].block0 && desc[lo].n == 0) lo++;
        const FTree &d = desc[lo];
        const uint64_t p = (b - d.block0) * LG::S + slot;
        K k = key_max<K>();
        V v = 0;
        if (p < d.n) {
            k = keys[d.in_off + p];
            v = vals[d.in_off + p];
            if (p + 1 < d.n && keys[d.in_off + p + 1] < k) f |= 1u;
        }
        unsigned char *blk = leaves + b * LG::BS;
        reinterpret_cast<K *>(blk)[slot] = k;
        reinterpret_cast<V *>(blk + kSectorBytes)[slot] = v;
    }
    unsigned int w = __reduce_or_sync(0xffffffffu, f);
    if ((threadIdx.x & 31) == 0 && w) atomicOr(flags, w);
}

// One level depth of every tree: entry j of level l of tree t (l = nlevels-1-
// depth) is the maximum of its child (a leaf block at depth 0, else the last
// separator of child node j on level l+1); padding entries are all-ones.
template <typename K, typename V>
__global__ void forest_level_kernel(const FTree *__restrict__ desc, const uint32_t *__restrict__ ptree,
                                    const uint64_t *__restrict__ pprefix,
                                    const uint64_t *__restrict__ pentries, uint32_t nitems,
                                    int depth, const unsigned char *__restrict__ leaves,
                                    K *__restrict__ seps) {
    using LG = LeafGeom<K, V>;
    constexpr int F = kLineBytes / (int)sizeof(K);
    const uint64_t total = pprefix[nitems];
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < total;
         i += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t lo = 0, len = nitems;
        while (len > 1) {
            const uint32_t half = len >> 1;
            lo = pprefix[lo + half] <= i ? lo + half : lo;
            len -= half;
        }
        const FTree &d = desc[ptree[lo]];
        const uint64_t j = i - pprefix[lo];
        const int l = d.nlevels - 1 - depth;
        K v = key_max<K>();
        if (j < pentries[lo]) {
            if (depth == 0)
                v = reinterpret_cast<const K *>(leaves + (d.block0 + j) * LG::BS)[LG::S - 1];
            else
                v = seps[d.sep0 + d.lvl_off[l + 1] + j * F + F - 1];
        }
        seps[d.sep0 + d.lvl_off[l] + j] = v;
    }
}

template <typename K>
__global__ void forest_max_kernel(const K *__restrict__ keys, FTree *__restrict__ desc,
                                  uint32_t ntrees) {
    for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < ntrees; t += gridDim.x * blockDim.x)
        desc[t].max_key = desc[t].n ? (uint64_t)keys[desc[t].in_off + desc[t].n - 1] : 0;
}

}  // namespace
}  // namespace bt

struct bt_forest {
    int device;
    int key_bytes, val_bytes;
    uint32_t num_trees;
    void *d_leaves = nullptr;
    void *d_seps = nullptr;
    bt::FTree *d_desc = nullptr;
    std::vector<bt::FTree> h_desc;
    // staged-root fanout: separator entries a work item may stage in shared
    // memory per descent it makes (bt_forest_set_stage_fanout)
    uint32_t stage_fanout = 16;
};

struct bt_forest_plan {
    const bt_forest *forest;
    bt::FItem *d_items = nullptr;
    uint64_t n_items = 0;
    unsigned long long *d_counter = nullptr;
    cudaStream_t cap = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
};

namespace bt {
namespace {

template <typename K, typename V>
bt_status forest_build_impl(bt_forest *f, const void *d_keys, const void *d_vals,
                            const uint64_t *off, cudaStream_t s) {
    using LG = LeafGeom<K, V>;
    constexpr int F = kLineBytes / (int)sizeof(K);
    const uint32_t T = f->num_trees;
    f->h_desc.assign(T, FTree());
    uint64_t blocks = 0, seps = 0;
    int maxdepth = 0;
    std::vector<std::vector<uint64_t>> ent(T);  // real entries per level, root first
    for (uint32_t t = 0; t < T; t++) {
        FTree &d = f->h_desc[t];
        std::memset(&d, 0, sizeof(d));
        d.n = off[t + 1] - off[t];
        d.in_off = off[t];
        d.block0 = blocks;
        d.sep0 = seps;
        if (d.n == 0) continue;
        const uint64_t nb = (d.n + LG::S - 1) / LG::S;
        std::vector<uint64_t> e_bu, n_bu;
        uint64_t e = nb;
        for (;;) {
            const uint64_t nodes = (e + F - 1) / F;
            e_bu.push_back(e);
            n_bu.push_back(nodes);
            if (nodes == 1) break;
            e = nodes;
        }
        const int L = (int)e_bu.size();
        if (L > kFMaxLevels) return fail(BT_ERR_INVALID_ARGUMENT, "a forest tree is too large");
        d.nlevels = L;
        uint64_t o = 0;
        ent[t].resize(L);
        for (int l = 0; l < L; l++) {
            d.lvl_off[l] = o;
            ent[t][l] = e_bu[L - 1 - l];
            o += n_bu[L - 1 - l] * F;
        }
        blocks += nb;
        seps += o;
        maxdepth = std::max(maxdepth, L);
    }
    if (blocks) {
        BT_CUDA(cudaMalloc(&f->d_leaves, blocks * LG::BS));
        BT_CUDA(cudaMemsetAsync(f->d_leaves, 0, blocks * LG::BS, s));
    }
    if (seps) BT_CUDA(cudaMalloc(&f->d_seps, seps * sizeof(K)));
    BT_CUDA(cudaMalloc((void **)&f->d_desc, T * sizeof(FTree)));
    BT_CUDA(cudaMemcpyAsync(f->d_desc, f->h_desc.data(), T * sizeof(FTree), cudaMemcpyHostToDevice, s));
    WsGuard g_flags(s);
    bt_status st = g_flags.alloc(sizeof(unsigned int));
    if (st != BT_OK) return st;
    unsigned int *d_flags = g_flags.as<unsigned int>();
    BT_CUDA(cudaMemsetAsync(d_flags, 0, sizeof(unsigned int), s));
    const unsigned grid = (unsigned)std::min<uint64_t>(std::max<uint64_t>(1, (blocks * LG::S + 255) / 256),
                                                       (uint64_t)sm_count() * 16);
    if (blocks) {
        count_launch();
        forest_leaf_kernel<K, V><<<grid, 256, 0, s>>>((const K *)d_keys, (const V *)d_vals, f->d_desc,
                                                      T, blocks, (unsigned char *)f->d_leaves, d_flags);
    }
    count_launch();
    forest_max_kernel<K><<<(T + 255) / 256, 256, 0, s>>>((const K *)d_keys, f->d_desc, T);
    // one pass per level depth, bottom up
    std::vector<uint32_t> ptree;
    std::vector<uint64_t> pprefix, pentries;
    for (int depth = 0; depth < maxdepth && st == BT_OK; depth++) {
        ptree.clear();
        pentries.clear();
        pprefix.assign(1, 0);
        for (uint32_t t = 0; t < T; t++) {
            const FTree &d = f->h_desc[t];
            if (d.nlevels <= depth) continue;
            const int l = d.nlevels - 1 - depth;
            const uint64_t padded = (l + 1 < d.nlevels ? d.lvl_off[l + 1] : 0) - d.lvl_off[l];
            const uint64_t pad_len = l + 1 < d.nlevels ? padded
                                                      : ((ent[t][l] + F - 1) / F) * F;
            ptree.push_back(t);
            pentries.push_back(ent[t][l]);
            pprefix.push_back(pprefix.back() + pad_len);
        }
        const uint32_t m = (uint32_t)ptree.size();
        uint32_t *d_pt = nullptr;
        uint64_t *d_pp = nullptr, *d_pe = nullptr;
        st = ws_alloc((void **)&d_pt, m * sizeof(uint32_t), s);
        if (st == BT_OK) st = ws_alloc((void **)&d_pp, (m + 1) * sizeof(uint64_t), s);
        if (st == BT_OK) st = ws_alloc((void **)&d_pe, m * sizeof(uint64_t), s);
        if (st == BT_OK) {
            cudaMemcpyAsync(d_pt, ptree.data(), m * sizeof(uint32_t), cudaMemcpyHostToDevice, s);
            cudaMemcpyAsync(d_pp, pprefix.data(), (m + 1) * sizeof(uint64_t), cudaMemcpyHostToDevice, s);
            cudaMemcpyAsync(d_pe, pentries.data(), m * sizeof(uint64_t), cudaMemcpyHostToDevice, s);
            const uint64_t total = pprefix.back();
            const unsigned g2 = (unsigned)std::min<uint64_t>(std::max<uint64_t>(1, (total + 255) / 256),
                                                             (uint64_t)sm_count() * 16);
            count_launch();
            forest_level_kernel<K, V><<<g2, 256, 0, s>>>(f->d_desc, d_pt, d_pp, d_pe, m, depth,
                                                         (const unsigned char *)f->d_leaves,
                                                         (K *)f->d_seps);
            // the host vectors are reused next pass: wait for the copies
            cudaStreamSynchronize(s);
        }
        ws_free(d_pt, s);
        ws_free(d_pp, s);
        ws_free(d_pe, s);
    }
    unsigned int flags = 0;
    BT_CUDA(cudaMemcpyAsync(&flags, d_flags, sizeof(flags), cudaMemcpyDeviceToHost, s));
    BT_CUDA(cudaMemcpyAsync(f->h_desc.data(), f->d_desc, T * sizeof(FTree), cudaMemcpyDeviceToHost, s));
    BT_CUDA(cudaStreamSynchronize(s));
    BT_CUDA(cudaGetLastError());
    if (st != BT_OK) return st;
    if (flags & 1u) return fail(BT_ERR_UNSORTED, "a forest tree's keys are not sorted ascending");
    return BT_OK;
}

// --------------------------------------------------------------- search ---

constexpr int kFThreads = 256;
constexpr int kFWarps = kFThreads / 32;
constexpr size_t kFStageBytes = 16 * 1024;  // separator level staged per work item

struct ForestDev {
    const FTree *desc;
    const unsigned char *leaves;
    const void *seps;
};

// One CTA per work item (one tree, up to `tile` queries of one kind), taken
// from a device queue so trees of very different sizes balance.  For an
// item with enough queries the CTA stages the deepest separator level of its
// tree that fits in 16 KB (chosen on the host: the item's slvl/sm); a binary
// search there resolves every level above it, the remaining levels and the
// leaf are walked by lane groups as in the single-tree kernels.
template <typename K, typename V, int G, int R>
__global__ void __launch_bounds__(kFThreads, 4)
forest_kernel(const __grid_constant__ ForestDev f, const FItem *__restrict__ items, uint64_t n_items,
              unsigned long long *__restrict__ counter, const K *__restrict__ q,
              V *__restrict__ out, const K *__restrict__ lo, const K *__restrict__ hi,
              uint64_t *__restrict__ counts) {
    __shared__ __align__(16) K s_lvl[kFStageBytes / sizeof(K)];
    __shared__ uint64_t s_res[kFWarps][64];
    __shared__ unsigned long long s_item;
    using LG = LeafGeom<K, V>;
    constexpr int NG = 32 / G;
    constexpr int I = G / R;
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int grp = lane / G;
    const int gl = lane % G;
    uint64_t *res = s_res[warp];
    const K *seps = static_cast<const K *>(f.seps);

    for (;;) {
        __syncthreads();  // the previous item's staged level is no longer read
        if (threadIdx.x == 0) s_item = atomicAdd(counter, 1ull);
        __syncthreads();
        const unsigned long long it = s_item;
        if (it >= n_items) break;
        const FItem w = items[it];
        const FTree &d = f.desc[w.tree];
        const uint64_t n = d.n;
        const int nl = d.nlevels;
        const K tmax = (K)d.max_key;
        const K *tseps = seps + d.sep0;
        const unsigned char *tleaves = f.leaves + d.block0 * LG::BS;
        const int sl = n > 0 ? w.slvl : -1;
        if (sl >= 0) {
            const K *src = tseps + d.lvl_off[sl];
            for (uint32_t i = threadIdx.x; i < w.sm; i += kFThreads) s_lvl[swz<K>(i)] = src[i];
            __syncthreads();
        }
        const int from = sl + 1;  // first level walked in global memory
        for (uint64_t sub = (uint64_t)warp * 32; sub < w.count; sub += kFWarps * 32) {
            const uint64_t base = w.begin + sub;
            const uint64_t end = w.begin + w.count;
            const uint64_t my = base + lane;
            if (w.kind == 0) {
                const K myq = my < end ? q[my] : (K)0;
                if (n == 0) {
                    if (my < end) out[my] = key_max<V>();
                    continue;
                }
                const K myqe = myq < tmax ? myq : tmax;
                const uint32_t mynode = sl >= 0 ? smem_bound<K>(s_lvl, w.sm, myqe, false) : 0u;
#pragma unroll
                for (int r = 0; r < R; r++) {
                    K qv[I], qe[I];
                    bool up[I];
                    uint32_t node[I];
#pragma unroll
                    for (int s = 0; s < I; s++) {
                        const int k = r * (NG * I) + s * NG + grp;
                        qv[s] = __shfl_sync(0xffffffffu, myq, k);
                        node[s] = __shfl_sync(0xffffffffu, mynode, k);
                        qe[s] = qv[s] < tmax ? qv[s] : tmax;
                        up[s] = false;
                    }
                    for (int lvl = from; lvl < nl; lvl++)
                        level_step<K, G, I>(tseps + d.lvl_off[lvl], qe, up, node, grp, gl);
                    leaf_point<K, V, G, I>(tleaves, node, qv, qe, tmax, grp, gl, [&](int s) -> V * {
                        const uint64_t qi = base + (uint64_t)(r * (NG * I) + s * NG + grp);
                        return qi < end ? out + qi : nullptr;
                    });
                }
            } else {
                // 64 descents: lower bounds of lo (d < 32), upper bounds of hi
                const bool v = my < end;
                const K a = v ? lo[my] : (K)0;
                const K b = v ? hi[my] : (K)0;
                if (n > 0) {
                    const K qa = a <= tmax ? a : tmax;
                    const K qb = b < tmax ? b : tmax;
                    const bool ub_upper = b < tmax;
                    const uint32_t na = sl >= 0 ? smem_bound<K>(s_lvl, w.sm, qa, false) : 0u;
                    const uint32_t nb = sl >= 0 ? smem_bound<K>(s_lvl, w.sm, qb, ub_upper) : 0u;
#pragma unroll
                    for (int r = 0; r < 2 * R; r++) {
                        const bool which = r >= R;
                        K qe[I];
                        bool up[I];
                        uint32_t node[I];
#pragma unroll
                        for (int s = 0; s < I; s++) {
                            const int k = (r % R) * (NG * I) + s * NG + grp;
                            qe[s] = __shfl_sync(0xffffffffu, which ? qb : qa, k);
                            node[s] = __shfl_sync(0xffffffffu, which ? nb : na, k);
                            up[s] = which ? __shfl_sync(0xffffffffu, (int)ub_upper, k) != 0 : false;
                        }
                        for (int lvl = from; lvl < nl; lvl++)
                            level_step<K, G, I>(tseps + d.lvl_off[lvl], qe, up, node, grp, gl);
                        int pos[I];
                        leaf_bound<K, V, G, I>(tleaves, node, qe, up, grp, gl, pos);
#pragma unroll
                        for (int s = 0; s < I; s++)
                            if (gl == 0)
                                res[(which ? 32 : 0) + (r % R) * (NG * I) + s * NG + grp] =
                                    (uint64_t)node[s] * LG::S + pos[s];
                    }
                }
                __syncwarp();
                if (v) {
                    uint64_t c = 0;
                    if (n > 0) {
                        const uint64_t lb = a <= tmax ? res[lane] : n;
                        const uint64_t ub = b < tmax ? res[32 + lane] : n;
                        c = (a <= b && ub > lb) ? ub - lb : 0;
                    }
                    counts[my] = c;
                }
                __syncwarp();
            }
        }
    }
}

struct PlanArgs {
    const void *q;
    void *out;
    const void *lo;
    const void *hi;
    uint64_t *counts;
};

template <typename K, typename V, int G, int R>
bt_status forest_capture(bt_forest_plan *p, const PlanArgs &a) {
    auto fn = forest_kernel<K, V, G, R>;
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kFThreads, 0) != cudaSuccess ||
        per_sm < 1)
        per_sm = 1;
    const uint64_t ctas = std::min<uint64_t>(std::max<uint64_t>(1, p->n_items), (uint64_t)sm_count() * per_sm);
    ForestDev fd{p->forest->d_desc, (const unsigned char *)p->forest->d_leaves, p->forest->d_seps};
    BT_CUDA(cudaStreamBeginCapture(p->cap, cudaStreamCaptureModeThreadLocal));
    cudaMemsetAsync(p->d_counter, 0, sizeof(unsigned long long), p->cap);
    fn<<<(unsigned)ctas, kFThreads, 0, p->cap>>>(fd, p->d_items, p->n_items, p->d_counter,
                                                 (const K *)a.q, (V *)a.out, (const K *)a.lo,
                                                 (const K *)a.hi, a.counts);
    const cudaError_t le = cudaGetLastError();
    const cudaError_t ee = cudaStreamEndCapture(p->cap, &p->graph);
    if (le != cudaSuccess) return cuda_fail(le, "forest kernel launch (capture)");
    if (ee != cudaSuccess) return cuda_fail(ee, "cudaStreamEndCapture");
    BT_CUDA(cudaGraphInstantiate(&p->exec, p->graph, 0));
    return BT_OK;
}

template <typename K, typename V>
bt_status forest_capture_cfg(bt_forest_plan *p, const PlanArgs &a, int g, int r) {
    if (g == 8 && r == 1) return forest_capture<K, V, 8, 1>(p, a);
    if (g == 8 && r == 2) return forest_capture<K, V, 8, 2>(p, a);
    if (g == 4 && r == 1) return forest_capture<K, V, 4, 1>(p, a);
    if (g == 4 && r == 2) return forest_capture<K, V, 4, 2>(p, a);
    if (g == 2 && r == 1) return forest_capture<K, V, 2, 1>(p, a);
    return fail(BT_ERR_INVALID_ARGUMENT, "unsupported (lanes, rounds) search configuration");
}

void free_plan(bt_forest_plan *p) {
    if (!p) return;
    if (p->exec) cudaGraphExecDestroy(p->exec);
    if (p->graph) cudaGraphDestroy(p->graph);
    if (p->d_items) cudaFree(p->d_items);
    if (p->d_counter) cudaFree(p->d_counter);
    if (p->cap) cudaStreamDestroy(p->cap);
    delete p;
}

}  // namespace
}  // namespace bt

extern "C" {

bt_status bt_forest_build(const void *d_keys, const void *d_vals, const uint64_t *h_off,
                          uint32_t num_trees, int key_bytes, int value_bytes, void *stream,
                          bt_forest **out) {
    using namespace bt;
    if (!out || !h_off) return fail(BT_ERR_INVALID_ARGUMENT, "out or offsets is NULL");
    *out = nullptr;
    if (num_trees == 0) return fail(BT_ERR_INVALID_ARGUMENT, "num_trees is 0");
    if ((key_bytes != 4 && key_bytes != 8) || (value_bytes != 4 && value_bytes != 8))
        return fail(BT_ERR_INVALID_ARGUMENT, "key_bytes and value_bytes must be 4 or 8");
    for (uint32_t t = 0; t < num_trees; t++)
        if (h_off[t + 1] < h_off[t]) return fail(BT_ERR_INVALID_ARGUMENT, "offsets must not decrease");
    if (h_off[num_trees] > 0 && (!d_keys || !d_vals))
        return fail(BT_ERR_INVALID_ARGUMENT, "keys or values is NULL");
    int dev = 0;
    BT_CUDA(cudaGetDevice(&dev));
    bt_status st = require_device(dev);
    if (st != BT_OK) return st;
    bt_forest *f = new bt_forest();
    f->device = dev;
    f->key_bytes = key_bytes;
    f->val_bytes = value_bytes;
    f->num_trees = num_trees;
    cudaStream_t s = (cudaStream_t)stream;
    if (key_bytes == 4)
        st = value_bytes == 4 ? forest_build_impl<uint32_t, uint32_t>(f, d_keys, d_vals, h_off, s)
                              : forest_build_impl<uint32_t, uint64_t>(f, d_keys, d_vals, h_off, s);
    else
        st = value_bytes == 4 ? forest_build_impl<uint64_t, uint32_t>(f, d_keys, d_vals, h_off, s)
                              : forest_build_impl<uint64_t, uint64_t>(f, d_keys, d_vals, h_off, s);
    if (st != BT_OK) {
        bt_forest_destroy(f);
        return st;
    }
    *out = f;
    return BT_OK;
}

bt_status bt_forest_destroy(bt_forest *f) {
    if (!f) return BT_OK;
    cudaDeviceSynchronize();
    if (f->d_leaves) cudaFree(f->d_leaves);
    if (f->d_seps) cudaFree(f->d_seps);
    if (f->d_desc) cudaFree(f->d_desc);
    delete f;
    return BT_OK;
}

bt_status bt_forest_plan_create(const bt_forest *f, const void *d_q, const uint64_t *h_qoff,
                                void *d_out, const void *d_lo, const void *d_hi,
                                const uint64_t *h_roff, uint64_t *d_counts, int lanes, int rounds,
                                uint32_t tile, bt_forest_plan **out) {
    using namespace bt;
    if (!f || !out || !h_qoff) return fail(BT_ERR_INVALID_ARGUMENT, "forest, out or offsets is NULL");
    *out = nullptr;
    if (tile == 0 || tile % 32) return fail(BT_ERR_INVALID_ARGUMENT, "tile must be a positive multiple of 32");
    if (search_cfg_index(lanes, rounds) < 0)
        return fail(BT_ERR_INVALID_ARGUMENT, "unsupported (lanes, rounds) search configuration");
    const uint32_t T = f->num_trees;
    std::vector<FItem> items;
    for (uint32_t t = 0; t < T; t++) {
        if (h_qoff[t + 1] < h_qoff[t]) return fail(BT_ERR_INVALID_ARGUMENT, "query offsets decrease");
        for (uint64_t b = h_qoff[t]; b < h_qoff[t + 1]; b += tile)
            items.push_back({t, 0u, b, std::min<uint64_t>(tile, h_qoff[t + 1] - b), -1, 0u});
    }
    if (h_qoff[T] > 0 && (!d_q || !d_out)) return fail(BT_ERR_INVALID_ARGUMENT, "queries or out is NULL");
    if (h_roff) {
        for (uint32_t t = 0; t < T; t++) {
            if (h_roff[t + 1] < h_roff[t]) return fail(BT_ERR_INVALID_ARGUMENT, "range offsets decrease");
            for (uint64_t b = h_roff[t]; b < h_roff[t + 1]; b += tile)
                items.push_back({t, 1u, b, std::min<uint64_t>(tile, h_roff[t + 1] - b), -1, 0u});
        }
        if (h_roff[T] > 0 && (!d_lo || !d_hi || !d_counts))
            return fail(BT_ERR_INVALID_ARGUMENT, "lo, hi or counts is NULL");
    }
    // The level each item stages: the deepest one that fits kFStageBytes and
    // is not much larger than the descents it saves (stage_fanout entries
    // per descent: the fanout of the shared-memory root the item's queries
    // search first).
    {
        const int kb = f->key_bytes;
        const uint64_t S = kSectorBytes / kb, F = kLineBytes / kb;
        for (FItem &it : items) {
            const FTree &d = f->h_desc[it.tree];
            if (d.n == 0) continue;
            const uint64_t descents = it.count * (it.kind == 0 ? 1 : 2);
            for (int l = d.nlevels - 1; l >= 0; l--) {
                const uint64_t nb = (d.n + S - 1) / S;
                const uint64_t ent = l + 1 < d.nlevels ? d.lvl_off[l + 1] - d.lvl_off[l]
                                                       : (nb + F - 1) / F * F;
                if (ent * kb <= kFStageBytes && ent <= (uint64_t)f->stage_fanout * descents) {
                    it.slvl = l;
                    it.sm = (uint32_t)ent;
                    break;
                }
            }
        }
    }
    // largest work items first: the queue ends with small ones, which balances the tail
    std::stable_sort(items.begin(), items.end(),
                     [](const FItem &x, const FItem &y) { return x.count > y.count; });
    int prev = 0;
    BT_CUDA(cudaGetDevice(&prev));
    BT_CUDA(cudaSetDevice(f->device));
    bt_forest_plan *p = new bt_forest_plan();
    p->forest = f;
    p->n_items = items.size();
    bt_status st = BT_OK;
    cudaError_t e = cudaStreamCreateWithFlags(&p->cap, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMalloc((void **)&p->d_counter, sizeof(unsigned long long));
    if (e == cudaSuccess && !items.empty()) e = cudaMalloc((void **)&p->d_items, items.size() * sizeof(FItem));
    if (e == cudaSuccess && !items.empty())
        e = cudaMemcpy(p->d_items, items.data(), items.size() * sizeof(FItem), cudaMemcpyHostToDevice);
    if (e != cudaSuccess) st = cuda_fail(e, "forest plan set-up");
    PlanArgs a{d_q, d_out, d_lo, d_hi, d_counts};
    if (st == BT_OK) {
        if (f->key_bytes == 4)
            st = f->val_bytes == 4 ? forest_capture_cfg<uint32_t, uint32_t>(p, a, lanes, rounds)
                                   : forest_capture_cfg<uint32_t, uint64_t>(p, a, lanes, rounds);
        else
            st = f->val_bytes == 4 ? forest_capture_cfg<uint64_t, uint32_t>(p, a, lanes, rounds)
                                   : forest_capture_cfg<uint64_t, uint64_t>(p, a, lanes, rounds);
    }
    cudaSetDevice(prev);
    if (st != BT_OK) {
        free_plan(p);
        return st;
    }
    *out = p;
    return BT_OK;
}

bt_status bt_forest_set_stage_fanout(bt_forest *f, uint32_t entries_per_descent) {
    using namespace bt;
    if (!f) return fail(BT_ERR_INVALID_ARGUMENT, "forest is NULL");
    if (entries_per_descent < 1 || entries_per_descent > 4096)
        return fail(BT_ERR_INVALID_ARGUMENT, "entries_per_descent must be 1..4096");
    f->stage_fanout = entries_per_descent;
    return BT_OK;
}

bt_status bt_forest_plan_run(bt_forest_plan *p, void *stream) {
    using namespace bt;
    if (!p) return fail(BT_ERR_INVALID_ARGUMENT, "plan is NULL");
    count_launch();
    BT_CUDA(cudaGraphLaunch(p->exec, (cudaStream_t)stream));
    return BT_OK;
}

bt_status bt_forest_plan_destroy(bt_forest_plan *p) {
    if (!p) return BT_OK;
    cudaStreamSynchronize(p->cap);
    bt::free_plan(p);
    return BT_OK;
}

}  // extern "C"
