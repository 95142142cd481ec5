// Learned position model: training kernels and the learned point search.
//
// No counterpart in the reference (its descent is always the page walk of
// BPTreeExactSearch.cu:39-68).  Two stages over the tree's (key, rank)
// pairs:
//   root   y = b2 + sum_j w2[j] * relu(w1[j] * x + b1[j]),  x = key normalised
//          to [0,1], y = rank normalised to [0,1); w1, w2 >= 0 keep it
//          monotone, so the segments it routes to are contiguous key ranges.
//          Trained by full-batch Adam on MSE with mlp_loss_grad_kernel /
//          adam_kernel below.
//   leaves rank = r_lo + icpt + slope * (key - base) per segment, fitted by
//          least squares; eps = max error over the segment's keys, measured
//          with the very same FP32 operations the search uses (explicit
//          round-to-nearest intrinsics, no contraction), so the bound holds
//          bit for bit.
// The search turns the predicted rank window into a window of entries on the
// separator level one above the bottom, scans those lines with the lane
// group, then descends normally.  If the scan cannot prove the lower bound is
// inside the window, that query takes the full descent (scalar, per lane).
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <vector>

#include "bt_search.cuh"

namespace bt {

struct LearnedState {
    float *d_mlp = nullptr;        // 3H+1
    SegParam *d_seg = nullptr;     // nseg
    unsigned long long *d_stats = nullptr;  // 2 counters
    LearnedDev dev;
};

void free_learned(LearnedState *s) {
    if (!s) return;
    if (s->d_mlp) cudaFree(s->d_mlp);
    if (s->d_seg) cudaFree(s->d_seg);
    if (s->d_stats) cudaFree(s->d_stats);
    delete s;
}

namespace {

// ---------------------------------------------------------------- model ---

// Root model in FP32 with explicit round-to-nearest operations (the same
// arithmetic in training-time assignment, eps measurement and search).
__device__ __forceinline__ float mlp_eval(const float *p, int H, float x) {
    float out = p[3 * H];
    for (int j = 0; j < H; j++) {
        const float h = __fadd_rn(__fmul_rn(p[j], x), p[H + j]);
        out = __fadd_rn(out, __fmul_rn(p[2 * H + j], fmaxf(h, 0.f)));
    }
    return out;
}

__device__ __forceinline__ float norm_key(uint64_t key, uint64_t kmin, float xscale) {
    return __fmul_rn(__ull2float_rn(key > kmin ? key - kmin : 0ull), xscale);
}

__device__ __forceinline__ uint32_t root_segment(const float *p, int H, uint32_t nseg, float x) {
    const float y = __fmul_rn(mlp_eval(p, H, x), (float)nseg);
    if (!(y > 0.f)) return 0;  // also catches NaN
    const float f = floorf(y);
    return f >= (float)nseg ? nseg - 1 : (uint32_t)f;
}

// Relative rank predicted by a leaf model for a key (FP32, round to
// nearest), clamped to the segment's rank range [0, cnt]: a key in the gap
// after the segment's last key (lognormal gaps can be 10^6 wide) must not be
// extrapolated along the line, its lower bound is at most the next segment's
// first rank.
__device__ __forceinline__ float leaf_pred(const SegParam &s, uint64_t key) {
    const uint64_t d = key > s.base ? key - s.base : 0ull;
    const float p = __fadd_rn(s.icpt, __fmul_rn(s.slope, __ull2float_rn(d)));
    return fminf(fmaxf(p, 0.f), (float)s.cnt);
}

template <typename K, typename V>
__device__ __forceinline__ K leaf_key(const unsigned char *leaves, uint64_t pos) {
    using LG = LeafGeom<K, V>;
    return reinterpret_cast<const K *>(leaves + (pos / LG::S) * LG::BS)[pos % LG::S];
}

// ------------------------------------------------------------- training ---

template <typename K, typename V>
__global__ void sample_kernel(const unsigned char *__restrict__ leaves, uint64_t n, uint64_t m,
                              uint64_t stride, uint64_t kmin, float xscale, float *__restrict__ x,
                              float *__restrict__ y) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < m;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t pos = i * stride;
        x[i] = norm_key((uint64_t)leaf_key<K, V>(leaves, pos), kmin, xscale);
        y[i] = (float)((double)pos / (double)n);
    }
}

// loss = mean((f(x) - y)^2) and its gradient w.r.t. the 3H+1 parameters,
// accumulated into loss[0] and grad[] (zeroed by the caller).
__global__ void __launch_bounds__(256)
mlp_loss_grad_kernel(const float *__restrict__ p, int H, const float *__restrict__ x,
                     const float *__restrict__ y, uint64_t n, float *__restrict__ loss,
                     float *__restrict__ grad) {
    __shared__ float sp[3 * kMaxHidden + 1];
    __shared__ float sg[3 * kMaxHidden + 2];
    const int np = 3 * H + 1;
    for (int k = threadIdx.x; k < np; k += blockDim.x) sp[k] = p[k];
    for (int k = threadIdx.x; k < np + 1; k += blockDim.x) sg[k] = 0.f;
    __syncthreads();
    float g[3 * kMaxHidden + 1];
    for (int k = 0; k < np; k++) g[k] = 0.f;
    float l = 0.f;
    const float scale = 2.f / (float)n;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const float xi = x[i];
        float out = sp[3 * H];
        for (int j = 0; j < H; j++) out += sp[2 * H + j] * fmaxf(sp[j] * xi + sp[H + j], 0.f);
        const float err = out - y[i];
        l += err * err;
        const float dout = scale * err;
        for (int j = 0; j < H; j++) {
            const float h = sp[j] * xi + sp[H + j];
            const float a = fmaxf(h, 0.f);
            g[2 * H + j] += dout * a;
            const float dh = h > 0.f ? dout * sp[2 * H + j] : 0.f;
            g[j] += dh * xi;
            g[H + j] += dh;
        }
        g[3 * H] += dout;
    }
    // warp sums, then one shared-memory atomic per warp and parameter
    for (int k = 0; k < np; k++) {
        float v = g[k];
        for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        if ((threadIdx.x & 31) == 0) atomicAdd(&sg[k], v);
    }
    for (int o = 16; o > 0; o >>= 1) l += __shfl_xor_sync(0xffffffffu, l, o);
    if ((threadIdx.x & 31) == 0) atomicAdd(&sg[np], l / (float)n);
    __syncthreads();
    for (int k = threadIdx.x; k < np; k += blockDim.x) atomicAdd(&grad[k], sg[k]);
    if (threadIdx.x == 0) atomicAdd(loss, sg[np]);
}

// One Adam step, then projection onto w1 >= 0, w2 >= 0 (monotone root).
__global__ void adam_kernel(float *p, const float *grad, float *m, float *v, int H, float lr,
                            int step) {
    const int k = threadIdx.x;
    if (k >= 3 * H + 1) return;
    const float b1 = 0.9f, b2 = 0.999f;
    const float g = grad[k];
    m[k] = b1 * m[k] + (1.f - b1) * g;
    v[k] = b2 * v[k] + (1.f - b2) * g * g;
    const float mh = m[k] / (1.f - powf(b1, (float)step));
    const float vh = v[k] / (1.f - powf(b2, (float)step));
    float w = p[k] - lr * mh / (sqrtf(vh) + 1e-8f);
    if (k < H || (k >= 2 * H && k < 3 * H)) w = fmaxf(w, 0.f);
    p[k] = w;
}

// r_lo[s] = first rank routed to segment >= s (r_lo[nseg] = n).  The root is
// monotone and keys ascend, so segments are contiguous rank ranges.
template <typename K, typename V>
__global__ void assign_kernel(const unsigned char *__restrict__ leaves, uint64_t n,
                              const float *__restrict__ p, int H, uint32_t nseg, uint64_t kmin,
                              float xscale, uint32_t *__restrict__ r_lo) {
    __shared__ float sp[3 * kMaxHidden + 1];
    for (int k = threadIdx.x; k < 3 * H + 1; k += blockDim.x) sp[k] = p[k];
    __syncthreads();
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t s = root_segment(sp, H, nseg,
                                        norm_key((uint64_t)leaf_key<K, V>(leaves, i), kmin, xscale));
        const uint32_t prev =
            i == 0 ? 0u
                   : root_segment(sp, H, nseg,
                                  norm_key((uint64_t)leaf_key<K, V>(leaves, i - 1), kmin, xscale)) + 1;
        for (uint32_t t = (i == 0 ? 0u : prev); t <= s; t++) r_lo[t] = (uint32_t)i;
        if (i == n - 1)
            for (uint32_t t = s + 1; t <= nseg; t++) r_lo[t] = (uint32_t)n;
    }
}

// Least-squares leaf models and their exact error bounds, one warp per segment.
template <typename K, typename V>
__global__ void fit_kernel(const unsigned char *__restrict__ leaves, uint64_t n, uint32_t nseg,
                           const uint32_t *__restrict__ r_lo, SegParam *__restrict__ seg) {
    const int lane = threadIdx.x & 31;
    for (uint64_t s = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5; s < nseg;
         s += ((uint64_t)gridDim.x * blockDim.x) >> 5) {
        const uint32_t a = r_lo[s], b = r_lo[s + 1];
        SegParam sp;
        sp.base = a < n ? (uint64_t)leaf_key<K, V>(leaves, a) : (uint64_t)leaf_key<K, V>(leaves, n - 1);
        sp.r_lo = a;
        sp.cnt = b - a;
        sp.pad = 0;
        double sx = 0, sy = 0, sxx = 0, sxy = 0;
        for (uint32_t i = a + lane; i < b; i += 32) {
            const uint64_t k = (uint64_t)leaf_key<K, V>(leaves, i);
            const double xv = (double)__ull2float_rn(k - sp.base);
            const double yv = (double)(i - a);
            sx += xv;
            sy += yv;
            sxx += xv * xv;
            sxy += xv * yv;
        }
        for (int o = 16; o > 0; o >>= 1) {
            sx += __shfl_xor_sync(0xffffffffu, sx, o);
            sy += __shfl_xor_sync(0xffffffffu, sy, o);
            sxx += __shfl_xor_sync(0xffffffffu, sxx, o);
            sxy += __shfl_xor_sync(0xffffffffu, sxy, o);
        }
        const double c = (double)(b - a);
        const double den = c * sxx - sx * sx;
        double slope = 0.0;
        if (c >= 2 && den > 0) slope = (c * sxy - sx * sy) / den;
        const double icpt = c > 0 ? (sy - slope * sx) / c : 0.0;
        sp.slope = (float)slope;
        sp.icpt = (float)icpt;
        // exact bound with the search's own arithmetic
        float e = 0.f;
        for (uint32_t i = a + lane; i < b; i += 32) {
            const float pr = leaf_pred(sp, (uint64_t)leaf_key<K, V>(leaves, i));
            e = fmaxf(e, fabsf(__fsub_rn(pr, (float)(i - a))));
        }
        for (int o = 16; o > 0; o >>= 1) e = fmaxf(e, __shfl_xor_sync(0xffffffffu, e, o));
        const float ce = ceilf(e);
        sp.eps = ce >= 4.0e9f ? 0xFFFFFFFFu : (uint32_t)ce;
        if (lane == 0) seg[s] = sp;
    }
}

// --------------------------------------------------------------- search ---

constexpr int kThreads = 256;
constexpr int kMaxWindowLines = 8;

// Full descent for one query by one thread (the fallback): binary search in
// each node line from global memory, then the leaf block.
template <typename K, typename V>
__device__ uint64_t scalar_lower_bound(const DevTree &t, K qe) {
    constexpr int F = kLineBytes / (int)sizeof(K);
    using LG = LeafGeom<K, V>;
    const K *gs = static_cast<const K *>(t.seps);
    uint64_t node = 0;
    for (int lvl = 0; lvl < t.nlevels; lvl++) {
        const K *line = gs + t.lvl_off[lvl] + node * F;
        int lo = 0, len = F;
        while (len > 1) {
            const int half = len >> 1;
            lo = line[lo + half - 1] < qe ? lo + half : lo;
            len -= half;
        }
        node = node * F + lo;
    }
    const K *kb = reinterpret_cast<const K *>(static_cast<const unsigned char *>(t.leaves) +
                                              node * LG::BS);
    int c = 0;
    for (int j = 0; j < LG::S; j++) c += kb[j] < qe;
    return node * LG::S + c;
}

template <typename K, typename V, int G, int R>
__global__ void __launch_bounds__(kThreads)
learned_kernel(const __grid_constant__ DevTree t, const __grid_constant__ LearnedDev m,
               const K *__restrict__ q, uint64_t nq, V *__restrict__ out) {
    __shared__ float sp[3 * kMaxHidden + 1];
    __shared__ uint8_t s_bad[kThreads];
    for (int k = threadIdx.x; k < 3 * m.hidden + 1; k += blockDim.x) sp[k] = m.mlp[k];
    __syncthreads();

    using LG = LeafGeom<K, V>;
    constexpr int F = kLineBytes / (int)sizeof(K);
    constexpr int KPL = F / G;
    constexpr int NG = 32 / G;
    constexpr int I = G / R;
    const int lane = threadIdx.x & 31;
    const int grp = lane / G;
    const int gl = lane % G;
    uint8_t *bad = s_bad + (threadIdx.x & ~31);
    const K tmax = (K)t.max_key;
    const unsigned char *leaves = static_cast<const unsigned char *>(t.leaves);
    const K *lvl_base = static_cast<const K *>(t.seps) + t.lvl_off[m.level];
    const uint64_t ntiles = (nq + 31) / 32;
    unsigned long long n_fallback = 0, n_window = 0;

    for (uint64_t tile = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5; tile < ntiles;
         tile += ((uint64_t)gridDim.x * blockDim.x) >> 5) {
        const uint64_t base = tile * 32;
        // phase 1: one lane per query, model -> window of entries on m.level
        const uint64_t my = base + lane;
        const K myq = my < nq ? q[my] : (K)0;
        const K myqe = myq < tmax ? myq : tmax;
        const uint32_t sid =
            root_segment(sp, m.hidden, m.nseg, norm_key((uint64_t)myqe, m.kmin, m.xscale));
        const SegParam sg = m.seg[sid];
        const float pr = leaf_pred(sg, (uint64_t)myqe);
        const double prc = fmin(fmax((double)pr, -1.0e12), 1.0e12);
        const int64_t A = (int64_t)sg.r_lo + (int64_t)floor(prc) - (int64_t)sg.eps - 1;
        const int64_t B = (int64_t)sg.r_lo + (int64_t)ceil(prc) + (int64_t)sg.eps + 1;
        const int64_t last = (int64_t)m.level_entries - 1;
        int64_t ja = (A < 0 ? 0 : A / (int64_t)m.kpe) - 1;
        int64_t jb = (B < 0 ? 0 : B / (int64_t)m.kpe) + 1;
        ja = ja < 0 ? 0 : (ja > last ? last : ja);
        jb = jb < ja ? ja : (jb > last ? last : jb);
        const uint32_t my_ja = (uint32_t)ja, my_jb = (uint32_t)jb;
        const int my_lines = (int)(my_jb / F - my_ja / F) + 1;
        bad[lane] = my_lines > kMaxWindowLines ? 1 : 0;
        __syncwarp();

        // phase 2: G lanes per query: scan the window, descend, leaf block
#pragma unroll
        for (int r = 0; r < R; r++) {
            K qv[I], qe[I];
            bool up[I];
            uint32_t node[I], wa[I], wb[I];
            bool sbad[I];
            int lines = 1;
#pragma unroll
            for (int s = 0; s < I; s++) {
                const int k = r * (NG * I) + s * NG + grp;
                qv[s] = __shfl_sync(0xffffffffu, myq, k);
                wa[s] = __shfl_sync(0xffffffffu, my_ja, k);
                wb[s] = __shfl_sync(0xffffffffu, my_jb, k);
                sbad[s] = bad[k] != 0;
                qe[s] = qv[s] < tmax ? qv[s] : tmax;
                up[s] = false;
                const int l = sbad[s] ? 1 : (int)(wb[s] / F - wa[s] / F) + 1;
                lines = l > lines ? l : lines;
            }
            lines = (int)__reduce_max_sync(0xffffffffu, (unsigned)lines);
            int cnt[I];
#pragma unroll
            for (int s = 0; s < I; s++) cnt[s] = 0;
            for (int w = 0; w < lines; w++) {
#pragma unroll
                for (int s = 0; s < I; s++) {
                    const uint32_t line = wa[s] / F + w;
                    const uint32_t e0 = line * F + gl * KPL;
                    if (!sbad[s] && line * F <= wb[s]) {
                        uint32_t c[KPL * sizeof(K) / 4];
                        load_bytes<KPL * (int)sizeof(K)>(lvl_base + (size_t)e0, c);
#pragma unroll
                        for (int k = 0; k < KPL; k++) {
                            const uint32_t e = e0 + k;
                            cnt[s] += (e >= wa[s] && e <= wb[s] && key_at<K>(c, k) < qe[s]) ? 1 : 0;
                        }
                    }
                }
            }
#pragma unroll
            for (int s = 0; s < I; s++) {
#pragma unroll
                for (int o = G / 2; o > 0; o >>= 1) cnt[s] += __shfl_xor_sync(0xffffffffu, cnt[s], o);
                const uint32_t width = wb[s] - wa[s] + 1;
                // the lower bound is proven inside [wa, wb] unless the scan is
                // empty with entries left of wa, or full with entries right of wb
                const bool outside = ((uint32_t)cnt[s] == 0 && wa[s] > 0) ||
                                     ((uint32_t)cnt[s] == width && wb[s] < (uint32_t)last);
                sbad[s] = sbad[s] || outside;
                node[s] = sbad[s] ? 0u : wa[s] + (uint32_t)cnt[s];
                if (gl == 0) bad[r * (NG * I) + s * NG + grp] = sbad[s] ? 1 : 0;
            }
            for (int lvl = m.level + 1; lvl < t.nlevels; lvl++)
                level_step<K, G, I>(static_cast<const K *>(t.seps) + t.lvl_off[lvl], qe, up, node,
                                    grp, gl);
            leaf_point<K, V, G, I>(leaves, node, qv, qe, tmax, grp, gl, [&](int s) -> V * {
                const uint64_t qi = base + (uint64_t)(r * (NG * I) + s * NG + grp);
                return (qi < nq && !sbad[s]) ? out + qi : nullptr;
            });
        }
        __syncwarp();
        // fallback: the owning lane runs the full descent for its own query
        const bool mine_bad = my < nq && bad[lane] != 0;
        if (mine_bad) {
            const uint64_t p = scalar_lower_bound<K, V>(t, myqe);
            const K k = leaf_key<K, V>(leaves, p);
            const bool found = myq <= tmax && k == myq;
            out[my] = found ? reinterpret_cast<const V *>(leaves + (p / LG::S) * LG::BS +
                                                          kSectorBytes)[p % LG::S]
                            : key_max<V>();
        }
        const unsigned fb = __ballot_sync(0xffffffffu, mine_bad);
        const unsigned valid = __ballot_sync(0xffffffffu, my < nq);
        n_fallback += __popc(fb);
        n_window += __popc(valid & ~fb);
        __syncwarp();
    }
    if (lane == 0 && m.stats) {
        atomicAdd(&m.stats[0], n_window);
        atomicAdd(&m.stats[1], n_fallback);
    }
}

template <typename K, typename V, int G, int R>
bt_status learned_launch(const bt_tree *t, const void *d_q, uint64_t nq, void *d_out,
                         cudaStream_t s) {
    auto fn = learned_kernel<K, V, G, R>;
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, kThreads, 0) != cudaSuccess ||
        per_sm < 1)
        per_sm = 1;
    uint64_t want = (nq + kThreads - 1) / kThreads;
    const uint64_t cap = (uint64_t)sm_count() * per_sm;
    const unsigned grid = (unsigned)std::max<uint64_t>(1, std::min(want, cap));
    count_launch();
    fn<<<grid, kThreads, 0, s>>>(t->dev, t->learned->dev, (const K *)d_q, nq, (V *)d_out);
    BT_CUDA(cudaGetLastError());
    return BT_OK;
}

template <typename K, typename V>
bt_status learned_cfg(const bt_tree *t, const void *d_q, uint64_t nq, void *d_out, cudaStream_t s) {
    switch (t->search_cfg) {
        case 0: return learned_launch<K, V, 8, 1>(t, d_q, nq, d_out, s);
        case 1: return learned_launch<K, V, 8, 2>(t, d_q, nq, d_out, s);
        case 2: return learned_launch<K, V, 4, 1>(t, d_q, nq, d_out, s);
        case 3: return learned_launch<K, V, 4, 2>(t, d_q, nq, d_out, s);
        default: return learned_launch<K, V, 2, 1>(t, d_q, nq, d_out, s);
    }
}

// ------------------------------------------------------------ training ----

struct DevBuf {
    void *p = nullptr;
    ~DevBuf() {
        if (p) cudaFree(p);
    }
};

unsigned grid_of(uint64_t n, int block, int per_sm = 8) {
    uint64_t g = (n + block - 1) / block;
    const uint64_t cap = (uint64_t)sm_count() * per_sm;
    return (unsigned)std::max<uint64_t>(1, std::min(g, cap));
}

template <typename K, typename V>
bt_status train_impl(bt_tree *t, const bt_learned_config &cfg, cudaStream_t s,
                     bt_learned_report *rep) {
    const uint64_t n = t->n;
    const int H = (int)cfg.hidden;
    const int np = 3 * H + 1;
    const uint32_t nseg = cfg.num_segments;
    const unsigned char *leaves = (const unsigned char *)t->d_leaves;
    // frees the new state on every early return; released on success
    struct Owner {
        LearnedState *p;
        ~Owner() { free_learned(p); }
    } own{new LearnedState()};
    LearnedState *st = own.p;
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, s);

    // normalisation of the root's input
    const uint64_t kmin = t->min_key;
    const double span = (double)(t->max_key - t->min_key);
    const float xscale = span > 0 ? (float)(1.0 / span) : 0.f;

    // training sample
    const uint64_t stride = std::max<uint64_t>(1, cfg.sample_stride ? cfg.sample_stride : n / (1u << 20));
    const uint64_t m = (n + stride - 1) / stride;
    DevBuf bx, by, bg, bm, bv, bl, brl;
    BT_CUDA(cudaMalloc(&bx.p, m * sizeof(float)));
    BT_CUDA(cudaMalloc(&by.p, m * sizeof(float)));
    BT_CUDA(cudaMalloc(&bg.p, (np + 1) * sizeof(float)));
    BT_CUDA(cudaMalloc(&bm.p, np * sizeof(float)));
    BT_CUDA(cudaMalloc(&bv.p, np * sizeof(float)));
    BT_CUDA(cudaMalloc(&brl.p, (nseg + 1) * sizeof(uint32_t)));
    BT_CUDA(cudaMalloc((void **)&st->d_mlp, np * sizeof(float)));
    BT_CUDA(cudaMalloc((void **)&st->d_seg, nseg * sizeof(SegParam)));
    BT_CUDA(cudaMalloc((void **)&st->d_stats, 2 * sizeof(unsigned long long)));
    BT_CUDA(cudaMemsetAsync(st->d_stats, 0, 2 * sizeof(unsigned long long), s));
    float *x = (float *)bx.p, *y = (float *)by.p, *grad = (float *)bg.p, *loss = grad + np;
    count_launch();
    sample_kernel<K, V><<<grid_of(m, 256), 256, 0, s>>>(leaves, n, m, stride, kmin, xscale, x, y);

    // initial root: hinges spread over [0, 1), output weights 1/H
    std::vector<float> p0(np);
    for (int j = 0; j < H; j++) {
        p0[j] = 1.f;
        p0[H + j] = -(float)j / (float)H;
        p0[2 * H + j] = 1.f / (float)H;
    }
    p0[3 * H] = 0.f;
    BT_CUDA(cudaMemcpyAsync(st->d_mlp, p0.data(), np * sizeof(float), cudaMemcpyHostToDevice, s));
    BT_CUDA(cudaMemsetAsync(bm.p, 0, np * sizeof(float), s));
    BT_CUDA(cudaMemsetAsync(bv.p, 0, np * sizeof(float), s));
    float l0 = 0.f, l1 = 0.f;
    const unsigned lg = grid_of(m, 256, 4);
    for (uint32_t it = 0; it <= cfg.iterations; it++) {
        BT_CUDA(cudaMemsetAsync(grad, 0, (np + 1) * sizeof(float), s));
        count_launch();
        mlp_loss_grad_kernel<<<lg, 256, 0, s>>>(st->d_mlp, H, x, y, m, loss, grad);
        if (it == 0) BT_CUDA(cudaMemcpyAsync(&l0, loss, sizeof(float), cudaMemcpyDeviceToHost, s));
        if (it == cfg.iterations) {
            BT_CUDA(cudaMemcpyAsync(&l1, loss, sizeof(float), cudaMemcpyDeviceToHost, s));
            break;
        }
        count_launch();
        adam_kernel<<<1, 128, 0, s>>>(st->d_mlp, grad, (float *)bm.p, (float *)bv.p, H,
                                      cfg.learning_rate, (int)it + 1);
    }

    // segments: assignment, least-squares fit, exact error bounds
    uint32_t *r_lo = (uint32_t *)brl.p;
    count_launch();
    assign_kernel<K, V><<<grid_of(n, 256), 256, 0, s>>>(leaves, n, st->d_mlp, H, nseg, kmin, xscale,
                                                      r_lo);
    count_launch();
    fit_kernel<K, V><<<grid_of((uint64_t)nseg * 32, 256), 256, 0, s>>>(leaves, n, nseg, r_lo,
                                                                     st->d_seg);
    BT_CUDA(cudaGetLastError());
    cudaEventRecord(e1, s);
    std::vector<SegParam> segs(nseg);
    BT_CUDA(cudaMemcpyAsync(segs.data(), st->d_seg, nseg * sizeof(SegParam), cudaMemcpyDeviceToHost, s));
    BT_CUDA(cudaStreamSynchronize(s));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);

    LearnedDev &d = st->dev;
    d.mlp = st->d_mlp;
    d.seg = st->d_seg;
    d.stats = st->d_stats;
    d.kmin = kmin;
    d.xscale = xscale;
    d.hidden = H;
    d.nseg = nseg;
    d.level = t->dev.nlevels >= 2 ? t->dev.nlevels - 2 : 0;
    uint64_t kpe = LeafGeom<K, V>::S;
    for (int l = t->dev.nlevels - 1; l > d.level; l--) kpe *= (uint64_t)(kLineBytes / sizeof(K));
    d.kpe = kpe;
    d.level_entries = t->lvl_entries[d.level];

    if (rep) {
        std::memset(rep, 0, sizeof(*rep));
        rep->root_loss_initial = l0;
        rep->root_loss_final = l1;
        rep->num_segments = nseg;
        rep->model_level = (uint32_t)d.level;
        rep->keys_per_entry = kpe;
        double esum = 0, lsum = 0;
        uint64_t emax = 0, used = 0;
        const int F = kLineBytes / (int)sizeof(K);
        for (uint32_t i = 0; i < nseg; i++) {
            const uint64_t cnt = (i + 1 < nseg ? segs[i + 1].r_lo : n) - segs[i].r_lo;
            if (!cnt) continue;
            used++;
            esum += segs[i].eps;
            emax = std::max<uint64_t>(emax, segs[i].eps);
            const double width_entries = (2.0 * segs[i].eps + 4.0) / (double)kpe + 3.0;
            lsum += std::ceil(width_entries / F);
        }
        rep->eps_mean = used ? esum / used : 0;
        rep->eps_max = emax;
        rep->window_lines_mean = used ? lsum / used : 0;
        rep->train_ms = ms;
    }
    if (t->learned) free_learned(t->learned);
    t->learned = st;
    own.p = nullptr;
    return BT_OK;
}

}  // namespace
}  // namespace bt

extern "C" {

bt_status bt_learned_train(bt_tree *t, const bt_learned_config *cfg_in, void *stream,
                           bt_learned_report *report) {
    using namespace bt;
    if (!t) return fail(BT_ERR_INVALID_ARGUMENT, "tree is NULL");
    if (t->n < 2) return fail(BT_ERR_INVALID_ARGUMENT, "a learned index needs at least 2 keys");
    if (t->n >= (1ull << 32)) return fail(BT_ERR_INVALID_ARGUMENT, "learned index supports n < 2^32");
    bt_learned_config cfg = {65536, 16, 400, 0, 0.01f};
    if (cfg_in) {
        if (cfg_in->num_segments) cfg.num_segments = cfg_in->num_segments;
        if (cfg_in->hidden) cfg.hidden = cfg_in->hidden;
        cfg.iterations = cfg_in->iterations;
        cfg.sample_stride = cfg_in->sample_stride;
        if (cfg_in->learning_rate > 0) cfg.learning_rate = cfg_in->learning_rate;
    }
    if (cfg.hidden > (uint32_t)kMaxHidden) return fail(BT_ERR_INVALID_ARGUMENT, "hidden must be <= 32");
    if (cfg.num_segments > (1u << 24)) return fail(BT_ERR_INVALID_ARGUMENT, "too many segments");
    int prev = 0;
    BT_CUDA(cudaGetDevice(&prev));
    if (prev != t->device) BT_CUDA(cudaSetDevice(t->device));
    cudaStream_t s = (cudaStream_t)stream;
    bt_status st;
    if (t->key_bytes == 4)
        st = t->val_bytes == 4 ? train_impl<uint32_t, uint32_t>(t, cfg, s, report)
                               : train_impl<uint32_t, uint64_t>(t, cfg, s, report);
    else
        st = t->val_bytes == 4 ? train_impl<uint64_t, uint32_t>(t, cfg, s, report)
                               : train_impl<uint64_t, uint64_t>(t, cfg, s, report);
    if (prev != t->device) cudaSetDevice(prev);
    return st;
}

bt_status bt_point_search_learned(const bt_tree *t, const void *d_q, uint64_t nq, void *d_out,
                                  void *stream) {
    using namespace bt;
    if (!t) return fail(BT_ERR_INVALID_ARGUMENT, "tree is NULL");
    if (!t->learned) return fail(BT_ERR_INVALID_ARGUMENT, "the tree has no trained learned index");
    if (nq == 0) return BT_OK;
    if (!d_q || !d_out) return fail(BT_ERR_INVALID_ARGUMENT, "queries or out is NULL");
    if (nq >= (1ull << 32)) return fail(BT_ERR_INVALID_ARGUMENT, "nq must be below 2^32");
    int prev = 0;
    BT_CUDA(cudaGetDevice(&prev));
    if (prev != t->device) BT_CUDA(cudaSetDevice(t->device));
    cudaStream_t s = (cudaStream_t)stream;
    bt_status st = BT_OK;
    cudaError_t e = cudaMemsetAsync(t->learned->d_stats, 0, 2 * sizeof(unsigned long long), s);
    if (e != cudaSuccess) st = cuda_fail(e, "cudaMemsetAsync");
    if (st == BT_OK) {
        if (t->key_bytes == 4)
            st = t->val_bytes == 4 ? learned_cfg<uint32_t, uint32_t>(t, d_q, nq, d_out, s)
                                   : learned_cfg<uint32_t, uint64_t>(t, d_q, nq, d_out, s);
        else
            st = t->val_bytes == 4 ? learned_cfg<uint64_t, uint32_t>(t, d_q, nq, d_out, s)
                                   : learned_cfg<uint64_t, uint64_t>(t, d_q, nq, d_out, s);
    }
    if (prev != t->device) cudaSetDevice(prev);
    return st;
}

bt_status bt_learned_last_stats(const bt_tree *t, uint64_t *windowed, uint64_t *fallback) {
    using namespace bt;
    if (!t || !t->learned) return fail(BT_ERR_INVALID_ARGUMENT, "the tree has no trained learned index");
    unsigned long long h[2] = {0, 0};
    BT_CUDA(cudaMemcpy(h, t->learned->d_stats, sizeof(h), cudaMemcpyDeviceToHost));
    if (windowed) *windowed = h[0];
    if (fallback) *fallback = h[1];
    return BT_OK;
}

bt_status bt_mlp_loss_grad(const float *d_params, uint32_t hidden, const float *d_x,
                           const float *d_y, uint64_t n, float *d_loss, float *d_grad,
                           void *stream) {
    using namespace bt;
    if (!d_params || !d_x || !d_y || !d_loss || !d_grad || n == 0)
        return fail(BT_ERR_INVALID_ARGUMENT, "null pointer or empty input");
    if (hidden == 0 || hidden > (uint32_t)kMaxHidden)
        return fail(BT_ERR_INVALID_ARGUMENT, "hidden must be 1..32");
    cudaStream_t s = (cudaStream_t)stream;
    BT_CUDA(cudaMemsetAsync(d_grad, 0, (3 * hidden + 1) * sizeof(float), s));
    BT_CUDA(cudaMemsetAsync(d_loss, 0, sizeof(float), s));
    count_launch();
    mlp_loss_grad_kernel<<<grid_of(n, 256, 4), 256, 0, s>>>(d_params, (int)hidden, d_x, d_y, n,
                                                            d_loss, d_grad);
    BT_CUDA(cudaGetLastError());
    return BT_OK;
}

}  // extern "C"
