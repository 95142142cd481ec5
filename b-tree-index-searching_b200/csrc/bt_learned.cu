// Learned index: build kernels (segmentation, root training, unit codes) and
// the learned point search.
//
// No counterpart in the reference: its descent is always the page walk of
// BPTreeExactSearch.cu:39-68, here the tree of bt_search.cu.  The learned
// index sends a point query straight to the 128-byte leaf unit holding its
// key, so the only DRAM read of a query is that unit; everything before it
// is on chip (shared memory and L2):
//
//   1. root (shared memory): a monotone MLP y = b2 + sum_j w2[j] *
//      ramp(w1[j] * x + b1[j]) (ramp = clamp to [0, 1]; w1, w2 >= 0) of the
//      normalised key predicts
//      the key's segment line among the nls lines; its worst error root_err
//      over the lines' first keys bounds a binary search over those keys,
//      staged in shared memory, to 2 * root_err + 3 entries.
//   2. segment line (one L2 read): four leaf models; the key's segment gives
//      a predicted rank p and its bound eps, so the key's rank lies in
//      [p - eps - 1, p + eps + 1].
//   3. code line (one L2 read; two for the queries whose count continues
//      into the neighbouring line, which wait in a per-warp queue for a
//      pass of their own): the thresholds between the leaf units of that
//      window; the thresholds at or below the key count the units to skip.
//   4. leaf unit (the DRAM read, by a lane quad: one request per unit): the
//      key's block(s) and values.
//
// Exactness.  Every bound used above is measured on the device with the
// search's own FP32 operations (explicit round-to-nearest intrinsics and
// fused multiply-adds, no implicit contraction), and every function of the key involved is monotone, so a
// bound measured at the keys holds for every query between them.  A query
// whose key lies just above a unit's threshold bucket lands one unit early
// and reads the next one; a query that would leave its window (impossible
// with correct bounds) takes the tree's full descent.  Results therefore
// always equal the plain search.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <vector>

#include "bt_search.cuh"

namespace bt {

struct LearnedState {
    float *d_mlp = nullptr;
    SegLine *d_seg = nullptr;
    CodeLine *d_codes = nullptr;
    void *d_stage = nullptr;
    unsigned long long *d_stats = nullptr;
    uint64_t bytes = 0;
    int shape = 1;  // search kernel shape (bt_learned_set_shape)
    LearnedDev dev;
};

void free_learned(LearnedState *s) {
    if (!s) return;
    cudaFree(s->d_mlp);
    cudaFree(s->d_seg);
    cudaFree(s->d_codes);
    cudaFree(s->d_stage);
    cudaFree(s->d_stats);
    delete s;
}

namespace {

constexpr uint64_t kPlaChunk = 1ull << 14;  // keys per segmentation thread
constexpr int kHullCap = 32;                 // points per convex hull
constexpr int kPlaThreads = 64;              // segmentation threads per CTA
constexpr int kPlaHullStride = 2 * kHullCap + 1;  // hull points per thread in shared memory
constexpr size_t kStageBudget = 160 * 1024;  // shared memory for the staged keys
constexpr int kMaxWalk = 8;                  // extra units read before the full descent
// Search CTA shapes (one CTA per SM: the staged keys), bt_learned_set_shape:
// 1 = 1024 threads, 2 = 768, 3 = 640, 4 = 512 (fewer threads, more
// registers per thread).
constexpr int kLearnedShapes = 4;
// Counters of a search (bt_learned_last_stats, bt_learned_last_lines): leaf
// units read beyond the first, full descents, code lines counted beyond the
// first.
constexpr int kLearnedStats = 3;

// ---------------------------------------------------------------- model ---

// Root model in FP32 with explicit round-to-nearest operations (the same
// arithmetic at training-time error measurement and in the search).
// Units are ramps, clamp(w1 x + b1, 0, 1): with w1, w2 >= 0 every term is
// non-decreasing in x under round-to-nearest (each fused multiply-add rounds
// a non-decreasing exact value once), so the network is monotone, and
// (unlike ReLUs with non-negative weights, whose sum is convex) a sum of
// ramps can follow a CDF that bends both ways.
//
// Evaluated from the parameters packed one float4 per unit, (w1, b1, w2, 0),
// with the units padded to a multiple of 4 by zero units (a zero unit adds
// exactly 0): one shared-memory load and two fused multiply-adds per unit.
constexpr int kMlpPack = 4;

__host__ __device__ constexpr int mlp_units4(int H) { return (H + kMlpPack - 1) / kMlpPack * kMlpPack; }

// Packs the flat parameters p = [w1[H], b1[H], w2[H], b2] into u[mlp_units4(H)]
// (+ b2 in *b2); called by every thread of the block with its own index.
__device__ __forceinline__ void pack_mlp(const float *p, int H, float4 *u, float *b2, int tid,
                                         int nth) {
    for (int k = tid; k < mlp_units4(H); k += nth)
        u[k] = k < H ? make_float4(p[k], p[H + k], p[2 * H + k], 0.f) : make_float4(0.f, 0.f, 0.f, 0.f);
    if (tid == 0) *b2 = p[3 * H];
}

__device__ __forceinline__ float mlp_eval4(const float4 *u, int H4, float b2, float x) {
    float out = b2;
    for (int j = 0; j < H4; j += kMlpPack) {
#pragma unroll
        for (int k = 0; k < kMlpPack; k++) {
            const float4 w = u[j + k];
            out = __fmaf_rn(w.z, __saturatef(__fmaf_rn(w.x, x, w.y)), out);
        }
    }
    return out;
}

__device__ __forceinline__ float norm_key(uint64_t key, uint64_t kmin, float xscale) {
    return __fmul_rn(__ull2float_rn(key > kmin ? key - kmin : 0ull), xscale);
}

// Segment line predicted by the root for normalised key x.
__device__ __forceinline__ int root_line(const float4 *u, int H4, float b2, uint32_t nls, float x) {
    const float y = __fmul_rn(mlp_eval4(u, H4, b2, x), (float)nls);
    if (!(y > 0.f)) return 0;  // also NaN
    const float f = floorf(y);
    return f >= (float)nls ? (int)nls - 1 : (int)f;
}

// Rank offset predicted by a leaf model, clamped to its rank range [0, cnt]
// (a key in the gap after the segment's last key must not be extrapolated
// along the line: its lower bound is the next segment's first rank).
__device__ __forceinline__ float seg_pred(float slope, float icpt, uint32_t cnt, uint64_t fk,
                                          uint64_t key) {
    const uint64_t d = key > fk ? key - fk : 0ull;
    const float p = __fadd_rn(icpt, __fmul_rn(slope, __ull2float_rn(d)));
    return fminf(fmaxf(p, 0.f), (float)cnt);
}

template <typename K, typename V>
__device__ __forceinline__ K leaf_key(const unsigned char *leaves, uint64_t pos) {
    using LG = LeafGeom<K, V>;
    return reinterpret_cast<const K *>(leaves + (pos / LG::S) * LG::BS)[pos % LG::S];
}

// Keys of one 128-byte leaf unit.
template <typename K, typename V>
__host__ __device__ constexpr int unit_keys() {
    return (kUnitBytes / LeafGeom<K, V>::BS) * LeafGeom<K, V>::S;
}

// ------------------------------------------------------- segmentation -----

struct PlaPt {
    uint64_t x;  // key - segment's first key
    int64_t y;   // rank - segment's first rank, +/- eps
};

// > 0 when b lies above the directed line o -> a (x increasing); exact.
__device__ __forceinline__ __int128 pla_cross(const PlaPt &o, const PlaPt &a, const PlaPt &b) {
    const __int128 ax = (__int128)a.x - (__int128)o.x, bx = (__int128)b.x - (__int128)o.x;
    const __int128 ay = (__int128)a.y - (__int128)o.y, by = (__int128)b.y - (__int128)o.y;
    return ax * by - ay * bx;
}

// Slope of the line through a and b and its value at x = 0, in double with
// explicit rounding (no contraction); flat for two points of one key.
__device__ __forceinline__ double pla_line_at0(const PlaPt &a, const PlaPt &b, double *slope) {
    if (b.x == a.x) {  // duplicate keys: a flat line through the middle
        *slope = 0.0;
        return __dmul_rn(__dadd_rn(__ll2double_rn(a.y), __ll2double_rn(b.y)), 0.5);
    }
    const double dx = __ull2double_rn(b.x - a.x);
    const double sl = __ddiv_rn(__dsub_rn(__ll2double_rn(b.y), __ll2double_rn(a.y)), dx);
    *slope = sl;
    return __dsub_rn(__ll2double_rn(a.y), __dmul_rn(sl, __ull2double_rn(a.x)));
}

// Error-bounded segmentation of the points (key[i], i) of one chunk of
// kPlaChunk keys, one thread per chunk: greedy maximal segments, each with a
// line within eps of all its points (the optimal streaming fit of O'Rourke,
// CACM 1981, as in the PGM-index, Ferragina & Vinciguerra, VLDB 2020).  An
// open segment keeps the upper convex hull of its lower points (x, y - eps),
// the lower convex hull of its upper points (x, y + eps), and the feasible
// lines of largest (M = Ma-Mb) and smallest (N = Na-Nb) slope; a point is
// feasible iff its lower point is not above M and its upper point not below
// N.  A segment also closes when a hull would exceed kHullCap points.
// COUNT: counts[c] = segments of chunk c.  Otherwise writes segment k of
// chunk c at offsets[c] + k: first rank and the mean of M and N as
// rank - first = icpt + slope * (key - first key).
template <typename K, typename V, bool COUNT>
__global__ void pla_kernel(const unsigned char *__restrict__ leaves, uint64_t n, uint32_t eps,
                           uint64_t nchunks, uint64_t *__restrict__ counts,
                           const uint64_t *__restrict__ offsets, uint32_t *__restrict__ starts,
                           double *__restrict__ slopes, double *__restrict__ icpts) {
    const uint64_t c = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    if (c >= nchunks) return;
    // the two hulls of this thread in shared memory (kPlaHullStride points
    // apart per thread: the padding spreads the threads over the banks)
    extern __shared__ PlaPt pla_sh[];
    PlaPt *lh = pla_sh + (size_t)threadIdx.x * kPlaHullStride;
    PlaPt *uh = lh + kHullCap;
    const int64_t e = (int64_t)eps;
    const uint64_t end = min(n, (c + 1) * kPlaChunk);
    uint64_t nseg = 0, out = COUNT ? 0 : offsets[c];
    uint64_t i = c * kPlaChunk;
    while (i < end) {
        const uint64_t s = i;
        const uint64_t x0 = (uint64_t)leaf_key<K, V>(leaves, s);
        int nl = 1, nu = 1;
        lh[0] = {0, -e};
        uh[0] = {0, e};
        PlaPt Ma = lh[0], Mb = uh[0], Na = uh[0], Nb = lh[0];
        uint64_t j = s + 1;
        if (j < end) {
            const PlaPt L = {(uint64_t)leaf_key<K, V>(leaves, j) - x0, 1 - e};
            const PlaPt U = {L.x, 1 + e};
            Mb = U;
            Nb = L;
            lh[nl++] = L;
            uh[nu++] = U;
            for (j = s + 2; j < end; j++) {
                const int64_t y = (int64_t)(j - s);
                const uint64_t x = (uint64_t)leaf_key<K, V>(leaves, j) - x0;
                const PlaPt L2 = {x, y - e}, U2 = {x, y + e};
                if (pla_cross(Ma, Mb, L2) > 0 || pla_cross(Na, Nb, U2) < 0) break;
                int nl2 = nl, nu2 = nu;
                while (nl2 >= 2 && pla_cross(lh[nl2 - 2], lh[nl2 - 1], L2) >= 0) nl2--;
                while (nu2 >= 2 && pla_cross(uh[nu2 - 2], uh[nu2 - 1], U2) <= 0) nu2--;
                if (nl2 >= kHullCap || nu2 >= kHullCap) break;
                if (pla_cross(Ma, Mb, U2) < 0) {  // M now pivots on U2
                    int b = 0;
                    for (int k = 1; k < nl; k++)
                        if (pla_cross(lh[b], U2, lh[k]) > 0) b = k;
                    Ma = lh[b];
                    Mb = U2;
                }
                if (pla_cross(Na, Nb, L2) > 0) {  // N now pivots on L2
                    int b = 0;
                    for (int k = 1; k < nu; k++)
                        if (pla_cross(uh[b], L2, uh[k]) < 0) b = k;
                    Na = uh[b];
                    Nb = L2;
                }
                lh[nl2] = L2;
                nl = nl2 + 1;
                uh[nu2] = U2;
                nu = nu2 + 1;
            }
        }
        if (!COUNT) {
            double sl = 0.0, ic = 0.0;
            if (j - s >= 2) {
                double sm, sn;
                const double m0 = pla_line_at0(Ma, Mb, &sm);
                const double n0 = pla_line_at0(Na, Nb, &sn);
                sl = __dmul_rn(__dadd_rn(sm, sn), 0.5);
                ic = __dmul_rn(__dadd_rn(m0, n0), 0.5);
            }
            starts[out] = (uint32_t)s;
            slopes[out] = sl;
            icpts[out] = ic;
            out++;
        }
        nseg++;
        i = j;
    }
    if (COUNT) counts[c] = nseg;
}

// Segment lines from the segmentation (one thread per line): first keys,
// ranks, FP32 lines (slope >= 0 keeps the prediction monotone).  eps is
// filled by seg_eps_kernel.
template <typename K, typename V>
__global__ void seg_fill_kernel(const unsigned char *__restrict__ leaves, uint64_t n,
                                uint32_t nseg, uint32_t nls, const uint32_t *__restrict__ starts,
                                const double *__restrict__ slopes, const double *__restrict__ icpts,
                                SegLine *__restrict__ seg) {
    for (uint32_t l = blockIdx.x * blockDim.x + threadIdx.x; l < nls; l += gridDim.x * blockDim.x) {
        SegLine sl;
        for (int k = 0; k < kSegPerLine; k++) {
            const uint32_t g = l * kSegPerLine + k;
            if (g < nseg) {
                const uint32_t a = starts[g];
                const uint32_t b = g + 1 < nseg ? starts[g + 1] : (uint32_t)n;
                sl.s[k].key = (uint64_t)leaf_key<K, V>(leaves, a);
                sl.s[k].r_lo = a;
                sl.s[k].cnt = b - a;
                sl.s[k].slope = __double2float_rn(fmax(slopes[g], 0.0));
                sl.s[k].icpt = __double2float_rn(icpts[g]);
            } else {
                sl.s[k].key = ~0ull;
                sl.s[k].r_lo = (uint32_t)n;
                sl.s[k].cnt = 0;
                sl.s[k].slope = 0.f;
                sl.s[k].icpt = 0.f;
            }
            sl.s[k].eps = 0;
            sl.s[k].pad = 0;
        }
        seg[l] = sl;
    }
}

// Exact error bound of every segment with the search's arithmetic, one warp
// per segment: eps = ceil(max |seg_pred(key_i) - (i - r_lo)|).
template <typename K, typename V>
__global__ void seg_eps_kernel(const unsigned char *__restrict__ leaves, uint32_t nseg,
                               SegLine *__restrict__ seg) {
    const int lane = threadIdx.x & 31;
    for (uint64_t g = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5; g < nseg;
         g += ((uint64_t)gridDim.x * blockDim.x) >> 5) {
        SegLine &sl = seg[g / kSegPerLine];
        const int k = (int)(g % kSegPerLine);
        const uint64_t fk = sl.s[k].key;
        const uint32_t a = sl.s[k].r_lo, cnt = sl.s[k].cnt;
        const float slope = sl.s[k].slope, icpt = sl.s[k].icpt;
        float err = 0.f;
        for (uint32_t i = lane; i < cnt; i += 32) {
            const float p = seg_pred(slope, icpt, cnt, fk, (uint64_t)leaf_key<K, V>(leaves, a + i));
            err = fmaxf(err, fabsf(__fsub_rn(p, (float)i)));
        }
        for (int o = 16; o > 0; o >>= 1) err = fmaxf(err, __shfl_xor_sync(0xffffffffu, err, o));
        if (lane == 0) {
            const float ce = ceilf(err);
            sl.s[k].eps = ce >= 4.0e9f ? 0xFFFFFFFFu : (uint32_t)ce;
        }
    }
}

// Staged keys (first key of every segment line) and the root's training
// pairs (x = normalised key, y = the line's centre in [0, 1)).  The staged
// array is stored already swizzled (entry l at slot swz(l), all-ones keys in
// the padding up to ns entries), so the search copies it to shared memory
// verbatim.
template <typename K>
__global__ void stage_kernel(const SegLine *__restrict__ seg, uint32_t nls, uint32_t ns,
                             uint64_t kmin, float xscale, K *__restrict__ stage,
                             float *__restrict__ x, float *__restrict__ y) {
    for (uint32_t l = blockIdx.x * blockDim.x + threadIdx.x; l < ns; l += gridDim.x * blockDim.x) {
        if (l >= nls) {
            stage[swz<K>(l)] = key_max<K>();
            continue;
        }
        const uint64_t k = seg[l].s[0].key;
        stage[swz<K>(l)] = (K)k;
        x[l] = norm_key(k, kmin, xscale);
        y[l] = (float)(((double)l + 0.5) / (double)nls);
    }
}

// Worst |root_line(x_l) - l| over the staged keys.
__global__ void root_err_kernel(const float *__restrict__ p, int H, const float *__restrict__ x,
                                uint32_t nls, unsigned int *__restrict__ err) {
    __shared__ float4 su[mlp_units4(kMaxHidden)];
    __shared__ float sb2;
    pack_mlp(p, H, su, &sb2, threadIdx.x, blockDim.x);
    __syncthreads();
    unsigned int e = 0;
    for (uint32_t l = blockIdx.x * blockDim.x + threadIdx.x; l < nls; l += gridDim.x * blockDim.x) {
        const int pl = root_line(su, mlp_units4(H), sb2, nls, x[l]);
        const int d = pl - (int)l;
        e = max(e, (unsigned int)(d < 0 ? -d : d));
    }
    for (int o = 16; o > 0; o >>= 1) e = max(e, __shfl_xor_sync(0xffffffffu, e, o));
    if ((threadIdx.x & 31) == 0) atomicMax(err, e);
}

// Code lines, one thread per line: thresholds j = 59 l .. 59 l + 58 (j <
// units - 1) between unit j and unit j + 1.  base = first key of the line's
// first unit; shift = the least for which every code fits kCodeMax; code =
// ((last key of unit j - base) >> shift) + 1, so T_j = base + (code <<
// shift) is the least multiple above unit j's keys.
template <typename K, typename V>
__global__ void code_kernel(const unsigned char *__restrict__ leaves, uint64_t n, uint64_t units,
                            uint64_t ncl, CodeLine *__restrict__ codes) {
    constexpr uint64_t KPU = unit_keys<K, V>();
    for (uint64_t l = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; l < ncl;
         l += (uint64_t)gridDim.x * blockDim.x) {
        const uint64_t j0 = l * kCodesPerLine;
        const uint64_t j1 = min(j0 + kCodesPerLine, units - 1);  // exclusive
        CodeLine cl;
        cl.base = (uint64_t)leaf_key<K, V>(leaves, j0 * KPU);
        const uint64_t top = (uint64_t)leaf_key<K, V>(leaves, min(j1 * KPU, n) - 1);
        const uint64_t span = top - cl.base;
        int sh = 0;
        while ((span >> sh) + 1 > kCodeMax) sh++;
        cl.shift = (uint16_t)sh;
        for (uint64_t j = j0; j < j0 + kCodesPerLine; j++) {
            uint16_t c = (uint16_t)kCodePad;
            if (j < j1) {
                const uint64_t last = (uint64_t)leaf_key<K, V>(leaves, (j + 1) * KPU - 1);
                c = (uint16_t)(((last - cl.base) >> sh) + 1);
            }
            cl.code[j - j0] = c;
        }
        codes[l] = cl;
    }
}

// ------------------------------------------------------------- search -----

// 32-byte load of an index line piece: read-only path, no L1 allocation,
// kept in L2 ahead of the streaming leaf reads (evict-last).
__device__ __forceinline__ uint64_t l2_evict_last() {
    uint64_t pol;
    asm("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(pol));
    return pol;
}

__device__ __forceinline__ void load_line32(const void *p, uint32_t (&w)[8],
                                            uint64_t pol = l2_evict_last()) {
    asm volatile(
        "ld.global.nc.L1::no_allocate.L2::cache_hint.v8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8], %9;"
        : "=r"(w[0]), "=r"(w[1]), "=r"(w[2]), "=r"(w[3]), "=r"(w[4]), "=r"(w[5]), "=r"(w[6]),
          "=r"(w[7])
        : "l"(p), "l"(pol));
}

// 32-byte load of a leaf-unit piece (touched once per query): evict-first.
__device__ __forceinline__ void load_unit32(const void *p, uint32_t (&w)[8],
                                            uint64_t pol = l2_evict_first()) {
    asm volatile(
        "ld.global.nc.L1::no_allocate.L2::cache_hint.v8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8], %9;"
        : "=r"(w[0]), "=r"(w[1]), "=r"(w[2]), "=r"(w[3]), "=r"(w[4]), "=r"(w[5]), "=r"(w[6]),
          "=r"(w[7])
        : "l"(p), "l"(pol));
}


// Last staged index in [a, b] whose key is below q (a when none: then a == 0
// by the root's bound).  Routing by "first key < q" sends a key equal to a
// segment's first key to the segment before, whose window reaches one rank
// past its end; with duplicate keys it finds the first occurrence.
template <typename K>
__device__ __forceinline__ uint32_t stage_search(const K *__restrict__ s, uint32_t a, uint32_t b,
                                                 K q) {
    uint32_t base = a, len = b - a + 1;
    while (len > 1) {
        const uint32_t half = len >> 1;
        base = s[swz<K>(base + half)] < q ? base + half : base;
        len -= half;
    }
    return base;
}

// Scalar full descent of the tree for one query (the fallback): writes its
// value, or all-ones on a miss, to *dst and, when hit is not null, 1 or 0 to
// *hit.
template <typename K, typename V>
__device__ __noinline__ void tree_point(const DevTree &t, K q, V *dst, uint8_t *hit) {
    using LG = LeafGeom<K, V>;
    const K tmax = (K)t.max_key;
    V v = key_max<V>();
    bool f = false;
    if (q <= tmax) {
        const uint32_t blk = block_lower_bound<K>(t, q);
        const unsigned char *b = static_cast<const unsigned char *>(t.leaves) + (size_t)blk * LG::BS;
        const K *kb = reinterpret_cast<const K *>(b);
        for (int i = 0; i < LG::S && !f; i++)
            if (kb[i] == q && (uint64_t)blk * LG::S + i < t.n) {
                v = reinterpret_cast<const V *>(b + kSectorBytes)[i];
                f = true;
            }
    }
    *dst = v;
    if (hit) *hit = f ? 1 : 0;
}

// 64-byte half of an index line: two 32-byte loads, evict-last in L2.
__device__ __forceinline__ void load_half_line(const unsigned char *p, uint32_t (&w)[16],
                                               uint64_t pol) {
    uint32_t a[8], b[8];
    load_line32(p, a, pol);
    load_line32(p + 32, b, pol);
#pragma unroll
    for (int i = 0; i < 8; i++) {
        w[i] = a[i];
        w[8 + i] = b[i];
    }
}

// Copies `bytes` (a multiple of 128) from global `src` into shared `dst` with
// bulk copies (cp.async.bulk, no multicast) completing on the mbarrier
// `bar`; every thread of the CTA calls it.  The wait is bounded: if the copy
// has not landed after kStageWaits polls, the CTA waits as long again (so
// no copy is left in flight when it moves on) and returns false -- the
// caller then answers its queries without the staged keys.
constexpr uint32_t kStageWaits = 1u << 22;

__device__ __forceinline__ bool stage_bulk(void *dst, const void *src, uint32_t bytes,
                                           unsigned long long *bar) {
    const uint32_t b = (uint32_t)__cvta_generic_to_shared(bar);
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(b) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(b), "r"(bytes)
                     : "memory");
        const uint32_t d = (uint32_t)__cvta_generic_to_shared(dst);
        for (uint32_t off = 0; off < bytes; off += 32768u) {
            const uint32_t nb = min(32768u, bytes - off);
            asm volatile(
                "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                    d + off),
                "l"(static_cast<const unsigned char *>(src) + off), "r"(nb), "r"(b)
                : "memory");
        }
    }
    uint32_t done = 0;
    for (uint32_t it = 0; it < kStageWaits && !done; it++)
        asm volatile(
            "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], 0; selp.u32 %0, 1, 0, p; }"
            : "=r"(done)
            : "r"(b)
            : "memory");
    if (!done) {  // wait once more for the copy in flight, then give up on it
        uint32_t late = 0;
        for (uint32_t it = 0; it < kStageWaits && !late; it++)
            asm volatile(
                "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], 0; selp.u32 %0, 1, 0, p; }"
                : "=r"(late)
                : "r"(b)
                : "memory");
    }
    return __syncthreads_and(done != 0) != 0;
}

// w[B + i] for i in 0..3 (B fixed): three selects.
template <int B, int N>
__device__ __forceinline__ uint32_t pick4(const uint32_t (&w)[N], int i) {
    const uint32_t lo = (i & 1) ? w[B + 1] : w[B];
    const uint32_t hi = (i & 1) ? w[B + 3] : w[B + 2];
    return (i & 2) ? hi : lo;
}

// w[B + 2 i] for i in 0..3 (B fixed).
template <int B, int N>
__device__ __forceinline__ uint32_t pick4s2(const uint32_t (&w)[N], int i) {
    const uint32_t lo = (i & 1) ? w[B + 2] : w[B];
    const uint32_t hi = (i & 1) ? w[B + 6] : w[B + 4];
    return (i & 2) ? hi : lo;
}

// Count of the thresholds of code line `line` at or below `key`, for the
// query of a lane pair (lane hl reads the 64-byte half hl; both lanes get
// the count).  Called by the whole warp; `act` false gives 0 and no load.
__device__ __forceinline__ uint32_t code_count(const CodeLine *__restrict__ codes, uint32_t line,
                                               bool act, uint64_t key, int hl, int p0, uint64_t pol) {
    uint32_t cw[16];
    if (act) {
        load_half_line(reinterpret_cast<const unsigned char *>(codes + line) + hl * 64, cw, pol);
    } else {
#pragma unroll
        for (int k = 0; k < 16; k++) cw[k] = 0;
    }
    const uint32_t b0 = __shfl_sync(0xffffffffu, cw[0], p0);
    const uint32_t b1 = __shfl_sync(0xffffffffu, cw[1], p0);
    const uint32_t shw = __shfl_sync(0xffffffffu, cw[2], p0);
    const uint64_t lbase = ((uint64_t)b1 << 32) | b0;
    // A line's codes never decrease, so those at or below the key's bucket
    // are a prefix of its 59 slots (lane 0 of the pair holds slots 0-26
    // after the base and the shift, lane 1 slots 27-58).
    uint32_t c = 0;
    if (act && key >= lbase) {
        const uint64_t d = (key - lbase) >> (shw & 0xFFFFu);
        const uint32_t qd = d >= kCodeMax ? kCodeMax : (uint32_t)d;
        // a word holds two 15-bit codes; in (0x8000 + qd) - code per half
        // no borrow crosses the halves, and bit 15 of a half is set iff
        // code <= qd
        const uint32_t qq2 = (qd | (qd << 16)) | 0x80008000u;
        // lane 0: words 0-1 hold the base and the low half of word 2 the
        // shift -- made codes that never count
        const uint32_t w0 = hl ? cw[0] : 0x7FFF7FFFu;
        const uint32_t w1 = hl ? cw[1] : 0x7FFF7FFFu;
        const uint32_t w2 = hl ? cw[2] : (cw[2] | 0x7FFFu);
        c = __popc((qq2 - w0) & 0x80008000u) + __popc((qq2 - w1) & 0x80008000u) +
            __popc((qq2 - w2) & 0x80008000u);
#pragma unroll
        for (int k = 3; k < 16; k++) c += __popc((qq2 - cw[k]) & 0x80008000u);
    }
    return c + __shfl_xor_sync(0xffffffffu, c, 1);
}

// Thresholds of the unit window [ua, ub) among the first c of line j0 / 59.
__device__ __forceinline__ uint32_t window_part(uint32_t ua, uint32_t ub, uint32_t j0, uint32_t c) {
    const uint32_t lo = max(ua, j0), hi = min(ub, j0 + c);
    return hi > lo ? hi - lo : 0u;
}

// A query whose unit window continues into the neighbouring code line, kept
// in its warp's shared-memory queue until 16 of them fill a pass.
struct Retry {
    uint64_t key;   // the query key (zero-extended)
    uint32_t qi;    // its index in the launch's batch (below 2^31)
    uint32_t pad;
    uint32_t ua, ub;
    uint32_t line;  // the code line still to count
    uint32_t skip;  // thresholds of the window at or below the key so far
};
constexpr int kRetryCap = 32;  // entries per warp (at most 15 + 16 at once)

// The leaf step of one pass: the query of every lane pair (live / unit / ub /
// key / qi, as held by the pair) is answered from its leaf unit, walking
// right past a threshold bucket.  Units are read by lane quads: quad g takes
// the queries of pairs g and 8 + g, lane part p of the quad bytes 32 p ..
// 32 p + 31 of the unit, so a unit is one request of one load instruction.
// Queries whose answer lies outside their window are answered by the tree's
// full descent.  Called by the whole warp.
template <typename K, typename V>
__device__ __forceinline__ void leaf_quads(const DevTree &t, uint32_t U, uint64_t pol, bool live,
                                           uint32_t unit, uint32_t ub, K key, uint32_t qi,
                                           V *__restrict__ out, uint8_t *__restrict__ fnd,
                                           uint32_t &n_extra, uint32_t &n_fallback) {
    using LG = LeafGeom<K, V>;
    constexpr int KPU = unit_keys<K, V>();
    constexpr int BPU = kUnitBytes / LG::BS;
    const int lane = threadIdx.x & 31, g = lane >> 2, part = lane & 3;
    const unsigned char *leaves = static_cast<const unsigned char *>(t.leaves);
    const uint64_t leaf_bytes = t.n_sectors * (uint64_t)LG::BS;
    // a key part holds the keys of block `blk` of the unit
    const bool key_part = (part * 32) % LG::BS == 0;
    const int blk = part * 32 / LG::BS;
    uint32_t un[2], ubq[2], qx[2];
    K qq[2];
    bool pend[2], lost_q[2];
#pragma unroll
    for (int h = 0; h < 2; h++) {
        const int src = 2 * (8 * h + g);  // lane 0 of the pair
        un[h] = __shfl_sync(0xffffffffu, unit, src);
        ubq[h] = __shfl_sync(0xffffffffu, ub, src);
        pend[h] = __shfl_sync(0xffffffffu, live ? 1u : 0u, src) != 0;
        lost_q[h] = false;
        qx[h] = __shfl_sync(0xffffffffu, qi, src);
        if constexpr (sizeof(K) == 8)
            qq[h] = ((K)__shfl_sync(0xffffffffu, (uint32_t)((uint64_t)key >> 32), src) << 32) |
                    __shfl_sync(0xffffffffu, (uint32_t)key, src);
        else
            qq[h] = (K)__shfl_sync(0xffffffffu, (uint32_t)key, src);
    }
    // a sub-query that is not pending keeps the words it last read: its
    // matches and keys are ignored below
    uint32_t u[2][8];
#pragma unroll
    for (int h = 0; h < 2; h++)
#pragma unroll
        for (int k = 0; k < 8; k++) u[h][k] = 0xFFFFFFFFu;
#pragma unroll 1
    for (int it = 0; it <= kMaxWalk; it++) {
#pragma unroll
        for (int h = 0; h < 2; h++) {
            const uint64_t off = (uint64_t)un[h] * kUnitBytes + part * 32;
            if (pend[h] && off < leaf_bytes) load_unit32(leaves + off, u[h], pol);
        }
        bool any = false;
#pragma unroll
        for (int h = 0; h < 2; h++) {
            const uint64_t r0 = (uint64_t)un[h] * KPU + (uint64_t)blk * LG::S;
            const bool last_unit = un[h] + 1 >= U;
            int pos = -1;
            K lastk = 0;
            if (key_part) {
#pragma unroll
                for (int i = LG::S - 1; i >= 0; i--)
                    if (key_at<K>(u[h], i) == qq[h]) pos = i;
                // the last unit's padding slots hold all-ones keys, which a
                // query may equal: a match there is no key
                if (last_unit && pos >= 0 && r0 + (uint64_t)pos >= t.n) pos = -1;
                lastk = key_at<K>(u[h], LG::S - 1);
            }
            // matches of the quad: the first key part with one answers
            // (block 0 before block 1: the first of equal keys)
            const unsigned mb = (__ballot_sync(0xffffffffu, pend[h] && pos >= 0) >> (4 * g)) & 0xFu;
            const bool found = mb != 0;
            const int kl = found ? __ffs(mb) - 1 : 0;
            const int mpos = __shfl_sync(0xffffffffu, pos, 4 * g + kl);
            // the unit's largest key (read only for units before the last,
            // whose blocks are full): the last key of its last block
            const int ll = 4 * g + (BPU == 2 ? 2 : 0);
            K ulast = (K)__shfl_sync(0xffffffffu, (uint32_t)lastk, ll);
            if constexpr (sizeof(K) == 8)
                ulast |= (K)__shfl_sync(0xffffffffu, (uint32_t)((uint64_t)lastk >> 32), ll) << 32;
            const bool beyond = pend[h] && !found && qq[h] > ulast && !last_unit;
            const bool walk = beyond && un[h] + 1 <= ubq[h];
            const bool lost = beyond && un[h] + 1 > ubq[h];
            if (pend[h] && !walk && !lost) {
                if (part == 0 && fnd) fnd[qx[h]] = found ? 1 : 0;
                if (!found) {
                    if (part == 0) out[qx[h]] = key_max<V>();
                } else {
                    // byte of the value within the unit: its block's value
                    // array follows the block's key sector
                    const int byte = (kl * 32 / LG::BS) * LG::BS + kSectorBytes + mpos * (int)sizeof(V);
                    if (byte / 32 == part) {
                        const int wi = (byte % 32) / 4;
                        V val;
                        if constexpr (sizeof(V) == 4) {
                            val = (wi & 4) ? pick4<4>(u[h], wi & 3) : pick4<0>(u[h], wi & 3);
                        } else {
                            const int i = wi >> 1;
                            val = ((uint64_t)pick4s2<1>(u[h], i) << 32) | pick4s2<0>(u[h], i);
                        }
                        out[qx[h]] = val;
                    }
                }
                pend[h] = false;
            } else if (walk) {
                un[h]++;
                if (part == 0 && it < kMaxWalk) n_extra++;
            }
            if (lost || (walk && it == kMaxWalk)) {
                lost_q[h] = true;  // outside the window: answered below
                pend[h] = false;
            }
            any |= pend[h];
        }
        if (!__any_sync(0xffffffffu, any)) break;
    }
#pragma unroll
    for (int h = 0; h < 2; h++) {
        if (lost_q[h] && part == 0) {  // the tree's full descent
            tree_point<K, V>(t, qq[h], out + qx[h], fnd ? fnd + qx[h] : nullptr);
            n_fallback++;
        }
    }
}

// One warp tile = 32 queries.  Phase 1 takes one lane per query (root
// network, then the staged keys: the query's segment line); the rest runs in
// two passes of 16 queries, a lane pair per query, each lane reading one
// 64-byte half of the segment line and of a code line.  A query counts the
// code line holding its predicted unit; when its window continues into the
// neighbouring line and that line's count is needed, the query waits in its
// warp's queue until 16 such queries make a pass of their own (so a pass
// always counts one line per query).  Leaf units are read by lane quads.
template <typename K, typename V, int T>
__global__ void __launch_bounds__(T, 1)
learned_kernel(const __grid_constant__ DevTree t, const __grid_constant__ LearnedDev m,
               const K *__restrict__ q, uint64_t nq, V *__restrict__ out,
               uint8_t *__restrict__ found) {
    constexpr int KPU = unit_keys<K, V>();  // keys per unit
    extern __shared__ uint4 smem_l[];
    __shared__ __align__(8) unsigned long long s_bar;
    __shared__ float4 s_mlp[mlp_units4(kMaxHidden)];
    __shared__ float s_b2;
    __shared__ Retry s_retry[T / 32][kRetryCap];
    K *s_stage = reinterpret_cast<K *>(smem_l);
    // the staged keys: one bulk copy of the (pre-swizzled) array, completing
    // on an mbarrier; the MLP parameters meanwhile by plain loads
    const bool staged = stage_bulk(s_stage, m.stage, m.stage_bytes, &s_bar);
    pack_mlp(m.mlp, (int)m.hidden, s_mlp, &s_b2, threadIdx.x, blockDim.x);
    __syncthreads();
    const int H4 = mlp_units4((int)m.hidden);
    const float b2 = s_b2;

    const int lane = threadIdx.x & 31;
    const int pr = lane >> 1, hl = lane & 1, p0 = pr * 2;
    const uint64_t pol_idx = l2_evict_last(), pol_leaf = l2_evict_first();
    const uint32_t U = (uint32_t)m.units;
    const uint64_t ntiles = (nq + 31) / 32;
    Retry *rq = s_retry[threadIdx.x >> 5];
    uint32_t qn = 0;  // entries in this warp's queue (the same in every lane)
    uint32_t n_extra = 0, n_fallback = 0, n_lines = 0;

    // Appends the queries of the pairs with `need` to the warp's queue (the
    // line word carries the direction of the walk in its top bit).
    auto enqueue = [&](bool need, uint64_t key, uint32_t qi, uint32_t ua, uint32_t ub,
                       uint32_t line_dir, uint32_t skip) {
        const unsigned qmask = __ballot_sync(0xffffffffu, hl == 0 && need);
        if (hl == 0 && need) {
            Retry e;
            e.key = key;
            e.qi = qi;
            e.ua = ua;
            e.ub = ub;
            e.line = line_dir;
            e.skip = skip;
            rq[qn + __popc(qmask & ((1u << lane) - 1u))] = e;
        }
        qn += __popc(qmask);
        __syncwarp();
    };
    // A pass of queued queries: pair pr takes entry first + pr (pr < cnt),
    // the top of the queue, and counts the entry's line; a window that
    // continues past that line as well goes back to the queue with the next
    // line, the others are answered from the leaf.
    auto retry_pass = [&](uint32_t first, uint32_t cnt) {
        const bool live = (uint32_t)pr < cnt;
        Retry e = {};
        if (live) e = rq[first + pr];
        __syncwarp();  // the entries are read before the queue is written again
        qn = first;
        const uint32_t line = e.line & 0x7FFFFFFFu;
        const bool right = (e.line >> 31) != 0;
        const uint32_t j0 = line * kCodesPerLine;
        const uint32_t c = code_count(m.codes, line, live, e.key, hl, p0, pol_idx);
        if (live && hl == 0) n_lines++;
        uint32_t skip = e.skip + window_part(e.ua, e.ub, j0, c);
        const uint32_t la = e.ua / kCodesPerLine, lb = (e.ub - 1) / kCodesPerLine;
        bool more;
        if (right) {
            more = live && line < lb && c >= kCodesPerLine;
        } else {
            more = live && line > la && c == 0;
            if (live && line > la && c > 0) skip += j0 - e.ua;
        }
        enqueue(more, e.key, e.qi, e.ua, e.ub, right ? ((line + 1) | 0x80000000u) : line - 1, skip);
        leaf_quads<K, V>(t, U, pol_leaf, live && !more, e.ua + skip, e.ub, (K)e.key, e.qi, out,
                         found, n_extra, n_fallback);
    };

    for (uint64_t tile = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5; tile < ntiles;
         tile += ((uint64_t)gridDim.x * blockDim.x) >> 5) {
        const uint64_t base = tile * 32;
        // ---- 1. root + staged keys: the query's segment line (one lane per query)
        const uint64_t my = base + lane;
        const K myq = my < nq ? q[my] : (K)0;
        if (!staged) {  // the staged keys never arrived: the tree's full descent
            if (my < nq) {
                tree_point<K, V>(t, myq, out + my, found ? found + my : nullptr);
                n_fallback++;
            }
            continue;
        }
        uint32_t my_sl;
        {
            const int pl = root_line(s_mlp, H4, b2, m.nls, norm_key((uint64_t)myq, m.kmin, m.xscale));
            const int e = (int)m.root_err + 1;
            const uint32_t a = (uint32_t)max(0, pl - e);
            const uint32_t b = (uint32_t)min((int)m.nls - 1, pl + e);
            my_sl = stage_search<K>(s_stage, a, b, myq);
        }
#pragma unroll 1
        for (int hf = 0; hf < 2; hf++) {
            const int k = hf * 16 + pr;
            const K qv = __shfl_sync(0xffffffffu, myq, k);
            const uint32_t qi = (uint32_t)(base + k);
            const bool live = base + k < nq;
            const uint32_t sl = __shfl_sync(0xffffffffu, my_sl, k);
            uint32_t w[16];
            if (live) {
                load_half_line(reinterpret_cast<const unsigned char *>(m.seg + sl) + hl * 64, w, pol_idx);
            } else {
#pragma unroll
                for (int i = 0; i < 16; i++) w[i] = 0;
            }
            // ---- 2. segment -> rank window -> unit window [ua, ub]
            // lane hl of the pair holds segments 2 hl (words 0-7) and 2 hl + 1
            // (words 8-15): key lo, key hi, r_lo, cnt, slope, icpt, eps, pad
            const uint64_t key = (uint64_t)qv;
            const bool b_lt = (((uint64_t)w[9] << 32) | w[8]) < key;
            const bool a_lt = (((uint64_t)w[1] << 32) | w[0]) < key;
            // segment c = how many of the line's keys 1..3 are below the key
            const uint32_t part = hl ? (a_lt ? 1u : 0u) + (b_lt ? 1u : 0u) : (b_lt ? 1u : 0u);
            const uint32_t c = part + __shfl_xor_sync(0xffffffffu, part, 1);
            // the lane holding segment c computes the window; the pair takes
            // its result
            const bool sb = (c & 1) != 0;
            const uint64_t fk = sb ? (((uint64_t)w[9] << 32) | w[8]) : (((uint64_t)w[1] << 32) | w[0]);
            const uint32_t r_lo = sb ? w[10] : w[2], cnt = sb ? w[11] : w[3];
            const float slope = __uint_as_float(sb ? w[12] : w[4]);
            const float icpt = __uint_as_float(sb ? w[13] : w[5]);
            const uint32_t eps = sb ? w[14] : w[6];
            const float p = seg_pred(slope, icpt, cnt, fk, key);  // in [0, cnt]
            // ranks [r_lo + floor(p) - eps - 1, r_lo + ceil(p) + eps + 1], clamped
            const uint32_t lo_r = r_lo + (uint32_t)floorf(p), hi_r = r_lo + (uint32_t)ceilf(p);
            const uint32_t ra = eps >= lo_r ? 0u : lo_r - eps - 1u;
            const uint32_t rb = hi_r + eps + 1u < hi_r ? 0xFFFFFFFFu : hi_r + eps + 1u;
            const int owner = p0 + (int)(c >> 1);
            const uint32_t ua = __shfl_sync(0xffffffffu, min(ra / (uint32_t)KPU, U - 1), owner);
            const uint32_t ub = max(ua, __shfl_sync(0xffffffffu, min(rb / (uint32_t)KPU, U - 1), owner));
            const uint32_t pu_raw = __shfl_sync(0xffffffffu, lo_r / (uint32_t)KPU, owner);
            // ---- 3. thresholds of the window at or below the key, counted on
            // the code line of the predicted unit first
            const bool has = live && ub > ua;
            const uint32_t pu = min(max(pu_raw, ua), ub > ua ? ub - 1 : ua);
            const uint32_t line = pu / kCodesPerLine, j0 = line * kCodesPerLine;
            const uint32_t la = ua / kCodesPerLine, lb = has ? (ub - 1) / kCodesPerLine : la;
            const uint32_t cl = code_count(m.codes, line, has, key, hl, p0, pol_idx);
            uint32_t skip = window_part(ua, ub, j0, cl);
            // The window's lines beside this one matter only where the count
            // may continue into them: left if none of this line's thresholds
            // is at or below the key (else every threshold left of it is),
            // right if all of them are.
            bool need = false, right = false;
            if (has) {
                if (cl == 0 && la < line) {
                    need = true;
                } else {
                    if (la < line) skip += j0 - ua;
                    if (lb > line && cl >= kCodesPerLine) need = right = true;
                }
            }
            // queue the queries that need the next line
            __syncwarp();
            enqueue(need, key, qi, ua, ub, right ? ((line + 1) | 0x80000000u) : line - 1, skip);
            // ---- 4. the leaf unit of the others
            leaf_quads<K, V>(t, U, pol_leaf, live && !need, ua + skip, ub, qv, qi, out, found,
                             n_extra, n_fallback);
            while (qn >= 16) retry_pass(qn - 16, 16);
        }
    }
    while (qn > 0) {  // the rest of the queue
        const uint32_t c = min(qn, 16u);
        retry_pass(qn - c, c);
    }
    if (m.stats && (n_extra | n_fallback | n_lines)) {
        atomicAdd(&m.stats[0], (unsigned long long)n_extra);
        atomicAdd(&m.stats[1], (unsigned long long)n_fallback);
        atomicAdd(&m.stats[2], (unsigned long long)n_lines);
    }
}

template <typename K, typename V, int T>
bt_status learned_launch_t(const bt_tree *t, const void *d_q, uint64_t nq, void *d_out,
                           uint8_t *d_found, cudaStream_t s) {
    const LearnedDev &m = t->learned->dev;
    auto fn = learned_kernel<K, V, T>;
    const size_t smem = (size_t)m.stage_bytes;
    // the largest dynamic shared-memory size this kernel was opened for, per
    // device (host threads may launch concurrently: atomic, and setting the
    // attribute twice is harmless)
    static std::atomic<int> set_for[64];
    const int dev = t->device;
    const bool cached = dev >= 0 && dev < 64;
    if (!cached || set_for[dev].load(std::memory_order_acquire) < (int)smem) {
        BT_CUDA(cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        if (cached) {
            int prev = set_for[dev].load(std::memory_order_relaxed);
            while (prev < (int)smem &&
                   !set_for[dev].compare_exchange_weak(prev, (int)smem, std::memory_order_release))
                ;
        }
    }
    // the kernel indexes its batch with 32-bit offsets: batches of 2^31
    // queries and more go as several launches
    constexpr uint64_t kChunk = 1ull << 31;
    for (uint64_t off = 0; off < nq; off += kChunk) {
        const uint64_t n = std::min(kChunk, nq - off);
        const uint64_t ntiles = (n + 31) / 32;
        const uint64_t want = (ntiles + T / 32 - 1) / (T / 32);
        const unsigned grid = (unsigned)std::max<uint64_t>(1, std::min<uint64_t>(want, sm_count()));
        count_launch();
        fn<<<grid, T, smem, s>>>(t->dev, m, (const K *)d_q + off, n, (V *)d_out + off,
                                 d_found ? d_found + off : nullptr);
        BT_CUDA(cudaGetLastError());
    }
    return BT_OK;
}

template <typename K, typename V>
bt_status learned_launch(const bt_tree *t, const void *d_q, uint64_t nq, void *d_out,
                         uint8_t *d_found, cudaStream_t s) {
    switch (t->learned->shape) {
        case 2: return learned_launch_t<K, V, 768>(t, d_q, nq, d_out, d_found, s);
        case 3: return learned_launch_t<K, V, 640>(t, d_q, nq, d_out, d_found, s);
        case 4: return learned_launch_t<K, V, 512>(t, d_q, nq, d_out, d_found, s);
        default: return learned_launch_t<K, V, 1024>(t, d_q, nq, d_out, d_found, s);
    }
}

// ------------------------------------------------------------- training ---

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
        for (int j = 0; j < H; j++) out += sp[2 * H + j] * fminf(fmaxf(sp[j] * xi + sp[H + j], 0.f), 1.f);
        const float err = out - y[i];
        l += err * err;
        const float dout = scale * err;
        for (int j = 0; j < H; j++) {
            const float h = sp[j] * xi + sp[H + j];
            const float a = fminf(fmaxf(h, 0.f), 1.f);
            g[2 * H + j] += dout * a;
            const float dh = (h > 0.f && h < 1.f) ? dout * sp[2 * H + j] : 0.f;
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

template <typename K, typename V>
bt_status train_impl(bt_tree *t, const bt_learned_config &cfg, cudaStream_t s,
                     bt_learned_report *rep) {
    using LG = LeafGeom<K, V>;
    const uint64_t n = t->n;
    const int H = (int)cfg.hidden;
    const int np = 3 * H + 1;
    const uint32_t kpu = (uint32_t)unit_keys<K, V>();
    const uint64_t units = (n + kpu - 1) / kpu;
    const unsigned char *leaves = (const unsigned char *)t->d_leaves;
    struct Owner {
        LearnedState *p;
        ~Owner() { free_learned(p); }
    } own{new LearnedState()};
    LearnedState *st = own.p;
    cudaEvent_t e0, e1;
    BT_CUDA(cudaEventCreate(&e0));
    BT_CUDA(cudaEventCreate(&e1));
    struct Ev {
        cudaEvent_t a, b;
        ~Ev() {
            cudaEventDestroy(a);
            cudaEventDestroy(b);
        }
    } evs{e0, e1};
    BT_CUDA(cudaEventRecord(e0, s));

    // ---- segmentation: the bound, then the segments
    const uint64_t nchunks = (n + kPlaChunk - 1) / kPlaChunk;
    DevBuf bcnt, boff, btot;
    BT_CUDA(cudaMalloc(&bcnt.p, nchunks * sizeof(uint64_t)));
    BT_CUDA(cudaMalloc(&boff.p, nchunks * sizeof(uint64_t)));
    BT_CUDA(cudaMalloc(&btot.p, sizeof(uint64_t)));
    uint64_t *cnt = (uint64_t *)bcnt.p, *off = (uint64_t *)boff.p, *tot = (uint64_t *)btot.p;
    const unsigned pg = (unsigned)((nchunks + kPlaThreads - 1) / kPlaThreads);
    const size_t pla_smem = (size_t)kPlaThreads * kPlaHullStride * sizeof(PlaPt);
    BT_CUDA(cudaFuncSetAttribute(pla_kernel<K, V, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)pla_smem));
    BT_CUDA(cudaFuncSetAttribute(pla_kernel<K, V, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)pla_smem));
    auto count_at = [&](uint32_t eps, uint64_t *total) -> bt_status {
        count_launch();
        pla_kernel<K, V, true><<<pg, kPlaThreads, pla_smem, s>>>(leaves, n, eps, nchunks, cnt, nullptr, nullptr,
                                                 nullptr, nullptr);
        BT_CUDA(cudaGetLastError());
        bt_status r = launch_scan_u64(cnt, off, nchunks, tot, s);
        if (r != BT_OK) return r;
        BT_CUDA(cudaMemcpyAsync(total, tot, sizeof(uint64_t), cudaMemcpyDeviceToHost, s));
        BT_CUDA(cudaStreamSynchronize(s));
        return BT_OK;
    };
    uint32_t eps = cfg.max_error;
    uint64_t nseg = 0;
    bt_status r;
    uint32_t counted = 0;  // the bound of the last count (its per-chunk offsets are in off)
    if (eps == 0) {
        // The least bound whose segmentation has at most num_segments
        // segments (the count does not grow with the bound).  The bracket
        // (lo, hi] -- count(lo) above the target, count(hi) at or below --
        // grows by 4x from 8, then narrows by interpolating log(count)
        // against log(bound), with a bisection step whenever an
        // interpolated step fails to halve it.
        const double tgt = (double)cfg.num_segments;
        uint32_t lo = 0, hi = 8;
        uint64_t c_lo = 0, c_hi = 0;
        for (;;) {
            if ((r = count_at(hi, &c_hi)) != BT_OK) return r;
            counted = hi;
            if (c_hi <= cfg.num_segments || hi >= (1u << 30)) break;
            lo = hi;
            c_lo = c_hi;
            hi = std::min<uint32_t>(hi * 4, 1u << 30);
        }
        bool bisect = false;
        while (hi - lo > 1) {
            uint32_t m = lo + (hi - lo) / 2;
            if (!bisect && lo > 0 && c_hi > 0 && c_lo > c_hi) {
                const double f = (std::log((double)c_lo) - std::log(tgt)) /
                                 (std::log((double)c_lo) - std::log((double)c_hi));
                const double lm = std::log((double)lo) + f * (std::log((double)hi) - std::log((double)lo));
                const double g = std::ceil(std::exp(lm));
                m = g <= (double)lo ? lo + 1 : g >= (double)hi ? hi - 1 : (uint32_t)g;
            }
            uint64_t c = 0;
            if ((r = count_at(m, &c)) != BT_OK) return r;
            counted = m;
            const uint32_t w = hi - lo;
            if (c <= cfg.num_segments) {
                hi = m;
                c_hi = c;
            } else {
                lo = m;
                c_lo = c;
            }
            bisect = !bisect && (hi - lo) * 2 > w;
        }
        eps = hi;
    }
    if (counted != eps && (r = count_at(eps, &nseg)) != BT_OK) return r;
    if (counted == eps) BT_CUDA(cudaMemcpy(&nseg, tot, sizeof(uint64_t), cudaMemcpyDeviceToHost));
    const uint32_t nls = (uint32_t)((nseg + kSegPerLine - 1) / kSegPerLine);
    const uint32_t row = 128;  // stage in whole bank rows (the swizzle permutes within rows)
    const uint64_t stage_bytes = ((uint64_t)nls * sizeof(K) + row - 1) / row * row;
    if (stage_bytes > kStageBudget)
        return fail(BT_ERR_NOT_SUPPORTED,
                    "the segmentation has " + std::to_string(nseg) +
                        " segments; their lines' first keys exceed the search's shared memory "
                        "(raise max_error or lower num_segments)");
    DevBuf bst, bsl, bic;
    BT_CUDA(cudaMalloc(&bst.p, nseg * sizeof(uint32_t)));
    BT_CUDA(cudaMalloc(&bsl.p, nseg * sizeof(double)));
    BT_CUDA(cudaMalloc(&bic.p, nseg * sizeof(double)));
    count_launch();
    pla_kernel<K, V, false><<<pg, kPlaThreads, pla_smem, s>>>(leaves, n, eps, nchunks, nullptr, off,
                                              (uint32_t *)bst.p, (double *)bsl.p, (double *)bic.p);
    BT_CUDA(cudaGetLastError());

    // ---- segment lines and their exact bounds
    BT_CUDA(cudaMalloc((void **)&st->d_seg, (size_t)nls * sizeof(SegLine)));
    count_launch();
    seg_fill_kernel<K, V><<<grid_of(nls, 256), 256, 0, s>>>(leaves, n, (uint32_t)nseg, nls,
                                                           (const uint32_t *)bst.p,
                                                           (const double *)bsl.p,
                                                           (const double *)bic.p, st->d_seg);
    count_launch();
    seg_eps_kernel<K, V><<<grid_of(nseg * 32, 256), 256, 0, s>>>(leaves, (uint32_t)nseg, st->d_seg);
    BT_CUDA(cudaGetLastError());

    // ---- staged keys and the root's training pairs
    const uint64_t kmin = t->min_key;
    const double span = (double)(t->max_key - t->min_key);
    const float xscale = span > 0 ? (float)(1.0 / span) : 0.f;
    BT_CUDA(cudaMalloc(&st->d_stage, stage_bytes));
    DevBuf bx, by, bg, bm, bv, berr;
    BT_CUDA(cudaMalloc(&bx.p, nls * sizeof(float)));
    BT_CUDA(cudaMalloc(&by.p, nls * sizeof(float)));
    BT_CUDA(cudaMalloc(&bg.p, (np + 1) * sizeof(float)));
    BT_CUDA(cudaMalloc(&bm.p, np * sizeof(float)));
    BT_CUDA(cudaMalloc(&bv.p, np * sizeof(float)));
    BT_CUDA(cudaMalloc(&berr.p, 2 * sizeof(unsigned int)));
    BT_CUDA(cudaMalloc((void **)&st->d_mlp, np * sizeof(float)));
    BT_CUDA(cudaMalloc((void **)&st->d_stats, kLearnedStats * sizeof(unsigned long long)));
    BT_CUDA(cudaMemsetAsync(st->d_stats, 0, kLearnedStats * sizeof(unsigned long long), s));
    BT_CUDA(cudaMemsetAsync(berr.p, 0, 2 * sizeof(unsigned int), s));
    float *x = (float *)bx.p, *y = (float *)by.p, *grad = (float *)bg.p, *loss = grad + np;
    unsigned int *err = (unsigned int *)berr.p;
    count_launch();
    stage_kernel<K><<<grid_of(stage_bytes / sizeof(K), 256), 256, 0, s>>>(
        st->d_seg, nls, (uint32_t)(stage_bytes / sizeof(K)), kmin, xscale, (K *)st->d_stage, x, y);

    // ---- root: ramps tiling [0, 1] in equal steps with output weights 1/H
    // (the identity y = x: the untrained network), then Adam
    std::vector<float> p0(np);
    for (int j = 0; j < H; j++) {
        p0[j] = (float)H;
        p0[H + j] = -(float)j;
        p0[2 * H + j] = 1.f / (float)H;
    }
    p0[3 * H] = 0.f;
    BT_CUDA(cudaMemcpyAsync(st->d_mlp, p0.data(), np * sizeof(float), cudaMemcpyHostToDevice, s));
    count_launch();
    root_err_kernel<<<grid_of(nls, 256, 4), 256, 0, s>>>(st->d_mlp, H, x, nls, err + 1);
    BT_CUDA(cudaMemsetAsync(bm.p, 0, np * sizeof(float), s));
    BT_CUDA(cudaMemsetAsync(bv.p, 0, np * sizeof(float), s));
    float l0 = 0.f, l1 = 0.f;
    const unsigned lg = grid_of(nls, 256, 4);
    for (uint32_t it = 0; it <= cfg.iterations; it++) {
        BT_CUDA(cudaMemsetAsync(grad, 0, (np + 1) * sizeof(float), s));
        count_launch();
        mlp_loss_grad_kernel<<<lg, 256, 0, s>>>(st->d_mlp, H, x, y, nls, loss, grad);
        if (it == 0) BT_CUDA(cudaMemcpyAsync(&l0, loss, sizeof(float), cudaMemcpyDeviceToHost, s));
        if (it == cfg.iterations) {
            BT_CUDA(cudaMemcpyAsync(&l1, loss, sizeof(float), cudaMemcpyDeviceToHost, s));
            break;
        }
        count_launch();
        adam_kernel<<<1, 128, 0, s>>>(st->d_mlp, grad, (float *)bm.p, (float *)bv.p, H,
                                      cfg.learning_rate, (int)it + 1);
    }
    count_launch();
    root_err_kernel<<<grid_of(nls, 256, 4), 256, 0, s>>>(st->d_mlp, H, x, nls, err);

    // ---- unit thresholds
    const uint64_t ncl = units > 1 ? (units - 1 + kCodesPerLine - 1) / kCodesPerLine : 0;
    BT_CUDA(cudaMalloc((void **)&st->d_codes, std::max<uint64_t>(1, ncl) * sizeof(CodeLine)));
    if (ncl) {
        count_launch();
        code_kernel<K, V><<<grid_of(ncl, 256), 256, 0, s>>>(leaves, n, units, ncl, st->d_codes);
    }
    BT_CUDA(cudaGetLastError());
    BT_CUDA(cudaEventRecord(e1, s));
    unsigned int herr[2] = {0, 0};
    std::vector<SegLine> segs(nls);
    BT_CUDA(cudaMemcpyAsync(herr, err, sizeof(herr), cudaMemcpyDeviceToHost, s));
    BT_CUDA(cudaMemcpyAsync(segs.data(), st->d_seg, nls * sizeof(SegLine), cudaMemcpyDeviceToHost, s));
    BT_CUDA(cudaStreamSynchronize(s));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);

    LearnedDev &d = st->dev;
    d.mlp = st->d_mlp;
    d.seg = st->d_seg;
    d.codes = st->d_codes;
    d.stage = st->d_stage;
    d.stats = st->d_stats;
    d.kmin = kmin;
    d.xscale = xscale;
    d.hidden = H;
    d.nseg = (uint32_t)nseg;
    d.nls = nls;
    d.root_err = herr[0];
    d.kpu = kpu;
    d.units = units;
    d.stage_bytes = (uint32_t)stage_bytes;
    st->bytes = (uint64_t)nls * sizeof(SegLine) + ncl * sizeof(CodeLine) + stage_bytes +
                np * sizeof(float);
    (void)LG::S;

    if (rep) {
        std::memset(rep, 0, sizeof(*rep));
        rep->root_loss_initial = l0;
        rep->root_loss_final = l1;
        rep->root_error = herr[0];
        rep->root_error_initial = herr[1];
        rep->num_segments = (uint32_t)nseg;
        rep->max_error = eps;
        double esum = 0, lsum = 0;
        uint64_t emax = 0;
        for (uint64_t g = 0; g < nseg; g++) {
            const SegLine &sl = segs[g / kSegPerLine];
            const int k = (int)(g % kSegPerLine);
            esum += sl.s[k].eps;
            emax = std::max<uint64_t>(emax, sl.s[k].eps);
            // window of 2 eps + 3 ranks: units it spans, then code lines
            const double win_units = (2.0 * sl.s[k].eps + 3.0) / kpu + 1.0;
            lsum += (double)sl.s[k].cnt * (1.0 + (win_units - 1.0) / kCodesPerLine);
        }
        rep->eps_mean = nseg ? esum / (double)nseg : 0;
        rep->eps_max = emax;
        rep->code_lines_mean = n ? lsum / (double)n : 0;
        rep->index_bytes = st->bytes;
        rep->keys_per_unit = kpu;
        rep->train_ms = ms;
    }
    if (t->learned) free_learned(t->learned);
    t->learned = st;
    own.p = nullptr;
    return BT_OK;
}

}  // namespace

bt_status launch_learned_search(const bt_tree *t, const void *d_q, uint64_t nq, void *d_out,
                                uint8_t *d_found, cudaStream_t s) {
    if (nq == 0) return BT_OK;
    if (t->key_bytes == 4)
        return t->val_bytes == 4 ? learned_launch<uint32_t, uint32_t>(t, d_q, nq, d_out, d_found, s)
                                 : learned_launch<uint32_t, uint64_t>(t, d_q, nq, d_out, d_found, s);
    return t->val_bytes == 4 ? learned_launch<uint64_t, uint32_t>(t, d_q, nq, d_out, d_found, s)
                             : learned_launch<uint64_t, uint64_t>(t, d_q, nq, d_out, d_found, s);
}

bt_status reset_learned_stats(const bt_tree *t, cudaStream_t s) {
    BT_CUDA(cudaMemsetAsync(t->learned->d_stats, 0, kLearnedStats * sizeof(unsigned long long), s));
    return BT_OK;
}

}  // namespace bt

extern "C" {

bt_status bt_learned_train(bt_tree *t, const bt_learned_config *cfg_in, void *stream,
                           bt_learned_report *report) {
    using namespace bt;
    if (!t) return fail(BT_ERR_INVALID_ARGUMENT, "tree is NULL");
    if (t->n < 2) return fail(BT_ERR_INVALID_ARGUMENT, "a learned index needs at least 2 keys");
    if (t->n >= (1ull << 32)) return fail(BT_ERR_INVALID_ARGUMENT, "learned index supports n < 2^32");
    bt_learned_config cfg = {65536, 0, 16, 400, 0.002f};
    if (cfg_in) {
        if (cfg_in->num_segments) cfg.num_segments = cfg_in->num_segments;
        cfg.max_error = cfg_in->max_error;
        if (cfg_in->hidden) cfg.hidden = cfg_in->hidden;
        cfg.iterations = cfg_in->iterations;
        if (cfg_in->learning_rate > 0) cfg.learning_rate = cfg_in->learning_rate;
    }
    if (cfg.hidden > (uint32_t)kMaxHidden) return fail(BT_ERR_INVALID_ARGUMENT, "hidden must be <= 32");
    if (cfg.max_error > (1u << 30)) return fail(BT_ERR_INVALID_ARGUMENT, "max_error too large");
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
    return bt_point_search(t, BT_POINT_LEARNED, d_q, nq, d_out, stream);
}

bt_status bt_learned_set_shape(bt_tree *t, uint32_t shape) {
    using namespace bt;
    if (!t || !t->learned) return fail(BT_ERR_INVALID_ARGUMENT, "the tree has no trained learned index");
    if (shape < 1 || shape > (uint32_t)kLearnedShapes)
        return fail(BT_ERR_INVALID_ARGUMENT, "shape must be 1..4");
    t->learned->shape = (int)shape;
    return BT_OK;
}

bt_status bt_learned_last_stats(const bt_tree *t, uint64_t *extra, uint64_t *fallback) {
    using namespace bt;
    if (!t || !t->learned) return fail(BT_ERR_INVALID_ARGUMENT, "the tree has no trained learned index");
    unsigned long long h[2] = {0, 0};
    BT_CUDA(cudaMemcpy(h, t->learned->d_stats, sizeof(h), cudaMemcpyDeviceToHost));
    if (extra) *extra = h[0];
    if (fallback) *fallback = h[1];
    return BT_OK;
}

bt_status bt_learned_last_lines(const bt_tree *t, uint64_t *extra_lines) {
    using namespace bt;
    if (!t || !t->learned) return fail(BT_ERR_INVALID_ARGUMENT, "the tree has no trained learned index");
    if (!extra_lines) return fail(BT_ERR_INVALID_ARGUMENT, "extra_lines is NULL");
    unsigned long long h[kLearnedStats] = {};
    BT_CUDA(cudaMemcpy(h, t->learned->d_stats, sizeof(h), cudaMemcpyDeviceToHost));
    *extra_lines = h[2];
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
