// Query grouping, exclusive scan and range-ID fill.
//
// Grouping reorders a query batch so that queries that walk the same part of
// the tree run next to each other (in the same CTAs, at the same time), which
// turns repeated node and leaf-sector reads into L1/L2 hits.  The reference
// does this with an MSD radix partition by 8-bit digits, iterated until every
// group holds at most GROUP_SEARCH_SIZE = 33,000 queries, with a host round
// trip per pass and per group (genGrouping, grouping.cu:1677-1851;
// radixGroupGPU :776; radixGroupSingleKernelGPU :1288), and one CTA per group.
//
// Here a group key of D bits is computed per query and the batch is sorted by
// it with D/8 stable LSD counting passes (histogram -> scan -> scatter), all
// on the device with no host round trip.  Each scatter carries the caller's
// index, so results are written straight back in the caller's order.
//   point : the top D bits of the key (relative to the tree's key width);
//   2D    : (top D/2 bits of start, top D/2 bits of end), row-major -- a true
//           2-D cell, where the reference buckets by the product of two
//           digits (bucketIdentify2d, grouping2d.cu:24-31);
//   Z     : the Morton interleave of those two D/2-bit coordinates, as the
//           reference interleaves start and end (calcuateZorder2d,
//           zOrder2d.cu:27-54) before grouping by the code.
// A pass is stable, so the order is deterministic (the reference's in-block
// atomicAdd scatter is not, grouping.cu:451-452).
#include <algorithm>
#include <atomic>
#include <vector>

#include "bt_internal.cuh"
#include "bt_sort.cuh"

namespace bt {
namespace {

constexpr int kPT = 512;             // partition threads per CTA
constexpr int kPWarps = kPT / 32;    // 16
constexpr int kIPL = 8;              // items per lane
constexpr int kPTile = kPT * kIPL;   // 4096 items per tile
constexpr int kPerWarp = 32 * kIPL;  // 256 items per warp sub-tile

struct GroupKeyParams {
    int kind;   // PartitionKind
    int shift;  // right shift applied to keys
    int cbits;  // bits per coordinate (2D/Z) or total bits (point)
};

__device__ __forceinline__ uint32_t spread16(uint32_t x) {
    x &= 0xFFFFu;
    x = (x | (x << 8)) & 0x00FF00FFu;
    x = (x | (x << 4)) & 0x0F0F0F0Fu;
    x = (x | (x << 2)) & 0x33333333u;
    x = (x | (x << 1)) & 0x55555555u;
    return x;
}

template <typename K>
__device__ __forceinline__ uint32_t group_key(K a, K b, const GroupKeyParams &p) {
    if (p.kind == kPartRadix) return (uint32_t)((uint64_t)a >> p.shift);  // caller takes the low byte
    const uint64_t lim = (1ull << p.cbits) - 1;
    uint64_t x = (uint64_t)a >> p.shift;
    x = x < lim ? x : lim;
    if (p.kind == kPartPoint) return (uint32_t)x;
    uint64_t y = (uint64_t)b >> p.shift;
    y = y < lim ? y : lim;
    if (p.kind == kPart2D) return (uint32_t)((x << p.cbits) | y);
    return spread16((uint32_t)x) | (spread16((uint32_t)y) << 1);
}

// Digit histogram of one tile: per-warp shared-memory histograms (atomics
// only collide inside a warp), summed per digit at the end.
template <typename K, bool HAS_B>
__global__ void __launch_bounds__(kPT)
part_hist_kernel(const K *__restrict__ a, const K *__restrict__ b, uint64_t n, GroupKeyParams gp,
                 int pass, uint32_t *__restrict__ counts, uint64_t ntiles) {
    __shared__ uint32_t h[kPWarps][256];
    for (int i = threadIdx.x; i < kPWarps * 256; i += kPT) (&h[0][0])[i] = 0;
    __syncthreads();
    const int w = threadIdx.x >> 5;
    const uint64_t t0 = (uint64_t)blockIdx.x * kPTile;
    K av[kIPL], bv[kIPL];
#pragma unroll
    for (int j = 0; j < kIPL; j++) {
        const uint64_t i = t0 + (uint64_t)j * kPT + threadIdx.x;
        av[j] = i < n ? a[i] : (K)0;
        bv[j] = (HAS_B && i < n) ? b[i] : (K)0;
    }
#pragma unroll
    for (int j = 0; j < kIPL; j++) {
        const uint64_t i = t0 + (uint64_t)j * kPT + threadIdx.x;
        if (i < n) atomicAdd(&h[w][(group_key<K>(av[j], bv[j], gp) >> (8 * pass)) & 0xFFu], 1u);
    }
    __syncthreads();
    for (int d = threadIdx.x; d < 256; d += kPT) {
        uint32_t c = 0;
#pragma unroll
        for (int ww = 0; ww < kPWarps; ww++) c += h[ww][d];
        counts[(uint64_t)d * ntiles + blockIdx.x] = c;
    }
}

// Exclusive scan of 256 values held one per thread by threads 0..255.
__device__ __forceinline__ uint32_t block_exscan256(uint32_t v, uint32_t *warp_tot) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_tot[w] = x;
    __syncwarp();
    return x - v;  // exclusive within the warp; caller adds the warp prefix
}

template <typename K, bool HAS_B>
__global__ void __launch_bounds__(kPT, 3)
part_scatter_kernel(const K *__restrict__ a, const K *__restrict__ b,
                    const uint32_t *__restrict__ perm_in, uint64_t n, GroupKeyParams gp, int pass,
                    const uint32_t *__restrict__ base, uint64_t ntiles, K *__restrict__ oa,
                    K *__restrict__ ob, uint32_t *__restrict__ operm) {
    __shared__ uint32_t cnt[kPWarps][256];
    __shared__ uint32_t tile_start[256];
    __shared__ uint32_t tile_base[256];  // global start of each digit's run of this tile
    __shared__ uint32_t digit_tot[256];  // items of each digit in this tile
    __shared__ uint32_t warp_tot[8];
    extern __shared__ __align__(16) unsigned char smem_raw[];
    K *sa = reinterpret_cast<K *>(smem_raw);
    K *sb = sa + kPTile;
    uint32_t *sp = reinterpret_cast<uint32_t *>(sb + (HAS_B ? kPTile : 0));
    uint8_t *sd = reinterpret_cast<uint8_t *>(sp + kPTile);

    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int i = threadIdx.x; i < kPWarps * 256; i += kPT) (&cnt[0][0])[i] = 0;
    if (threadIdx.x < 256) tile_base[threadIdx.x] = base[(uint64_t)threadIdx.x * ntiles + blockIdx.x];
    __syncthreads();

    const uint64_t t0 = (uint64_t)blockIdx.x * kPTile;
    K av[kIPL], bv[kIPL];
    uint32_t pv[kIPL], dg[kIPL], rk[kIPL];
#pragma unroll
    for (int j = 0; j < kIPL; j++) {
        const uint64_t i = t0 + (uint64_t)w * kPerWarp + (uint64_t)j * 32 + lane;
        dg[j] = 0xFFFFFFFFu;
        av[j] = 0;
        bv[j] = 0;
        pv[j] = 0;
        if (i < n) {
            av[j] = a[i];
            if (HAS_B) bv[j] = b[i];
            pv[j] = perm_in ? perm_in[i] : (uint32_t)i;
            dg[j] = (group_key<K>(av[j], bv[j], gp) >> (8 * pass)) & 0xFFu;
        }
    }
    // Stable rank of every item among the same-digit items of this warp's
    // sub-tile (item order = j-major, then lane).  The peer masks do not
    // depend on the counters: take them all first.
    const unsigned lt = (1u << lane) - 1u;
    unsigned mm[kIPL];
#pragma unroll
    for (int j = 0; j < kIPL; j++) mm[j] = __match_any_sync(0xffffffffu, dg[j]);
    // Rows in order: each row's leader of a digit adds the row's count to the
    // warp's counter and hands the old value to its peers (the next row's
    // atomic comes after this row's shuffle, so the order is the item order).
#pragma unroll
    for (int j = 0; j < kIPL; j++) {
        const unsigned m = mm[j];
        const int leader = __ffs(m) - 1;
        uint32_t c = 0;
        if (dg[j] != 0xFFFFFFFFu && lane == leader) c = atomicAdd(&cnt[w][dg[j]], (uint32_t)__popc(m));
        c = __shfl_sync(0xffffffffu, c, leader);
        rk[j] = c + __popc(m & lt);
    }
    __syncthreads();
    // Per digit: exclusive prefix over the 16 warps, and the tile total.
    // Warp ww handles digits 16 ww .. 16 ww + 15, half a lane-row each of
    // the warps 0-7 and 8-15.
    {
        const int d = 16 * w + (lane & 15);
        const int h = lane >> 4;
        uint32_t v[kPWarps / 2], run = 0;
#pragma unroll
        for (int k = 0; k < kPWarps / 2; k++) v[k] = cnt[(kPWarps / 2) * h + k][d];
        uint32_t half_tot = 0;
#pragma unroll
        for (int k = 0; k < kPWarps / 2; k++) half_tot += v[k];
        const uint32_t other = __shfl_xor_sync(0xffffffffu, half_tot, 16);
        run = h ? other : 0u;
#pragma unroll
        for (int k = 0; k < kPWarps / 2; k++) {
            cnt[(kPWarps / 2) * h + k][d] = run;
            run += v[k];
        }
        if (h == 0) digit_tot[d] = half_tot + other;
    }
    __syncthreads();
    uint32_t tot = threadIdx.x < 256 ? digit_tot[threadIdx.x] : 0u;
    uint32_t ex = 0;
    if (threadIdx.x < 256) ex = block_exscan256(tot, warp_tot);
    __syncthreads();
    if (threadIdx.x < 256) {
        uint32_t wp = 0;
        for (int ww = 0; ww < (threadIdx.x >> 5); ww++) wp += warp_tot[ww];
        tile_start[threadIdx.x] = ex + wp;
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < kIPL; j++) {
        if (dg[j] != 0xFFFFFFFFu) {
            const uint32_t lp = tile_start[dg[j]] + cnt[w][dg[j]] + rk[j];
            sa[lp] = av[j];
            if (HAS_B) sb[lp] = bv[j];
            sp[lp] = pv[j];
            sd[lp] = (uint8_t)dg[j];
        }
    }
    __syncthreads();
    const uint32_t tn = (uint32_t)min((uint64_t)kPTile, n - t0);
    for (uint32_t lp = threadIdx.x; lp < tn; lp += kPT) {
        const uint32_t d = sd[lp];
        const uint64_t g = (uint64_t)tile_base[d] + (lp - tile_start[d]);
        oa[g] = sa[lp];
        if (HAS_B) ob[g] = sb[lp];
        operm[g] = sp[lp];
    }
}

// ------------------------------------------- single-pass partition ----
//
// The kernels above take three launches per pass (tile histograms, a global
// scan of the tile x digit table, the scatter), read the keys twice per pass
// and load each tile's 256 digit bases from a table laid out digit-major
// (256 scattered reads per tile).  The path below makes one read of the keys
// for the global digit counts of every pass, then one scatter launch per
// pass: tiles are taken in launch order from a counter, and each tile learns
// where its digits start from the tiles before it by decoupled look-back
// (Merrill & Garland, "Single-pass parallel prefix scan with decoupled
// look-back", 2016; used per digit in the onesweep radix sort of Adinets &
// Merrill, 2022): it publishes its digit counts, then walks back over its
// predecessors' published values until it meets an inclusive prefix.

constexpr int kMaxPasses = 8;
constexpr unsigned long long kStAgg = 1ull << 62;   // tile aggregate published
constexpr unsigned long long kStInc = 2ull << 62;   // inclusive prefix published
constexpr unsigned long long kStVal = (1ull << 62) - 1;
constexpr uint32_t kLookbackSpins = 1u << 22;       // polls of one predecessor before giving up

// Look-backs that gave up (a predecessor never published: impossible while
// tiles are taken in order, as they are here); read by
// bt_partition_lookback_timeouts.
__device__ unsigned int g_lookback_timeouts = 0;

__device__ __forceinline__ unsigned long long ld_acquire_u64(const unsigned long long *p) {
    unsigned long long v;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void st_release_u64(unsigned long long *p, unsigned long long v) {
    asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

// Digit of pass p of an item: byte p of its group key (of the key itself for
// the radix sort).
template <typename K>
__device__ __forceinline__ uint32_t pass_digit(K a, K b, const GroupKeyParams &gp, int p) {
    if (gp.kind == kPartRadix) return (uint32_t)(((uint64_t)a >> (8 * p)) & 0xFFu);
    return (group_key<K>(a, b, gp) >> (8 * p)) & 0xFFu;
}

// hist[p * 256 + d] += items whose pass-p digit is d, for every pass, in one
// read of the items (the digits do not depend on the order the passes leave).
template <typename K, bool HAS_B>
__global__ void __launch_bounds__(kPT)
part_hist_all_kernel(const K *__restrict__ a, const K *__restrict__ b, uint64_t n,
                     GroupKeyParams gp, int passes, uint32_t *__restrict__ hist) {
    constexpr int C = 4;  // copies, so that one hot digit is not one hot counter
    __shared__ uint32_t h[C][kMaxPasses * 256];
    for (int i = threadIdx.x; i < C * kMaxPasses * 256; i += kPT) (&h[0][0])[i] = 0;
    __syncthreads();
    uint32_t *hc = h[(threadIdx.x >> 5) & (C - 1)];
    for (uint64_t i = blockIdx.x * (uint64_t)kPT + threadIdx.x; i < n; i += (uint64_t)gridDim.x * kPT) {
        const K av = a[i];
        const K bv = HAS_B ? b[i] : (K)0;
        for (int p = 0; p < passes; p++) atomicAdd(&hc[p * 256 + pass_digit<K>(av, bv, gp, p)], 1u);
    }
    __syncthreads();
    for (int i = threadIdx.x; i < passes * 256; i += kPT) {
        uint32_t c = 0;
#pragma unroll
        for (int k = 0; k < C; k++) c += h[k][i];
        if (c) atomicAdd(&hist[i], c);
    }
}

// One pass of the stable partition: the tile taken from *tile_ctr (in launch
// order) is ranked exactly as in part_scatter_kernel, its digit bases come
// from the global digit starts (exclusive scan of hist) plus the look-back
// over the tiles before it, and it is written out through shared memory.
template <typename K, bool HAS_B>
__global__ void __launch_bounds__(kPT, 3)
part_onesweep_kernel(const K *__restrict__ a, const K *__restrict__ b,
                     const uint32_t *__restrict__ perm_in, uint64_t n, GroupKeyParams gp, int pass,
                     const uint32_t *__restrict__ hist, unsigned int *__restrict__ tile_ctr,
                     unsigned long long *__restrict__ status, K *__restrict__ oa,
                     K *__restrict__ ob, uint32_t *__restrict__ operm) {
    __shared__ uint32_t cnt[kPWarps][256];
    __shared__ uint32_t tile_start[256];
    __shared__ uint32_t tile_base[256];
    __shared__ uint32_t digit_tot[256];
    __shared__ uint32_t warp_tot[8];
    __shared__ uint32_t s_tile;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    K *sa = reinterpret_cast<K *>(smem_raw);
    K *sb = sa + kPTile;
    uint32_t *sp = reinterpret_cast<uint32_t *>(sb + (HAS_B ? kPTile : 0));
    uint8_t *sd = reinterpret_cast<uint8_t *>(sp + kPTile);

    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int i = threadIdx.x; i < kPWarps * 256; i += kPT) (&cnt[0][0])[i] = 0;
    if (threadIdx.x == 0) s_tile = atomicAdd(tile_ctr, 1u);
    // global start of every digit: exclusive scan of this pass's counts
    uint32_t gstart = 0;
    if (threadIdx.x < 256) gstart = block_exscan256(hist[pass * 256 + threadIdx.x], warp_tot);
    __syncthreads();
    if (threadIdx.x < 256) {
        uint32_t wp = 0;
        for (int ww = 0; ww < (threadIdx.x >> 5); ww++) wp += warp_tot[ww];
        gstart += wp;
    }
    const uint64_t tile = s_tile;
    const uint64_t t0 = tile * kPTile;
    K av[kIPL], bv[kIPL];
    uint32_t pv[kIPL], dg[kIPL], rk[kIPL];
#pragma unroll
    for (int j = 0; j < kIPL; j++) {
        const uint64_t i = t0 + (uint64_t)w * kPerWarp + (uint64_t)j * 32 + lane;
        dg[j] = 0xFFFFFFFFu;
        av[j] = 0;
        bv[j] = 0;
        pv[j] = 0;
        if (i < n) {
            av[j] = a[i];
            if (HAS_B) bv[j] = b[i];
            pv[j] = perm_in ? perm_in[i] : (uint32_t)i;
            dg[j] = pass_digit<K>(av[j], bv[j], gp, pass);
        }
    }
    const unsigned lt = (1u << lane) - 1u;
    unsigned mm[kIPL];
#pragma unroll
    for (int j = 0; j < kIPL; j++) mm[j] = __match_any_sync(0xffffffffu, dg[j]);
#pragma unroll
    for (int j = 0; j < kIPL; j++) {
        const unsigned m = mm[j];
        const int leader = __ffs(m) - 1;
        uint32_t c = 0;
        if (dg[j] != 0xFFFFFFFFu && lane == leader) c = atomicAdd(&cnt[w][dg[j]], (uint32_t)__popc(m));
        c = __shfl_sync(0xffffffffu, c, leader);
        rk[j] = c + __popc(m & lt);
    }
    __syncthreads();
    {
        const int d = 16 * w + (lane & 15);
        const int h = lane >> 4;
        uint32_t v[kPWarps / 2];
#pragma unroll
        for (int k = 0; k < kPWarps / 2; k++) v[k] = cnt[(kPWarps / 2) * h + k][d];
        uint32_t half_tot = 0;
#pragma unroll
        for (int k = 0; k < kPWarps / 2; k++) half_tot += v[k];
        const uint32_t other = __shfl_xor_sync(0xffffffffu, half_tot, 16);
        uint32_t run = h ? other : 0u;
#pragma unroll
        for (int k = 0; k < kPWarps / 2; k++) {
            cnt[(kPWarps / 2) * h + k][d] = run;
            run += v[k];
        }
        if (h == 0) digit_tot[d] = half_tot + other;
    }
    __syncthreads();
    // publish this tile's counts, then sum the predecessors' (look-back)
    if (threadIdx.x < 256) {
        const int d = threadIdx.x;
        const uint32_t agg = digit_tot[d];
        unsigned long long *mine = status + tile * 256 + d;
        unsigned long long prefix = 0;
        if (tile == 0) {
            st_release_u64(mine, kStInc | agg);
        } else {
            st_release_u64(mine, kStAgg | agg);
            uint64_t tp = tile - 1;
            uint32_t spins = 0;
            for (;;) {
                const unsigned long long v = ld_acquire_u64(status + tp * 256 + d);
                const unsigned long long f = v & ~kStVal;
                if (f == 0) {
                    if (++spins > kLookbackSpins) {  // never in a correct launch; bounded anyway
                        atomicAdd(&g_lookback_timeouts, 1u);
                        break;
                    }
                    __nanosleep(32);
                    continue;
                }
                spins = 0;
                prefix += v & kStVal;
                if (f == kStInc || tp == 0) break;
                tp--;
            }
            st_release_u64(mine, kStInc | (prefix + agg));
        }
        tile_base[d] = gstart + (uint32_t)prefix;
    }
    uint32_t tot = threadIdx.x < 256 ? digit_tot[threadIdx.x] : 0u;
    uint32_t ex = 0;
    if (threadIdx.x < 256) ex = block_exscan256(tot, warp_tot + 0);
    __syncthreads();
    if (threadIdx.x < 256) {
        uint32_t wp = 0;
        for (int ww = 0; ww < (threadIdx.x >> 5); ww++) wp += warp_tot[ww];
        tile_start[threadIdx.x] = ex + wp;
    }
    __syncthreads();
#pragma unroll
    for (int j = 0; j < kIPL; j++) {
        if (dg[j] != 0xFFFFFFFFu) {
            const uint32_t lp = tile_start[dg[j]] + cnt[w][dg[j]] + rk[j];
            sa[lp] = av[j];
            if (HAS_B) sb[lp] = bv[j];
            sp[lp] = pv[j];
            sd[lp] = (uint8_t)dg[j];
        }
    }
    __syncthreads();
    const uint32_t tn = t0 < n ? (uint32_t)min((uint64_t)kPTile, n - t0) : 0u;
    for (uint32_t lp = threadIdx.x; lp < tn; lp += kPT) {
        const uint32_t d = sd[lp];
        const uint64_t g = (uint64_t)tile_base[d] + (lp - tile_start[d]);
        oa[g] = sa[lp];
        if (HAS_B) ob[g] = sb[lp];
        operm[g] = sp[lp];
    }
}

// ---------------------------------------------------------------- scan ----

constexpr int kST = 512;
constexpr int kSIPT = 8;
constexpr int kSTile = kST * kSIPT;

template <typename T>
__device__ __forceinline__ T block_exscan(T v, T *s_warp, T *total) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    T x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        T y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) s_warp[w] = x;
    __syncthreads();
    if (w == 0) {
        T y = lane < (kST / 32) ? s_warp[lane] : (T)0;
        T z = y;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            T u = __shfl_up_sync(0xffffffffu, z, o);
            if (lane >= o) z += u;
        }
        if (lane < (kST / 32)) s_warp[lane] = z - y;
        if (lane == 31) *total = z;
    }
    __syncthreads();
    return x - v + s_warp[w];
}

template <typename T>
__global__ void __launch_bounds__(kST) scan_reduce_kernel(const T *__restrict__ in, uint64_t n,
                                                          T *__restrict__ sums) {
    __shared__ T s_warp[kST / 32];
    __shared__ T total;
    const uint64_t t0 = (uint64_t)blockIdx.x * kSTile + (uint64_t)threadIdx.x * kSIPT;
    T acc = 0;
#pragma unroll
    for (int j = 0; j < kSIPT; j++)
        if (t0 + j < n) acc += in[t0 + j];
    block_exscan<T>(acc, s_warp, &total);
    if (threadIdx.x == 0) sums[blockIdx.x] = total;
}

template <typename T>
__global__ void __launch_bounds__(kST)
scan_down_kernel(const T *__restrict__ in, uint64_t n, const T *__restrict__ offs,
                 T *__restrict__ out, T *__restrict__ grand_total) {
    __shared__ T s_warp[kST / 32];
    __shared__ T total;
    const uint64_t t0 = (uint64_t)blockIdx.x * kSTile + (uint64_t)threadIdx.x * kSIPT;
    T v[kSIPT];
    T acc = 0;
#pragma unroll
    for (int j = 0; j < kSIPT; j++) {
        v[j] = (t0 + j < n) ? in[t0 + j] : (T)0;
        acc += v[j];
    }
    T run = block_exscan<T>(acc, s_warp, &total) + (offs ? offs[blockIdx.x] : (T)0);
#pragma unroll
    for (int j = 0; j < kSIPT; j++) {
        if (t0 + j < n) out[t0 + j] = run;
        run += v[j];
    }
    if (grand_total && blockIdx.x == gridDim.x - 1 && threadIdx.x == 0)
        *grand_total = total + (offs ? offs[blockIdx.x] : (T)0);
}

// Scratch elements scan_run needs for n inputs (block sums and offsets of
// every recursion level).
uint64_t scan_ws_elems(uint64_t n) {
    uint64_t total = 0;
    while (n > (uint64_t)kSTile) {
        n = (n + kSTile - 1) / kSTile;
        total += 2 * n;
    }
    return total;
}

// Exclusive scan d_out = scan(d_in) with caller-provided scratch (ws of
// scan_ws_elems(n) elements); *d_total (optional) receives the sum.
template <typename T>
bt_status scan_run(const T *d_in, T *d_out, uint64_t n, T *d_total, T *ws, cudaStream_t s) {
    if (n == 0) {
        if (d_total) BT_CUDA(cudaMemsetAsync(d_total, 0, sizeof(T), s));
        return BT_OK;
    }
    const uint64_t nb = (n + kSTile - 1) / kSTile;
    if (nb == 1) {
        count_launch();
        scan_down_kernel<T><<<1, kST, 0, s>>>(d_in, n, nullptr, d_out, d_total);
        BT_CUDA(cudaGetLastError());
        return BT_OK;
    }
    T *sums = ws, *offs = ws + nb;
    count_launch();
    scan_reduce_kernel<T><<<(unsigned)nb, kST, 0, s>>>(d_in, n, sums);
    bt_status st = scan_run<T>(sums, offs, nb, nullptr, ws + 2 * nb, s);
    if (st != BT_OK) return st;
    count_launch();
    scan_down_kernel<T><<<(unsigned)nb, kST, 0, s>>>(d_in, n, offs, d_out, d_total);
    BT_CUDA(cudaGetLastError());
    return BT_OK;
}

template <typename T>
bt_status scan_impl(const T *d_in, T *d_out, uint64_t n, T *d_total, cudaStream_t s) {
    const uint64_t we = scan_ws_elems(n);
    T *ws = nullptr;
    if (we) {
        bt_status st = ws_alloc((void **)&ws, we * sizeof(T), s);
        if (st != BT_OK) return st;
    }
    bt_status st = scan_run<T>(d_in, d_out, n, d_total, ws, s);
    ws_free(ws, s);
    return st;
}

// -------------------------------------------------------- partition host --

// Dynamic shared memory of part_scatter_kernel<K, HAS_B> and its one-time
// raise above the 48 KB default (per device and instantiation; function
// attributes are per device, and the server's worker and user threads may
// partition at once).
template <typename K, bool HAS_B>
constexpr size_t scatter_smem() {
    return (size_t)kPTile * (sizeof(K) * (HAS_B ? 2 : 1) + sizeof(uint32_t) + 1);
}

template <typename K, bool HAS_B>
bt_status scatter_smem_attr() {
    static std::atomic<bool> done[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev >= 0 && dev < 64 && done[dev].load(std::memory_order_acquire)) return BT_OK;
    BT_CUDA(cudaFuncSetAttribute(part_scatter_kernel<K, HAS_B>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)scatter_smem<K, HAS_B>()));
    if (dev >= 0 && dev < 64) done[dev].store(true, std::memory_order_release);
    return BT_OK;
}

template <typename K, bool HAS_B>
bt_status onesweep_smem_attr() {
    static std::atomic<bool> done[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev >= 0 && dev < 64 && done[dev].load(std::memory_order_acquire)) return BT_OK;
    BT_CUDA(cudaFuncSetAttribute(part_onesweep_kernel<K, HAS_B>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)scatter_smem<K, HAS_B>()));
    if (dev >= 0 && dev < 64) done[dev].store(true, std::memory_order_release);
    return BT_OK;
}

// Workspace of the single-pass partition: digit counts of every pass, one
// tile counter per pass, the look-back status of one pass.
struct SweepWs {
    uint32_t *hist;
    unsigned int *ctr;
    unsigned long long *status;
    static size_t bytes(uint64_t ntiles) {
        return kMaxPasses * 256 * sizeof(uint32_t) + 256 + ntiles * 256 * sizeof(unsigned long long);
    }
    void carve(unsigned char *p) {
        hist = reinterpret_cast<uint32_t *>(p);
        ctr = reinterpret_cast<unsigned int *>(p + kMaxPasses * 256 * sizeof(uint32_t));
        status = reinterpret_cast<unsigned long long *>(p + kMaxPasses * 256 * sizeof(uint32_t) + 256);
    }
};

// Stable partition of n items by `passes` digits: pass p reads (ia, ib, ip)
// and writes (oa[p], ob[p], op[p]); the histogram of every pass comes from
// one read of the input.
template <typename K, bool HAS_B>
bt_status sweep_passes(const K *a, const K *b, uint64_t n, GroupKeyParams gp, int passes,
                       K *const *oa, K *const *ob, uint32_t *const *op, SweepWs ws,
                       cudaStream_t s) {
    const uint64_t ntiles = (n + kPTile - 1) / kPTile;
    BT_CUDA(cudaMemsetAsync(ws.hist, 0, kMaxPasses * 256 * sizeof(uint32_t) + 256, s));
    bt_status st = onesweep_smem_attr<K, HAS_B>();
    if (st != BT_OK) return st;
    count_launch();
    part_hist_all_kernel<K, HAS_B>
        <<<(unsigned)std::min<uint64_t>(ntiles, (uint64_t)sm_count() * 4), kPT, 0, s>>>(
            a, b, n, gp, passes, ws.hist);
    const K *ia = a, *ib = b;
    const uint32_t *ip = nullptr;
    for (int p = 0; p < passes; p++) {
        BT_CUDA(cudaMemsetAsync(ws.status, 0, ntiles * 256 * sizeof(unsigned long long), s));
        count_launch();
        part_onesweep_kernel<K, HAS_B><<<(unsigned)ntiles, kPT, scatter_smem<K, HAS_B>(), s>>>(
            ia, ib, ip, n, gp, p, ws.hist, ws.ctr + p, ws.status, oa[p], HAS_B ? ob[p] : nullptr,
            op[p]);
        BT_CUDA(cudaGetLastError());
        ia = oa[p];
        ib = HAS_B ? ob[p] : nullptr;
        ip = op[p];
    }
    return BT_OK;
}

template <typename K, bool HAS_B>
bt_status partition_impl(const bt_tree *t, int kind, const K *d_a, const K *d_b, uint64_t nq,
                         K *out_a, K *out_b, uint32_t *out_perm, cudaStream_t s) {
    GroupKeyParams gp;
    gp.kind = kind;
    const int kb = bitlen64(t->max_key);
    int dbits;
    if (kind == kPartPoint) {
        dbits = kPointGroupBits;
        gp.cbits = dbits;
    } else {
        dbits = kRangeGroupBits * 2;  // two coordinates
        gp.cbits = kRangeGroupBits;
    }
    gp.shift = std::max(0, kb - gp.cbits);
    const int passes = (dbits + 7) / 8;
    const uint64_t ntiles = (nq + kPTile - 1) / kPTile;
    if (ntiles * 256 >= (1ull << 32)) return fail(BT_ERR_INVALID_ARGUMENT, "batch too large");

    // One workspace: digit counts, scan scratch and, for two passes, one
    // intermediate copy of the payload.  (The look-back path of
    // sweep_passes was measured slower here -- one or two passes, 2^24
    // queries: 0.325 ms against 0.239 -- so grouping keeps tile histograms,
    // one scan and the scatter; the device sort, with four or eight passes
    // served by one histogram read, uses sweep_passes.)
    const uint64_t ncounts = ntiles * 256;
    const uint64_t scan_we = scan_ws_elems(ncounts);
    const size_t pp_bytes = passes > 1 ? nq * (sizeof(K) * (HAS_B ? 2 : 1) + sizeof(uint32_t)) + 512 : 0;
    const size_t cbytes = ((ncounts + scan_we) * sizeof(uint32_t) + 255) / 256 * 256;
    unsigned char *ws = nullptr;
    bt_status st = ws_alloc((void **)&ws, cbytes + pp_bytes, s);
    if (st != BT_OK) return st;
    uint32_t *counts = reinterpret_cast<uint32_t *>(ws);
    uint32_t *scan_ws = counts + ncounts;
    K *oa[2] = {out_a, out_a}, *ob[2] = {out_b, out_b};
    uint32_t *op[2] = {out_perm, out_perm};
    if (passes > 1) {  // pass 0 into the intermediate copy, pass 1 into the caller's arrays
        unsigned char *pp = ws + cbytes;
        oa[0] = reinterpret_cast<K *>(pp);
        pp += (nq * sizeof(K) + 255) / 256 * 256;
        if (HAS_B) {
            ob[0] = reinterpret_cast<K *>(pp);
            pp += (nq * sizeof(K) + 255) / 256 * 256;
        }
        op[0] = reinterpret_cast<uint32_t *>(pp);
    }
    if (passes > 2) st = fail(BT_ERR_INTERNAL, "partition supports at most two passes");
    if (st == BT_OK) st = scatter_smem_attr<K, HAS_B>();
    const K *ia = d_a, *ib = d_b;
    const uint32_t *ip = nullptr;
    for (int p = 0; p < passes && st == BT_OK; p++) {
        count_launch();
        part_hist_kernel<K, HAS_B><<<(unsigned)ntiles, kPT, 0, s>>>(ia, ib, nq, gp, p, counts, ntiles);
        st = scan_run<uint32_t>(counts, counts, ncounts, nullptr, scan_ws, s);
        if (st != BT_OK) break;
        count_launch();
        part_scatter_kernel<K, HAS_B><<<(unsigned)ntiles, kPT, scatter_smem<K, HAS_B>(), s>>>(
            ia, ib, ip, nq, gp, p, counts, ntiles, oa[p], ob[p], op[p]);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) st = cuda_fail(e, "partition kernels");
        ia = oa[p];
        ib = ob[p];
        ip = op[p];
    }
    ws_free(ws, s);
    return st;
}

template <typename V>
__global__ void gather_kernel(const V *__restrict__ in, const uint32_t *__restrict__ idx, uint64_t n,
                              V *__restrict__ out) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x)
        out[i] = in[idx[i]];
}

// LSD radix sort of keys carrying the input index: pass p partitions by
// byte p of the key (stable), so after the last pass the keys are sorted and
// equal keys keep their input order; then values are gathered by index.
template <typename K, typename V>
bt_status sort_pairs_impl(const K *d_keys, const V *d_vals, uint64_t n, K *out_keys, V *out_vals,
                          cudaStream_t s) {
    const int passes = (int)sizeof(K);
    const uint64_t ntiles = (n + kPTile - 1) / kPTile;
    const size_t sweep_bytes = (SweepWs::bytes(ntiles) + 255) / 256 * 256;
    const size_t kbytes = (n * sizeof(K) + 255) / 256 * 256;
    const size_t pbytes = (n * sizeof(uint32_t) + 255) / 256 * 256;
    unsigned char *ws = nullptr;
    bt_status st = ws_alloc((void **)&ws, sweep_bytes + 2 * (kbytes + pbytes), s);
    if (st != BT_OK) return st;
    SweepWs sw;
    sw.carve(ws);
    unsigned char *pp = ws + sweep_bytes;
    K *tk[2] = {reinterpret_cast<K *>(pp), reinterpret_cast<K *>(pp + kbytes + pbytes)};
    uint32_t *tp[2] = {reinterpret_cast<uint32_t *>(pp + kbytes),
                       reinterpret_cast<uint32_t *>(pp + 2 * kbytes + pbytes)};
    K *ok[kMaxPasses];
    uint32_t *op[kMaxPasses];
    for (int p = 0; p < passes; p++) {
        ok[p] = p == passes - 1 ? out_keys : tk[p & 1];
        op[p] = tp[p & 1];
    }
    GroupKeyParams gp;
    gp.kind = kPartRadix;
    gp.cbits = 8;
    gp.shift = 0;
    st = sweep_passes<K, false>(d_keys, nullptr, n, gp, passes, ok, nullptr, op, sw, s);
    if (st == BT_OK) {
        count_launch();
        gather_kernel<V><<<(unsigned)std::min<uint64_t>((n + 255) / 256, (uint64_t)sm_count() * 16), 256, 0, s>>>(
            d_vals, op[passes - 1], n, out_vals);
        cudaError_t e = cudaGetLastError();
        if (e != cudaSuccess) st = cuda_fail(e, "value gather");
    }
    ws_free(ws, s);
    return st;
}

bt_status order_u16_impl(const uint32_t *d_keys, uint64_t n, uint32_t *d_perm, cudaStream_t s) {
    const uint64_t ntiles = (n + kPTile - 1) / kPTile;
    const size_t sweep_bytes = (SweepWs::bytes(ntiles) + 255) / 256 * 256;
    const size_t b = (n * sizeof(uint32_t) + 255) / 256 * 256;
    unsigned char *ws = nullptr;
    bt_status st = ws_alloc((void **)&ws, sweep_bytes + 3 * b, s);
    if (st != BT_OK) return st;
    SweepWs sw;
    sw.carve(ws);
    uint32_t *k0 = reinterpret_cast<uint32_t *>(ws + sweep_bytes);
    uint32_t *k1 = reinterpret_cast<uint32_t *>(ws + sweep_bytes + b);
    uint32_t *p0 = reinterpret_cast<uint32_t *>(ws + sweep_bytes + 2 * b);
    uint32_t *ok[2] = {k0, k1};
    uint32_t *op[2] = {p0, d_perm};
    GroupKeyParams gp;
    gp.kind = kPartRadix;
    gp.cbits = 8;
    gp.shift = 0;
    st = sweep_passes<uint32_t, false>(d_keys, nullptr, n, gp, 2, ok, nullptr, op, sw, s);
    ws_free(ws, s);
    return st;
}

// Single-pass point partition into caller-provided memory (no allocation):
// counts and scan scratch come from `ws` (partition_ws_bytes bytes).
template <typename K>
bt_status partition_point_prealloc(const bt_tree *t, const K *d_q, uint64_t nq, K *out_q,
                                   uint32_t *out_perm, unsigned char *ws, cudaStream_t s) {
    GroupKeyParams gp;
    gp.kind = kPartPoint;
    gp.cbits = kPointGroupBits;
    gp.shift = std::max(0, bitlen64(t->max_key) - gp.cbits);
    const uint64_t ntiles = (nq + kPTile - 1) / kPTile;
    const uint64_t ncounts = ntiles * 256;
    uint32_t *counts = reinterpret_cast<uint32_t *>(ws);
    uint32_t *scan_ws = counts + ncounts;
    const size_t smem = scatter_smem<K, false>();
    auto scat = part_scatter_kernel<K, false>;
    bt_status sa = scatter_smem_attr<K, false>();
    if (sa != BT_OK) return sa;
    count_launch();
    part_hist_kernel<K, false><<<(unsigned)ntiles, kPT, 0, s>>>(d_q, nullptr, nq, gp, 0, counts, ntiles);
    bt_status st = scan_run<uint32_t>(counts, counts, ncounts, nullptr, scan_ws, s);
    if (st != BT_OK) return st;
    count_launch();
    scat<<<(unsigned)ntiles, kPT, smem, s>>>(d_q, nullptr, nullptr, nq, gp, 0, counts, ntiles, out_q,
                                             nullptr, out_perm);
    BT_CUDA(cudaGetLastError());
    return BT_OK;
}

// --------------------------------------------------------- range fill ----

// One warp per query: ids[off .. off+cnt) = values of positions lb .. lb+cnt
// (read from the leaf blocks, S values per block).
template <typename K, typename V>
__global__ void __launch_bounds__(256)
range_fill_kernel(const unsigned char *__restrict__ leaves, const uint64_t *__restrict__ lb,
                  const uint64_t *__restrict__ cnt, const uint64_t *__restrict__ off, uint64_t nq,
                  V *__restrict__ ids) {
    using LG = LeafGeom<K, V>;
    const int lane = threadIdx.x & 31;
    const uint64_t warp = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5;
    const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t i = warp; i < nq; i += nw) {
        const uint64_t c = cnt[i], l = lb[i], o = off[i];
        for (uint64_t k = lane; k < c; k += 32) {
            const uint64_t p = l + k;
            ids[o + k] = reinterpret_cast<const V *>(leaves + (p / LG::S) * LG::BS +
                                                     kSectorBytes)[p % LG::S];
        }
    }
}

// Sorts each query's ID segment when values do not ascend with keys, in
// three tiers by length.  Up to kWarpSortCap values: one warp sorts the
// segment in registers (warp_sort_small, a bitonic network) and writes it
// back.  Up to kSortCap: one CTA per segment, bitonic network in shared
// memory; the warp pass lists these segments.  Longer: listed afterwards and
// sorted one CTA each by a bitonic network over a padded copy in global
// memory.
constexpr int kSortCap = 4096;
constexpr unsigned int kMedListCap = 1u << 16;
constexpr int kWSortThreads = 256;

// stat[0]: segments of kWarpSortCap < c <= kSortCap (listed in med_list up
// to kMedListCap); stat[1]: set if a segment is longer than kSortCap.  With
// skip_small, segments of up to kWarpSortCap values are already sorted.
template <typename V>
__global__ void __launch_bounds__(kWSortThreads)
warp_segment_sort_kernel(const uint64_t *__restrict__ cnt, const uint64_t *__restrict__ off,
                         uint64_t nq, V *__restrict__ ids, unsigned int *__restrict__ stat,
                         uint64_t *__restrict__ med_list, bool skip_small) {
    const int lane = threadIdx.x & 31;
    const uint64_t nw = ((uint64_t)gridDim.x * blockDim.x) >> 5;
    for (uint64_t i = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5; i < nq; i += nw) {
        const uint64_t c = cnt[i];
        if (c < 2) continue;
        if (c > (uint64_t)kWarpSortCap) {
            if (lane == 0) {
                if (c > (uint64_t)kSortCap) {
                    atomicOr(&stat[1], 1u);
                } else {
                    const unsigned int k = atomicAdd(&stat[0], 1u);
                    if (k < kMedListCap) med_list[k] = i;
                }
            }
            continue;
        }
        if (skip_small) continue;
        V *seg = ids + off[i];
        warp_sort_small<V>(seg, seg, (uint32_t)c, lane);
    }
}

// One CTA per medium segment: the listed ones (list != null, n entries), or
// every segment with kWarpSortCap < c <= kSortCap (list == null, n = nq).
template <typename V>
__global__ void __launch_bounds__(512)
segment_sort_kernel(const uint64_t *__restrict__ cnt, const uint64_t *__restrict__ off,
                    const uint64_t *__restrict__ list, uint64_t n, V *__restrict__ ids) {
    __shared__ V buf[kSortCap];
    for (uint64_t li = blockIdx.x; li < n; li += gridDim.x) {
        const uint64_t i = list ? list[li] : li;
        const uint64_t c = cnt[i];
        if (c <= (uint64_t)kWarpSortCap || c > (uint64_t)kSortCap) continue;
        uint32_t p2 = 1;
        while (p2 < c) p2 <<= 1;
        V *seg = ids + off[i];
        for (uint32_t k = threadIdx.x; k < p2; k += blockDim.x) buf[k] = k < c ? seg[k] : key_max<V>();
        __syncthreads();
        for (uint32_t size = 2; size <= p2; size <<= 1) {
            for (uint32_t stride = size >> 1; stride > 0; stride >>= 1) {
                for (uint32_t k = threadIdx.x; k < p2; k += blockDim.x) {
                    const uint32_t partner = k ^ stride;
                    if (partner > k) {
                        const bool asc = (k & size) == 0;
                        const V x = buf[k], y = buf[partner];
                        if ((x > y) == asc) {
                            buf[k] = y;
                            buf[partner] = x;
                        }
                    }
                }
                __syncthreads();
            }
        }
        for (uint32_t k = threadIdx.x; k < c; k += blockDim.x) seg[k] = buf[k];
        __syncthreads();
    }
}

// Segments longer than kSortCap: list them (index, offset, count).
__global__ void list_long_segments(const uint64_t *__restrict__ cnt, const uint64_t *__restrict__ off,
                                   uint64_t nq, unsigned int *__restrict__ n_long,
                                   uint64_t *__restrict__ list, unsigned int max_list) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < nq;
         i += (uint64_t)gridDim.x * blockDim.x) {
        if (cnt[i] > (uint64_t)kSortCap) {
            const unsigned int k = atomicAdd(n_long, 1u);
            if (k < max_list) {
                list[2 * k] = off[i];
                list[2 * k + 1] = cnt[i];
            }
        }
    }
}

// One CTA sorts one long segment: copy into a power-of-two scratch padded
// with all-ones, bitonic network in global (L2-resident) memory, copy back.
template <typename V>
__global__ void __launch_bounds__(1024)
long_segment_sort(V *__restrict__ ids, uint64_t off, uint64_t c, V *__restrict__ tmp, uint64_t p2) {
    for (uint64_t k = threadIdx.x; k < p2; k += blockDim.x) tmp[k] = k < c ? ids[off + k] : key_max<V>();
    __syncthreads();
    for (uint64_t size = 2; size <= p2; size <<= 1) {
        for (uint64_t stride = size >> 1; stride > 0; stride >>= 1) {
            for (uint64_t k = threadIdx.x; k < p2; k += blockDim.x) {
                const uint64_t partner = k ^ stride;
                if (partner > k) {
                    const bool asc = (k & size) == 0;
                    const V x = tmp[k], y = tmp[partner];
                    if ((x > y) == asc) {
                        tmp[k] = y;
                        tmp[partner] = x;
                    }
                }
            }
            __syncthreads();
        }
    }
    for (uint64_t k = threadIdx.x; k < c; k += blockDim.x) ids[off + k] = tmp[k];
}

}  // namespace

bt_status launch_partition(const bt_tree *t, int kind, const void *d_a, const void *d_b,
                           uint64_t nq, void *d_out_a, void *d_out_b, uint32_t *d_perm,
                           cudaStream_t s) {
    if (nq == 0) return BT_OK;
    if (nq >= (1ull << 32)) return fail(BT_ERR_INVALID_ARGUMENT, "grouped batches need nq < 2^32");
    const bool hb = kind != kPartPoint;
    if (t->key_bytes == 4)
        return hb ? partition_impl<uint32_t, true>(t, kind, (const uint32_t *)d_a,
                                                   (const uint32_t *)d_b, nq, (uint32_t *)d_out_a,
                                                   (uint32_t *)d_out_b, d_perm, s)
                  : partition_impl<uint32_t, false>(t, kind, (const uint32_t *)d_a, nullptr, nq,
                                                    (uint32_t *)d_out_a, nullptr, d_perm, s);
    return hb ? partition_impl<uint64_t, true>(t, kind, (const uint64_t *)d_a,
                                               (const uint64_t *)d_b, nq, (uint64_t *)d_out_a,
                                               (uint64_t *)d_out_b, d_perm, s)
              : partition_impl<uint64_t, false>(t, kind, (const uint64_t *)d_a, nullptr, nq,
                                                (uint64_t *)d_out_a, nullptr, d_perm, s);
}

bt_status launch_sort_pairs(int key_bytes, int value_bytes, const void *d_keys, const void *d_vals,
                            uint64_t n, void *out_keys, void *out_vals, cudaStream_t s) {
    if (n == 0) return BT_OK;
    if (n >= (1ull << 32)) return fail(BT_ERR_INVALID_ARGUMENT, "sort needs fewer than 2^32 pairs");
    if (key_bytes == 4)
        return value_bytes == 4
                   ? sort_pairs_impl<uint32_t, uint32_t>((const uint32_t *)d_keys, (const uint32_t *)d_vals, n,
                                                         (uint32_t *)out_keys, (uint32_t *)out_vals, s)
                   : sort_pairs_impl<uint32_t, uint64_t>((const uint32_t *)d_keys, (const uint64_t *)d_vals, n,
                                                         (uint32_t *)out_keys, (uint64_t *)out_vals, s);
    return value_bytes == 4
               ? sort_pairs_impl<uint64_t, uint32_t>((const uint64_t *)d_keys, (const uint32_t *)d_vals, n,
                                                     (uint64_t *)out_keys, (uint32_t *)out_vals, s)
               : sort_pairs_impl<uint64_t, uint64_t>((const uint64_t *)d_keys, (const uint64_t *)d_vals, n,
                                                     (uint64_t *)out_keys, (uint64_t *)out_vals, s);
}

bt_status launch_order_u16(const uint32_t *d_keys, uint64_t n, uint32_t *d_perm, cudaStream_t s) {
    if (n == 0) return BT_OK;
    if (n >= (1ull << 32)) return fail(BT_ERR_INVALID_ARGUMENT, "ordering needs n < 2^32");
    return order_u16_impl(d_keys, n, d_perm, s);
}

size_t partition_point_ws_bytes(uint64_t nq) {
    const uint64_t ncounts = ((nq + kPTile - 1) / kPTile) * 256;
    return (ncounts + scan_ws_elems(ncounts)) * sizeof(uint32_t);
}

bt_status launch_partition_point_prealloc(const bt_tree *t, const void *d_q, uint64_t nq,
                                          void *out_q, uint32_t *out_perm, void *ws,
                                          cudaStream_t s) {
    if (nq == 0) return BT_OK;
    if (t->key_bytes == 4)
        return partition_point_prealloc<uint32_t>(t, (const uint32_t *)d_q, nq, (uint32_t *)out_q,
                                                  out_perm, (unsigned char *)ws, s);
    return partition_point_prealloc<uint64_t>(t, (const uint64_t *)d_q, nq, (uint64_t *)out_q,
                                              out_perm, (unsigned char *)ws, s);
}

bt_status launch_scan_u64(const uint64_t *d_in, uint64_t *d_out, uint64_t n, uint64_t *d_total,
                          cudaStream_t s) {
    return scan_impl<uint64_t>(d_in, d_out, n, d_total, s);
}

bt_status launch_range_fill(const bt_tree *t, const uint64_t *d_lb, const uint64_t *d_counts,
                            const uint64_t *d_offsets, uint64_t nq, void *d_ids, cudaStream_t s) {
    if (nq == 0 || t->n == 0) return BT_OK;
    const unsigned grid = (unsigned)std::min<uint64_t>((nq + 7) / 8, (uint64_t)sm_count() * 8);
    count_launch();
    const unsigned char *lv = (const unsigned char *)t->d_leaves;
    if (t->key_bytes == 4 && t->val_bytes == 4)
        range_fill_kernel<uint32_t, uint32_t><<<grid, 256, 0, s>>>(lv, d_lb, d_counts, d_offsets,
                                                                   nq, (uint32_t *)d_ids);
    else if (t->key_bytes == 4)
        range_fill_kernel<uint32_t, uint64_t><<<grid, 256, 0, s>>>(lv, d_lb, d_counts, d_offsets,
                                                                   nq, (uint64_t *)d_ids);
    else if (t->val_bytes == 4)
        range_fill_kernel<uint64_t, uint32_t><<<grid, 256, 0, s>>>(lv, d_lb, d_counts, d_offsets,
                                                                   nq, (uint32_t *)d_ids);
    else
        range_fill_kernel<uint64_t, uint64_t><<<grid, 256, 0, s>>>(lv, d_lb, d_counts, d_offsets,
                                                                   nq, (uint64_t *)d_ids);
    BT_CUDA(cudaGetLastError());
    if (t->values_sorted) return BT_OK;
    return launch_segment_sort(t, d_counts, d_offsets, nq, d_ids, s);
}

bt_status launch_segment_sort(const bt_tree *t, const uint64_t *d_counts, const uint64_t *d_offsets,
                              uint64_t nq, void *d_ids, cudaStream_t s, bool small_sorted) {
    if (nq == 0) return BT_OK;
    WsGuard g_stat(s), g_med(s);
    bt_status st = g_stat.alloc(2 * sizeof(unsigned int));
    if (st == BT_OK) st = g_med.alloc(kMedListCap * sizeof(uint64_t));
    if (st != BT_OK) return st;
    unsigned int *stat = g_stat.as<unsigned int>();
    uint64_t *med = g_med.as<uint64_t>();
    BT_CUDA(cudaMemsetAsync(stat, 0, 2 * sizeof(unsigned int), s));
    const unsigned gw = (unsigned)std::min<uint64_t>((nq + kWSortThreads / 32 - 1) / (kWSortThreads / 32),
                                                     (uint64_t)sm_count() * 8);
    count_launch();
    if (t->val_bytes == 4)
        warp_segment_sort_kernel<uint32_t><<<gw, kWSortThreads, 0, s>>>(d_counts, d_offsets, nq,
                                                                        (uint32_t *)d_ids, stat, med,
                                                                        small_sorted);
    else
        warp_segment_sort_kernel<uint64_t><<<gw, kWSortThreads, 0, s>>>(d_counts, d_offsets, nq,
                                                                        (uint64_t *)d_ids, stat, med,
                                                                        small_sorted);
    unsigned int h[2] = {0, 0};
    BT_CUDA(cudaMemcpyAsync(h, stat, sizeof(h), cudaMemcpyDeviceToHost, s));
    BT_CUDA(cudaStreamSynchronize(s));
    if (h[0] > 0) {
        // medium segments: the list, or (if it overflowed) every segment
        const bool listed = h[0] <= kMedListCap;
        const uint64_t n = listed ? h[0] : nq;
        const unsigned g2 = (unsigned)std::min<uint64_t>(n, (uint64_t)sm_count() * 4);
        count_launch();
        if (t->val_bytes == 4)
            segment_sort_kernel<uint32_t><<<g2, 512, 0, s>>>(d_counts, d_offsets, listed ? med : nullptr,
                                                             n, (uint32_t *)d_ids);
        else
            segment_sort_kernel<uint64_t><<<g2, 512, 0, s>>>(d_counts, d_offsets, listed ? med : nullptr,
                                                             n, (uint64_t *)d_ids);
        BT_CUDA(cudaGetLastError());
    }
    if (!h[1]) return BT_OK;
    // some segments exceed the shared-memory sort: list and sort them one CTA each
    const unsigned int max_list = 1u << 16;
    WsGuard g_list(s);
    st = g_list.alloc(2 * (size_t)max_list * sizeof(uint64_t));
    if (st != BT_OK) return st;
    unsigned int *flag = stat;
    uint64_t *d_list = g_list.as<uint64_t>();
    BT_CUDA(cudaMemsetAsync(flag, 0, sizeof(unsigned int), s));
    count_launch();
    list_long_segments<<<(unsigned)std::min<uint64_t>((nq + 255) / 256, 4096), 256, 0, s>>>(
        d_counts, d_offsets, nq, flag, d_list, max_list);
    unsigned int n_long = 0;
    BT_CUDA(cudaMemcpyAsync(&n_long, flag, sizeof(n_long), cudaMemcpyDeviceToHost, s));
    BT_CUDA(cudaStreamSynchronize(s));
    if (n_long > max_list)
        return fail(BT_ERR_NOT_SUPPORTED, "more than 65536 result sets exceed 4096 unsorted values");
    std::vector<uint64_t> list(2 * (size_t)n_long);
    BT_CUDA(cudaMemcpyAsync(list.data(), d_list, list.size() * sizeof(uint64_t),
                            cudaMemcpyDeviceToHost, s));
    BT_CUDA(cudaStreamSynchronize(s));
    const size_t vb = (size_t)t->val_bytes;
    for (unsigned int k = 0; k < n_long && st == BT_OK; k++) {
        const uint64_t off = list[2 * k], c = list[2 * k + 1];
        uint64_t p2 = 1;
        while (p2 < c) p2 <<= 1;
        WsGuard g_tmp(s);
        st = g_tmp.alloc(p2 * vb);
        if (st != BT_OK) break;
        count_launch();
        if (vb == 4)
            long_segment_sort<uint32_t><<<1, 1024, 0, s>>>((uint32_t *)d_ids, off, c, g_tmp.as<uint32_t>(), p2);
        else
            long_segment_sort<uint64_t><<<1, 1024, 0, s>>>((uint64_t *)d_ids, off, c, g_tmp.as<uint64_t>(), p2);
    }
    BT_CUDA(cudaGetLastError());
    return st;
}

}  // namespace bt

extern "C" {

uint64_t bt_partition_lookback_timeouts(void) {
    unsigned int v = 0;
    if (cudaMemcpyFromSymbol(&v, bt::g_lookback_timeouts, sizeof(v)) != cudaSuccess) return ~0ull;
    return v;
}

}  // extern "C"
