// Memory-system probes for the benchmark (lib/libbt_probe.so).
//
// A measurement aid only: no search path uses this library, and the engine
// (lib/libbtree_b200.so) does not link it.  bench.py loads it to set the
// search kernels against what the GPU sustains for their access shapes.
//
//   btp_measure_gather  random reads of 32-, 64- or 128-byte blocks (16-byte
//                       lanes, L1 bypassed) over a region: the ceiling of a
//                       kernel that makes one random DRAM read per query.
//   btp_measure_chain   per query, 1 or 2 random 128-byte line reads from an
//                       L2-sized array (the L2-resident part of an index;
//                       sizes are rounded down to powers of two),
//                       then one random block read from a large region whose
//                       address depends on the loaded line (the leaf read).
//                       Shows how the random DRAM rate holds up while a given
//                       footprint of index lines is read from L2 beside it.
//   btp_measure_hops    per query, `hops` DEPENDENT random 128-byte line reads
//                       from an L2-sized array (each address depends on the
//                       line before), then one dependent random 128-byte read
//                       from a large region, in one of three forms: a lane
//                       per query with 32-byte register loads, a lane pair
//                       per query (64 bytes per lane), or a lane per query
//                       whose lines arrive in its own shared-memory slot by
//                       bulk copies (cp.async.bulk, completing on a per-lane
//                       mbarrier; no multicast), a lane quad per query, or
//                       lane pairs for the lines and quads for the last read.
//
// All functions allocate their own buffers, flush L2 with a 512 MiB write
// between passes and return the best of three timed passes.  The extern "C"
// declarations are below; they are not part of the engine's C ABI.
#include <cuda_runtime.h>
#include <stdint.h>

#include <algorithm>
#include <cstdio>

namespace {

__device__ __forceinline__ uint64_t splitmix64(uint64_t x) {
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

__device__ __forceinline__ uint4 ld_nc_na(const void *p) {
    uint4 x;
    asm volatile("ld.global.nc.L1::no_allocate.v4.b32 {%0,%1,%2,%3}, [%4];"
                 : "=r"(x.x), "=r"(x.y), "=r"(x.z), "=r"(x.w)
                 : "l"(p));
    return x;
}

__device__ __forceinline__ uint4 ld_evict_first(const void *p) {
    uint64_t pol;
    asm("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol));
    uint4 x;
    asm volatile("ld.global.nc.L1::no_allocate.L2::cache_hint.v4.b32 {%0,%1,%2,%3}, [%4], %5;"
                 : "=r"(x.x), "=r"(x.y), "=r"(x.z), "=r"(x.w)
                 : "l"(p), "l"(pol));
    return x;
}

__global__ void index_kernel(uint32_t *idx, uint64_t n, uint64_t nblocks, uint64_t seed) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x)
        idx[i] = (uint32_t)(splitmix64(seed + i) % nblocks);
}

template <int G>
__global__ void __launch_bounds__(256)
gather_kernel(const unsigned char *__restrict__ buf, const uint32_t *__restrict__ idx, uint64_t n,
              int bshift, uint32_t *__restrict__ sink) {
    const uint64_t tid = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x / G;
    const int gl = (int)(tid % G);
    uint32_t acc = 0;
    for (uint64_t i = tid / G; i < n; i += stride) {
        const uint4 x = ld_nc_na(buf + ((uint64_t)idx[i] << bshift) + gl * 16);
        acc ^= x.x ^ x.y ^ x.z ^ x.w;
    }
    if (acc == 0x9E3779B9u) sink[0] = acc;  // keeps the loads live
}

// 8 lanes per query, I queries in flight per 8-lane group.  Lane l reads
// bytes 16l..16l+15 of each 128-byte index line; the leaf block index mixes
// in the loaded words (masked by `mask`, zero at run time) so the leaf read
// cannot issue before the line arrives.  Leaf reads: LB = 64 (lanes 0-3) or
// 128 bytes (all 8 lanes), evict-first in L2 like the search kernels' leaves.
template <int CL, int LB, int I>
__global__ void __launch_bounds__(256)
chain_kernel(const unsigned char *__restrict__ lines, uint64_t nlines,
             const unsigned char *__restrict__ leaves, uint64_t nblocks, uint64_t n,
             uint32_t mask, uint64_t seed, uint32_t *__restrict__ sink) {
    const uint64_t tid = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    const uint64_t groups = (uint64_t)gridDim.x * blockDim.x / 8;
    const int gl = (int)(tid % 8);
    uint32_t acc = 0;
    for (uint64_t i0 = (tid / 8) * I; i0 < n; i0 += groups * I) {
        uint32_t w[I];
#pragma unroll
        for (int s = 0; s < I; s++) {
            const uint64_t h = splitmix64(seed + i0 + s);
            w[s] = 0;
            if (CL > 0 && nlines) {
                const uint64_t li = h & (nlines - 1);
#pragma unroll
                for (int c = 0; c < CL; c++) {
                    const uint64_t l = li + c < nlines ? li + c : li;
                    const uint4 x = ld_nc_na(lines + l * 128 + gl * 16);
                    w[s] ^= x.x ^ x.y ^ x.z ^ x.w;
                }
            }
        }
#pragma unroll
        for (int s = 0; s < I; s++) {
            const uint64_t h2 = splitmix64(~(seed + i0 + s));
            const uint64_t b = (h2 ^ (uint64_t)(w[s] & mask)) & (nblocks - 1);
            if (LB == 128 || gl < LB / 16) {
                const uint4 y = ld_evict_first(leaves + b * LB + gl * 16);
                acc ^= y.x ^ y.y ^ y.z ^ y.w;
            }
        }
    }
    if (acc == 0x9E3779B9u) sink[0] = acc;
}

__device__ __forceinline__ void ld_line32(const void *p, uint32_t (&w)[8], uint64_t pol) {
    asm volatile(
        "ld.global.nc.L1::no_allocate.L2::cache_hint.v8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8], %9;"
        : "=r"(w[0]), "=r"(w[1]), "=r"(w[2]), "=r"(w[3]), "=r"(w[4]), "=r"(w[5]), "=r"(w[6]),
          "=r"(w[7])
        : "l"(p), "l"(pol));
}

__device__ __forceinline__ uint32_t xor8(const uint32_t (&w)[8]) {
    return w[0] ^ w[1] ^ w[2] ^ w[3] ^ w[4] ^ w[5] ^ w[6] ^ w[7];
}

// XOR of `words` 32-byte pieces at p (registers, one lane).
__device__ __forceinline__ uint32_t load_xor(const unsigned char *p, int pieces, uint64_t pol) {
    uint32_t acc = 0;
    for (int c = 0; c < pieces; c++) {
        uint32_t w[8];
        ld_line32(p + 32 * c, w, pol);
        acc ^= xor8(w);
    }
    return acc;
}

constexpr uint32_t kHopWaits = 1u << 20;

// Bounded wait for phase `par` of the mbarrier at shared address b; false if
// it did not complete within kHopWaits polls.
__device__ __forceinline__ bool bar_wait(uint32_t b, uint32_t par) {
    uint32_t done = 0;
    for (uint32_t it = 0; it < kHopWaits && !done; it++)
        asm volatile(
            "{ .reg .pred p; mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2; selp.u32 %0, 1, 0, p; }"
            : "=r"(done)
            : "r"(b), "r"(par)
            : "memory");
    return done != 0;
}

// One 128-byte bulk copy global -> this lane's slot, completing on its mbarrier.
__device__ __forceinline__ void bulk128(uint32_t slot, const void *src, uint32_t b) {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], 128;" ::"r"(b) : "memory");
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], 128, [%2];" ::"r"(slot),
        "l"(src), "r"(b)
        : "memory");
}

// MODE 0: a lane per query, register loads (4 x 32 bytes per line).
// MODE 1: a lane pair per query, 64 bytes per lane.
// MODE 2: a lane per query, bulk copies into a 128-byte shared slot per lane.
// MODE 3: a lane quad per query, 32 bytes per lane.
// MODE 4: lane pairs for the line hops, lane quads for the final read.
// Line addresses depend on the previous line's words (masked by `mask`, zero
// at run time), so the reads of a query form a chain of hops + 1.
template <int MODE, int HOPS>
__global__ void __launch_bounds__(256)
hop_kernel(const unsigned char *__restrict__ lines, uint64_t nlines,
           const unsigned char *__restrict__ leaves, uint64_t nunits, uint64_t n, uint32_t mask,
           uint64_t seed, uint32_t *__restrict__ sink) {
    uint64_t pol_l, pol_f;
    asm("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(pol_l));
    asm("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(pol_f));
    const uint64_t tid = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    const uint64_t nth = (uint64_t)gridDim.x * blockDim.x;
    uint32_t acc = 0;
    if constexpr (MODE == 2) {
        extern __shared__ __align__(128) unsigned char slots[];
        __shared__ __align__(8) unsigned long long bars[256];
        const uint32_t b = (uint32_t)__cvta_generic_to_shared(&bars[threadIdx.x]);
        const uint32_t slot = (uint32_t)__cvta_generic_to_shared(slots + threadIdx.x * 128);
        const uint4 *sp = reinterpret_cast<const uint4 *>(slots + threadIdx.x * 128);
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(b) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        __syncwarp();
        uint32_t par = 0;
        for (uint64_t i = tid; i < n; i += nth) {
            const uint64_t h = splitmix64(seed + i);
            uint64_t li = h & (nlines - 1);
            uint32_t w = 0;
            for (int hop = 0; hop <= HOPS; hop++) {
                const unsigned char *src =
                    hop < HOPS ? lines + li * 128
                               : leaves + ((splitmix64(~(seed + i)) ^ (w & mask)) & (nunits - 1)) * 128;
                bulk128(slot, src, b);
                if (!bar_wait(b, par)) {  // record, wait out the copy, stop
                    atomicOr(sink + 1, 1u);
                    bar_wait(b, par);
                    return;
                }
                par ^= 1;
                const uint4 x = sp[threadIdx.x & 7];
                w = x.x ^ x.y ^ x.z ^ x.w;
                if (hop < HOPS) li = (splitmix64(h + hop + 1) ^ (w & mask)) & (nlines - 1);
            }
            acc ^= w;
        }
    } else if constexpr (MODE == 4) {
        // lane pairs for the hops; the final read by lane quads (a quad per
        // query, 32 bytes per lane), the pair's address moved by shuffles
        const int part = (int)(threadIdx.x & 1);
        const int lane = (int)(threadIdx.x & 31);
        const uint64_t warp = tid >> 5, nwarps = nth >> 5;
        for (uint64_t base = warp * 16; base < n; base += nwarps * 16) {
            const uint64_t i0 = base + (lane >> 1);
            const bool live = i0 < n;
            const uint64_t h = splitmix64(seed + i0);
            uint64_t li = h & (nlines - 1);
            uint32_t w = 0;
            for (int hop = 0; hop < HOPS; hop++) {
                if (live) w = load_xor(lines + li * 128 + part * 64, 2, pol_l);
                w ^= __shfl_xor_sync(0xffffffffu, w, 1);
                li = (splitmix64(h + hop + 1) ^ (w & mask)) & (nlines - 1);
            }
            const uint64_t leaf = (splitmix64(~(seed + i0)) ^ (w & mask)) & (nunits - 1);
            for (int sub = 0; sub < 2; sub++) {
                const int src = 2 * (8 * sub + (lane >> 2));
                const uint64_t lf = ((uint64_t)__shfl_sync(0xffffffffu, (uint32_t)(leaf >> 32), src) << 32) |
                                    __shfl_sync(0xffffffffu, (uint32_t)leaf, src);
                if (base + 8 * sub + (lane >> 2) < n) {
                    uint32_t y[8];
                    ld_line32(leaves + lf * 128 + (lane & 3) * 32, y, pol_f);
                    acc ^= xor8(y);
                }
            }
        }
    } else {
        const int per = MODE == 0 ? 1 : MODE == 1 ? 2 : 4;  // lanes per query
        const int part = (int)(threadIdx.x & (per - 1));
        const int pieces = MODE == 0 ? 4 : MODE == 1 ? 2 : 1;
        for (uint64_t i0 = tid / per; i0 < n; i0 += nth / per) {
            const uint64_t h = splitmix64(seed + i0);
            uint64_t li = h & (nlines - 1);
            uint32_t w = 0;
            for (int hop = 0; hop <= HOPS; hop++) {
                const unsigned char *src =
                    hop < HOPS ? lines + li * 128
                               : leaves + ((splitmix64(~(seed + i0)) ^ (w & mask)) & (nunits - 1)) * 128;
                w = load_xor(src + part * (128 / per), pieces, hop < HOPS ? pol_l : pol_f);
                if (MODE == 1) w ^= __shfl_xor_sync(0x3u << (threadIdx.x & 30), w, 1);  // the group loops alike
                if (MODE == 3) {
                    const unsigned qm = 0xFu << (threadIdx.x & 28);
                    w ^= __shfl_xor_sync(qm, w, 1);
                    w ^= __shfl_xor_sync(qm, w, 2);
                }
                if (hop < HOPS) li = (splitmix64(h + hop + 1) ^ (w & mask)) & (nlines - 1);
            }
            acc ^= w;
        }
    }
    if (acc == 0x9E3779B9u) sink[0] = acc;
}

int sm_count() {
    int dev = 0, n = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
    return n > 0 ? n : 1;
}

struct Bufs {
    unsigned char *a = nullptr, *b = nullptr, *flush = nullptr;
    uint32_t *idx = nullptr, *sink = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    ~Bufs() {
        if (e0) cudaEventDestroy(e0);
        if (e1) cudaEventDestroy(e1);
        cudaFree(a);
        cudaFree(b);
        cudaFree(flush);
        cudaFree(idx);
        cudaFree(sink);
    }
};

constexpr size_t kFlushBytes = 512ull << 20;

// Best of three timed passes of launch(), each after an L2 flush; one
// untimed pass first (warm_after_flush: also one untimed pass after each
// flush, so an L2-sized array is resident when the timed pass starts).
template <typename F>
cudaError_t time_best(Bufs &b, F launch, bool warm_after_flush, float *best) {
    cudaError_t e = cudaEventCreate(&b.e0);
    if (e == cudaSuccess) e = cudaEventCreate(&b.e1);
    *best = 0;
    for (int rep = 0; rep < 4 && e == cudaSuccess; rep++) {
        e = cudaMemsetAsync(b.flush, rep, kFlushBytes, 0);
        if (e != cudaSuccess) break;
        if (warm_after_flush) launch();
        cudaEventRecord(b.e0, 0);
        launch();
        cudaEventRecord(b.e1, 0);
        e = cudaEventSynchronize(b.e1);
        float ms = 0;
        if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, b.e0, b.e1);
        if (e == cudaSuccess && rep > 0 && (*best == 0 || ms < *best)) *best = ms;
    }
    if (e == cudaSuccess) e = cudaGetLastError();
    return e;
}

thread_local char g_err[256];

int fail(const char *what, cudaError_t e) {
    snprintf(g_err, sizeof(g_err), "%s: %s", what, e == cudaSuccess ? "" : cudaGetErrorString(e));
    return 1;
}

}  // namespace

extern "C" {

// Detail of the last failure of a probe call on this thread.
__attribute__((visibility("default"))) const char *btp_last_error(void) { return g_err; }

// Random block reads per second (blocks of 32, 64 or 128 bytes, uniformly
// random over region_bytes).  Returns 0 on success.
__attribute__((visibility("default"))) int btp_measure_gather(uint64_t region_bytes,
                                                              uint64_t n_reads,
                                                              uint32_t block_bytes,
                                                              double *reads_per_s) {
    if (!reads_per_s) return fail("reads_per_s is NULL", cudaSuccess);
    *reads_per_s = 0;
    if (block_bytes != 32 && block_bytes != 64 && block_bytes != 128)
        return fail("block_bytes must be 32, 64 or 128", cudaSuccess);
    const uint64_t nblocks = region_bytes / block_bytes;
    if (nblocks == 0 || nblocks > (1ull << 32) || n_reads == 0 || n_reads > (1ull << 30))
        return fail("region or read count out of range", cudaSuccess);
    Bufs b;
    cudaError_t e = cudaMalloc(&b.a, nblocks * block_bytes);
    if (e == cudaSuccess) e = cudaMalloc(&b.idx, n_reads * sizeof(uint32_t));
    if (e == cudaSuccess) e = cudaMalloc(&b.sink, sizeof(uint32_t));
    if (e == cudaSuccess) e = cudaMalloc(&b.flush, kFlushBytes);
    if (e == cudaSuccess) e = cudaMemset(b.a, 1, nblocks * block_bytes);
    if (e != cudaSuccess) return fail("allocation", e);
    const unsigned grid = (unsigned)sm_count() * 8;
    index_kernel<<<grid, 256>>>(b.idx, n_reads, nblocks, 12345);
    const int bshift = block_bytes == 32 ? 5 : block_bytes == 64 ? 6 : 7;
    float best = 0;
    e = time_best(b, [&] {
        if (block_bytes == 32) gather_kernel<2><<<grid, 256>>>(b.a, b.idx, n_reads, bshift, b.sink);
        else if (block_bytes == 64) gather_kernel<4><<<grid, 256>>>(b.a, b.idx, n_reads, bshift, b.sink);
        else gather_kernel<8><<<grid, 256>>>(b.a, b.idx, n_reads, bshift, b.sink);
    }, false, &best);
    if (e != cudaSuccess) return fail("gather probe", e);
    *reads_per_s = best > 0 ? (double)n_reads / (best * 1e-3) : 0.0;
    return 0;
}

// Queries per second of the chain "1 or 2 random 128-byte lines from an
// array of line_bytes (0: none), then one dependent random leaf_read-byte
// block (64 or 128) from a region of leaf_bytes".  in_flight = queries per
// 8-lane group (1 or 2).  warm: the timed pass follows an untimed one after
// each flush, so the line array starts resident in L2.  Returns 0 on success.
__attribute__((visibility("default"))) int btp_measure_chain(uint64_t line_bytes,
                                                             uint64_t leaf_bytes,
                                                             uint64_t n_queries,
                                                             uint32_t leaf_read,
                                                             uint32_t lines_per_query,
                                                             uint32_t in_flight, int warm,
                                                             double *queries_per_s) {
    if (!queries_per_s) return fail("queries_per_s is NULL", cudaSuccess);
    *queries_per_s = 0;
    if (leaf_read != 64 && leaf_read != 128) return fail("leaf_read must be 64 or 128", cudaSuccess);
    if (lines_per_query > 2 || (lines_per_query > 0 && line_bytes < 128))
        return fail("lines_per_query must be 0, 1 or 2 (with line_bytes >= 128)", cudaSuccess);
    if (in_flight != 1 && in_flight != 2) return fail("in_flight must be 1 or 2", cudaSuccess);
    // power-of-two counts: the kernel indexes with masks (a 64-bit modulo
    // per query would make the probe instruction bound)
    auto pow2_floor = [](uint64_t v) { return v ? 1ull << (63 - __builtin_clzll(v)) : 0ull; };
    const uint64_t nlines = lines_per_query ? pow2_floor(line_bytes / 128) : 0;
    const uint64_t nblocks = pow2_floor(leaf_bytes / leaf_read);
    if (nblocks == 0 || n_queries == 0 || n_queries > (1ull << 30) || nlines > (1ull << 32))
        return fail("sizes out of range", cudaSuccess);
    Bufs b;
    cudaError_t e = cudaMalloc(&b.b, nblocks * leaf_read);
    if (e == cudaSuccess && nlines) e = cudaMalloc(&b.a, nlines * 128);
    if (e == cudaSuccess) e = cudaMalloc(&b.sink, sizeof(uint32_t));
    if (e == cudaSuccess) e = cudaMalloc(&b.flush, kFlushBytes);
    if (e == cudaSuccess) e = cudaMemset(b.b, 1, nblocks * leaf_read);
    if (e == cudaSuccess && nlines) e = cudaMemset(b.a, 3, nlines * 128);
    if (e != cudaSuccess) return fail("allocation", e);
    const unsigned grid = (unsigned)sm_count() * 8;
    const uint32_t mask = 0;  // the dependency is kept, the address is not changed
    auto run = [&](auto kern) {
        kern<<<grid, 256>>>(b.a, nlines, b.b, nblocks, n_queries, mask, 777, b.sink);
    };
    float best = 0;
    e = time_best(b, [&] {
        const int key = (int)lines_per_query * 100 + (leaf_read == 128 ? 10 : 0) + (int)in_flight;
        switch (key) {
            case 1: run(chain_kernel<0, 64, 1>); break;
            case 2: run(chain_kernel<0, 64, 2>); break;
            case 11: run(chain_kernel<0, 128, 1>); break;
            case 12: run(chain_kernel<0, 128, 2>); break;
            case 101: run(chain_kernel<1, 64, 1>); break;
            case 102: run(chain_kernel<1, 64, 2>); break;
            case 111: run(chain_kernel<1, 128, 1>); break;
            case 112: run(chain_kernel<1, 128, 2>); break;
            case 201: run(chain_kernel<2, 64, 1>); break;
            case 202: run(chain_kernel<2, 64, 2>); break;
            case 211: run(chain_kernel<2, 128, 1>); break;
            default: run(chain_kernel<2, 128, 2>); break;
        }
    }, warm != 0, &best);
    if (e != cudaSuccess) return fail("chain probe", e);
    *queries_per_s = best > 0 ? (double)n_queries / (best * 1e-3) : 0.0;
    return 0;
}

// Queries per second of the chain "hops dependent random 128-byte lines
// from an array of line_bytes, then one dependent random 128-byte read from
// a region of leaf_bytes" (both rounded down to powers of two), read in form
// `mode`: 0 = a lane per query with register loads, 1 = a lane pair per
// query, 2 = a lane per query with bulk copies into shared memory, 3 = a
// lane quad per query, 4 = lane pairs for the lines and quads for the last
// read.  The line
// array starts each timed pass resident in L2.  Returns 0 on success; a bulk
// wait that gives up is reported as a failure.
__attribute__((visibility("default"))) int btp_measure_hops(uint64_t line_bytes, uint64_t leaf_bytes,
                                                            uint64_t n_queries, uint32_t hops,
                                                            uint32_t mode, double *queries_per_s) {
    if (!queries_per_s) return fail("queries_per_s is NULL", cudaSuccess);
    *queries_per_s = 0;
    if (hops > 3 || mode > 4) return fail("hops must be 0..3 and mode 0..4", cudaSuccess);
    auto pow2_floor = [](uint64_t v) { return v ? 1ull << (63 - __builtin_clzll(v)) : 0ull; };
    const uint64_t nlines = pow2_floor(line_bytes / 128);
    const uint64_t nunits = pow2_floor(leaf_bytes / 128);
    if (nlines == 0 || nunits == 0 || n_queries == 0 || n_queries > (1ull << 30))
        return fail("sizes out of range", cudaSuccess);
    Bufs b;
    cudaError_t e = cudaMalloc(&b.b, nunits * 128);
    if (e == cudaSuccess) e = cudaMalloc(&b.a, nlines * 128);
    if (e == cudaSuccess) e = cudaMalloc(&b.sink, 2 * sizeof(uint32_t));
    if (e == cudaSuccess) e = cudaMalloc(&b.flush, kFlushBytes);
    if (e == cudaSuccess) e = cudaMemset(b.b, 1, nunits * 128);
    if (e == cudaSuccess) e = cudaMemset(b.a, 3, nlines * 128);
    if (e == cudaSuccess) e = cudaMemset(b.sink, 0, 2 * sizeof(uint32_t));
    if (e != cudaSuccess) return fail("allocation", e);
    const unsigned grid = (unsigned)sm_count() * 8;
    const size_t smem = mode == 2 ? 256 * 128 : 0;
    auto run = [&](auto kern) {
        kern<<<grid, 256, smem>>>(b.a, nlines, b.b, nunits, n_queries, 0u, 777, b.sink);
    };
    float best = 0;
    e = time_best(b, [&] {
        switch (mode * 10 + hops) {
            case 0: run(hop_kernel<0, 0>); break;
            case 1: run(hop_kernel<0, 1>); break;
            case 2: run(hop_kernel<0, 2>); break;
            case 3: run(hop_kernel<0, 3>); break;
            case 10: run(hop_kernel<1, 0>); break;
            case 11: run(hop_kernel<1, 1>); break;
            case 12: run(hop_kernel<1, 2>); break;
            case 13: run(hop_kernel<1, 3>); break;
            case 20: run(hop_kernel<2, 0>); break;
            case 21: run(hop_kernel<2, 1>); break;
            case 22: run(hop_kernel<2, 2>); break;
            case 23: run(hop_kernel<2, 3>); break;
            case 30: run(hop_kernel<3, 0>); break;
            case 31: run(hop_kernel<3, 1>); break;
            case 32: run(hop_kernel<3, 2>); break;
            case 33: run(hop_kernel<3, 3>); break;
            case 40: run(hop_kernel<4, 0>); break;
            case 41: run(hop_kernel<4, 1>); break;
            case 42: run(hop_kernel<4, 2>); break;
            default: run(hop_kernel<4, 3>); break;
        }
    }, true, &best);
    if (e != cudaSuccess) return fail("hop probe", e);
    uint32_t flags[2] = {0, 0};
    e = cudaMemcpy(flags, b.sink, sizeof(flags), cudaMemcpyDeviceToHost);
    if (e != cudaSuccess) return fail("hop probe", e);
    if (flags[1]) return fail("hop probe: a bulk-copy wait gave up", cudaSuccess);
    *queries_per_s = best > 0 ? (double)n_queries / (best * 1e-3) : 0.0;
    return 0;
}

}  // extern "C"
