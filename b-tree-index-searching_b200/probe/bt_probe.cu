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
//
// Both functions allocate their own buffers, flush L2 with a 512 MiB write
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

}  // extern "C"
