// Random-gather ceiling of the current GPU (declared in btree_b200.h).
//
// A point search that misses the cache costs one read of one leaf block at a
// random address.  Such reads are limited by the number of random DRAM
// accesses the GPU sustains, not by its copy bandwidth: on a B200 a 64-byte
// random read reaches about 45 G reads/s (2.9 TB/s of useful bytes) against
// 6.5 TB/s for a streaming copy.  This probe measures that ceiling with the
// search's own access shape -- blocks of 32, 64 or 128 bytes read by 16-byte
// lanes, L1 bypassed -- so a search kernel's throughput can be set against
// it.  It allocates its own buffers; it is a measurement aid, not part of any
// search path.
#include <algorithm>

#include "bt_internal.cuh"

namespace bt {
namespace {

__device__ __forceinline__ uint64_t splitmix64(uint64_t x) {
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

__global__ void probe_index_kernel(uint32_t *idx, uint64_t n, uint64_t nblocks, uint64_t seed) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x)
        idx[i] = (uint32_t)(splitmix64(seed + i) % nblocks);
}

template <int G>
__global__ void __launch_bounds__(256)
probe_gather_kernel(const unsigned char *__restrict__ buf, const uint32_t *__restrict__ idx,
                    uint64_t n, int bshift, uint32_t *__restrict__ sink) {
    const uint64_t tid = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x / G;
    const int gl = (int)(tid % G);
    uint32_t acc = 0;
    for (uint64_t i = tid / G; i < n; i += stride) {
        uint4 x;
        asm volatile("ld.global.nc.L1::no_allocate.v4.b32 {%0,%1,%2,%3}, [%4];"
                     : "=r"(x.x), "=r"(x.y), "=r"(x.z), "=r"(x.w)
                     : "l"(buf + ((uint64_t)idx[i] << bshift) + gl * 16));
        acc ^= x.x ^ x.y ^ x.z ^ x.w;
    }
    if (acc == 0x9E3779B9u) sink[0] = acc;  // keeps the loads live
}

}  // namespace
}  // namespace bt

extern "C" {

bt_status bt_measure_gather(uint64_t region_bytes, uint64_t n_reads, uint32_t block_bytes,
                            double *reads_per_s) {
    using namespace bt;
    if (!reads_per_s) return fail(BT_ERR_INVALID_ARGUMENT, "reads_per_s is NULL");
    *reads_per_s = 0;
    if (block_bytes != 32 && block_bytes != 64 && block_bytes != 128)
        return fail(BT_ERR_INVALID_ARGUMENT, "block_bytes must be 32, 64 or 128");
    const uint64_t nblocks = region_bytes / block_bytes;
    if (nblocks == 0 || nblocks > (1ull << 32) || n_reads == 0 || n_reads > (1ull << 30))
        return fail(BT_ERR_INVALID_ARGUMENT, "region or read count out of range");
    int dev = 0;
    BT_CUDA(cudaGetDevice(&dev));
    bt_status st = require_device(dev);
    if (st != BT_OK) return st;
    unsigned char *buf = nullptr;
    uint32_t *idx = nullptr, *sink = nullptr;
    unsigned char *flush = nullptr;
    const size_t flush_bytes = 512ull << 20;  // larger than L2
    cudaEvent_t a = nullptr, b = nullptr;
    cudaError_t e = cudaMalloc(&buf, nblocks * block_bytes);
    if (e == cudaSuccess) e = cudaMalloc(&idx, n_reads * sizeof(uint32_t));
    if (e == cudaSuccess) e = cudaMalloc(&sink, sizeof(uint32_t));
    if (e == cudaSuccess) e = cudaMalloc(&flush, flush_bytes);
    if (e == cudaSuccess) e = cudaMemset(buf, 1, nblocks * block_bytes);
    if (e == cudaSuccess) e = cudaEventCreate(&a);
    if (e == cudaSuccess) e = cudaEventCreate(&b);
    float best = 0;
    if (e == cudaSuccess) {
        count_launch();
        probe_index_kernel<<<sm_count() * 8, 256>>>(idx, n_reads, nblocks, 12345);
        const int bshift = block_bytes == 32 ? 5 : block_bytes == 64 ? 6 : 7;
        const unsigned grid = (unsigned)sm_count() * 8;
        for (int rep = 0; rep < 4 && e == cudaSuccess; rep++) {
            e = cudaMemsetAsync(flush, rep, flush_bytes, 0);
            if (e != cudaSuccess) break;
            cudaEventRecord(a, 0);
            count_launch();
            if (block_bytes == 32) probe_gather_kernel<2><<<grid, 256>>>(buf, idx, n_reads, bshift, sink);
            else if (block_bytes == 64) probe_gather_kernel<4><<<grid, 256>>>(buf, idx, n_reads, bshift, sink);
            else probe_gather_kernel<8><<<grid, 256>>>(buf, idx, n_reads, bshift, sink);
            cudaEventRecord(b, 0);
            e = cudaEventSynchronize(b);
            float ms = 0;
            if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, a, b);
            if (e == cudaSuccess && rep > 0 && (best == 0 || ms < best)) best = ms;  // rep 0 warms up
        }
    }
    if (a) cudaEventDestroy(a);
    if (b) cudaEventDestroy(b);
    cudaFree(buf);
    cudaFree(idx);
    cudaFree(sink);
    cudaFree(flush);
    if (e != cudaSuccess) return cuda_fail(e, "random-gather probe");
    *reads_per_s = best > 0 ? (double)n_reads / (best * 1e-3) : 0.0;
    return BT_OK;
}

}  // extern "C"
