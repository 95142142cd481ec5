// Grouped point search that allocates no memory.
//
// bt_point_search(BT_POINT_GROUPED) takes its scratch -- the grouped copy of
// the queries, the permutation back to the caller's order and the
// partition's digit counts -- from a stream-ordered memory pool.  Some
// callers cannot let a library allocate device memory: a serving process or
// framework whose device memory is entirely reserved by its own allocator
// (an extra cudaMalloc either fails or breaks its memory budget), or a
// latency-critical path where an allocation call may block or synchronize.
// bt_point_search_grouped_noalloc serves them: its scratch is the fixed
// array below, linked into this library, so the call itself allocates
// nothing.
//
// Limits and sharing:
//   * at most kNoallocMaxQueries (2^18) queries per call; larger batches are
//     rejected with BT_ERR_INVALID_ARGUMENT (split them, or use
//     bt_point_search);
//   * the array lives on every GPU that loads this library, until exit
//     (kNoallocScratchBytes, 4 MiB);
//   * all calls on a device share it, and it keeps the last call's contents.
//     Nothing in it has to start at zero: every call overwrites all the bytes
//     it reads.  Calls that overlap on the GPU (different streams, or
//     different host threads, without ordering between them) race on it.
//   * the first call on each device looks up the array's device address
//     (cudaGetSymbolAddress) with that device current; make that first call
//     before any stream capture.  The address is cached for the life of the
//     process, so it does not survive a cudaDeviceReset of that device.
#include <mutex>

#include "bt_internal.cuh"

namespace bt {
namespace {

constexpr uint64_t kNoallocMaxQueries = 1ull << 18;
constexpr size_t kNoallocScratchBytes = 4u << 20;

// Scratch of the no-allocation search.  In host code this name is only a
// stand-in for the symbol, not a device address: kernels receive the address
// obtained by cudaGetSymbolAddress below.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoallocScratchBytes];

std::mutex g_mu;
void *g_scratch_addr[64] = {};

// Device address of g_noalloc_scratch on the current device (looked up once
// per device).
bt_status scratch_address(int dev, void **out) {
    if (dev < 0 || dev >= 64) return fail(BT_ERR_NOT_SUPPORTED, "device index out of range");
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_scratch_addr[dev]) {
        void *p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress(no-allocation scratch)");
        g_scratch_addr[dev] = p;
    }
    *out = g_scratch_addr[dev];
    return BT_OK;
}

size_t align256(size_t x) { return (x + 255) / 256 * 256; }

}  // namespace
}  // namespace bt

extern "C" {

bt_status bt_point_search_grouped_noalloc(const bt_tree *t, const void *d_queries, uint64_t nq,
                                          void *d_out, void *stream) {
    using namespace bt;
    if (!t) return fail(BT_ERR_INVALID_ARGUMENT, "tree is NULL");
    if (nq == 0) return BT_OK;
    if (!d_queries || !d_out) return fail(BT_ERR_INVALID_ARGUMENT, "queries or out is NULL");
    if (nq > kNoallocMaxQueries)
        return fail(BT_ERR_INVALID_ARGUMENT,
                    "bt_point_search_grouped_noalloc takes at most 262144 queries per call "
                    "(its fixed scratch is 4 MiB); split the batch or use bt_point_search");
    int prev = 0;
    BT_CUDA(cudaGetDevice(&prev));
    if (prev != t->device) BT_CUDA(cudaSetDevice(t->device));
    cudaStream_t s = (cudaStream_t)stream;
    bt_status st = BT_OK;
    if (t->n == 0) {
        st = launch_point_search(t, d_queries, nullptr, nq, d_out, s);
    } else {
        void *base = nullptr;
        st = scratch_address(t->device, &base);
        if (st == BT_OK) {
            // grouped queries | permutation | partition counts and scan scratch
            unsigned char *p = static_cast<unsigned char *>(base);
            const size_t q_bytes = align256(nq * (size_t)t->key_bytes);
            const size_t perm_bytes = align256(nq * sizeof(uint32_t));
            const size_t need = q_bytes + perm_bytes + partition_point_ws_bytes(nq);
            if (need > kNoallocScratchBytes) {
                st = fail(BT_ERR_INTERNAL, "no-allocation scratch layout exceeds its array");
            } else {
                void *grouped = p;
                uint32_t *perm = reinterpret_cast<uint32_t *>(p + q_bytes);
                void *ws = p + q_bytes + perm_bytes;
                st = launch_partition_point_prealloc(t, d_queries, nq, grouped, perm, ws, s);
                if (st == BT_OK) st = launch_point_search(t, grouped, perm, nq, d_out, s);
            }
        }
    }
    if (prev != t->device) cudaSetDevice(prev);
    return st;
}

}  // extern "C"
