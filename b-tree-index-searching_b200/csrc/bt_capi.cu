// C ABI entry points for search (declared in include/btree_b200.h).
#include <algorithm>
#include <cstring>
#include <mutex>

#include "bt_internal.cuh"

namespace bt {
namespace {

struct DeviceGuard {
    int prev = -1;
    bool changed = false;
    explicit DeviceGuard(int d) {
        cudaGetDevice(&prev);
        if (prev != d) {
            cudaSetDevice(d);
            changed = true;
        }
    }
    ~DeviceGuard() {
        if (changed) cudaSetDevice(prev);
    }
};

bt_status check_tree(const bt_tree *t) {
    if (!t) return fail(BT_ERR_INVALID_ARGUMENT, "tree is NULL");
    return BT_OK;
}

// Non-blocking streams per device for the host-buffer pipelines, one per
// buffer slot.  Chunk i runs on slot i % kPipeSlots: its H2D copy waits only
// for the D2H copy of chunk i - kPipeSlots, so with three slots the
// host-to-device engine keeps copying while the device-to-host engine drains
// the two chunks before (PCIe carries both directions at once).
constexpr int kPipeSlots = 3;
struct PipeStreams {
    cudaStream_t s[kPipeSlots] = {};
    bool ready = false;
};
std::mutex g_pipe_mu;
PipeStreams g_pipe[64];

bt_status pipe_streams(int dev, cudaStream_t (&out)[kPipeSlots]) {
    std::lock_guard<std::mutex> lk(g_pipe_mu);
    PipeStreams &p = g_pipe[dev];
    if (!p.ready) {
        for (int i = 0; i < kPipeSlots; i++)
            BT_CUDA(cudaStreamCreateWithFlags(&p.s[i], cudaStreamNonBlocking));
        p.ready = true;
    }
    for (int i = 0; i < kPipeSlots; i++) out[i] = p.s[i];
    return BT_OK;
}

bt_status point_device(const bt_tree *t, int mode, const void *d_q, uint64_t nq, void *d_out,
                       cudaStream_t s, uint8_t *d_found = nullptr) {
    if (mode == BT_POINT_BASIC || t->n == 0)
        return launch_point_search(t, d_q, nullptr, nq, d_out, s, d_found);
    if (mode == BT_POINT_LEARNED) return launch_learned_search(t, d_q, nq, d_out, d_found, s);
    void *gq = nullptr;
    uint32_t *perm = nullptr;
    bt_status st = ws_alloc(&gq, nq * t->key_bytes, s);
    if (st == BT_OK) st = ws_alloc((void **)&perm, nq * sizeof(uint32_t), s);
    if (st == BT_OK) st = launch_partition(t, kPartPoint, d_q, nullptr, nq, gq, nullptr, perm, s);
    if (st == BT_OK) st = launch_point_search(t, gq, perm, nq, d_out, s, d_found);
    ws_free(gq, s);
    ws_free(perm, s);
    return st;
}

bt_status count_device(const bt_tree *t, int mode, const void *d_lo, const void *d_hi, uint64_t nq,
                       uint64_t *d_counts, uint64_t *d_lb, cudaStream_t s) {
    if (mode == BT_RANGE_BASIC || t->n == 0)
        return launch_bounds(t, d_lo, d_hi, nullptr, nq, d_counts, d_lb, s);
    const int kind = mode == BT_RANGE_GROUPED_2D ? kPart2D : kPartZ;
    void *ga = nullptr, *gb = nullptr;
    uint32_t *perm = nullptr;
    bt_status st = ws_alloc(&ga, nq * t->key_bytes, s);
    if (st == BT_OK) st = ws_alloc(&gb, nq * t->key_bytes, s);
    if (st == BT_OK) st = ws_alloc((void **)&perm, nq * sizeof(uint32_t), s);
    if (st == BT_OK) st = launch_partition(t, kind, d_lo, d_hi, nq, ga, gb, perm, s);
    if (st == BT_OK) st = launch_bounds(t, ga, gb, perm, nq, d_counts, d_lb, s);
    ws_free(ga, s);
    ws_free(gb, s);
    ws_free(perm, s);
    return st;
}

bool valid_point_mode(int m) {
    return m == BT_POINT_BASIC || m == BT_POINT_GROUPED || m == BT_POINT_LEARNED;
}
bool valid_range_mode(int m) {
    return m == BT_RANGE_BASIC || m == BT_RANGE_GROUPED_2D || m == BT_RANGE_ZORDER;
}

// Host-buffer pipeline: chunks alternate between two streams; each chunk is
// H2D -> kernels -> D2H on its stream, so copies of one chunk overlap the
// kernels of the other.  `run` issues the kernels of one chunk.
template <typename Run>
bt_status host_pipeline(const bt_tree *t, cudaStream_t caller, uint64_t nq, uint64_t chunk,
                        int n_in, const void *const *h_in, const size_t *in_w, void *h_out,
                        size_t out_w, Run run) {
    cudaStream_t ps[kPipeSlots];
    bt_status st = pipe_streams(t->device, ps);
    if (st != BT_OK) return st;
    cudaEvent_t ev;
    BT_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    cudaEventRecord(ev, caller);
    for (int i = 0; i < kPipeSlots; i++) cudaStreamWaitEvent(ps[i], ev, 0);
    void *din[kPipeSlots][2] = {};
    void *dout[kPipeSlots] = {};
    const uint64_t cap = std::min(chunk, nq);
    for (int i = 0; i < kPipeSlots && st == BT_OK; i++) {
        for (int k = 0; k < n_in && st == BT_OK; k++) st = ws_alloc(&din[i][k], cap * in_w[k], ps[i]);
        if (st == BT_OK) st = ws_alloc(&dout[i], cap * out_w, ps[i]);
    }
    for (uint64_t c0 = 0, ci = 0; c0 < nq && st == BT_OK; c0 += chunk, ci++) {
        const int slot = (int)(ci % kPipeSlots);
        cudaStream_t s = ps[slot];
        const uint64_t m = std::min(chunk, nq - c0);
        for (int k = 0; k < n_in && st == BT_OK; k++) {
            cudaError_t e = cudaMemcpyAsync(din[slot][k], (const char *)h_in[k] + c0 * in_w[k],
                                            m * in_w[k], cudaMemcpyHostToDevice, s);
            if (e != cudaSuccess) st = cuda_fail(e, "cudaMemcpyAsync H2D");
        }
        if (st == BT_OK) st = run(din[slot], m, dout[slot], s);
        if (st == BT_OK) {
            cudaError_t e = cudaMemcpyAsync((char *)h_out + c0 * out_w, dout[slot], m * out_w,
                                            cudaMemcpyDeviceToHost, s);
            if (e != cudaSuccess) st = cuda_fail(e, "cudaMemcpyAsync D2H");
        }
    }
    for (int i = 0; i < kPipeSlots; i++) {
        for (int k = 0; k < n_in; k++) ws_free(din[i][k], ps[i]);
        ws_free(dout[i], ps[i]);
    }
    cudaError_t es = cudaSuccess;
    for (int i = 0; i < kPipeSlots; i++) {
        const cudaError_t e = cudaStreamSynchronize(ps[i]);
        if (es == cudaSuccess) es = e;
    }
    cudaEventDestroy(ev);
    if (st != BT_OK) return st;
    if (es != cudaSuccess) return cuda_fail(es, "cudaStreamSynchronize");
    return BT_OK;
}

uint64_t pipeline_chunk(uint64_t nq) {
    // Eight chunks or more for large batches (copy/compute overlap), but not
    // below 2M queries (per-chunk launch and grouping overheads; the grouped
    // search's window kernel starts at 2^21 queries).
    const uint64_t c = (nq + 7) / 8;
    return std::max<uint64_t>(c, std::min<uint64_t>(nq, 1ull << 21));
}

}  // namespace
}  // namespace bt

extern "C" {

bt_status bt_point_search(const bt_tree *t, int mode, const void *d_queries, uint64_t nq,
                          void *d_out, void *stream) {
    using namespace bt;
    bt_status st = check_tree(t);
    if (st != BT_OK) return st;
    if (!valid_point_mode(mode)) return fail(BT_ERR_INVALID_ARGUMENT, "unknown point mode");
    if (mode == BT_POINT_LEARNED && !t->learned)
        return fail(BT_ERR_INVALID_ARGUMENT, "the tree has no trained learned index");
    if (nq == 0) return BT_OK;
    if (!d_queries || !d_out) return fail(BT_ERR_INVALID_ARGUMENT, "queries or out is NULL");
    if (nq >= (1ull << 32)) return fail(BT_ERR_INVALID_ARGUMENT, "nq must be below 2^32");
    DeviceGuard g(t->device);
    if (mode == BT_POINT_LEARNED) {
        st = reset_learned_stats(t, (cudaStream_t)stream);
        if (st != BT_OK) return st;
    }
    return point_device(t, mode, d_queries, nq, d_out, (cudaStream_t)stream);
}

bt_status bt_point_search_found(const bt_tree *t, int mode, const void *d_queries, uint64_t nq,
                                void *d_out, uint8_t *d_found, void *stream) {
    using namespace bt;
    bt_status st = check_tree(t);
    if (st != BT_OK) return st;
    if (!valid_point_mode(mode)) return fail(BT_ERR_INVALID_ARGUMENT, "unknown point mode");
    if (mode == BT_POINT_LEARNED && !t->learned)
        return fail(BT_ERR_INVALID_ARGUMENT, "the tree has no trained learned index");
    if (nq == 0) return BT_OK;
    if (!d_queries || !d_out || !d_found)
        return fail(BT_ERR_INVALID_ARGUMENT, "queries, out or found is NULL");
    if (nq >= (1ull << 32)) return fail(BT_ERR_INVALID_ARGUMENT, "nq must be below 2^32");
    DeviceGuard g(t->device);
    if (mode == BT_POINT_LEARNED) {
        st = reset_learned_stats(t, (cudaStream_t)stream);
        if (st != BT_OK) return st;
    }
    return point_device(t, mode, d_queries, nq, d_out, (cudaStream_t)stream, d_found);
}

bt_status bt_point_search_host(const bt_tree *t, int mode, const void *h_queries, uint64_t nq,
                               void *h_out, void *stream) {
    using namespace bt;
    bt_status st = check_tree(t);
    if (st != BT_OK) return st;
    if (!valid_point_mode(mode)) return fail(BT_ERR_INVALID_ARGUMENT, "unknown point mode");
    if (mode == BT_POINT_LEARNED && !t->learned)
        return fail(BT_ERR_INVALID_ARGUMENT, "the tree has no trained learned index");
    if (nq == 0) return BT_OK;
    if (!h_queries || !h_out) return fail(BT_ERR_INVALID_ARGUMENT, "queries or out is NULL");
    if (nq >= (1ull << 32)) return fail(BT_ERR_INVALID_ARGUMENT, "nq must be below 2^32");
    DeviceGuard g(t->device);
    if (mode == BT_POINT_LEARNED) {
        st = reset_learned_stats(t, (cudaStream_t)stream);
        if (st != BT_OK) return st;
    }
    const void *ins[1] = {h_queries};
    const size_t w[1] = {(size_t)t->key_bytes};
    return host_pipeline(t, (cudaStream_t)stream, nq, pipeline_chunk(nq), 1, ins, w, h_out,
                         (size_t)t->val_bytes,
                         [&](void *const *din, uint64_t m, void *dout, cudaStream_t s) {
                             return point_device(t, mode, din[0], m, dout, s);
                         });
}

bt_status bt_group_queries(const bt_tree *t, const void *d_queries, uint64_t nq, void *d_grouped,
                           uint32_t *d_perm, void *stream) {
    using namespace bt;
    bt_status st = check_tree(t);
    if (st != BT_OK) return st;
    if (nq == 0) return BT_OK;
    if (!d_queries || !d_grouped || !d_perm)
        return fail(BT_ERR_INVALID_ARGUMENT, "queries, grouped or perm is NULL");
    if (nq >= (1ull << 32)) return fail(BT_ERR_INVALID_ARGUMENT, "nq must be below 2^32");
    DeviceGuard g(t->device);
    return launch_partition(t, kPartPoint, d_queries, nullptr, nq, d_grouped, nullptr, d_perm,
                            (cudaStream_t)stream);
}

bt_status bt_point_search_grouped_batch(const bt_tree *t, const void *d_grouped,
                                        const uint32_t *d_perm, uint64_t nq, void *d_out,
                                        void *stream) {
    using namespace bt;
    bt_status st = check_tree(t);
    if (st != BT_OK) return st;
    if (nq == 0) return BT_OK;
    if (!d_grouped || !d_perm || !d_out)
        return fail(BT_ERR_INVALID_ARGUMENT, "grouped, perm or out is NULL");
    if (nq >= (1ull << 32)) return fail(BT_ERR_INVALID_ARGUMENT, "nq must be below 2^32");
    DeviceGuard g(t->device);
    return launch_point_search(t, d_grouped, d_perm, nq, d_out, (cudaStream_t)stream);
}

bt_status bt_range_count(const bt_tree *t, int mode, const void *d_lo, const void *d_hi,
                         uint64_t nq, uint64_t *d_counts, void *stream) {
    using namespace bt;
    bt_status st = check_tree(t);
    if (st != BT_OK) return st;
    if (!valid_range_mode(mode)) return fail(BT_ERR_INVALID_ARGUMENT, "unknown range mode");
    if (nq == 0) return BT_OK;
    if (!d_lo || !d_hi || !d_counts) return fail(BT_ERR_INVALID_ARGUMENT, "lo, hi or counts is NULL");
    if (nq >= (1ull << 32)) return fail(BT_ERR_INVALID_ARGUMENT, "nq must be below 2^32");
    DeviceGuard g(t->device);
    return count_device(t, mode, d_lo, d_hi, nq, d_counts, nullptr, (cudaStream_t)stream);
}

bt_status bt_range_search(const bt_tree *t, int mode, const void *d_lo, const void *d_hi,
                          uint64_t nq, uint64_t *d_counts, uint64_t *d_offsets, void *d_ids,
                          uint64_t ids_capacity, uint64_t *h_total, void *stream) {
    using namespace bt;
    bt_status st = check_tree(t);
    if (st != BT_OK) return st;
    if (!valid_range_mode(mode)) return fail(BT_ERR_INVALID_ARGUMENT, "unknown range mode");
    if (!h_total) return fail(BT_ERR_INVALID_ARGUMENT, "h_total is NULL");
    *h_total = 0;
    if (nq == 0) return BT_OK;
    if (!d_lo || !d_hi || !d_counts || !d_offsets)
        return fail(BT_ERR_INVALID_ARGUMENT, "lo, hi, counts or offsets is NULL");
    if (nq >= (1ull << 32)) return fail(BT_ERR_INVALID_ARGUMENT, "nq must be below 2^32");
    DeviceGuard g(t->device);
    cudaStream_t s = (cudaStream_t)stream;
    uint64_t *lb = nullptr, *d_total = nullptr;
    st = ws_alloc((void **)&lb, nq * sizeof(uint64_t), s);
    if (st == BT_OK) st = ws_alloc((void **)&d_total, sizeof(uint64_t), s);
    if (st == BT_OK) st = count_device(t, mode, d_lo, d_hi, nq, d_counts, lb, s);
    if (st == BT_OK) st = launch_scan_u64(d_counts, d_offsets, nq, d_total, s);
    uint64_t total = 0;
    if (st == BT_OK) {
        cudaError_t e = cudaMemcpyAsync(&total, d_total, sizeof(total), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) st = cuda_fail(e, "total hits read-back");
    }
    if (st == BT_OK) {
        *h_total = total;
        if (total > ids_capacity) {
            st = fail(BT_ERR_CAPACITY, "ids_capacity is below the total hit count");
        } else if (total > 0) {
            if (!d_ids) st = fail(BT_ERR_INVALID_ARGUMENT, "ids is NULL");
            else st = launch_range_fill(t, lb, d_counts, d_offsets, nq, d_ids, s);
        }
    }
    ws_free(lb, s);
    ws_free(d_total, s);
    return st;
}

bt_status bt_range_count_host(const bt_tree *t, int mode, const void *h_lo, const void *h_hi,
                              uint64_t nq, uint64_t *h_counts, void *stream) {
    using namespace bt;
    bt_status st = check_tree(t);
    if (st != BT_OK) return st;
    if (!valid_range_mode(mode)) return fail(BT_ERR_INVALID_ARGUMENT, "unknown range mode");
    if (nq == 0) return BT_OK;
    if (!h_lo || !h_hi || !h_counts) return fail(BT_ERR_INVALID_ARGUMENT, "lo, hi or counts is NULL");
    if (nq >= (1ull << 32)) return fail(BT_ERR_INVALID_ARGUMENT, "nq must be below 2^32");
    DeviceGuard g(t->device);
    const void *ins[2] = {h_lo, h_hi};
    const size_t w[2] = {(size_t)t->key_bytes, (size_t)t->key_bytes};
    return host_pipeline(t, (cudaStream_t)stream, nq, pipeline_chunk(nq), 2, ins, w, h_counts,
                         sizeof(uint64_t),
                         [&](void *const *din, uint64_t m, void *dout, cudaStream_t s) {
                             return count_device(t, mode, din[0], din[1], m, (uint64_t *)dout,
                                                 nullptr, s);
                         });
}

}  // extern "C"
