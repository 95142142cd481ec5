// Continuous-batching request loop (declared in include/btree_b200.h).
//
// The reference serves one batch per synchronous host call: it allocates,
// copies, launches, synchronizes and frees inside the call
// (BPTreeExactSearch.cu:409-484), so a second batch waits for the whole
// first one.  Here a worker thread owns a set of slots -- a stream, a
// completion event and device buffers for max_batch queries each; the number
// of slots is what the memory budget admits.  Requests queue on the host and
// are cut into jobs of at most max_batch queries.  Whenever a slot is free the
// worker issues the next job on it (H2D copy, search kernel, D2H copy, event),
// so jobs of requests that arrive while others are running start at once and
// overlap on the device with the jobs already in flight.  A request completes
// when its last job's event has fired; its latency is measured from submit to
// that observation.
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "bt_internal.cuh"

namespace {

using Clock = std::chrono::steady_clock;

double now_us() {
    return std::chrono::duration<double, std::micro>(Clock::now().time_since_epoch()).count();
}

struct Request {
    const unsigned char *hq;
    unsigned char *hout;
    uint64_t nq;
    uint64_t jobs_total;
    uint64_t jobs_issued = 0;
    uint64_t jobs_done = 0;
    double t_submit = 0, t_done = 0;
    bool done = false;
};

struct Slot {
    cudaStream_t stream = nullptr;
    cudaEvent_t event = nullptr;
    void *dq = nullptr;
    void *dout = nullptr;
    Request *req = nullptr;  // null when free
};

}  // namespace

struct bt_server {
    const bt_tree *tree;
    int mode;
    uint64_t max_batch;
    std::vector<Slot> slots;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<Request *> pending;  // requests with jobs not yet issued
    std::unordered_map<uint64_t, Request *> tickets;
    uint64_t next_ticket = 1;
    bool stop = false;
    bt_status error = BT_OK;
    std::string error_msg;
    uint32_t in_flight = 0, max_in_flight = 0;
    uint64_t completed = 0, jobs = 0;
    std::thread worker;
};

namespace {

bt_status run_job(bt_server *s, Slot &sl, const void *dq, uint64_t m) {
    const bt_tree *t = s->tree;
    switch (s->mode) {
        case BT_SERVE_LEARNED:
            return bt_point_search_learned(t, dq, m, sl.dout, sl.stream);
        case BT_SERVE_GROUPED:
            return bt_point_search(t, BT_POINT_GROUPED, dq, m, sl.dout, sl.stream);
        default:
            return bt_point_search(t, BT_POINT_BASIC, dq, m, sl.dout, sl.stream);
    }
}

void worker_loop(bt_server *s) {
    cudaSetDevice(s->tree->device);
    const size_t kb = (size_t)s->tree->key_bytes, vb = (size_t)s->tree->val_bytes;
    std::unique_lock<std::mutex> lk(s->mu);
    for (;;) {
        // reap finished jobs
        for (Slot &sl : s->slots) {
            if (!sl.req) continue;
            const cudaError_t q = cudaEventQuery(sl.event);
            if (q == cudaErrorNotReady) continue;
            if (q != cudaSuccess && s->error == BT_OK) {
                s->error = BT_ERR_CUDA;
                s->error_msg = cudaGetErrorString(q);
            }
            Request *r = sl.req;
            sl.req = nullptr;
            s->in_flight--;
            if (++r->jobs_done == r->jobs_total) {
                r->t_done = now_us();
                r->done = true;
                s->completed++;
                s->cv_done.notify_all();
            }
        }
        // admit: the next job of the oldest pending request into each free slot
        for (Slot &sl : s->slots) {
            if (sl.req || s->pending.empty()) continue;
            Request *r = s->pending.front();
            const uint64_t off = r->jobs_issued * s->max_batch;
            const uint64_t m = std::min<uint64_t>(s->max_batch, r->nq - off);
            if (++r->jobs_issued == r->jobs_total) s->pending.pop_front();
            sl.req = r;
            s->in_flight++;
            s->jobs++;
            if (s->in_flight > s->max_in_flight) s->max_in_flight = s->in_flight;
            cudaError_t e = cudaMemcpyAsync(sl.dq, r->hq + off * kb, m * kb, cudaMemcpyHostToDevice,
                                            sl.stream);
            bt_status st = e == cudaSuccess ? run_job(s, sl, sl.dq, m) : BT_ERR_CUDA;
            if (st == BT_OK)
                e = cudaMemcpyAsync(r->hout + off * vb, sl.dout, m * vb, cudaMemcpyDeviceToHost,
                                    sl.stream);
            if (st == BT_OK && e == cudaSuccess) e = cudaEventRecord(sl.event, sl.stream);
            if ((st != BT_OK || e != cudaSuccess) && s->error == BT_OK) {
                s->error = st != BT_OK ? st : BT_ERR_CUDA;
                s->error_msg = st != BT_OK ? bt_last_error() : cudaGetErrorString(e);
                cudaEventRecord(sl.event, sl.stream);  // so the job still retires
            }
        }
        if (s->stop && s->pending.empty() && s->in_flight == 0) break;
        if (s->in_flight == 0 && s->pending.empty()) {
            s->cv_work.wait(lk);
        } else {
            // jobs on the device: poll their events without holding the lock long
            lk.unlock();
            std::this_thread::yield();
            lk.lock();
        }
    }
}

}  // namespace

extern "C" {

bt_status bt_server_create(const bt_tree *t, const bt_server_config *cfg_in, bt_server **out) {
    using namespace bt;
    if (!t || !out) return fail(BT_ERR_INVALID_ARGUMENT, "tree or out is NULL");
    *out = nullptr;
    bt_server_config cfg = {8, 256ull << 20, 65536, BT_SERVE_BASIC};
    if (cfg_in) {
        if (cfg_in->slots) cfg.slots = cfg_in->slots;
        if (cfg_in->memory_budget_bytes) cfg.memory_budget_bytes = cfg_in->memory_budget_bytes;
        if (cfg_in->max_batch) cfg.max_batch = cfg_in->max_batch;
        cfg.mode = cfg_in->mode;
    }
    if (cfg.mode < BT_SERVE_BASIC || cfg.mode > BT_SERVE_LEARNED)
        return fail(BT_ERR_INVALID_ARGUMENT, "unknown serve mode");
    if (cfg.mode == BT_SERVE_LEARNED && !t->learned)
        return fail(BT_ERR_INVALID_ARGUMENT, "learned serving needs a trained model");
    const uint64_t per_slot = (uint64_t)cfg.max_batch * (t->key_bytes + t->val_bytes) + 512;
    const uint64_t fit = cfg.memory_budget_bytes / per_slot;
    if (fit == 0) return fail(BT_ERR_CAPACITY, "memory budget below one slot");
    const uint32_t nslots = (uint32_t)std::min<uint64_t>(cfg.slots, fit);
    int prev = 0;
    BT_CUDA(cudaGetDevice(&prev));
    BT_CUDA(cudaSetDevice(t->device));
    bt_server *s = new bt_server();
    s->tree = t;
    s->mode = cfg.mode;
    s->max_batch = cfg.max_batch;
    s->slots.resize(nslots);
    bt_status st = BT_OK;
    for (Slot &sl : s->slots) {
        cudaError_t e = cudaStreamCreateWithFlags(&sl.stream, cudaStreamNonBlocking);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&sl.event, cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaMalloc(&sl.dq, (size_t)cfg.max_batch * t->key_bytes);
        if (e == cudaSuccess) e = cudaMalloc(&sl.dout, (size_t)cfg.max_batch * t->val_bytes);
        if (e != cudaSuccess) {
            st = cuda_fail(e, "server slot set-up");
            break;
        }
    }
    cudaSetDevice(prev);
    if (st != BT_OK) {
        for (Slot &sl : s->slots) {
            if (sl.dq) cudaFree(sl.dq);
            if (sl.dout) cudaFree(sl.dout);
            if (sl.event) cudaEventDestroy(sl.event);
            if (sl.stream) cudaStreamDestroy(sl.stream);
        }
        delete s;
        return st;
    }
    s->worker = std::thread(worker_loop, s);
    *out = s;
    return BT_OK;
}

bt_status bt_server_submit(bt_server *s, const void *hq, uint64_t nq, void *hout, uint64_t *ticket) {
    using namespace bt;
    if (!s || !ticket) return fail(BT_ERR_INVALID_ARGUMENT, "server or ticket is NULL");
    if (nq > 0 && (!hq || !hout)) return fail(BT_ERR_INVALID_ARGUMENT, "queries or out is NULL");
    Request *r = new Request();
    r->hq = (const unsigned char *)hq;
    r->hout = (unsigned char *)hout;
    r->nq = nq;
    r->jobs_total = (nq + s->max_batch - 1) / s->max_batch;
    r->t_submit = now_us();
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->error != BT_OK) {
        delete r;
        return fail(s->error, s->error_msg);
    }
    *ticket = s->next_ticket++;
    s->tickets[*ticket] = r;
    if (r->jobs_total == 0) {
        r->done = true;
        r->t_done = r->t_submit;
        s->completed++;
    } else {
        s->pending.push_back(r);
        s->cv_work.notify_one();
    }
    return BT_OK;
}

bt_status bt_server_wait(bt_server *s, uint64_t ticket, double *latency_us) {
    using namespace bt;
    if (!s) return fail(BT_ERR_INVALID_ARGUMENT, "server is NULL");
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->tickets.find(ticket);
    if (it == s->tickets.end()) return fail(BT_ERR_INVALID_ARGUMENT, "unknown or already waited ticket");
    Request *r = it->second;
    s->cv_done.wait(lk, [&] { return r->done || s->error != BT_OK; });
    if (!r->done) return fail(s->error, s->error_msg);
    if (latency_us) *latency_us = r->t_done - r->t_submit;
    s->tickets.erase(it);
    delete r;
    if (s->error != BT_OK) return fail(s->error, s->error_msg);
    return BT_OK;
}

bt_status bt_server_get_stats(bt_server *s, bt_server_stats *st) {
    using namespace bt;
    if (!s || !st) return fail(BT_ERR_INVALID_ARGUMENT, "server or stats is NULL");
    std::lock_guard<std::mutex> lk(s->mu);
    st->slots = (uint32_t)s->slots.size();
    st->max_in_flight = s->max_in_flight;
    st->completed = s->completed;
    st->jobs = s->jobs;
    return BT_OK;
}

bt_status bt_server_destroy(bt_server *s) {
    if (!s) return BT_OK;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
        s->cv_work.notify_one();
    }
    if (s->worker.joinable()) s->worker.join();
    cudaSetDevice(s->tree->device);
    for (Slot &sl : s->slots) {
        cudaStreamSynchronize(sl.stream);
        cudaFree(sl.dq);
        cudaFree(sl.dout);
        cudaEventDestroy(sl.event);
        cudaStreamDestroy(sl.stream);
    }
    for (auto &kv : s->tickets) delete kv.second;
    delete s;
    return BT_OK;
}

bt_status bt_server_replay(bt_server *s, uint64_t nreq, const uint64_t *nq,
                           const void *const *hq, void *const *hout, const double *arrival_us,
                           double *latency_us, double *wall_us) {
    using namespace bt;
    if (!s || (nreq && (!nq || !hq || !hout || !arrival_us || !latency_us)))
        return fail(BT_ERR_INVALID_ARGUMENT, "null argument");
    std::vector<uint64_t> tk(nreq);
    const double t0 = now_us();
    for (uint64_t i = 0; i < nreq; i++) {
        while (now_us() - t0 < arrival_us[i]) {
        }
        bt_status st = bt_server_submit(s, hq[i], nq[i], hout[i], &tk[i]);
        if (st != BT_OK) return st;
    }
    for (uint64_t i = 0; i < nreq; i++) {
        bt_status st = bt_server_wait(s, tk[i], &latency_us[i]);
        if (st != BT_OK) return st;
    }
    if (wall_us) *wall_us = now_us() - t0;
    return BT_OK;
}

}  // extern "C"
