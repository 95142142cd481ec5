// Runtime helpers: error state, device checks, the engine's memory pool.
#include <atomic>
#include <mutex>
#include <string>

#include "bt_internal.cuh"

namespace bt {

namespace {
thread_local std::string g_last_error;

struct DeviceState {
    bool pool_ready = false;
    cudaMemPool_t pool = nullptr;
    int sms = 0;
    int checked = 0;  // 0 unknown, 1 ok, -1 unsupported
};
std::mutex g_mu;
DeviceState g_dev[64];
}  // namespace

std::atomic<uint64_t> g_launches{0};
std::atomic<uint64_t> g_ws_allocs{0};  // ws_alloc calls (bt_workspace_allocations)

void count_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }

void set_error(const std::string &msg) { g_last_error = msg; }

bt_status fail(bt_status s, const std::string &msg) {
    g_last_error = msg;
    return s;
}

bt_status cuda_fail(cudaError_t e, const char *what) {
    g_last_error = std::string(what) + ": " + cudaGetErrorString(e);
    return e == cudaErrorMemoryAllocation ? BT_ERR_OUT_OF_MEMORY : BT_ERR_CUDA;
}

static int current_device() {
    int d = 0;
    cudaGetDevice(&d);
    return d;
}

bt_status require_device(int device) {
    if (device < 0 || device >= 64) return fail(BT_ERR_NOT_SUPPORTED, "device index out of range");
    std::lock_guard<std::mutex> lk(g_mu);
    DeviceState &st = g_dev[device];
    if (st.checked == 0) {
        cudaDeviceProp p;
        cudaError_t e = cudaGetDeviceProperties(&p, device);
        if (e != cudaSuccess) return cuda_fail(e, "cudaGetDeviceProperties");
        st.sms = p.multiProcessorCount;
        st.checked = (p.major == 10) ? 1 : -1;
    }
    if (st.checked < 0)
        return fail(BT_ERR_NOT_SUPPORTED, "this library is built for sm_100a (B200) only");
    return BT_OK;
}

int sm_count() {
    int d = current_device();
    if (d < 0 || d >= 64) return 148;
    std::lock_guard<std::mutex> lk(g_mu);
    if (g_dev[d].sms == 0) {
        int v = 0;
        cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, d);
        g_dev[d].sms = v > 0 ? v : 148;
    }
    return g_dev[d].sms;
}

bt_status ws_alloc(void **p, size_t bytes, cudaStream_t s) {
    *p = nullptr;
    g_ws_allocs.fetch_add(1, std::memory_order_relaxed);
    if (bytes == 0) bytes = 256;
    int d = current_device();
    cudaMemPool_t pool;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        DeviceState &st = g_dev[d];
        if (!st.pool_ready) {
            cudaMemPoolProps props = {};
            props.allocType = cudaMemAllocationTypePinned;
            props.handleTypes = cudaMemHandleTypeNone;
            props.location.type = cudaMemLocationTypeDevice;
            props.location.id = d;
            cudaError_t e = cudaMemPoolCreate(&st.pool, &props);
            if (e != cudaSuccess) return cuda_fail(e, "cudaMemPoolCreate");
            uint64_t keep = UINT64_MAX;  // keep freed blocks cached for the next call
            cudaMemPoolSetAttribute(st.pool, cudaMemPoolAttrReleaseThreshold, &keep);
            st.pool_ready = true;
        }
        pool = st.pool;
    }
    cudaError_t e = cudaMallocFromPoolAsync(p, bytes, pool, s);
    if (e != cudaSuccess) return cuda_fail(e, "cudaMallocFromPoolAsync");
    return BT_OK;
}

void ws_free(void *p, cudaStream_t s) {
    if (p) cudaFreeAsync(p, s);
}

}  // namespace bt

extern "C" {

int bt_version(void) { return BT_VERSION_NUMBER; }

const char *bt_status_string(bt_status s) {
    switch (s) {
        case BT_OK: return "ok";
        case BT_ERR_INVALID_ARGUMENT: return "invalid argument";
        case BT_ERR_UNSORTED: return "build keys are not sorted ascending";
        case BT_ERR_OUT_OF_MEMORY: return "out of device memory";
        case BT_ERR_CUDA: return "CUDA runtime error";
        case BT_ERR_CAPACITY: return "output buffer too small";
        case BT_ERR_NOT_SUPPORTED: return "not supported on this device";
        case BT_ERR_TIMEOUT: return "bounded device wait timed out";
        case BT_ERR_INTERNAL: return "device-side consistency check failed";
    }
    return "unknown status";
}

const char *bt_last_error(void) { return bt::g_last_error.c_str(); }

uint64_t bt_kernel_launches(void) { return bt::g_launches.load(std::memory_order_relaxed); }

uint64_t bt_workspace_allocations(void) { return bt::g_ws_allocs.load(std::memory_order_relaxed); }

}  // extern "C"
