// Harness around the reference implementation's own sources -- TEST
// INFRASTRUCTURE ONLY (parity pinning and the "reference kernels on this GPU"
// baseline).  It is compiled together with the reference's .cu files, where
// they lie, by oracle/Makefile into oracle/_ref/libbtref.so.  The engine never
// links it.
//
// The reference's host wrappers discard their outputs
// (BPTreeExactSearch.cu:483, BtreeRangeSearch.cu:915-916), so this harness
// calls the reference's public build and grouping functions and launches the
// reference's kernels itself, with the launch shapes the wrappers use, and
// copies the results back.
//
// Inputs this harness refuses, because the reference faults or reads out of
// bounds on them (found by reading its code, never run):
//   * n not a multiple of PAGESIZE: main.cu:126-129 claims PAGESIZE keys for
//     the last leaf and assignDataToLeaf reads past the arrays
//     (BPTree.cu:107,113-116);
//   * fewer than 1024 queries for the ungrouped kernels: the grid is
//     floor(n/1024) blocks (BPTreeExactSearch.cu:437);
//   * a range with start > end: the leaf walk runs off the list
//     (BtreeRangeSearch.cu:337-346);
//   * an all-zero query batch in the grouped paths (interval 0 in
//     zOrder2d.cu:129, no grouping pass in grouping.cu:1744).
#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <vector>

#include "utils.h"
#include "BPTree.h"
#include "grouping.h"
#include "grouping2d.h"
#include "zOrder2d.h"

// Kernels defined in the reference's translation units.
__global__ void kernelSearchingNaiveOneStep(const ulli *, BTPage *, const ulli *, ulli, ulli *);
__global__ void kernelSearchingKeyGroupTwoStep(const ulli *, BTPage *, const ulli *, ulli *, ulli *,
                                               ulli, ulli *);
__global__ void kernelSearchingKeyRangeGroupStateTwo(const ulli *, BTPage *, const ulli *, ulli,
                                                     ulli *);
__global__ void kernelGenerateSearchResult(const ulli *, const ulli *, ulli, const ulli *,
                                           const ulli *, ulli *, ulli *, BTPage *);
__global__ void kernelSearchingKeyRangeGroupStateTwoGrouping(const ulli *, BTPage *, const ulli *,
                                                             ulli, ulli *, ulli, ulli *, ulli *);
__global__ void kernelGenerateSearchResultGrouping(const ulli *, const ulli *, ulli, const ulli *,
                                                   const ulli *, ulli *, ulli *, BTPage *, ulli *,
                                                   ulli *, ulli);

namespace {
ulli *g_root = nullptr;       // device u64[1] holding the root page index
BTPage *g_pool = nullptr;     // the reference's page pool
ulli *g_cur_page = nullptr;   // managed page counter
const ulli kBlock = 1024;     // BLOCK_SIZE of the search files
const ulli kMaxBlocks = 65535;

int check(cudaError_t e) {
    if (e != cudaSuccess) {
        fprintf(stderr, "refh: %s\n", cudaGetErrorString(e));
        return 1;
    }
    return 0;
}

struct Timer {
    cudaEvent_t a, b;
    Timer() { cudaEventCreate(&a); cudaEventCreate(&b); cudaEventRecord(a, 0); }
    float stop() {
        float ms = 0.f;
        cudaEventRecord(b, 0);
        cudaEventSynchronize(b);
        cudaEventElapsedTime(&ms, a, b);
        cudaEventDestroy(a);
        cudaEventDestroy(b);
        return ms;
    }
};

ulli basic_blocks(ulli n) { return (n / kBlock) > kMaxBlocks ? kMaxBlocks : n / kBlock; }

// Group-list launch used by all grouped reference kernels.
struct Groups {
    ulli *d_count = nullptr, *d_prefix = nullptr;
    ulli num = 0;
    Groups(const std::vector<ulli> &count, const std::vector<ulli> &prefix) {
        num = count.size();
        cudaMalloc((void **)&d_count, sizeof(ulli) * num);
        cudaMalloc((void **)&d_prefix, sizeof(ulli) * num);
        cudaMemcpy(d_count, count.data(), sizeof(ulli) * num, cudaMemcpyHostToDevice);
        cudaMemcpy(d_prefix, prefix.data(), sizeof(ulli) * num, cudaMemcpyHostToDevice);
    }
    ~Groups() { cudaFree(d_count); cudaFree(d_prefix); }
    ulli blocks() const { return num > kMaxBlocks ? kMaxBlocks : num; }
};
}  // namespace

extern "C" {

void refh_free(void) {
    if (g_pool) cudaFree(g_pool);
    if (g_cur_page) cudaFree(g_cur_page);
    if (g_root) cudaFree(g_root);
    g_pool = nullptr;
    g_cur_page = nullptr;
    g_root = nullptr;
}

// Build through the reference's genBPlusTree with main.cu's leaf plan.
int refh_build(const uint64_t *keys, const uint64_t *data, uint64_t n) {
    if (n == 0 || n % PAGESIZE != 0) return 2;
    refh_free();
    cudaSetDevice(0);
    ulli *d_k = nullptr, *d_d = nullptr;
    if (check(cudaMalloc((void **)&d_k, n * 8)) || check(cudaMalloc((void **)&d_d, n * 8))) return 1;
    cudaMemcpy(d_k, keys, n * 8, cudaMemcpyHostToDevice);
    cudaMemcpy(d_d, data, n * 8, cudaMemcpyHostToDevice);
    std::vector<ulli> groupList, groupPrefix;
    for (ulli i = 0; i < n; i += PAGESIZE) {  // main.cu:126-129
        groupList.push_back(PAGESIZE);
        groupPrefix.push_back(i);
    }
    ulli level = 0, size = 0, *index = nullptr;
    // genBPlusTree frees d_k and d_d (BPTree.cu:210-211).
    genBPlusTree(d_k, d_d, n, groupList, groupPrefix, g_root, level, index, size, g_pool,
                 g_cur_page);
    return check(cudaDeviceSynchronize());
}

uint64_t refh_root(void) {
    ulli r = 0;
    if (g_root) cudaMemcpy(&r, g_root, 8, cudaMemcpyDeviceToHost);
    return r;
}

// kernelSearchingNaiveOneStep with the launch of BPTreeExactSearch.cu:437-444.
int refh_point_basic(const uint64_t *q, uint64_t nq, uint64_t *out, float *ms) {
    if (!g_pool || nq < kBlock) return 2;
    ulli *d_q = nullptr, *d_o = nullptr;
    cudaMalloc((void **)&d_q, nq * 8);
    cudaMalloc((void **)&d_o, nq * 8);
    cudaMemcpy(d_q, q, nq * 8, cudaMemcpyHostToDevice);
    cudaMemset(d_o, 0, nq * 8);
    Timer t;
    kernelSearchingNaiveOneStep<<<basic_blocks(nq), kBlock>>>(g_root, g_pool, d_q, nq, d_o);
    float e = t.stop();
    if (ms) *ms = e;
    int rc = check(cudaGetLastError());
    cudaMemcpy(out, d_o, nq * 8, cudaMemcpyDeviceToHost);
    cudaFree(d_q);
    cudaFree(d_o);
    return rc;
}

// The grouped point search of SearchingBTreeGPUCombineStep
// (BPTreeExactSearch.cu:602-723): genGrouping, then
// kernelSearchingKeyGroupTwoStep one block per group.  q is overwritten with
// the grouped order (as the reference does, :613) and out is in that order.
int refh_point_grouped(uint64_t *q, uint64_t nq, uint64_t *out, float *ms) {
    if (!g_pool || nq == 0) return 2;
    std::vector<ulli> groupList, groupPrefix;
    ulli *d_grouped = (ulli *)genGrouping((ulli *)q, nq, groupList, groupPrefix, GROUP_SEARCH_SIZE);
    cudaMemcpy(q, d_grouped, nq * 8, cudaMemcpyDeviceToHost);
    Groups g(groupList, groupPrefix);
    ulli *d_o = nullptr;
    cudaMalloc((void **)&d_o, nq * 8);
    cudaMemset(d_o, 0, nq * 8);
    Timer t;
    kernelSearchingKeyGroupTwoStep<<<g.blocks(), kBlock>>>(g_root, g_pool, d_grouped, g.d_prefix,
                                                            g.d_count, g.num, d_o);
    float e = t.stop();
    if (ms) *ms = e;
    int rc = check(cudaGetLastError());
    cudaMemcpy(out, d_o, nq * 8, cudaMemcpyDeviceToHost);
    cudaFree(d_o);
    cudaFree(d_grouped);
    return rc;
}

// kernelSearchingKeyRangeGroupStateTwo alone: (pos << 32) | leaf per query.
int refh_range_endpoints(const uint64_t *q, uint64_t nq, uint64_t *out) {
    if (!g_pool || nq < kBlock) return 2;
    ulli *d_q = nullptr, *d_o = nullptr;
    cudaMalloc((void **)&d_q, nq * 8);
    cudaMalloc((void **)&d_o, nq * 8);
    cudaMemcpy(d_q, q, nq * 8, cudaMemcpyHostToDevice);
    kernelSearchingKeyRangeGroupStateTwo<<<basic_blocks(nq), kBlock>>>(g_root, g_pool, d_q, nq, d_o);
    int rc = check(cudaDeviceSynchronize());
    cudaMemcpy(out, d_o, nq * 8, cudaMemcpyDeviceToHost);
    cudaFree(d_q);
    cudaFree(d_o);
    return rc;
}

static int ranges_ok(const uint64_t *lo, const uint64_t *hi, uint64_t nq) {
    for (uint64_t i = 0; i < nq; i++)
        if (lo[i] > hi[i]) return 0;
    return 1;
}

// SearchingBTreeGPURange (BtreeRangeSearch.cu:786-925), returning the counts.
int refh_range_basic(const uint64_t *lo, const uint64_t *hi, uint64_t nq, uint64_t *counts,
                     float *ms) {
    if (!g_pool || nq < kBlock || !ranges_ok(lo, hi, nq)) return 2;
    ulli *d_lo, *d_hi, *d_elo, *d_ehi, *d_cnt, *d_off;
    cudaMalloc((void **)&d_lo, nq * 8);
    cudaMalloc((void **)&d_hi, nq * 8);
    cudaMalloc((void **)&d_elo, nq * 8);
    cudaMalloc((void **)&d_ehi, nq * 8);
    cudaMalloc((void **)&d_cnt, nq * 8 * DOB_PAGE_SIZE);
    cudaMalloc((void **)&d_off, nq * 8);
    cudaMemcpy(d_lo, lo, nq * 8, cudaMemcpyHostToDevice);
    cudaMemcpy(d_hi, hi, nq * 8, cudaMemcpyHostToDevice);
    cudaMemset(d_cnt, 0, nq * 8 * DOB_PAGE_SIZE);
    ulli b = basic_blocks(nq);
    Timer t;
    kernelSearchingKeyRangeGroupStateTwo<<<b, kBlock>>>(g_root, g_pool, d_lo, nq, d_elo);
    kernelSearchingKeyRangeGroupStateTwo<<<b, kBlock>>>(g_root, g_pool, d_hi, nq, d_ehi);
    kernelGenerateSearchResult<<<b, kBlock>>>(d_lo, d_hi, nq, d_elo, d_ehi, d_cnt, d_off, g_pool);
    float e = t.stop();
    if (ms) *ms = e;
    int rc = check(cudaGetLastError());
    cudaMemcpy(counts, d_cnt, nq * 8, cudaMemcpyDeviceToHost);
    cudaFree(d_lo); cudaFree(d_hi); cudaFree(d_elo); cudaFree(d_ehi); cudaFree(d_cnt); cudaFree(d_off);
    return rc;
}

// SearchingBTreeGPURangeWithGrouping (mode 1, BtreeRangeSearch.cu:377-575) or
// ...WithGroupingZorder (mode 2, :578-783), returning the counts.  lo and hi
// are overwritten with the grouped order; counts are in that order.
int refh_range_grouped(int mode, uint64_t *lo, uint64_t *hi, uint64_t nq, uint64_t *counts,
                       float *ms) {
    if (!g_pool || nq == 0 || !ranges_ok(lo, hi, nq)) return 2;
    std::vector<ulli> groupList, groupPrefix;
    ulli *g_lo = nullptr, *g_hi = nullptr;
    if (mode == 1) {
        genGrouping2d((ulli *)lo, (ulli *)hi, nq, groupList, g_lo, g_hi, groupPrefix,
                      GROUP_SEARCH_SIZE);
    } else if (mode == 2) {
        ulli *z = nullptr, *gz = nullptr;
        genGrouping2dZ((ulli *)lo, (ulli *)hi, z, nq);
        genGroupingWithTwodata(z, (ulli *)lo, (ulli *)hi, nq, gz, g_lo, g_hi, groupList,
                               groupPrefix, GROUP_SEARCH_SIZE);
        delete[] z;
        delete[] gz;
    } else {
        return 2;
    }
    for (uint64_t i = 0; i < nq; i++) {
        lo[i] = g_lo[i];
        hi[i] = g_hi[i];
    }
    delete[] g_lo;
    delete[] g_hi;
    Groups g(groupList, groupPrefix);
    ulli *d_lo, *d_hi, *d_elo, *d_ehi, *d_cnt, *d_off;
    cudaMalloc((void **)&d_lo, nq * 8);
    cudaMalloc((void **)&d_hi, nq * 8);
    cudaMalloc((void **)&d_elo, nq * 8);
    cudaMalloc((void **)&d_ehi, nq * 8);
    cudaMalloc((void **)&d_cnt, nq * 8 * DOB_PAGE_SIZE);
    cudaMalloc((void **)&d_off, nq * 8);
    cudaMemcpy(d_lo, lo, nq * 8, cudaMemcpyHostToDevice);
    cudaMemcpy(d_hi, hi, nq * 8, cudaMemcpyHostToDevice);
    cudaMemset(d_cnt, 0, nq * 8 * DOB_PAGE_SIZE);
    Timer t;
    kernelSearchingKeyRangeGroupStateTwoGrouping<<<g.blocks(), kBlock>>>(
        g_root, g_pool, d_lo, nq, d_elo, g.num, g.d_prefix, g.d_count);
    kernelSearchingKeyRangeGroupStateTwoGrouping<<<g.blocks(), kBlock>>>(
        g_root, g_pool, d_hi, nq, d_ehi, g.num, g.d_prefix, g.d_count);
    kernelGenerateSearchResultGrouping<<<g.blocks(), kBlock>>>(d_lo, d_hi, nq, d_elo, d_ehi, d_cnt,
                                                              d_off, g_pool, g.d_prefix, g.d_count,
                                                              g.num);
    float e = t.stop();
    if (ms) *ms = e;
    int rc = check(cudaGetLastError());
    cudaMemcpy(counts, d_cnt, nq * 8, cudaMemcpyDeviceToHost);
    cudaFree(d_lo); cudaFree(d_hi); cudaFree(d_elo); cudaFree(d_ehi); cudaFree(d_cnt); cudaFree(d_off);
    return rc;
}

}  // extern "C"
