// btree -- the reference program's command line, served by this engine.
//
// Same arguments and flow as the reference's main.cu (main.cu:20-355):
//
//   btree inputSize keyFile dataFile                         build only
//   btree inputSize keyFile dataFile querySize queryFile     point searches
//   btree inputSize keyFile dataFile querySize startFile endFile   ranges
//
// Files hold raw host-endian u64 values with no header (main.cu:33-55).
// The pairs are uploaded, sorted on the device (bt_sort_pairs in place of
// the reference's cub::DeviceRadixSort::SortPairs, main.cu:109-118) and
// handed to genBPlusTree, which frees them (BPTree.cu:209-211).  Then, as in
// main.cu:189-215, SearchingBTreeGPUCombineStep on the query file and
// SearchingBTreeGPUOnlyOneState on a fresh read of it; or, as in
// main.cu:307-355, the three range searches, each on fresh reads of the
// start and end files.  Every call goes through the reference's own C++ API
// (include/btree_b200_compat.h), so this program is also the check that a
// reference caller runs on the engine unchanged.
//
// One addition: when the environment variable BTREE_RESULTS_DIR names a
// directory, the outputs the reference computes and discards are written
// there as raw u64 files (combine_results.bin and combine_keys.bin: the
// results and the caller's query array after the grouped call, both in
// grouped order; naive_results.bin; range_basic.bin, range_2d.bin,
// range_zorder.bin: per-range counts).
#include <cuda_runtime.h>

#include <cerrno>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <string>
#include <vector>

#include "btree_b200_compat.h"

namespace {

bool read_u64(const char *path, ulli *dst, ulli n) {
    std::ifstream f(path, std::ios::binary | std::ios::in);
    if (f.fail()) {
        std::cerr << "Error: " << strerror(errno) << std::endl;
        return false;
    }
    f.read(reinterpret_cast<char *>(dst), (std::streamsize)(sizeof(ulli) * n));
    if ((ulli)f.gcount() != sizeof(ulli) * n) {
        std::cerr << "Error: " << path << " holds fewer than " << n << " values" << std::endl;
        return false;
    }
    return true;
}

void dump(const char *name, const ulli *p, ulli n) {
    const char *dir = std::getenv("BTREE_RESULTS_DIR");
    if (!dir || !*dir) return;
    const std::string path = std::string(dir) + "/" + name;
    FILE *f = std::fopen(path.c_str(), "wb");
    if (!f) {
        std::cerr << "Error: cannot write " << path << std::endl;
        std::exit(1);
    }
    if (n && std::fwrite(p, sizeof(ulli), n, f) != n) {
        std::cerr << "Error: short write to " << path << std::endl;
        std::exit(1);
    }
    std::fclose(f);
}

void dump_last(const char *name) {
    ulli n = 0;
    const ulli *r = bt_compat_last_results(&n);
    dump(name, r, n);
}

void cuda_or_exit(cudaError_t e, const char *what) {
    if (e != cudaSuccess) {
        std::cerr << "GPUassert: " << what << ": " << cudaGetErrorString(e) << std::endl;
        std::exit((int)e);
    }
}

}  // namespace

int main(int argc, char *argv[]) {
    if (argc < 4) {
        std::cerr << "usage:" << argv[0] << " inputSize fileNameKey filenameData" << std::endl;
        return -1;
    }
    if (std::strlen(argv[1]) > 18) {
        std::cerr << "Error inputSize greater than long long" << std::endl;
        return -1;
    }
    std::cout << "Init Algorithm with PageSize " << PAGESIZE << std::endl;
    const ulli inputSize = std::strtoull(argv[1], nullptr, 10);
    std::vector<ulli> input(inputSize), inputData(inputSize);
    if (!read_u64(argv[2], input.data(), inputSize) ||
        !read_u64(argv[3], inputData.data(), inputSize))
        return -1;
    std::cout << "Init problem complete." << std::endl;
    std::cout << "Problem Size: " << inputSize / 1000000 << " Million Key" << std::endl;

    // upload and sort the (key, data) pairs; genBPlusTree takes the sorted
    // arrays and frees them
    cuda_or_exit(cudaSetDevice(0), "cudaSetDevice");
    ulli *d_in = nullptr, *d_in_data = nullptr, *d_out = nullptr, *d_out_data = nullptr;
    const size_t bytes = sizeof(ulli) * (inputSize ? inputSize : 1);
    cuda_or_exit(cudaMalloc(&d_in, bytes), "cudaMalloc");
    cuda_or_exit(cudaMalloc(&d_in_data, bytes), "cudaMalloc");
    cuda_or_exit(cudaMalloc(&d_out, bytes), "cudaMalloc");
    cuda_or_exit(cudaMalloc(&d_out_data, bytes), "cudaMalloc");
    cuda_or_exit(cudaMemcpy(d_in, input.data(), sizeof(ulli) * inputSize, cudaMemcpyHostToDevice),
                 "cudaMemcpy");
    cuda_or_exit(cudaMemcpy(d_in_data, inputData.data(), sizeof(ulli) * inputSize,
                            cudaMemcpyHostToDevice),
                 "cudaMemcpy");
    const bt_status st = bt_sort_pairs(d_in, d_in_data, inputSize, 8, 8, d_out, d_out_data, nullptr);
    if (st != BT_OK) {
        std::cerr << "GPUassert: sort: " << bt_status_string(st) << " (" << bt_last_error() << ")"
                  << std::endl;
        return (int)st;
    }
    cuda_or_exit(cudaDeviceSynchronize(), "sort");
    cudaFree(d_in);
    cudaFree(d_in_data);

    std::vector<ulli> groupList, groupPrefix;  // the reference's leaf plan; unused by the engine
    for (ulli i = 0; i < inputSize; i += PAGESIZE) {
        groupList.push_back(PAGESIZE);
        groupPrefix.push_back(i);
    }
    ulli *dev_btree = nullptr;
    ulli treeLevel = 0;
    ulli *btreeIndex = nullptr;
    ulli bTreeSize = 0;
    BTPage *dev_globalPointer = nullptr;
    ulli *dev_currentPage = nullptr;
    std::cout << "Data sorted and building the Tree." << std::endl;
    genBPlusTree(d_out, d_out_data, inputSize, groupList, groupPrefix, dev_btree, treeLevel,
                 btreeIndex, bTreeSize, dev_globalPointer, dev_currentPage);

    if (argc == 6) {
        const ulli nq = std::strtoull(argv[4], nullptr, 10);
        std::vector<ulli> input_key(nq ? nq : 1);
        std::cout << "=================================================================" << std::endl;
        if (!read_u64(argv[5], input_key.data(), nq)) return -1;
        std::cout << "Init Searching key complete." << std::endl;
        std::cout << "Problem Key Size: " << nq / 1000000 << " Million Key" << std::endl;
        ulli *result0 = (ulli *)SearchingBTreeGPUCombineStep(input_key.data(), nq, dev_btree,
                                                             dev_globalPointer);
        dump("combine_results.bin", result0, nq);
        dump("combine_keys.bin", input_key.data(), nq);
        delete[] result0;
        std::cout << "=================================================================" << std::endl;
        if (!read_u64(argv[5], input_key.data(), nq)) return -1;
        std::cout << "Init Searching key complete." << std::endl;
        std::cout << "Problem Key Size: " << nq / 1000000 << " Million Key" << std::endl;
        SearchingBTreeGPUOnlyOneState(input_key.data(), nq, dev_btree, dev_globalPointer);
        dump_last("naive_results.bin");
        std::cout << "-----------------------------------------------------------------" << std::endl;
    }
    if (argc == 7) {
        const ulli nq = std::strtoull(argv[4], nullptr, 10);
        std::vector<ulli> start(nq ? nq : 1), end(nq ? nq : 1);
        auto reload = [&] { return read_u64(argv[5], start.data(), nq) && read_u64(argv[6], end.data(), nq); };
        if (!reload()) return -1;
        std::cout << "Init Searching key complete." << std::endl;
        std::cout << "Problem Key Size: " << nq / 1000000 << " Million Key" << std::endl;
        SearchingBTreeGPURange(start.data(), end.data(), nq, dev_btree, dev_globalPointer);
        dump_last("range_basic.bin");
        std::cout << ">>>>>>>>>>>>>>>>>>>>>>>>>>>>>>>>>>>>>>>>>>>>>>>>>>>>>>>>>>>>>>>>" << std::endl;
        if (!reload()) return -1;
        SearchingBTreeGPURangeWithGrouping(start.data(), end.data(), nq, dev_btree, dev_globalPointer);
        dump_last("range_2d.bin");
        std::cout << "=================================================================" << std::endl;
        if (!reload()) return -1;
        SearchingBTreeGPURangeWithGroupingZorder(start.data(), end.data(), nq, dev_btree,
                                                 dev_globalPointer);
        dump_last("range_zorder.bin");
        std::cout << "-----------------------------------------------------------------" << std::endl;
        std::cout << std::endl;
    }
    return 0;
}
