// Internal definitions shared by the engine's translation units.
//
// Tree layout in HBM (one allocation per array, 256-byte aligned):
//
//   leaves  the sorted keys and their values in leaf blocks.  Block b holds
//           keys b*S .. b*S+S-1 (S = 32 / sizeof(key): one 32-byte DRAM
//           sector) followed by the same positions' values, the block padded
//           to a power of two (64 bytes, or 128 for 4-byte keys with 8-byte
//           values).  A point-search hit needs one block: its key sector and
//           value sector come in the same 64-byte DRAM access.  Unused key
//           slots of the last block hold the all-ones key.
//   seps    separator levels, stored root first.  Level t holds nodes of
//           F = 128 / sizeof(key) separators (one 128-byte line).  A
//           separator is the maximum key of the node (or leaf block) below
//           it, as in the reference's internal pages (BPTree.cu:54-55).
//
// Child j of node i at level t is node i*F + j of level t+1; the children of
// the bottom level are leaf blocks.  No pointers are stored.  A search for
// q <= max_key takes, at every level, the first separator >= q (lower bound)
// or > q (upper bound); padding separators are all-ones and never win.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "../../include/btree_b200.h"

#define BT_VERSION_NUMBER 10000

namespace bt {

constexpr int kLineBytes = 128;   // internal node size
constexpr int kSectorBytes = 32;  // leaf sector size
constexpr int kMaxLevels = 24;

// Shared-memory budget for the separator level a search CTA stages (the
// deepest level that fits is staged and binary-searched per query).
constexpr size_t kSmemTopBudget = 96 * 1024;

// Leaf block geometry for key type K and value type V.
template <typename K, typename V>
struct LeafGeom {
    static constexpr int S = kSectorBytes / (int)sizeof(K);  // keys per block
    static constexpr int VB = S * (int)sizeof(V);             // value bytes per block
    static constexpr int BS = (kSectorBytes + VB) <= 64 ? 64 : 128;  // block stride
};

inline int leaf_stride(int key_bytes, int val_bytes) {
    const int vb = (kSectorBytes / key_bytes) * val_bytes;
    return (kSectorBytes + vb) <= 64 ? 64 : 128;
}

struct DevTree {
    const void *leaves;
    const void *seps;
    uint64_t n;
    uint64_t max_key;
    uint64_t n_sectors;
    uint64_t lvl_off[kMaxLevels];  // element offset of level t in seps (t = 0 is the root)
    int nlevels;
    int smem_level;                // level staged in shared memory (resolves levels 0..smem_level)
    uint32_t smem_entries;         // its real separators
    uint32_t smem_bytes;           // bytes staged (a multiple of 16)
};

// ---- learned index (see bt_learned.cu) ----------------------------------

constexpr int kSegPerLine = 4;      // segments per segment line
constexpr int kCodesPerLine = 59;   // thresholds per code line
constexpr int kUnitBytes = 128;     // a leaf unit: the 128-byte aligned piece of the leaf array

// One segment (leaf model): it covers the keys [key, next segment's key),
// ranks r_lo .. r_lo + cnt - 1; rank ~ r_lo + clamp(icpt + slope * (q -
// key), 0, cnt) within eps of the truth for every key of the segment.
struct SegRec {
    uint64_t key;
    uint32_t r_lo, cnt;
    float slope, icpt;
    uint32_t eps, pad;
};

// Four consecutive segments in one 128-byte line, 32 bytes each, so that
// each lane of a pair reading a 64-byte half holds two whole segments.
// Unused slots of the last line: key all-ones, r_lo = n, cnt = 0.
struct SegLine {
    SegRec s[kSegPerLine];
};

// Thresholds between consecutive leaf units, 59 per 128-byte line.
// Threshold j separates unit j from unit j + 1: T_j = base + (code << shift)
// is the smallest such value above the largest key of unit j, so q >= T_j
// iff q >= base and ((q - base) >> shift) >= code.  Codes are 15-bit values
// (at most kCodeMax; kCodePad marks a slot past the last threshold), so that
// two of them in a 32-bit word compare against the key in one subtraction.
constexpr uint32_t kCodeMax = 0x7FFEu;
constexpr uint32_t kCodePad = 0x7FFFu;

struct CodeLine {
    uint64_t base;
    uint16_t shift;
    uint16_t code[kCodesPerLine];
};

constexpr int kMaxHidden = 32;

// Device view of a trained learned index.
struct LearnedDev {
    const float *mlp;        // root parameters (3*hidden+1)
    const SegLine *seg;      // segment lines
    const CodeLine *codes;   // code lines
    const void *stage;       // first key of every segment line (key type), nls entries
    unsigned long long *stats;  // [extra leaf-unit reads, full-descent fallbacks] of the last search
    uint64_t kmin;           // root input: x = (key - kmin) * xscale
    float xscale;
    int hidden;
    uint32_t nseg;           // segments
    uint32_t nls;            // segment lines
    uint32_t root_err;       // |root's line prediction - line| <= root_err at every staged key
    uint32_t kpu;            // keys per leaf unit
    uint64_t units;          // leaf units
    uint32_t stage_bytes;    // shared-memory bytes of the staged keys (whole bank rows)
};

struct LearnedState;

}  // namespace bt

struct bt_tree {
    int device;
    int key_bytes;
    int val_bytes;
    uint64_t n;
    uint64_t n_sectors;
    void *d_leaves;
    void *d_seps;
    uint64_t seps_elems;
    uint64_t lvl_nodes[bt::kMaxLevels];
    uint64_t lvl_entries[bt::kMaxLevels];
    uint64_t min_key, max_key;
    int values_sorted;
    int search_cfg;  // index into the search kernels' (lanes, rounds) table
    bt::DevTree dev;
    bt::LearnedState *learned;  // trained learned index, or null
};

namespace bt {

// Thread-local error detail, set by fail().
void set_error(const std::string &msg);
bt_status fail(bt_status s, const std::string &msg);
bt_status cuda_fail(cudaError_t e, const char *what);

#define BT_CUDA(call)                                            \
    do {                                                         \
        cudaError_t e__ = (call);                                \
        if (e__ != cudaSuccess) return ::bt::cuda_fail(e__, #call); \
    } while (0)

// Stream-ordered allocation from the engine's own memory pool on the
// current device (cached between calls, never returned to other users).
bt_status ws_alloc(void **p, size_t bytes, cudaStream_t s);
void ws_free(void *p, cudaStream_t s);

// A workspace allocation returned to the pool (stream-ordered) when the
// guard leaves scope, on every path out of the function.
struct WsGuard {
    void *p = nullptr;
    cudaStream_t s;
    explicit WsGuard(cudaStream_t st) : s(st) {}
    WsGuard(const WsGuard &) = delete;
    WsGuard &operator=(const WsGuard &) = delete;
    ~WsGuard() {
        if (p) ws_free(p, s);
    }
    bt_status alloc(size_t bytes) { return ws_alloc(&p, bytes, s); }
    template <typename T>
    T *as() const { return static_cast<T *>(p); }
};

// Counts one kernel launch (bt_kernel_launches).
void count_launch();
// Number of SMs of the current device (cached).
int sm_count();
// Checks the current device is sm_100 class.
bt_status require_device(int device);

template <typename K>
__host__ __device__ constexpr K key_max() {
    return (K)~(K)0;
}

inline int bitlen64(uint64_t v) {
    int b = 0;
    while (v) {
        v >>= 1;
        b++;
    }
    return b;
}

// Host launchers implemented in the .cu files.
bt_status launch_point_search(const bt_tree *t, const void *d_q, const uint32_t *d_perm,
                              uint64_t nq, void *d_out, cudaStream_t s,
                              uint8_t *d_found = nullptr);
bt_status launch_bounds(const bt_tree *t, const void *d_lo, const void *d_hi,
                        const uint32_t *d_perm, uint64_t nq, uint64_t *d_counts,
                        uint64_t *d_lb, cudaStream_t s);
bt_status launch_partition(const bt_tree *t, int kind, const void *d_a, const void *d_b,
                           uint64_t nq, void *d_out_a, void *d_out_b, uint32_t *d_perm,
                           cudaStream_t s);
bt_status launch_scan_u64(const uint64_t *d_in, uint64_t *d_out, uint64_t n, uint64_t *d_total,
                          cudaStream_t s);
// Point-query partition into caller memory: ws must hold
// partition_point_ws_bytes(nq) bytes; nothing is allocated.
size_t partition_point_ws_bytes(uint64_t nq);
bt_status launch_partition_point_prealloc(const bt_tree *t, const void *d_q, uint64_t nq,
                                          void *out_q, uint32_t *out_perm, void *ws,
                                          cudaStream_t s);
bt_status launch_range_fill(const bt_tree *t, const uint64_t *d_lb, const uint64_t *d_counts,
                            const uint64_t *d_offsets, uint64_t nq, void *d_ids, cudaStream_t s);
// Stable sort of n (key, value) pairs by key on the device: LSD radix sort
// with 8-bit digits (key_bytes passes of the partition kernels, carrying the
// input index), then one gather of the values.  Equal keys keep their input
// order.  n < 2^32; outputs must not alias inputs.
bt_status launch_sort_pairs(int key_bytes, int value_bytes, const void *d_keys, const void *d_vals,
                            uint64_t n, void *out_keys, void *out_vals, cudaStream_t s);
// Stable order of n 16-bit keys (the low halves of d_keys): d_perm[g] = the
// index of the item in position g (two 8-bit passes of the partition).
bt_status launch_order_u16(const uint32_t *d_keys, uint64_t n, uint32_t *d_perm, cudaStream_t s);
// Sorts each segment ids[offsets[i] .. + counts[i]) ascending (value width
// of t).  small_sorted: segments of up to 256 values are sorted already.
bt_status launch_segment_sort(const bt_tree *t, const uint64_t *d_counts, const uint64_t *d_offsets,
                              uint64_t nseg, void *d_ids, cudaStream_t s, bool small_sorted = false);

// (lanes per query, rounds) -> index of the search configuration table in
// bt_search.cu, or -1.
int search_cfg_index(int lanes, int rounds);
int default_search_cfg(int key_bytes);
int search_cfg_lanes(int cfg);
int search_cfg_rounds(int cfg);

void free_learned(bt::LearnedState *s);
// Learned point search of d_q into d_out on s (the tree has a learned index;
// the counters of bt_learned_last_stats accumulate).
bt_status launch_learned_search(const bt_tree *t, const void *d_q, uint64_t nq, void *d_out,
                                uint8_t *d_found, cudaStream_t s);
// Zeroes those counters (stream-ordered).
bt_status reset_learned_stats(const bt_tree *t, cudaStream_t s);

// Partition kinds for launch_partition.
enum PartitionKind { kPartPoint = 0, kPart2D = 1, kPartZ = 2, kPartRadix = 3 };
// Digit bits used by the grouping passes.
constexpr int kPointGroupBits = 8;
constexpr int kRangeGroupBits = 8;

}  // namespace bt
