/*
 * btree_b200.h -- C ABI of the B200 B+tree index engine.
 *
 * This is the engine's real interface: plain pointers, sizes and status
 * codes, no C++ types.  It replaces the reference's C++ host API
 * (BPTree.h:26-55, grouping.h:6-28, grouping2d.h:8-10, zOrder2d.h:8); the
 * C++ compatibility shim with the reference's exact signatures is in
 * btree_b200_compat.h and is implemented on top of these functions.
 *
 * Conventions (all functions):
 *   - Every call returns a bt_status; nothing calls exit().  A thread-local
 *     message with details is available from bt_last_error().
 *   - `stream` is a cudaStream_t passed as void* (NULL = legacy default
 *     stream).  Device-pointer calls are asynchronous on that stream unless
 *     stated otherwise; host-pointer calls (suffix _host) return after the
 *     results are in host memory.
 *   - The caller keeps ownership of every buffer it passes.
 *   - Results always come back in the caller's query order, also for the
 *     grouped modes (the reference returns grouped order instead,
 *     BPTreeExactSearch.cu:613,722).
 *   - Keys are unsigned integers of 4 or 8 bytes, values of 4 or 8 bytes.
 *     A point-search miss yields the all-ones value of the value width
 *     (INVALID_DATA, BPTree.h:12, for 8-byte values).
 *   - Duplicate keys are allowed.  A point search returns the value at the
 *     first occurrence (std::lower_bound), a range search counts every
 *     occurrence.
 */
#ifndef BTREE_B200_H
#define BTREE_B200_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define BT_API __attribute__((visibility("default")))
#else
#define BT_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef enum bt_status {
    BT_OK = 0,
    BT_ERR_INVALID_ARGUMENT = 1, /* null pointer, bad width, bad mode, size limit */
    BT_ERR_UNSORTED = 2,         /* build keys are not in ascending order */
    BT_ERR_OUT_OF_MEMORY = 3,    /* device allocation failed */
    BT_ERR_CUDA = 4,             /* a CUDA runtime call failed */
    BT_ERR_CAPACITY = 5,         /* the caller's output buffer is too small */
    BT_ERR_NOT_SUPPORTED = 6,    /* no sm_100 device, or feature not built */
    BT_ERR_TIMEOUT = 7,          /* a bounded device wait gave up */
    BT_ERR_INTERNAL = 8          /* a device-side consistency check failed */
} bt_status;

typedef enum bt_point_mode {
    BT_POINT_BASIC = 0,  /* SearchingBTreeGPUOnlyOneState, BPTreeExactSearch.cu:409 */
    BT_POINT_GROUPED = 1, /* SearchingBTreeGPUCombineStep, BPTreeExactSearch.cu:602 */
    BT_POINT_LEARNED = 2  /* through the tree's learned index (bt_learned_train); no
                             counterpart in the reference */
} bt_point_mode;

typedef enum bt_range_mode {
    BT_RANGE_BASIC = 0,      /* SearchingBTreeGPURange, BtreeRangeSearch.cu:786 */
    BT_RANGE_GROUPED_2D = 1, /* SearchingBTreeGPURangeWithGrouping, BtreeRangeSearch.cu:377 */
    BT_RANGE_ZORDER = 2      /* SearchingBTreeGPURangeWithGroupingZorder, BtreeRangeSearch.cu:578 */
} bt_range_mode;

typedef struct bt_tree bt_tree;

typedef struct bt_info {
    uint64_t num_keys;
    uint32_t key_bytes;
    uint32_t value_bytes;
    uint32_t num_levels;   /* separator levels above the leaf sectors */
    uint32_t fanout;       /* separators per internal node (one 128-byte line) */
    uint32_t leaf_keys;    /* keys per leaf sector (one 32-byte sector) */
    uint32_t smem_levels;  /* top levels resolved by the shared-memory binary search */
    uint64_t device_bytes; /* HBM held by the tree */
    uint64_t min_key;
    uint64_t max_key;
    int32_t device;
    int32_t values_sorted;      /* values ascend with keys (range IDs need no sort) */
    uint32_t lanes_per_query;   /* search kernel configuration (see bt_set_search_config) */
    uint32_t rounds;
} bt_info;

/* Library version as MAJOR*10000 + MINOR*100 + PATCH. */
BT_API int bt_version(void);
/* Static string for a status code. */
BT_API const char *bt_status_string(bt_status s);
/* Details of the last failure on the calling thread ("" if none). */
BT_API const char *bt_last_error(void);

/*
 * Bulk build from keys sorted ascending (device memory) and their values.
 * Replaces genBPlusTree (BPTree.cu:127-306) together with the leaf plan of
 * main.cu:126-129.  Unlike the reference, the inputs are not freed and are
 * not referenced after the call returns (the tree keeps its own copy).
 * Synchronizes `stream` (it reads back the sortedness check).
 * n == 0 builds an empty tree (every search misses).
 */
BT_API bt_status bt_build(const void *d_sorted_keys, const void *d_values, uint64_t n,
                   int key_bytes, int value_bytes, void *stream, bt_tree **out);

/* Same, from host memory (pageable or pinned). */
BT_API bt_status bt_build_host(const void *h_sorted_keys, const void *h_values, uint64_t n,
                        int key_bytes, int value_bytes, void *stream, bt_tree **out);

/*
 * Stable sort of n (key, value) pairs by key on the device into separate
 * output arrays (which must not alias the inputs): an LSD radix sort with
 * 8-bit digits; equal keys keep their input order.  Replaces the
 * cub::DeviceRadixSort::SortPairs call the reference's main.cu runs before
 * its build (main.cu:109-118).  n < 2^32.  Asynchronous on `stream`.
 */
BT_API bt_status bt_sort_pairs(const void *d_keys, const void *d_values, uint64_t n, int key_bytes,
                               int value_bytes, void *d_keys_out, void *d_values_out, void *stream);

/* bt_build from unsorted device pairs: bt_sort_pairs into engine scratch,
 * then bt_build (the reference's main.cu:109-129 sequence). */
BT_API bt_status bt_build_unsorted(const void *d_keys, const void *d_values, uint64_t n,
                                   int key_bytes, int value_bytes, void *stream, bt_tree **out);

/*
 * Build from the reference program's input files: `keys_path` and
 * `values_path` each hold at least n raw host-endian 64-bit values with no
 * header (the files main.cu:33-55 reads); the pairs need not be sorted.
 * Reads both, uploads them, sorts on the device and builds (main.cu:64-129
 * with genBPlusTree).  u64 keys and values.  Synchronous.
 */
BT_API bt_status bt_build_from_files(const char *keys_path, const char *values_path, uint64_t n,
                                     void *stream, bt_tree **out);

/*
 * Tree image (no counterpart in the reference, which rebuilds from its input
 * files every run): bt_save writes the built leaf blocks, separator levels
 * and their descriptor to one file; bt_load reads it back onto the current
 * device as a tree that searches exactly like the saved one (its search
 * configuration is the default; a trained learned model is not saved).
 * The image is raw device layout: read it on a machine of the same
 * endianness.  Both are synchronous.
 */
BT_API bt_status bt_save(const bt_tree *tree, const char *path);
BT_API bt_status bt_load(const char *path, void *stream, bt_tree **out);

/* Free every device resource of a tree.  NULL is accepted. */
BT_API bt_status bt_destroy(bt_tree *tree);

BT_API bt_status bt_get_info(const bt_tree *tree, bt_info *info);

/*
 * Search-kernel configuration of a tree: lanes of a warp that share one query
 * on the levels below shared memory (2, 4 or 8) and the number of rounds in
 * which a warp's 32 queries pass through those levels (1 or 2; each lane
 * group keeps lanes/rounds queries in flight).  Supported pairs: (8,1) (8,2)
 * (4,1) (4,2) (2,1).  Results do not depend on it; speed does.  The
 * reference has no such knob (one thread per query, BPTreeExactSearch.cu:31);
 * the autotuner sets it.
 */
BT_API bt_status bt_set_search_config(bt_tree *tree, int lanes_per_query, int rounds);

/*
 * Point search: d_out[i] = value of key d_queries[i], or all-ones on a miss.
 * Replaces kernelSearchingNaiveOneStep (BPTreeExactSearch.cu:25, mode
 * BASIC) and genGrouping + kernelSearchingKeyGroupTwoStep
 * (grouping.cu:1677, BPTreeExactSearch.cu:207, mode GROUPED).
 * Queries have key_bytes each, outputs value_bytes each; nq < 2^32.
 */
BT_API bt_status bt_point_search(const bt_tree *tree, int mode, const void *d_queries, uint64_t nq,
                          void *d_out, void *stream);

/*
 * Point search with a found flag per query: as bt_point_search, and
 * d_found[i] = 1 when key d_queries[i] is in the tree, else 0 (one byte per
 * query).  The flag tells a stored value of all-ones from a miss, which the
 * value alone cannot (the reference returns INVALID_DATA, BPTree.h:12, for
 * both).  Same modes and limits as bt_point_search.
 */
BT_API bt_status bt_point_search_found(const bt_tree *tree, int mode, const void *d_queries,
                                       uint64_t nq, void *d_out, uint8_t *d_found, void *stream);

/* Same with host buffers; copies are pipelined with the search in chunks.
 * Returns when h_out is filled. */
BT_API bt_status bt_point_search_host(const bt_tree *tree, int mode, const void *h_queries,
                               uint64_t nq, void *h_out, void *stream);

/*
 * The grouping step alone (genGrouping, grouping.cu:1677): writes the
 * queries in grouped order to d_grouped and, for each grouped slot, the
 * caller's index of that query to d_perm (u32).  The order is a stable
 * partition by the top bits of the key, deterministic for a given tree.
 */
BT_API bt_status bt_group_queries(const bt_tree *tree, const void *d_queries, uint64_t nq,
                           void *d_grouped, uint32_t *d_perm, void *stream);

/*
 * Search a batch already grouped by bt_group_queries: d_out[d_perm[i]] =
 * value of d_grouped[i].  This is the search stage of BT_POINT_GROUPED on
 * its own, for callers that group once and search repeatedly (and the
 * kernel a benchmark times alone).  d_perm must be a permutation of 0..nq-1.
 */
BT_API bt_status bt_point_search_grouped_batch(const bt_tree *tree, const void *d_grouped,
                                               const uint32_t *d_perm, uint64_t nq, void *d_out,
                                               void *stream);

/*
 * Grouped point search that allocates no device memory (no counterpart in
 * the reference).  Same results as bt_point_search(BT_POINT_GROUPED), for
 * callers that cannot let a library allocate -- a process whose device
 * memory is reserved by its own allocator, or a latency-critical path where
 * an allocation could block.  Its scratch is a fixed 4 MiB array inside the
 * library (present on every GPU that loads it, until exit), so nq is limited
 * to 262144 per call (larger batches: BT_ERR_INVALID_ARGUMENT).  All calls on
 * a device share that array: calls that overlap on the GPU race.  The first
 * call on each device looks up the array's address; make it before any
 * stream capture.  The address is kept for the life of the process: after a
 * cudaDeviceReset (which ends the context it belongs to) this entry point
 * must not be called again on that device.
 */
BT_API bt_status bt_point_search_grouped_noalloc(const bt_tree *tree, const void *d_queries,
                                                 uint64_t nq, void *d_out, void *stream);

/*
 * Range count over inclusive intervals [d_lo[i], d_hi[i]]: d_counts[i] = number
 * of keys k with lo <= k <= hi (0 when lo > hi).  Replaces
 * kernelSearchingKeyRangeGroupStateTwo + kernelGenerateSearchResult
 * (BtreeRangeSearch.cu:215,297) and their grouped twins (:33,:123), whose
 * counts the reference never returns.  mode selects the query reordering
 * (bt_range_mode); results do not depend on it.
 */
BT_API bt_status bt_range_count(const bt_tree *tree, int mode, const void *d_lo, const void *d_hi,
                         uint64_t nq, uint64_t *d_counts, void *stream);

/*
 * Range search with hit IDs: counts as above, d_offsets = exclusive scan of
 * the counts, and d_ids[d_offsets[i] .. + d_counts[i]) = the values of the
 * hit keys of query i, sorted ascending.  *h_total receives the total hit
 * count.  If it exceeds ids_capacity (in values) the call returns
 * BT_ERR_CAPACITY with counts, offsets and *h_total filled and d_ids
 * untouched.  Synchronizes `stream` (it reads the total back).
 */
BT_API bt_status bt_range_search(const bt_tree *tree, int mode, const void *d_lo, const void *d_hi,
                          uint64_t nq, uint64_t *d_counts, uint64_t *d_offsets, void *d_ids,
                          uint64_t ids_capacity, uint64_t *h_total, void *stream);

/*
 * Rectangle search over 2-D points (an extension beyond the reference's path; the reference only
 * reorders 1-D range queries by a Z-order of (start, end), zOrder2d.cu:27-54).
 * The tree's keys are 32-bit Morton codes of (x, y) in u16 (x in the even
 * bits, y in the odd bits), its values point IDs; rectangle i is
 * [x0,x1] x [y0,y1] inclusive.  Outputs as bt_range_search: counts, offsets
 * and, for each rectangle, the IDs of the points inside sorted ascending.
 * Each box is covered by at most 16 aligned square cells (each cell is one
 * contiguous run of Morton codes, found by a lower and an upper bound);
 * cells inside the box count whole, the keys of cells on its edge are
 * tested one by one.
 * BT_ERR_INVALID_ARGUMENT unless the tree has 4-byte keys;
 * BT_ERR_NOT_SUPPORTED from 2^31 points on.
 */
BT_API bt_status bt_rect_search(const bt_tree *tree, const uint16_t *d_x0, const uint16_t *d_y0,
                                const uint16_t *d_x1, const uint16_t *d_y1, uint64_t nr,
                                uint64_t *d_counts, uint64_t *d_offsets, void *d_ids,
                                uint64_t ids_capacity, uint64_t *h_total, void *stream);

/* bt_rect_search with the boxes processed in a grouped order (no counterpart
 * in the reference; its 2-D and Z-order groupings reorder 1-D range queries,
 * grouping2d.cu:24-31, zOrder2d.cu:27-54): mode BT_RANGE_GROUPED_2D orders
 * them by the 256 x 256 cell of their corner (x0, y0) row by row,
 * BT_RANGE_ZORDER by the Morton code of that cell, BT_RANGE_BASIC keeps the
 * input order.  Boxes of one cell then run together and share their keys in
 * cache.  Outputs are the same in every mode, in the caller's order. */
BT_API bt_status bt_rect_search_mode(const bt_tree *tree, int mode, const uint16_t *d_x0,
                                     const uint16_t *d_y0, const uint16_t *d_x1,
                                     const uint16_t *d_y1, uint64_t nr, uint64_t *d_counts,
                                     uint64_t *d_offsets, void *d_ids, uint64_t ids_capacity,
                                     uint64_t *h_total, void *stream);

/* Range count with host buffers (pipelined like bt_point_search_host). */
BT_API bt_status bt_range_count_host(const bt_tree *tree, int mode, const void *h_lo,
                              const void *h_hi, uint64_t nq, uint64_t *h_counts,
                              void *stream);

/* ---- learned position model (an extension beyond the reference's path; the reference has no
 * counterpart: its descent is always the page walk of
 * BPTreeExactSearch.cu:39-68) ------------------------------------------ */

/*
 * A learned index over the tree's sorted (key, rank) pairs that sends each
 * point query to the one 128-byte piece of the leaf array ("leaf unit")
 * holding its key, with the upper separator levels replaced by a model small
 * enough to stay on chip:
 *  - leaf models: an error-bounded piecewise-linear segmentation of
 *    (key, rank) -- greedy maximal segments, each with a line within
 *    `max_error` ranks of all its keys (the optimal streaming fit of
 *    O'Rourke 1981, the segmentation of the PGM-index, Ferragina &
 *    Vinciguerra 2020), computed on the GPU; a segment's bound eps is then
 *    re-measured with the exact FP32 arithmetic of the search;
 *  - root: a monotone MLP (1 input, `hidden` ramp units clamp(w1 x + b1, 0,
 *    1), 1 output; input and output weights kept >= 0) from the normalised
 *    key to the position of the key's segment among the segment lines (4
 *    segments per 128-byte line), started as the identity and trained on the
 *    GPU by full-batch Adam with this library's own forward/backward kernels;
 *    its worst error over the lines' first keys bounds a shared-memory search
 *    over those keys;
 *  - unit thresholds: one 15-bit code per leaf-unit boundary (59 per
 *    128-byte line with a 64-bit base and a shift), an exact separator
 *    between the units' key ranges.
 * A query: the root and a short shared-memory search give the segment line
 * (one L2 read), the segment's line and eps a window of ranks, the code line
 * of the predicted unit (one L2 read; the neighbouring line too for the
 * queries whose count continues there) the leaf unit, which is the only
 * DRAM read.
 * A query whose key lies past the unit's last key reads the next unit; one
 * that leaves the window takes the tree's full descent: results are always
 * the plain search's.
 */
typedef struct bt_learned_config {
    uint32_t num_segments;  /* target segment count: max_error is raised until
                               the segmentation needs at most this many (default 65536) */
    uint32_t max_error;     /* segmentation bound in ranks; 0 = chosen from num_segments.
                               When set, num_segments is ignored */
    uint32_t hidden;        /* root hidden units, 1..32 (default 16) */
    uint32_t iterations;    /* root training steps (default 400) */
    float learning_rate;    /* Adam step size (default 0.002) */
} bt_learned_config;

typedef struct bt_learned_report {
    float root_loss_initial;  /* MSE of the root before training */
    float root_loss_final;    /* ... and after */
    uint32_t root_error;      /* root's worst line-position error after training */
    uint32_t root_error_initial; /* ... and of the untrained root */
    uint32_t num_segments;    /* segments of the segmentation */
    uint32_t max_error;       /* the segmentation's bound */
    uint64_t eps_max;         /* largest measured segment bound (FP32 search arithmetic) */
    double eps_mean;          /* mean measured segment bound */
    double code_lines_mean;   /* mean code lines a query's window spans (over the keys) */
    uint64_t index_bytes;     /* device bytes of the model, segment lines and codes */
    uint32_t keys_per_unit;   /* keys in one 128-byte leaf unit */
    uint32_t pad;
    double train_ms;          /* device time of the whole build */
} bt_learned_report;

/* Build the learned index of `tree` (replacing a previous one).  cfg may be
 * NULL for defaults; report may be NULL.  BT_ERR_NOT_SUPPORTED when the
 * segment lines' first keys do not fit the search's shared memory (more than
 * about 2^16 segments for u64 keys: raise max_error).  Synchronizes `stream`. */
BT_API bt_status bt_learned_train(bt_tree *tree, const bt_learned_config *cfg, void *stream,
                                  bt_learned_report *report);

/* Point search through the learned index: bt_point_search(BT_POINT_LEARNED)
 * (same results as the other modes).  BT_ERR_INVALID_ARGUMENT if the tree has
 * no trained index. */
BT_API bt_status bt_point_search_learned(const bt_tree *tree, const void *d_queries, uint64_t nq,
                                         void *d_out, void *stream);

/* Shape of the learned search kernel (one CTA per SM): 1 = 1024-thread CTAs
 * (the default), 2 = 768, 3 = 640, 4 = 512.  Fewer threads leave more
 * registers to each.  Results do not depend on it; the autotuner picks the
 * fastest. */
BT_API bt_status bt_learned_set_shape(bt_tree *tree, uint32_t shape);

/* Counters of the last learned search on this tree: leaf units read beyond
 * the first one (keys just past a unit's threshold) and queries that took
 * the full tree descent. */
BT_API bt_status bt_learned_last_stats(const bt_tree *tree, uint64_t *extra_unit_reads,
                                       uint64_t *fallback);

/* Code lines the last learned search on this tree counted beyond each
 * query's first (queries whose rank window continues into a neighbouring
 * line and whose count had to go on there). */
BT_API bt_status bt_learned_last_lines(const bt_tree *tree, uint64_t *extra_code_lines);

/*
 * The root model's training kernels, exposed so their gradients can be
 * checked: for params p (3*hidden+1 floats: w1[hidden], b1[hidden],
 * w2[hidden], b2) and n points (x[i], y[i]) in device memory, writes
 * loss = mean((f(x)-y)^2) to d_loss[0] and dloss/dp to d_grad (device).
 */
BT_API bt_status bt_mlp_loss_grad(const float *d_params, uint32_t hidden, const float *d_x,
                                  const float *d_y, uint64_t n, float *d_loss, float *d_grad,
                                  void *stream);

/* ---- batched forest of uneven trees (an extension beyond the reference's path; in the
 * reference each tree is its own genBPlusTree + search host calls) ------ */

typedef struct bt_forest bt_forest;
typedef struct bt_forest_plan bt_forest_plan;

/*
 * Build num_trees independent trees at once.  Tree t's keys (sorted
 * ascending) and values are d_keys/d_values[h_offsets[t] .. h_offsets[t+1]),
 * device memory; h_offsets is a host array of num_trees+1 entries.  Empty
 * trees are allowed.  All trees share one leaf array and one separator array
 * (same layout as a single tree) plus a per-tree descriptor table.
 */
BT_API bt_status bt_forest_build(const void *d_keys, const void *d_values, const uint64_t *h_offsets,
                                 uint32_t num_trees, int key_bytes, int value_bytes, void *stream,
                                 bt_forest **out);
BT_API bt_status bt_forest_destroy(bt_forest *forest);

/*
 * A reusable search plan over fixed buffers: point queries of tree t are
 * d_queries[h_q_offsets[t] .. h_q_offsets[t+1]) with results in d_out at the
 * same positions; range queries of tree t are [d_lo[i], d_hi[i]] for i in
 * h_r_offsets[t] .. h_r_offsets[t+1] with counts in d_counts[i] (h_r_offsets
 * may be NULL for no ranges).  The plan cuts every tree's queries into work
 * items of `tile` queries and records one persistent kernel launch, in which
 * warps take items from a device queue, as a CUDA graph (captured on a
 * private stream when the plan is made).  lanes_per_query / rounds as in
 * bt_set_search_config.
 */
BT_API bt_status bt_forest_plan_create(const bt_forest *forest, const void *d_queries,
                                       const uint64_t *h_q_offsets, void *d_out, const void *d_lo,
                                       const void *d_hi, const uint64_t *h_r_offsets,
                                       uint64_t *d_counts, int lanes_per_query, int rounds,
                                       uint32_t tile, bt_forest_plan **out);
/*
 * Fanout of the shared-memory root of the forest search, used by the plans
 * made after the call: each work item stages in shared memory the deepest
 * separator level of its tree that fits 16 KB and has at most
 * entries_per_descent entries per descent the item makes (default 16), and
 * one binary search there replaces every level above it.  A larger value
 * stages deeper levels for fewer queries.  Node lines themselves stay 128
 * bytes (16 u64 or 32 u32 separators); the reference's fixed fanout is
 * PAGESIZE = 5000 (BPTree.h:8).  The autotuner (autotune.tune_forest) picks
 * it with the tile and lanes per query.  Results do not depend on it.
 */
BT_API bt_status bt_forest_set_stage_fanout(bt_forest *forest, uint32_t entries_per_descent);
/* Launch the plan's graph on `stream` (asynchronous). */
BT_API bt_status bt_forest_plan_run(bt_forest_plan *plan, void *stream);
BT_API bt_status bt_forest_plan_destroy(bt_forest_plan *plan);

/* ---- continuous-batching request loop (an extension beyond the reference's path; the reference
 * runs one synchronous batch per host call, BPTreeExactSearch.cu:409-484) */

typedef struct bt_server bt_server;

typedef enum bt_serve_mode {
    BT_SERVE_BASIC = 0,   /* bt_point_search basic */
    BT_SERVE_GROUPED = 1, /* bt_point_search grouped */
    BT_SERVE_LEARNED = 2  /* bt_point_search_learned (needs a trained model) */
} bt_serve_mode;

typedef struct bt_server_config {
    uint32_t slots;               /* concurrent device jobs wanted (default 8) */
    uint64_t memory_budget_bytes; /* device memory for job buffers (default 256 MiB) */
    uint32_t max_batch;           /* queries per job; larger requests are split (default 65536) */
    int32_t mode;                 /* bt_serve_mode */
} bt_server_config;

typedef struct bt_server_stats {
    uint32_t slots;          /* slots the memory budget admitted */
    uint32_t max_in_flight;  /* most jobs on the device at once so far */
    uint64_t completed;      /* requests completed */
    uint64_t jobs;           /* device jobs issued */
} bt_server_stats;

/*
 * A server answering point-query requests on one tree.  A worker thread
 * admits requests chunk by chunk into free slots -- each slot a stream with
 * its own device buffers, the number of slots bounded by the memory budget --
 * as soon as one frees up, so requests that arrive while others run are
 * admitted at once and their copies and kernels overlap on the device.
 * Host buffers must stay valid until the request completes; pinned host
 * memory lets the copies run asynchronously.
 */
BT_API bt_status bt_server_create(const bt_tree *tree, const bt_server_config *cfg,
                                  bt_server **out);
/* Queue a request (non-blocking); *ticket identifies it. */
BT_API bt_status bt_server_submit(bt_server *srv, const void *h_queries, uint64_t nq, void *h_out,
                                  uint64_t *ticket);
/* Block until the request is answered; *latency_us = submit-to-completion
 * time.  Each ticket can be waited for once. */
BT_API bt_status bt_server_wait(bt_server *srv, uint64_t ticket, double *latency_us);
BT_API bt_status bt_server_get_stats(bt_server *srv, bt_server_stats *stats);
/* Waits for all outstanding work, then frees the server. */
BT_API bt_status bt_server_destroy(bt_server *srv);
/*
 * Load generator: submits nreq requests at their arrival times (arrival_us,
 * microseconds after the call starts, ascending), waits for all, and fills
 * latency_us[i]; *wall_us receives the total time.
 */
BT_API bt_status bt_server_replay(bt_server *srv, uint64_t nreq, const uint64_t *nq,
                                  const void *const *h_queries, void *const *h_outs,
                                  const double *arrival_us, double *latency_us, double *wall_us);

/* Number of kernel launches this library has issued in this process (all
 * devices, all threads).  Lets a caller count the device work behind a call. */
BT_API uint64_t bt_kernel_launches(void);

/* Number of scratch allocations this library has made from its memory pool
 * in this process (all devices, all threads).  Lets a caller check that a
 * call allocated nothing. */
BT_API uint64_t bt_workspace_allocations(void);

/* Number of times a grouping or sorting pass on the current device gave up
 * waiting for the digit counts of an earlier tile (its look-back is bounded;
 * a correct launch never gives up, and a pass that did has wrong output).
 * Synchronous; all-ones if it cannot be read. */
BT_API uint64_t bt_partition_lookback_timeouts(void);

#ifdef __cplusplus
}
#endif

#endif /* BTREE_B200_H */
