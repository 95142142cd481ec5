/*
 * CPU oracle for the B+tree index search path.
 *
 * TEST INFRASTRUCTURE ONLY.  Nothing in the shipped library links, loads or
 * calls this code; only tests/, __graft_entry__.smoke() and bench.py's CPU
 * baseline leg use it, and only to check results (or as the timed CPU baseline).
 *
 * Two families of functions live here:
 *
 *  1. orc_*  : ground truth.  Plain binary search over the sorted key array
 *              (std::lower_bound / std::upper_bound semantics).  Point search
 *              returns values[lower_bound(q)] on an exact match, else the
 *              all-ones sentinel of the value width (the reference's
 *              INVALID_DATA, BPTree.h:12).  Range search over the inclusive
 *              interval [lo, hi] returns upper_bound(hi) - lower_bound(lo)
 *              hits and the values of those keys, sorted ascending.
 *
 *  2. refc_* : a literal CPU restatement of the reference's page-based tree
 *              (fanout PAGESIZE = 5000, BPTree.h:6-23) and of its kernels,
 *              including their quirks, so that divergences between the
 *              reference and the ground truth can be explained case by case.
 *              Each function cites the reference file:line it follows.
 *
 * All functions are thread-safe; `nthreads` <= 0 means "all OpenMP threads".
 */
#ifndef BT_ORACLE_H
#define BT_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- ground truth ---------------------------------------------------------- */

/* Point search.  key_bytes/val_bytes in {4, 8}.  out has val_bytes per query. */
int orc_point_search(const void *keys, const void *vals, uint64_t n,
                     int key_bytes, int val_bytes,
                     const void *queries, uint64_t nq, void *out, int nthreads);

/* Range counts for inclusive [lo[i], hi[i]]; lo > hi gives 0. */
int orc_range_count(const void *keys, uint64_t n, int key_bytes,
                    const void *lo, const void *hi, uint64_t nq,
                    uint64_t *counts, int nthreads);

/* Range hit IDs: ids[offsets[i] .. offsets[i]+counts[i]) = values of the hit
 * keys of query i, sorted ascending.  offsets must be the exclusive scan of
 * the counts from orc_range_count. */
int orc_range_ids(const void *keys, const void *vals, uint64_t n,
                  int key_bytes, int val_bytes,
                  const void *lo, const void *hi, uint64_t nq,
                  const uint64_t *offsets, void *ids, int nthreads);

/* lower_bound / upper_bound positions (for property tests). */
int orc_bounds(const void *keys, uint64_t n, int key_bytes,
               const void *queries, uint64_t nq, int upper,
               uint64_t *pos, int nthreads);

/* Rectangle search over Z-ordered points (x, y in u16, z = interleave).
 * Points are given sorted by (z, id).  Rectangle i is [x0,x1] x [y0,y1]
 * inclusive.  counts[i] = hits; with ids != NULL, ids[offsets[i]..] = the hit
 * point IDs sorted ascending. */
int orc_rect_search(const uint32_t *z_sorted, const uint32_t *ids_sorted, uint64_t n,
                    const uint16_t *x0, const uint16_t *y0,
                    const uint16_t *x1, const uint16_t *y1, uint64_t nq,
                    uint64_t *counts, const uint64_t *offsets, uint32_t *ids,
                    int nthreads);

/* 32-bit Morton interleave of (x, y): x in even bits, y in odd bits. */
uint32_t orc_morton2_u16(uint16_t x, uint16_t y);

/* Error-bounded piecewise-linear segmentation of the points (key[i], i),
 * i in [0, n) (keys ascending and unique, key_bytes 4 or 8): greedy maximal
 * segments, each admitting a line within eps of all its points (the optimal
 * streaming fit of O'Rourke 1981 as in the PGM-index, Ferragina &
 * Vinciguerra 2020).  A segment never crosses a multiple of `chunk` (0: no
 * limit) and is closed when either convex hull would exceed hull_cap
 * points.  For the first max_out segments writes the start index and, when
 * non-NULL, the line rank - start = icpt + slope * (key - key[start]): the
 * mean of the steepest and the flattest feasible line (slope 0, icpt 0 for
 * a one-point segment).  Returns the number of segments.  Restates the
 * engine's GPU segmentation (its chunking and hull cap included). */
uint64_t orc_pla_segments(const void *keys, uint64_t n, int key_bytes, uint32_t eps,
                          uint64_t chunk, int hull_cap, uint64_t *starts, double *slopes,
                          double *icpts, uint64_t max_out);

/* ---- literal restatement of the reference ------------------------------ */

#define REFC_PAGESIZE 5000
#define REFC_INVALID 0xFFFFFFFFFFFFFFFFull

typedef struct refc_tree refc_tree;

/* Build the reference's page tree from sorted (key, data) pairs, following
 * genBPlusTree (BPTree.cu:127-306): leaves of PAGESIZE consecutive pairs
 * (assignDataToLeaf, BPTree.cu:73-125) and internal pages of
 * (child.max, child page index) built bottom-up (kernelMaxIntermidatePage,
 * BPTree.cu:28-70).  `leaf_sizes`/nleaves is the caller's groupList
 * (main.cu:126-129 always passes PAGESIZE per group); pass NULL for
 * ceil(n / PAGESIZE) groups of PAGESIZE with an exact last group.
 * Reads of pairs at index >= n return 0 (the reference reads past its
 * arrays there, quirk of main.cu:126-129). */
refc_tree *refc_build(const uint64_t *keys, const uint64_t *data, uint64_t n,
                      const uint64_t *leaf_sizes, uint64_t nleaves);
void refc_free(refc_tree *t);
uint64_t refc_root(const refc_tree *t);
uint64_t refc_num_pages(const refc_tree *t);

/* kernelSearchingNaiveOneStep, BPTreeExactSearch.cu:25-105. */
int refc_point_basic(const refc_tree *t, const uint64_t *q, uint64_t nq,
                     uint64_t *out, int nthreads);
/* kernelSearchingKeyGroupTwoStep, BPTreeExactSearch.cu:207-294 (leaf
 * compares data[] instead of key[], :269-276). */
int refc_point_grouped(const refc_tree *t, const uint64_t *q, uint64_t nq,
                       uint64_t *out, int nthreads);
/* kernelSearchingKeyRangeGroupStateTwo, BtreeRangeSearch.cu:215-294, and
 * its grouped twin :33-119 (identical per-query result): (pos << 32) | leaf. */
int refc_range_endpoint(const refc_tree *t, const uint64_t *q, uint64_t nq,
                        uint64_t *out, int nthreads);
/* kernelGenerateSearchResult, BtreeRangeSearch.cu:297-374 (grouped = 0), or
 * kernelGenerateSearchResultGrouping, :123-211 (grouped = 1, compares data[]). */
int refc_range_count(const refc_tree *t, const uint64_t *lo, const uint64_t *hi,
                     const uint64_t *ep_lo, const uint64_t *ep_hi, uint64_t nq,
                     int grouped, uint64_t *counts, int nthreads);

/* bucketIdentify, grouping.cu:25-29 (8-bit digits, pass 0 = top byte). */
int refc_bucket(uint64_t v, int pass);
/* bucketIdentify2d, grouping2d.cu:24-31 (3-bit stride, 4-bit digit, product). */
int refc_bucket2d(uint64_t a, uint64_t b, int pass);
/* calcuateZorder2d, zOrder2d.cu:27-54. */
uint64_t refc_zorder(uint64_t a, uint64_t b, int ix, int iy);
/* the grouping interval of genGrouping2dZ, zOrder2d.cu:129-130. */
int refc_zorder_interval(uint64_t max_value);

#ifdef __cplusplus
}
#endif

#endif
