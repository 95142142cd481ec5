/*
 * btree_b200_compat.h -- the reference's C++ host API, served by this engine.
 *
 * Byte-identical declarations to the reference's BPTree.h:26-55 (with the
 * types of utils.h:4 and the constants and page struct of BPTree.h:6-23), so
 * a caller written against the reference -- its main.cu, for instance --
 * links against libbtree_b200.so instead of BPTree.cu, BPTreeExactSearch.cu,
 * BtreeRangeSearch.cu and the grouping files, unchanged.  The page struct is
 * declared only so that the mangled names match (an unnamed struct with a
 * typedef name mangles as that name); the engine stores no BTPage.
 *
 * Observable conventions kept from the reference:
 *   - genBPlusTree takes ownership of, and frees, both device input arrays
 *     (BPTree.cu:209-211), writes the root index into a new device u64[1]
 *     (:272-273), returns the tree handle through dev_globalPointer_in
 *     (:275) and a managed u64 page counter through dev_currentPage_in
 *     (:276), leaves treeLevel_out, btreeIndex_out and bTreeSize_out
 *     untouched (:277-278) and prints "Building the Tree <seconds>" (:258).
 *     The handle is not a device pointer to pages: pass it back, do not
 *     dereference it (the reference's callers never do, main.cu:142-355).
 *   - SearchingBTreeGPUOnlyOneState returns NULL (BPTreeExactSearch.cu:483).
 *   - SearchingBTreeGPUCombineStep overwrites input_key with the grouped
 *     order (:613) and returns a new[] array of results in that order (:722);
 *     free it with delete[].
 *   - The three range functions return NULL and hand no counts to the caller
 *     (BtreeRangeSearch.cu:574,782,924).
 *   - Every call runs on device 0, synchronously, on the legacy default
 *     stream, and prints the reference's timing lines; a failure prints a
 *     message and exits the process (gpuAssert, BPTreeExactSearch.cu:864-871).
 *
 * Deliberate differences: results are exact (lower_bound semantics) where the
 * reference's grouped point search compares data[] instead of key[]
 * (BPTreeExactSearch.cu:269-276) and its range counts drop keys at leaf
 * boundaries (BtreeRangeSearch.cu:329,350).  The groupList/groupPrefix leaf
 * plan is not needed and is ignored (the reference's own plan claims
 * PAGESIZE keys for a partial last leaf, main.cu:126-129).
 *
 * Extra entry points (no counterpart in the reference; they give callers the
 * results the reference computes and discards):
 *   bt_compat_last_results -- outputs of the last search call made through
 *     this header, in the order described above;
 *   bt_compat_tree -- the C-ABI tree behind a genBPlusTree handle.
 */
#ifndef BTREE_B200_COMPAT_H
#define BTREE_B200_COMPAT_H

#include <vector>

#include "btree_b200.h"

typedef unsigned long long int ulli;

#define PAGE_ALLOCATION 200041
#define PAGESIZE 5000
#define GROUP_SEARCH_SIZE 33000
#define DOB_PAGE_SIZE 1
#define INVALID_DATA 0xffffffffffffffff

typedef struct {
    ulli key[PAGESIZE];
    ulli data[PAGESIZE];
    bool leafFlag;
    int size;
    ulli max;
    ulli min;
    int previous;
    int next;
} BTPage;

BT_API void *genBPlusTree(ulli *devInputKey, ulli *devInput, ulli inputSize,
                          std::vector<ulli> groupList, std::vector<ulli> groupPrefix,
                          ulli *&dev_btree_out, ulli &treeLevel_out, ulli *&btreeIndex_out,
                          ulli &bTreeSize_out, BTPage *&dev_globalPointer_in,
                          ulli *&dev_currentPage_in);

BT_API void *SearchingBTreeGPUOnlyOneState(ulli *input_key, ulli inputSize, ulli *dev_Btree,
                                           BTPage *dev_globalPointer);

BT_API void *SearchingBTreeGPUCombineStep(ulli *input_key, ulli inputSize, ulli *dev_Btree,
                                          BTPage *dev_globalPointer);

BT_API void *SearchingBTreeGPURange(ulli *input_key_start, ulli *input_key_end, ulli inputSize,
                                    ulli *dev_Btree, BTPage *dev_globalPointer);

BT_API void *SearchingBTreeGPURangeWithGrouping(ulli *input_key_start, ulli *input_key_end,
                                                ulli inputSize, ulli *dev_Btree,
                                                BTPage *dev_globalPointer);

BT_API void *SearchingBTreeGPURangeWithGroupingZorder(ulli *input_key_start, ulli *input_key_end,
                                                      ulli inputSize, ulli *dev_Btree,
                                                      BTPage *dev_globalPointer);

extern "C" {
/* Outputs of the last search made through this header (point: values;
 * range: counts), *n receives their number.  Valid until the next call. */
BT_API const ulli *bt_compat_last_results(ulli *n);
/* The C-ABI tree behind a genBPlusTree handle (NULL if unknown). */
BT_API bt_tree *bt_compat_tree(BTPage *dev_globalPointer);
}

#endif /* BTREE_B200_COMPAT_H */
