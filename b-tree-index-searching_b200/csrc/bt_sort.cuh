// Warp-level sort of short value lists (up to 256 values), shared by the
// segment sort of range/rectangle results and the rectangle fill pass.
//
// The values sit in registers in striped order -- value e = m * 32 + lane in
// v[m] of lane `lane` -- padded with all-ones to 32 * E.  A bitonic network
// over the 32 * E slots: compare-exchange partners at distance < 32 are in
// other lanes of the same register (one shuffle), partners at distance >= 32
// in other registers of the same lane (no data movement).  Loads and stores
// in striped order are coalesced.
#pragma once

#include "bt_internal.cuh"

namespace bt {

template <typename V, int E>
__device__ __forceinline__ void warp_bitonic_sort(V (&v)[E], int lane) {
    constexpr int N = 32 * E;
#pragma unroll
    for (int size = 2; size <= N; size <<= 1) {
#pragma unroll
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            if (stride >= 32) {
#pragma unroll
                for (int m = 0; m < E; m++) {
                    const int pm = m ^ (stride >> 5);
                    if (pm > m) {
                        const bool asc = ((m * 32 + lane) & size) == 0;
                        const V a = v[m], b = v[pm];
                        const bool sw = asc ? (a > b) : (a < b);
                        v[m] = sw ? b : a;
                        v[pm] = sw ? a : b;
                    }
                }
            } else {
                const bool lower = (lane & stride) == 0;
#pragma unroll
                for (int m = 0; m < E; m++) {
                    const V o = __shfl_xor_sync(0xffffffffu, v[m], stride);
                    const bool asc = ((m * 32 + lane) & size) == 0;
                    const V lo = v[m] < o ? v[m] : o;
                    const V hi = v[m] < o ? o : v[m];
                    v[m] = (lower == asc) ? lo : hi;
                }
            }
        }
    }
}

// dst[0..c) = src[0..c) sorted ascending, c <= 32 * E; src may equal dst.
// Every lane of the warp must call it.
template <typename V, int E>
__device__ __forceinline__ void warp_sort_copy(const V *src, V *dst, uint32_t c, int lane) {
    V v[E];
#pragma unroll
    for (int m = 0; m < E; m++) {
        const uint32_t e = m * 32u + lane;
        v[m] = e < c ? src[e] : key_max<V>();
    }
    __syncwarp();  // every load is done before any store (in-place use)
    warp_bitonic_sort<V, E>(v, lane);
#pragma unroll
    for (int m = 0; m < E; m++) {
        const uint32_t e = m * 32u + lane;
        if (e < c) dst[e] = v[m];
    }
}

constexpr int kWarpSortCap = 256;

// As warp_sort_copy, choosing the register count from c (<= kWarpSortCap).
template <typename V>
__device__ __forceinline__ void warp_sort_small(const V *src, V *dst, uint32_t c, int lane) {
    if (c <= 32) warp_sort_copy<V, 1>(src, dst, c, lane);
    else if (c <= 64) warp_sort_copy<V, 2>(src, dst, c, lane);
    else if (c <= 128) warp_sort_copy<V, 4>(src, dst, c, lane);
    else warp_sort_copy<V, 8>(src, dst, c, lane);
}

}  // namespace bt
