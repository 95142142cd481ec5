// Rectangle search over Z-ordered 2-D points (declared in btree_b200.h).
//
// Keys are 32-bit Morton codes z = interleave(x, y) (x in the even bits).
// Every point of the box [x0,x1] x [y0,y1] has its code in
// [zmin, zmax] = [Z(x0,y0), Z(x1,y1)] (interleaving is monotone in each
// coordinate), but that interval also holds many points outside the box.
// One warp per rectangle scans the sorted keys 32 at a time from
// lower_bound(zmin), tests each decoded (x, y) against the box, and when the
// window's last key lies outside the box jumps to lower_bound(BIGMIN) --
// BIGMIN being the smallest code above it that lies inside the box (Tropf &
// Herzog, "Multidimensional range search in dynamically balanced trees",
// 1981) -- so long outside runs cost one descent instead of a scan.  A count
// pass, an exclusive scan and a fill pass produce CSR output; the IDs of each
// box are then sorted.
#include <algorithm>

#include "bt_search.cuh"

namespace bt {
namespace {

constexpr int kRThreads = 256;

__device__ __forceinline__ uint32_t compact16(uint32_t v) {
    v &= 0x55555555u;
    v = (v | (v >> 1)) & 0x33333333u;
    v = (v | (v >> 2)) & 0x0F0F0F0Fu;
    v = (v | (v >> 4)) & 0x00FF00FFu;
    v = (v | (v >> 8)) & 0x0000FFFFu;
    return v;
}

__device__ __forceinline__ uint32_t spread16d(uint32_t v) {
    v &= 0xFFFFu;
    v = (v | (v << 8)) & 0x00FF00FFu;
    v = (v | (v << 4)) & 0x0F0F0F0Fu;
    v = (v | (v << 2)) & 0x33333333u;
    v = (v | (v << 1)) & 0x55555555u;
    return v;
}

__device__ __forceinline__ bool in_box(uint32_t z, uint32_t x0, uint32_t y0, uint32_t x1,
                                       uint32_t y1) {
    const uint32_t x = compact16(z), y = compact16(z >> 1);
    return x >= x0 && x <= x1 && y >= y0 && y <= y1;
}

// Smallest Morton code > z inside the box [zmin, zmax] (both corners' codes),
// or 0xFFFFFFFF if there is none; z must lie inside [zmin, zmax] and outside
// the box.  Bits are visited from the top; at each bit the (z, zmin, zmax)
// pattern decides whether the box lies entirely above z in that subtree, splits
// it (narrowing zmin or zmax to one half of the dimension), or ends the walk.
__device__ uint32_t bigmin(uint32_t z, uint32_t zmin, uint32_t zmax) {
    uint32_t best = 0xFFFFFFFFu;
    for (int b = 31; b >= 0; b--) {
        const uint32_t m = 1u << b;
        const uint32_t low = ((b & 1) ? 0xAAAAAAAAu : 0x55555555u) & (m - 1u);  // lower bits, same dim
        const int zb = (z & m) != 0, lb = (zmin & m) != 0, hb = (zmax & m) != 0;
        if (!zb && !lb && hb) {
            best = (zmin | m) & ~low;   // the upper half starts here
            zmax = (zmax & ~m) | low;   // keep looking in the lower half
        } else if (!zb && lb && hb) {
            return zmin;                // the whole box is above z here
        } else if (zb && !lb && !hb) {
            return best;                // z is above the box here
        } else if (zb && !lb && hb) {
            zmin = (zmin | m) & ~low;   // continue in the upper half
        } else if (lb && !hb) {
            return best;                // empty box in this dimension
        }
    }
    return best;
}

// First position with key >= q (q <= max key) by the whole warp: the lanes
// binary-search the staged level together (same path), then walk the global
// levels with all 32 lanes on one node line, then the leaf block.
template <typename V>
__device__ __forceinline__ uint64_t warp_lower_bound(const DevTree &t, const uint32_t *s_lvl,
                                                     uint32_t q) {
    const uint32_t tmax = (uint32_t)t.max_key;
    if (q > tmax) return t.n;
    uint32_t qe[1] = {q};
    bool up[1] = {false};
    uint32_t node[1] = {smem_bound<uint32_t>(s_lvl, t.smem_entries, q, false)};
    const int lane = threadIdx.x & 31;
    walk_global<uint32_t, 32, 1>(t, qe, up, node, 0, lane);
    int pos[1];
    leaf_bound<uint32_t, V, 32, 1>(static_cast<const unsigned char *>(t.leaves), node, qe, up, 0,
                                   lane, pos);
    return (uint64_t)node[0] * LeafGeom<uint32_t, V>::S + pos[0];
}

// FILL = false: counts[i] = points in box i.  FILL = true: write their IDs
// at ids[offsets[i] ..] (in key order; sorted afterwards).
template <typename V, bool FILL>
__global__ void __launch_bounds__(kRThreads)
rect_kernel(const __grid_constant__ DevTree t, const uint16_t *__restrict__ x0s,
            const uint16_t *__restrict__ y0s, const uint16_t *__restrict__ x1s,
            const uint16_t *__restrict__ y1s, uint64_t nr, uint64_t *__restrict__ counts,
            const uint64_t *__restrict__ offsets, V *__restrict__ ids) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    uint32_t *s_lvl = reinterpret_cast<uint32_t *>(smem_raw);
    stage_level<uint32_t>(s_lvl, t);
    __syncthreads();
    using LG = LeafGeom<uint32_t, V>;
    const int lane = threadIdx.x & 31;
    const unsigned char *leaves = static_cast<const unsigned char *>(t.leaves);
    const unsigned lt = (1u << lane) - 1u;
    for (uint64_t i = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5; i < nr;
         i += ((uint64_t)gridDim.x * blockDim.x) >> 5) {
        const uint32_t x0 = x0s[i], y0 = y0s[i], x1 = x1s[i], y1 = y1s[i];
        uint64_t c = 0;
        if (x0 <= x1 && y0 <= y1 && t.n > 0) {
            const uint32_t zmin = spread16d(x0) | (spread16d(y0) << 1);
            const uint32_t zmax = spread16d(x1) | (spread16d(y1) << 1);
            const uint64_t base_out = FILL ? offsets[i] : 0;
            uint64_t pos = warp_lower_bound<V>(t, s_lvl, zmin);
            while (pos < t.n) {
                const uint64_t p = pos + lane;
                const bool valid = p < t.n;
                const uint32_t k = valid ? reinterpret_cast<const uint32_t *>(
                                               leaves + (p / LG::S) * LG::BS)[p % LG::S]
                                         : 0xFFFFFFFFu;
                const bool in_range = valid && k <= zmax;
                const bool inside = in_range && in_box(k, x0, y0, x1, y1);
                const unsigned hit = __ballot_sync(0xffffffffu, inside);
                if (FILL && inside)
                    ids[base_out + c + __popc(hit & lt)] = reinterpret_cast<const V *>(
                        leaves + (p / LG::S) * LG::BS + kSectorBytes)[p % LG::S];
                c += __popc(hit);
                if (__ballot_sync(0xffffffffu, in_range) != 0xffffffffu) break;  // past zmax or n
                const uint32_t last = __shfl_sync(0xffffffffu, k, 31);
                if (hit >> 31) {  // the window ends inside the box: keep scanning
                    pos += 32;
                    continue;
                }
                const uint32_t bm = bigmin(last, zmin, zmax);
                if (bm == 0xFFFFFFFFu || bm > zmax) break;
                // bm > last, so the new position is past this window
                pos = warp_lower_bound<V>(t, s_lvl, bm);
            }
        }
        if (!FILL && lane == 0) counts[i] = c;
    }
}

template <typename V>
bt_status rect_impl(const bt_tree *t, const uint16_t *x0, const uint16_t *y0, const uint16_t *x1,
                    const uint16_t *y1, uint64_t nr, uint64_t *counts, uint64_t *offsets,
                    void *ids, uint64_t cap, uint64_t *h_total, cudaStream_t s) {
    const size_t smem = t->dev.smem_bytes;
    auto kc = rect_kernel<V, false>;
    auto kf = rect_kernel<V, true>;
    if (smem > 48 * 1024) {
        BT_CUDA(cudaFuncSetAttribute(kc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        BT_CUDA(cudaFuncSetAttribute(kf, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    }
    int per_sm = 1;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kc, kRThreads, smem);
    const unsigned grid = (unsigned)std::max<uint64_t>(
        1, std::min<uint64_t>((nr + 7) / 8, (uint64_t)sm_count() * std::max(per_sm, 1)));
    count_launch();
    kc<<<grid, kRThreads, smem, s>>>(t->dev, x0, y0, x1, y1, nr, counts, nullptr, nullptr);
    BT_CUDA(cudaGetLastError());
    uint64_t *d_total = nullptr;
    bt_status st = ws_alloc((void **)&d_total, sizeof(uint64_t), s);
    if (st != BT_OK) return st;
    st = launch_scan_u64(counts, offsets, nr, d_total, s);
    uint64_t total = 0;
    if (st == BT_OK) {
        cudaError_t e = cudaMemcpyAsync(&total, d_total, sizeof(total), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) st = cuda_fail(e, "rectangle total read-back");
    }
    ws_free(d_total, s);
    if (st != BT_OK) return st;
    *h_total = total;
    if (total > cap) return fail(BT_ERR_CAPACITY, "ids_capacity is below the total hit count");
    if (total == 0) return BT_OK;
    if (!ids) return fail(BT_ERR_INVALID_ARGUMENT, "ids is NULL");
    count_launch();
    kf<<<grid, kRThreads, smem, s>>>(t->dev, x0, y0, x1, y1, nr, counts, offsets, (V *)ids);
    BT_CUDA(cudaGetLastError());
    return launch_segment_sort(t, counts, offsets, nr, ids, s);
}

}  // namespace
}  // namespace bt

extern "C" {

bt_status bt_rect_search(const bt_tree *t, const uint16_t *x0, const uint16_t *y0,
                         const uint16_t *x1, const uint16_t *y1, uint64_t nr, uint64_t *counts,
                         uint64_t *offsets, void *ids, uint64_t cap, uint64_t *h_total,
                         void *stream) {
    using namespace bt;
    if (!t) return fail(BT_ERR_INVALID_ARGUMENT, "tree is NULL");
    if (!h_total) return fail(BT_ERR_INVALID_ARGUMENT, "h_total is NULL");
    *h_total = 0;
    if (t->key_bytes != 4)
        return fail(BT_ERR_INVALID_ARGUMENT, "rectangle search needs 32-bit Morton-code keys");
    if (nr == 0) return BT_OK;
    if (!x0 || !y0 || !x1 || !y1 || !counts || !offsets)
        return fail(BT_ERR_INVALID_ARGUMENT, "a rectangle or output array is NULL");
    int prev = 0;
    BT_CUDA(cudaGetDevice(&prev));
    if (prev != t->device) BT_CUDA(cudaSetDevice(t->device));
    cudaStream_t s = (cudaStream_t)stream;
    const bt_status st =
        t->val_bytes == 4 ? rect_impl<uint32_t>(t, x0, y0, x1, y1, nr, counts, offsets, ids, cap, h_total, s)
                          : rect_impl<uint64_t>(t, x0, y0, x1, y1, nr, counts, offsets, ids, cap, h_total, s);
    if (prev != t->device) cudaSetDevice(prev);
    return st;
}

}  // extern "C"
