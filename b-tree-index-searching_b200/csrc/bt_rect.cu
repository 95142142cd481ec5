// Rectangle search over Z-ordered 2-D points (declared in btree_b200.h).
//
// Keys are 32-bit Morton codes z = interleave(x, y) (x in the even bits).  An
// aligned square cell of side 2^c ([X, X + 2^c) x [Y, Y + 2^c), X and Y
// multiples of 2^c) holds exactly the codes of one interval
// [Z(X,Y), Z(X,Y) + 4^c), so its points are one contiguous run of the sorted
// keys.  Each box [x0,x1] x [y0,y1] is covered by the aligned cells of the
// smallest c that needs at most 16 of them; one warp per box finds the run
// of every cell with 32 descents in one round (lanes 0-15: lower bound of a
// cell's first code, lanes 16-31: upper bound of its last), the same
// two-phase descent as the point search.  Cells inside the box count their
// whole run; the runs of the cells on the box's edge are scanned by the warp
// together, 32 keys at a time, testing each decoded (x, y).  A count pass
// (which also stores every cell's run), an exclusive scan and a fill pass
// produce CSR output; the IDs of each box are then sorted.
//
// About 1.3x the box's area in codes is scanned; the alternative of scanning
// [Z(x0,y0), Z(x1,y1)] and jumping over outside stretches (BIGMIN, Tropf &
// Herzog 1981) pays one dependent root-to-leaf descent per jump.
#include <algorithm>

#include "bt_search.cuh"
#include "bt_sort.cuh"

namespace bt {
namespace {

constexpr int kRThreads = 512;
constexpr int kRWarps = kRThreads / 32;
constexpr int kMaxCells = 16;

__device__ __forceinline__ uint32_t spread16d(uint32_t v) {
    v &= 0xFFFFu;
    v = (v | (v << 8)) & 0x00FF00FFu;
    v = (v | (v << 4)) & 0x0F0F0F0Fu;
    v = (v | (v << 2)) & 0x33333333u;
    v = (v | (v << 1)) & 0x55555555u;
    return v;
}

// A box in code space.  Spreading a coordinate's bits apart is strictly
// monotone, so x in [x0, x1] holds exactly when the code's x bits (the even
// ones) lie in [spread(x0), spread(x1)]; likewise y in the odd bits.
struct ZBox {
    uint32_t x0, x1, y0, y1;
    __device__ __forceinline__ ZBox(uint32_t bx0, uint32_t by0, uint32_t bx1, uint32_t by1)
        : x0(spread16d(bx0)), x1(spread16d(bx1)), y0(spread16d(by0) << 1), y1(spread16d(by1) << 1) {}
    __device__ __forceinline__ bool holds(uint32_t z) const {
        const uint32_t zx = z & 0x55555555u, zy = z & 0xAAAAAAAAu;
        return zx >= x0 && zx <= x1 && zy >= y0 && zy <= y1;
    }
};

// The cover of one box: cells of side 2^c, nx per row; cell j of the lane.
struct Cell {
    uint32_t zs, ze;  // first and last code of the cell
    bool valid;       // j < number of cells
    bool full;        // the cell lies inside the box
};

__device__ __forceinline__ Cell box_cell(uint32_t x0, uint32_t y0, uint32_t x1, uint32_t y1, int j) {
    // A side of s cells of size 2^c spans at least s / 2^c cells, so every
    // c below floor(log2(s)) - 4 needs more than 16: start there.
    const uint32_t s = max(x1 - x0, y1 - y0) + 1u;
    int c = max(0, 31 - __clz((int)s) - 4);
    uint32_t nx = (x1 >> c) - (x0 >> c) + 1, ny = (y1 >> c) - (y0 >> c) + 1;
    while (nx * ny > (uint32_t)kMaxCells) {  // c = 16 gives one cell; nx, ny <= 32 here
        c++;
        nx = (x1 >> c) - (x0 >> c) + 1;
        ny = (y1 >> c) - (y0 >> c) + 1;
    }
    Cell cell;
    cell.valid = (uint32_t)j < nx * ny;
    const uint32_t X = ((x0 >> c) + (uint32_t)j % nx) << c;
    const uint32_t Y = ((y0 >> c) + (uint32_t)j / nx) << c;
    const uint32_t side = (1u << c) - 1u;  // c <= 16
    cell.zs = spread16d(X) | (spread16d(Y) << 1);
    cell.ze = (uint32_t)((uint64_t)cell.zs + (1ull << (2 * c)) - 1ull);
    cell.full = X >= x0 && X + side <= x1 && Y >= y0 && Y + side <= y1;
    return cell;
}

// The cover's cells merged into runs: cells taken in Z order, a cell joining
// the run before it when its codes continue that run's (last code + 1 ==
// first code) and it is of the same kind (inside the box, or on its edge).
// A run is one contiguous stretch of codes, so its points are one stretch of
// the sorted keys: two bounds per run instead of two per cell.  Lane r < 16
// receives run r (valid for r < the returned count); lanes >= 16 receive
// run r - 16 as well.  `ord` is 16 words of per-warp scratch.
__device__ __forceinline__ int box_runs(uint32_t x0, uint32_t y0, uint32_t x1, uint32_t y1,
                                        int lane, uint32_t *ord, Cell &run) {
    const int j = lane % kMaxCells;
    const Cell c = box_cell(x0, y0, x1, y1, j);
    // Z rank of this cell among the valid ones (codes of distinct cells differ)
    int rank = 0;
#pragma unroll
    for (int k = 0; k < kMaxCells; k++) {
        const uint32_t zk = __shfl_sync(0xffffffffu, c.zs, k);
        const bool vk = __shfl_sync(0xffffffffu, (int)c.valid, k) != 0;
        rank += (vk && zk < c.zs) ? 1 : 0;
    }
    if (lane < kMaxCells && c.valid) ord[rank] = (uint32_t)j;
    __syncwarp();
    const int nvalid = __popc(__ballot_sync(0xffffffffu, lane < kMaxCells && c.valid));
    // the cell of rank r (lane r), and of rank r - 1
    const int r = j;
    const int src = r < nvalid ? (int)ord[r] : 0;
    const int prv = (r > 0 && r <= nvalid) ? (int)ord[r - 1] : 0;
    __syncwarp();
    const uint32_t zs = __shfl_sync(0xffffffffu, c.zs, src);
    const uint32_t ze = __shfl_sync(0xffffffffu, c.ze, src);
    const bool full = __shfl_sync(0xffffffffu, (int)c.full, src) != 0;
    const uint32_t pze = __shfl_sync(0xffffffffu, c.ze, prv);
    const bool pfull = __shfl_sync(0xffffffffu, (int)c.full, prv) != 0;
    const bool in = r < nvalid;
    const bool starts = in && (r == 0 || pze + 1u != zs || pfull != full);
    const unsigned sm = __ballot_sync(0xffffffffu, lane < kMaxCells && starts);
    const int nruns = __popc(sm);
    // run k: from the k-th start to the cell before the (k+1)-th start
    const int k = j;
    const unsigned fa = __fns(sm, 0, k + 1), fb = __fns(sm, 0, k + 2);  // ~0u: none
    const int first = fa == ~0u ? 0 : (int)fa;
    const int last = fa == ~0u ? 0 : (fb == ~0u ? nvalid - 1 : (int)fb - 1);
    run.zs = __shfl_sync(0xffffffffu, zs, first);
    run.ze = __shfl_sync(0xffffffffu, ze, last < 0 ? 0 : last);
    run.full = __shfl_sync(0xffffffffu, (int)full, first) != 0;
    run.valid = k < nruns;
    return nruns;
}

// Exclusive prefix sum over the warp.
__device__ __forceinline__ uint32_t warp_excl_scan(uint32_t v, int lane, uint32_t &total) {
    uint32_t x = v;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, d);
        if (lane >= d) x += y;
    }
    total = __shfl_sync(0xffffffffu, x, 31);
    return x - v;
}

// Lower bounds of the codes held by lanes c < nc (lane c receives the first
// key position at or above its code; n when the code is above every key):
// 4 lanes per descent, I descents in flight per lane group, so up to 8 I
// codes in one round.  res is 32 words of per-warp scratch.
template <typename V, int I>
__device__ __forceinline__ uint32_t code_lower_bounds(const DevTree &t, const uint32_t *s_lvl,
                                                      uint32_t *res, uint32_t code, bool have,
                                                      int lane) {
    using LG = LeafGeom<uint32_t, V>;
    constexpr int G = 4, NG = 32 / G;
    const int grp = lane / G, gl = lane % G;
    const uint32_t tmax = (uint32_t)t.max_key;
    const uint32_t qa = code < tmax ? code : tmax;
    const uint32_t nd = have ? smem_bound<uint32_t>(s_lvl, t.smem_entries, qa, false) : 0u;
    uint32_t qe[I], node[I];
    bool ups[I];
#pragma unroll
    for (int s = 0; s < I; s++) {
        const int k = s * NG + grp;
        qe[s] = __shfl_sync(0xffffffffu, qa, k);
        node[s] = __shfl_sync(0xffffffffu, nd, k);
        ups[s] = false;
    }
    walk_global<uint32_t, G, I>(t, qe, ups, node, grp, gl);
    int pos[I];
    leaf_bound<uint32_t, V, G, I>(static_cast<const unsigned char *>(t.leaves), node, qe, ups, grp,
                                  gl, pos);
#pragma unroll
    for (int s = 0; s < I; s++)
        if (gl == 0) res[s * NG + grp] = node[s] * (uint32_t)LG::S + (uint32_t)pos[s];
    __syncwarp();
    const uint32_t v = res[lane];
    __syncwarp();
    return code > tmax ? (uint32_t)t.n : v;
}

// Key positions of the box's runs: run r (lane r < nruns) holds the keys
// [lower(zs_r), lower(ze_r + 1)).  When run r + 1 starts at ze_r + 1 the two
// bounds are one descent, so the distinct boundary codes (at most 2 nruns,
// in Z order) are gathered first and each is descended once.  Lane r < 16
// receives lo = the first key position of run r and hi = the position after
// its last key.
template <typename V>
__device__ __forceinline__ void run_bounds(const DevTree &t, const uint32_t *s_lvl, uint32_t *res,
                                           const Cell &run, int nruns, int lane, uint32_t &lo,
                                           uint32_t &hi) {
    const bool rv = lane < nruns;
    const uint32_t nzs = __shfl_sync(0xffffffffu, run.zs, (lane + 1) & 31);
    const bool top = run.ze == 0xFFFFFFFFu;  // no code above: the run ends with the keys
    const bool own_end = rv && !top && !(lane + 1 < nruns && nzs == run.ze + 1u);
    uint32_t nc;
    const uint32_t at = warp_excl_scan(rv ? 1u + (own_end ? 1u : 0u) : 0u, lane, nc);
    if (rv) {
        res[at] = run.zs;
        if (own_end) res[at + 1] = run.ze + 1u;
    }
    __syncwarp();
    const bool have = (uint32_t)lane < nc;
    const uint32_t code = have ? res[lane] : 0u;
    __syncwarp();
    const uint32_t lb = nc <= 8    ? code_lower_bounds<V, 1>(t, s_lvl, res, code, have, lane)
                        : nc <= 16 ? code_lower_bounds<V, 2>(t, s_lvl, res, code, have, lane)
                                   : code_lower_bounds<V, 4>(t, s_lvl, res, code, have, lane);
    lo = __shfl_sync(0xffffffffu, lb, at & 31);
    // the code after run r's: its own end, or the next run's start
    const uint32_t nx = __shfl_sync(0xffffffffu, lb, (at + 1) & 31);
    hi = top ? (uint32_t)t.n : nx;
}

// Cell (0..15) whose run holds item k of the concatenated runs, given each
// lane's exclusive offset `off` (cells past the last hold offset = total).
__device__ __forceinline__ int find_cell(uint32_t off, uint32_t k) {
    int j = 0;
#pragma unroll
    for (int step = kMaxCells / 2; step >= 1; step >>= 1) {
        const uint32_t o = __shfl_sync(0xffffffffu, off, j + step);
        if (o <= k) j += step;
    }
    return j;
}

template <typename V>
__device__ __forceinline__ const unsigned char *block_of(const unsigned char *leaves, uint32_t p) {
    using LG = LeafGeom<uint32_t, V>;
    return leaves + (size_t)(p / LG::S) * LG::BS;
}

// Count pass: counts[i] = points in box i; runs[i * 16 + j] = (first key
// position, length) of cell j's run.
template <typename V>
__global__ void __launch_bounds__(kRThreads, 2)
rect_count_kernel(const __grid_constant__ DevTree t, const uint16_t *__restrict__ x0s,
                  const uint16_t *__restrict__ y0s, const uint16_t *__restrict__ x1s,
                  const uint16_t *__restrict__ y1s, const uint32_t *__restrict__ order, uint64_t nr,
                  uint64_t *__restrict__ counts, uint2 *__restrict__ runs) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    uint32_t *s_lvl = reinterpret_cast<uint32_t *>(smem_raw);
    uint32_t *res = reinterpret_cast<uint32_t *>(smem_raw + (((size_t)t.smem_bytes + 15) / 16 * 16)) +
                    (threadIdx.x >> 5) * 32;
    stage_level<uint32_t>(s_lvl, t);
    __syncthreads();
    using LG = LeafGeom<uint32_t, V>;
    const int lane = threadIdx.x & 31;
    const unsigned char *leaves = static_cast<const unsigned char *>(t.leaves);
    for (uint64_t g = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5; g < nr;
         g += ((uint64_t)gridDim.x * blockDim.x) >> 5) {
        // box i in position g of the processing order; runs follow that order
        const uint64_t i = order ? (uint64_t)order[g] : g;
        const uint32_t x0 = x0s[i], y0 = y0s[i], x1 = x1s[i], y1 = y1s[i];
        if (x0 > x1 || y0 > y1) {  // empty box (warp-uniform)
            if (lane == 0) counts[i] = 0;
            if (lane < kMaxCells) runs[g * kMaxCells + lane] = make_uint2(0u, 0u);
            continue;
        }
        const ZBox box(x0, y0, x1, y1);
        Cell cell;
        const int nruns = box_runs(x0, y0, x1, y1, lane, res, cell);
        uint32_t b, ub;
        run_bounds<V>(t, s_lvl, res, cell, nruns, lane, b, ub);
        const uint32_t len = (lane < kMaxCells && cell.valid && ub > b) ? ub - b : 0u;
        uint32_t total;
        // whole runs of the cells inside the box; edge cells are scanned
        warp_excl_scan(cell.full ? len : 0u, lane, total);
        uint64_t c = total;
        uint32_t P;
        const uint32_t poff = warp_excl_scan(cell.full ? 0u : len, lane, P);
        for (uint32_t base = 0; base < P; base += 64) {  // two loads in flight per lane
            uint32_t key[2];
            bool act[2];
#pragma unroll
            for (int h = 0; h < 2; h++) {
                const uint32_t k = base + 32 * h + lane;
                const int jc = find_cell(poff, k);
                const uint32_t p = __shfl_sync(0xffffffffu, b, jc) + (k - __shfl_sync(0xffffffffu, poff, jc));
                act[h] = k < P;
                key[h] = act[h] ? reinterpret_cast<const uint32_t *>(block_of<V>(leaves, p))[p % LG::S] : 0u;
            }
#pragma unroll
            for (int h = 0; h < 2; h++) c += __popc(__ballot_sync(0xffffffffu, act[h] && box.holds(key[h])));
        }
        if (lane == 0) counts[i] = c;
        // the fill pass reads each run's kind from its length's top bit
        if (lane < kMaxCells) runs[g * kMaxCells + lane] = make_uint2(b, len | (cell.full ? 0x80000000u : 0u));
    }
}

// Fill pass: the IDs of box i's points at ids[offsets[i] ..].  A box with at
// most kWarpSortCap points gathers them in shared memory and writes them
// sorted (warp_sort_small); larger ones are written cell by cell and sorted
// afterwards.
template <typename V>
__global__ void __launch_bounds__(kRThreads)
rect_fill_kernel(const __grid_constant__ DevTree t, const uint16_t *__restrict__ x0s,
                 const uint16_t *__restrict__ y0s, const uint16_t *__restrict__ x1s,
                 const uint16_t *__restrict__ y1s, const uint32_t *__restrict__ order, uint64_t nr,
                 const uint2 *__restrict__ runs,
                 const uint64_t *__restrict__ counts, const uint64_t *__restrict__ offsets,
                 V *__restrict__ ids) {
    __shared__ V s_buf[kRWarps][kWarpSortCap];
    using LG = LeafGeom<uint32_t, V>;
    const int lane = threadIdx.x & 31;
    const unsigned lt = (1u << lane) - 1u;
    V *buf = s_buf[threadIdx.x >> 5];
    const unsigned char *leaves = static_cast<const unsigned char *>(t.leaves);
    for (uint64_t g = (blockIdx.x * (uint64_t)blockDim.x + threadIdx.x) >> 5; g < nr;
         g += ((uint64_t)gridDim.x * blockDim.x) >> 5) {
        const uint64_t i = order ? (uint64_t)order[g] : g;
        const uint32_t x0 = x0s[i], y0 = y0s[i], x1 = x1s[i], y1 = y1s[i];
        const uint64_t cnt = counts[i];
        if (x0 > x1 || y0 > y1 || cnt == 0) continue;
        const ZBox box(x0, y0, x1, y1);
        const uint2 rr = lane < kMaxCells ? runs[g * kMaxCells + lane] : make_uint2(0u, 0u);
        const bool run_full = (rr.y & 0x80000000u) != 0;
        const uint2 run = make_uint2(rr.x, rr.y & 0x7FFFFFFFu);
        const bool buffered = cnt <= (uint64_t)kWarpSortCap;
        V *dst = buffered ? buf : ids + offsets[i];
        uint32_t T;
        const uint32_t off = warp_excl_scan(run.y, lane, T);
        uint32_t out = 0;
        for (uint32_t base = 0; base < T; base += 64) {  // two chunks' loads in flight
            uint32_t key[2];
            V val[2];
            bool act[2], full[2];
#pragma unroll
            for (int h = 0; h < 2; h++) {
                const uint32_t k = base + 32 * h + lane;
                const int jc = find_cell(off, k);
                const uint32_t p = __shfl_sync(0xffffffffu, run.x, jc) + (k - __shfl_sync(0xffffffffu, off, jc));
                full[h] = __shfl_sync(0xffffffffu, (int)run_full, jc) != 0;
                act[h] = k < T;
                const unsigned char *blk = block_of<V>(leaves, p);
                key[h] = act[h] && !full[h] ? reinterpret_cast<const uint32_t *>(blk)[p % LG::S] : 0u;
                val[h] = act[h] ? reinterpret_cast<const V *>(blk + kSectorBytes)[p % LG::S] : (V)0;
            }
#pragma unroll
            for (int h = 0; h < 2; h++) {
                const bool inside = act[h] && (full[h] || box.holds(key[h]));
                const unsigned hit = __ballot_sync(0xffffffffu, inside);
                if (inside) dst[out + __popc(hit & lt)] = val[h];
                out += __popc(hit);
            }
        }
        if (buffered) {
            __syncwarp();
            warp_sort_small<V>(buf, ids + offsets[i], (uint32_t)cnt, lane);
            __syncwarp();
        }
    }
}

// Group key of every box: the 256 x 256 cell of its corner (x0, y0), as a
// row-major cell index (2-D grouping) or the Morton code of the cell (Z-order
// grouping) -- the two reorderings the reference applies to its 1-D range
// queries (grouping2d.cu, zOrder2d.cu:27-54), here on the boxes themselves.
__global__ void rect_group_key_kernel(const uint16_t *__restrict__ x0s,
                                      const uint16_t *__restrict__ y0s, uint64_t nr, int zorder,
                                      uint32_t *__restrict__ key) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < nr;
         i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t cx = (uint32_t)x0s[i] >> 8, cy = (uint32_t)y0s[i] >> 8;
        key[i] = zorder ? (spread16d(cx) | (spread16d(cy) << 1)) : ((cy << 8) | cx);
    }
}

template <typename V>
bt_status rect_impl(const bt_tree *t, int mode, const uint16_t *x0, const uint16_t *y0,
                    const uint16_t *x1, const uint16_t *y1, uint64_t nr, uint64_t *counts,
                    uint64_t *offsets, void *ids, uint64_t cap, uint64_t *h_total, cudaStream_t s) {
    const size_t smem = ((size_t)t->dev.smem_bytes + 15) / 16 * 16 + (size_t)kRWarps * 32 * sizeof(uint32_t);
    auto kc = rect_count_kernel<V>;
    auto kf = rect_fill_kernel<V>;
    if (smem > 48 * 1024)
        BT_CUDA(cudaFuncSetAttribute(kc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int per_sm = 1;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kc, kRThreads, smem);
    const unsigned grid = (unsigned)std::max<uint64_t>(
        1, std::min<uint64_t>((nr + kRWarps - 1) / kRWarps, (uint64_t)sm_count() * std::max(per_sm, 1)));
    WsGuard g_runs(s), g_total(s), g_order(s), g_key(s);
    bt_status st = g_runs.alloc(nr * kMaxCells * sizeof(uint2));
    if (st == BT_OK) st = g_total.alloc(sizeof(uint64_t));
    if (st != BT_OK) return st;
    uint2 *runs = g_runs.as<uint2>();
    uint64_t *d_total = g_total.as<uint64_t>();
    const uint32_t *order = nullptr;
    if (mode != BT_RANGE_BASIC) {  // process the boxes in grouped order
        st = g_order.alloc(nr * sizeof(uint32_t));
        if (st == BT_OK) st = g_key.alloc(nr * sizeof(uint32_t));
        if (st != BT_OK) return st;
        count_launch();
        rect_group_key_kernel<<<(unsigned)std::min<uint64_t>((nr + 255) / 256, (uint64_t)sm_count() * 8),
                                256, 0, s>>>(x0, y0, nr, mode == BT_RANGE_ZORDER, g_key.as<uint32_t>());
        BT_CUDA(cudaGetLastError());
        st = launch_order_u16(g_key.as<uint32_t>(), nr, g_order.as<uint32_t>(), s);
        if (st != BT_OK) return st;
        order = g_order.as<uint32_t>();
    }
    count_launch();
    kc<<<grid, kRThreads, smem, s>>>(t->dev, x0, y0, x1, y1, order, nr, counts, runs);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) st = cuda_fail(e, "rectangle count pass");
    if (st == BT_OK) st = launch_scan_u64(counts, offsets, nr, d_total, s);
    uint64_t total = 0;
    if (st == BT_OK) {
        e = cudaMemcpyAsync(&total, d_total, sizeof(total), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) st = cuda_fail(e, "rectangle total read-back");
    }
    if (st == BT_OK) {
        *h_total = total;
        if (total > cap) {
            st = fail(BT_ERR_CAPACITY, "ids_capacity is below the total hit count");
        } else if (total > 0 && !ids) {
            st = fail(BT_ERR_INVALID_ARGUMENT, "ids is NULL");
        } else if (total > 0) {
            const unsigned fgrid = (unsigned)std::max<uint64_t>(
                1, std::min<uint64_t>((nr + kRWarps - 1) / kRWarps, (uint64_t)sm_count() * 4));
            count_launch();
            kf<<<fgrid, kRThreads, 0, s>>>(t->dev, x0, y0, x1, y1, order, nr, runs, counts, offsets,
                                           (V *)ids);
            e = cudaGetLastError();
            if (e != cudaSuccess) st = cuda_fail(e, "rectangle fill pass");
            if (st == BT_OK) st = launch_segment_sort(t, counts, offsets, nr, ids, s, true);
        }
    }
    return st;
}

}  // namespace
}  // namespace bt

extern "C" {

bt_status bt_rect_search(const bt_tree *t, const uint16_t *x0, const uint16_t *y0,
                         const uint16_t *x1, const uint16_t *y1, uint64_t nr, uint64_t *counts,
                         uint64_t *offsets, void *ids, uint64_t cap, uint64_t *h_total,
                         void *stream) {
    return bt_rect_search_mode(t, BT_RANGE_BASIC, x0, y0, x1, y1, nr, counts, offsets, ids, cap,
                               h_total, stream);
}

bt_status bt_rect_search_mode(const bt_tree *t, int mode, const uint16_t *x0, const uint16_t *y0,
                              const uint16_t *x1, const uint16_t *y1, uint64_t nr,
                              uint64_t *counts, uint64_t *offsets, void *ids, uint64_t cap,
                              uint64_t *h_total, void *stream) {
    using namespace bt;
    if (!t) return fail(BT_ERR_INVALID_ARGUMENT, "tree is NULL");
    if (mode != BT_RANGE_BASIC && mode != BT_RANGE_GROUPED_2D && mode != BT_RANGE_ZORDER)
        return fail(BT_ERR_INVALID_ARGUMENT, "unknown rectangle mode");
    if (nr >= (1ull << 32)) return fail(BT_ERR_INVALID_ARGUMENT, "nr must be below 2^32");
    if (!h_total) return fail(BT_ERR_INVALID_ARGUMENT, "h_total is NULL");
    *h_total = 0;
    if (t->key_bytes != 4)
        return fail(BT_ERR_INVALID_ARGUMENT, "rectangle search needs 32-bit Morton-code keys");
    if (t->n >= (1ull << 31))
        return fail(BT_ERR_NOT_SUPPORTED, "rectangle search needs fewer than 2^31 points");
    if (nr == 0) return BT_OK;
    if (!x0 || !y0 || !x1 || !y1 || !counts || !offsets)
        return fail(BT_ERR_INVALID_ARGUMENT, "a rectangle or output array is NULL");
    int prev = 0;
    BT_CUDA(cudaGetDevice(&prev));
    if (prev != t->device) BT_CUDA(cudaSetDevice(t->device));
    cudaStream_t s = (cudaStream_t)stream;
    if (t->n == 0) {  // no points: every box is empty
        cudaError_t e = cudaMemsetAsync(counts, 0, nr * sizeof(uint64_t), s);
        if (e == cudaSuccess) e = cudaMemsetAsync(offsets, 0, nr * sizeof(uint64_t), s);
        if (prev != t->device) cudaSetDevice(prev);
        return e == cudaSuccess ? BT_OK : cuda_fail(e, "rectangle search on an empty tree");
    }
    const bt_status st =
        t->val_bytes == 4
            ? rect_impl<uint32_t>(t, mode, x0, y0, x1, y1, nr, counts, offsets, ids, cap, h_total, s)
            : rect_impl<uint64_t>(t, mode, x0, y0, x1, y1, nr, counts, offsets, ids, cap, h_total, s);
    if (prev != t->device) cudaSetDevice(prev);
    return st;
}

}  // extern "C"
