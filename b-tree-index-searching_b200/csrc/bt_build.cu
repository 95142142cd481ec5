// Bulk build: sorted (key, value) arrays -> leaf blocks + separator levels.  Replaces genBPlusTree (BPTree.cu:127-306): the reference copies
// PAGESIZE pairs per leaf page (assignDataToLeaf, BPTree.cu:73-125) and builds
// (child.max, child index) pages per level with a host-synchronized loop
// (kernelMaxIntermidatePage, BPTree.cu:28-70, :218-243).  Here the leaf level
// is the sorted array itself, cut into 32-byte key sectors with their values
// alongside, and each separator level is one strided gather of the level
// below; nothing is pointer-linked, so the whole build is a few streaming
// passes with no host round trip between levels.
#include <algorithm>
#include <cstdio>
#include <cstring>
#include <vector>

#include "bt_internal.cuh"

namespace bt {
namespace {

// One thread per leaf position: copy keys and values into their leaf block
// (all-ones keys pad the last block), check the ascending order of keys
// (bit 0) and values (bit 1), and emit the bottom separator level (the last
// key of every block).
template <typename K, typename V>
__global__ void __launch_bounds__(256)
copy_pad_kernel(const K *__restrict__ keys, const V *__restrict__ vals, uint64_t n,
                uint64_t n_pos, unsigned char *__restrict__ leaves, K *__restrict__ bottom_sep,
                unsigned int *__restrict__ flags) {
    using LG = LeafGeom<K, V>;
    unsigned int f = 0;
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n_pos;
         i += (uint64_t)gridDim.x * blockDim.x) {
        K k = key_max<K>();
        V v = 0;
        if (i < n) {
            k = keys[i];
            v = vals[i];
            if (i + 1 < n) {
                if (keys[i + 1] < k) f |= 1u;
                if (vals[i + 1] < v) f |= 2u;
            }
        }
        const uint64_t b = i / LG::S;
        const int j = (int)(i % LG::S);
        unsigned char *blk = leaves + b * LG::BS;
        reinterpret_cast<K *>(blk)[j] = k;
        reinterpret_cast<V *>(blk + kSectorBytes)[j] = v;
        if constexpr (kSectorBytes + LG::VB < LG::BS) {
            // the block's padding after its values (zero, so tree images are
            // deterministic)
            constexpr int PW = (LG::BS - kSectorBytes - LG::VB) / 4;
            if (j < PW) reinterpret_cast<uint32_t *>(blk + kSectorBytes + LG::VB)[j] = 0u;
        }
        if (j == LG::S - 1) bottom_sep[b] = k;
    }
    unsigned int w = __reduce_or_sync(0xffffffffu, f);
    if ((threadIdx.x & 31) == 0 && w) atomicOr(flags, w);
}

// dst[j] = src[j*F + F-1] for j < entries (maximum of node j of the level
// below), all-ones for the padding up to nodes*F.
template <typename K>
__global__ void __launch_bounds__(256)
level_kernel(const K *__restrict__ src, uint64_t entries, uint64_t padded, K *__restrict__ dst) {
    constexpr int F = kLineBytes / sizeof(K);
    for (uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; j < padded;
         j += (uint64_t)gridDim.x * blockDim.x)
        dst[j] = j < entries ? src[j * F + F - 1] : key_max<K>();
}

template <typename K>
__global__ void pad_kernel(K *__restrict__ dst, uint64_t from, uint64_t to) {
    for (uint64_t j = from + blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; j < to;
         j += (uint64_t)gridDim.x * blockDim.x)
        dst[j] = key_max<K>();
}

unsigned grid_for(uint64_t n, int block) {
    uint64_t g = (n + block - 1) / block;
    uint64_t cap = (uint64_t)sm_count() * 16;
    if (g > cap) g = cap;
    return (unsigned)std::max<uint64_t>(1, g);
}

template <typename K, typename V>
bt_status build_impl(bt_tree *t, const void *d_keys, const void *d_vals, cudaStream_t s) {
    constexpr int S = kSectorBytes / sizeof(K);
    constexpr int F = kLineBytes / sizeof(K);
    const uint64_t n = t->n;
    t->n_sectors = (n + S - 1) / S;
    const uint64_t n_pos = t->n_sectors * S;

    // Level geometry, bottom-up, then stored root first.
    uint64_t ent_bu[kMaxLevels], nod_bu[kMaxLevels];
    int L = 0;
    uint64_t entries = t->n_sectors;
    for (;;) {
        if (L >= kMaxLevels) return fail(BT_ERR_INVALID_ARGUMENT, "too many keys");
        uint64_t nodes = (entries + F - 1) / F;
        ent_bu[L] = entries;
        nod_bu[L] = nodes;
        L++;
        if (nodes == 1) break;
        entries = nodes;
    }
    DevTree &dt = t->dev;
    dt.nlevels = L;
    uint64_t off = 0;
    for (int lvl = 0; lvl < L; lvl++) {
        t->lvl_entries[lvl] = ent_bu[L - 1 - lvl];
        t->lvl_nodes[lvl] = nod_bu[L - 1 - lvl];
        dt.lvl_off[lvl] = off;
        off += t->lvl_nodes[lvl] * F;
    }
    t->seps_elems = off;

    const size_t leaf_bytes = t->n_sectors * (size_t)LeafGeom<K, V>::BS;
    BT_CUDA(cudaMalloc(&t->d_leaves, leaf_bytes));
    BT_CUDA(cudaMalloc(&t->d_seps, t->seps_elems * sizeof(K)));
    WsGuard g_flags(s);
    bt_status st = g_flags.alloc(sizeof(unsigned int));
    if (st != BT_OK) return st;
    unsigned int *d_flags = g_flags.as<unsigned int>();
    BT_CUDA(cudaMemsetAsync(d_flags, 0, sizeof(unsigned int), s));

    K *seps = (K *)t->d_seps;
    K *bottom = seps + dt.lvl_off[L - 1];
    count_launch();
    copy_pad_kernel<K, V><<<grid_for(n_pos, 256), 256, 0, s>>>(
        (const K *)d_keys, (const V *)d_vals, n, n_pos, (unsigned char *)t->d_leaves, bottom,
        d_flags);
    const uint64_t bottom_pad = t->lvl_nodes[L - 1] * F;
    if (bottom_pad > t->n_sectors) {
        count_launch();
        pad_kernel<K><<<grid_for(bottom_pad - t->n_sectors, 256), 256, 0, s>>>(
            bottom, t->n_sectors, bottom_pad);
    }
    for (int lvl = L - 2; lvl >= 0; lvl--) {
        const uint64_t padded = t->lvl_nodes[lvl] * F;
        count_launch();
        level_kernel<K><<<grid_for(padded, 256), 256, 0, s>>>(
            seps + dt.lvl_off[lvl + 1], t->lvl_entries[lvl], padded, seps + dt.lvl_off[lvl]);
    }
    BT_CUDA(cudaGetLastError());

    unsigned int flags = 0;
    K kmin = 0, kmax = 0;
    BT_CUDA(cudaMemcpyAsync(&flags, d_flags, sizeof(flags), cudaMemcpyDeviceToHost, s));
    const unsigned char *lv = (const unsigned char *)t->d_leaves;
    BT_CUDA(cudaMemcpyAsync(&kmin, lv, sizeof(K), cudaMemcpyDeviceToHost, s));
    BT_CUDA(cudaMemcpyAsync(&kmax,
                            lv + ((n - 1) / S) * LeafGeom<K, V>::BS + ((n - 1) % S) * sizeof(K),
                            sizeof(K), cudaMemcpyDeviceToHost, s));
    BT_CUDA(cudaStreamSynchronize(s));
    if (flags & 1u) return fail(BT_ERR_UNSORTED, "build keys are not sorted ascending");
    t->values_sorted = (flags & 2u) ? 0 : 1;
    t->min_key = (uint64_t)kmin;
    t->max_key = (uint64_t)kmax;

    dt.leaves = t->d_leaves;
    dt.seps = t->d_seps;
    dt.n = n;
    dt.max_key = t->max_key;
    dt.n_sectors = t->n_sectors;
    // The deepest separator level whose real entries fit the shared-memory
    // budget; a binary search over it resolves every level above it at once.
    int sl = 0;
    while (sl + 1 <= L - 1 && t->lvl_entries[sl + 1] * sizeof(K) <= kSmemTopBudget) sl++;
    dt.smem_level = sl;
    dt.smem_entries = (uint32_t)t->lvl_entries[sl];
    // whole 128-byte bank rows, so the swizzle stays inside the staged region
    dt.smem_bytes = (uint32_t)(((t->lvl_entries[sl] * sizeof(K)) + 127) / 128 * 128);
    return BT_OK;
}

template <typename K>
bt_status build_k(bt_tree *t, const void *dk, const void *dv, cudaStream_t s) {
    return t->val_bytes == 4 ? build_impl<K, uint32_t>(t, dk, dv, s)
                             : build_impl<K, uint64_t>(t, dk, dv, s);
}

void free_tree(bt_tree *t) {
    if (!t) return;
    if (t->learned) free_learned(t->learned);
    if (t->d_leaves) cudaFree(t->d_leaves);
    if (t->d_seps) cudaFree(t->d_seps);
    delete t;
}

}  // namespace
}  // namespace bt

extern "C" {

bt_status bt_build(const void *d_sorted_keys, const void *d_values, uint64_t n, int key_bytes,
                   int value_bytes, void *stream, bt_tree **out) {
    using namespace bt;
    if (!out) return fail(BT_ERR_INVALID_ARGUMENT, "out is NULL");
    *out = nullptr;
    if (key_bytes != 4 && key_bytes != 8)
        return fail(BT_ERR_INVALID_ARGUMENT, "key_bytes must be 4 or 8");
    if (value_bytes != 4 && value_bytes != 8)
        return fail(BT_ERR_INVALID_ARGUMENT, "value_bytes must be 4 or 8");
    if (n > 0 && (!d_sorted_keys || !d_values))
        return fail(BT_ERR_INVALID_ARGUMENT, "keys or values pointer is NULL");
    // leaf block and node indices are 32-bit in the search kernels
    if (n >= (1ull << 34)) return fail(BT_ERR_INVALID_ARGUMENT, "n must be below 2^34");
    int dev = 0;
    BT_CUDA(cudaGetDevice(&dev));
    bt_status st = require_device(dev);
    if (st != BT_OK) return st;
    bt_tree *t = new bt_tree();
    std::memset(t, 0, sizeof(*t));
    t->device = dev;
    t->key_bytes = key_bytes;
    t->val_bytes = value_bytes;
    t->n = n;
    t->values_sorted = 1;
    t->search_cfg = default_search_cfg(key_bytes);
    if (n > 0) {
        cudaStream_t s = (cudaStream_t)stream;
        st = key_bytes == 4 ? build_k<uint32_t>(t, d_sorted_keys, d_values, s)
                            : build_k<uint64_t>(t, d_sorted_keys, d_values, s);
        if (st != BT_OK) {
            free_tree(t);
            return st;
        }
    }
    *out = t;
    return BT_OK;
}

bt_status bt_sort_pairs(const void *d_keys, const void *d_values, uint64_t n, int key_bytes,
                        int value_bytes, void *d_keys_out, void *d_values_out, void *stream) {
    using namespace bt;
    if ((key_bytes != 4 && key_bytes != 8) || (value_bytes != 4 && value_bytes != 8))
        return fail(BT_ERR_INVALID_ARGUMENT, "key_bytes and value_bytes must be 4 or 8");
    if (n == 0) return BT_OK;
    if (!d_keys || !d_values || !d_keys_out || !d_values_out)
        return fail(BT_ERR_INVALID_ARGUMENT, "a key or value pointer is NULL");
    if (d_keys_out == d_keys || d_values_out == d_values)
        return fail(BT_ERR_INVALID_ARGUMENT, "outputs must not alias the inputs");
    int dev = 0;
    BT_CUDA(cudaGetDevice(&dev));
    bt_status st = require_device(dev);
    if (st != BT_OK) return st;
    return launch_sort_pairs(key_bytes, value_bytes, d_keys, d_values, n, d_keys_out, d_values_out,
                             (cudaStream_t)stream);
}

bt_status bt_build_unsorted(const void *d_keys, const void *d_values, uint64_t n, int key_bytes,
                            int value_bytes, void *stream, bt_tree **out) {
    using namespace bt;
    if (!out) return fail(BT_ERR_INVALID_ARGUMENT, "out is NULL");
    *out = nullptr;
    if ((key_bytes != 4 && key_bytes != 8) || (value_bytes != 4 && value_bytes != 8))
        return fail(BT_ERR_INVALID_ARGUMENT, "key_bytes and value_bytes must be 4 or 8");
    if (n == 0) return bt_build(nullptr, nullptr, 0, key_bytes, value_bytes, stream, out);
    if (!d_keys || !d_values) return fail(BT_ERR_INVALID_ARGUMENT, "keys or values pointer is NULL");
    int dev = 0;
    BT_CUDA(cudaGetDevice(&dev));
    bt_status st = require_device(dev);
    if (st != BT_OK) return st;
    cudaStream_t s = (cudaStream_t)stream;
    void *sk = nullptr, *sv = nullptr;
    st = ws_alloc(&sk, n * key_bytes, s);
    if (st == BT_OK) st = ws_alloc(&sv, n * value_bytes, s);
    if (st == BT_OK) st = launch_sort_pairs(key_bytes, value_bytes, d_keys, d_values, n, sk, sv, s);
    if (st == BT_OK) st = bt_build(sk, sv, n, key_bytes, value_bytes, stream, out);
    ws_free(sk, s);
    ws_free(sv, s);
    return st;
}

bt_status bt_build_host(const void *h_sorted_keys, const void *h_values, uint64_t n,
                        int key_bytes, int value_bytes, void *stream, bt_tree **out) {
    using namespace bt;
    if (!out) return fail(BT_ERR_INVALID_ARGUMENT, "out is NULL");
    *out = nullptr;
    if ((key_bytes != 4 && key_bytes != 8) || (value_bytes != 4 && value_bytes != 8))
        return fail(BT_ERR_INVALID_ARGUMENT, "key_bytes and value_bytes must be 4 or 8");
    if (n == 0) return bt_build(nullptr, nullptr, 0, key_bytes, value_bytes, stream, out);
    if (!h_sorted_keys || !h_values)
        return fail(BT_ERR_INVALID_ARGUMENT, "keys or values pointer is NULL");
    cudaStream_t s = (cudaStream_t)stream;
    void *dk = nullptr, *dv = nullptr;
    bt_status st = ws_alloc(&dk, n * key_bytes, s);
    if (st == BT_OK) st = ws_alloc(&dv, n * value_bytes, s);
    if (st == BT_OK) {
        cudaError_t e = cudaMemcpyAsync(dk, h_sorted_keys, n * key_bytes, cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(dv, h_values, n * value_bytes, cudaMemcpyHostToDevice, s);
        if (e != cudaSuccess) st = cuda_fail(e, "cudaMemcpyAsync");
    }
    if (st == BT_OK) st = bt_build(dk, dv, n, key_bytes, value_bytes, stream, out);
    ws_free(dk, s);
    ws_free(dv, s);
    return st;
}

// ---- tree image: the built arrays and their descriptor in one file --------

namespace {

constexpr char kImageMagic[8] = {'B', 'T', 'B', '2', '0', '0', 'I', 'M'};
constexpr uint32_t kImageVersion = 1;

struct ImageHeader {
    char magic[8];
    uint32_t version;
    int32_t key_bytes, val_bytes, values_sorted;
    uint64_t n, n_sectors, seps_elems, min_key, max_key;
    uint64_t lvl_nodes[bt::kMaxLevels], lvl_entries[bt::kMaxLevels], lvl_off[bt::kMaxLevels];
    int32_t nlevels, smem_level;
    uint32_t smem_entries, smem_bytes;
    uint64_t leaf_bytes, sep_bytes;
};

// Copies `bytes` between a device buffer and a file through a host bounce
// buffer of at most 64 MiB.
bt_status stream_file(FILE *f, void *dptr, uint64_t bytes, bool write) {
    using namespace bt;
    const uint64_t chunk = std::min<uint64_t>(bytes, 64ull << 20);
    std::vector<unsigned char> buf(chunk ? chunk : 1);
    for (uint64_t o = 0; o < bytes; o += chunk) {
        const uint64_t m = std::min(chunk, bytes - o);
        if (write) {
            BT_CUDA(cudaMemcpy(buf.data(), (const unsigned char *)dptr + o, m, cudaMemcpyDeviceToHost));
            if (fwrite(buf.data(), 1, m, f) != m) return fail(BT_ERR_INVALID_ARGUMENT, "tree image: write failed");
        } else {
            if (fread(buf.data(), 1, m, f) != m) return fail(BT_ERR_INVALID_ARGUMENT, "tree image: file is truncated");
            BT_CUDA(cudaMemcpy((unsigned char *)dptr + o, buf.data(), m, cudaMemcpyHostToDevice));
        }
    }
    return BT_OK;
}

}  // namespace

bt_status bt_build_from_files(const char *keys_path, const char *values_path, uint64_t n,
                              void *stream, bt_tree **out) {
    using namespace bt;
    if (!keys_path || !values_path || !out) return fail(BT_ERR_INVALID_ARGUMENT, "path or out is NULL");
    *out = nullptr;
    if (n == 0) return bt_build(nullptr, nullptr, 0, 8, 8, stream, out);
    std::vector<uint64_t> hk(n), hv(n);
    const char *paths[2] = {keys_path, values_path};
    std::vector<uint64_t> *bufs[2] = {&hk, &hv};
    for (int i = 0; i < 2; i++) {
        FILE *f = fopen(paths[i], "rb");
        if (!f) return fail(BT_ERR_INVALID_ARGUMENT, std::string("cannot open ") + paths[i]);
        const size_t got = fread(bufs[i]->data(), sizeof(uint64_t), n, f);
        fclose(f);
        if (got != n)
            return fail(BT_ERR_INVALID_ARGUMENT, std::string(paths[i]) + " holds fewer than n values");
    }
    int dev = 0;
    BT_CUDA(cudaGetDevice(&dev));
    bt_status st = require_device(dev);
    if (st != BT_OK) return st;
    cudaStream_t s = (cudaStream_t)stream;
    WsGuard gk(s), gv(s);
    st = gk.alloc(n * sizeof(uint64_t));
    if (st == BT_OK) st = gv.alloc(n * sizeof(uint64_t));
    if (st != BT_OK) return st;
    BT_CUDA(cudaMemcpyAsync(gk.p, hk.data(), n * sizeof(uint64_t), cudaMemcpyHostToDevice, s));
    BT_CUDA(cudaMemcpyAsync(gv.p, hv.data(), n * sizeof(uint64_t), cudaMemcpyHostToDevice, s));
    st = bt_build_unsorted(gk.p, gv.p, n, 8, 8, stream, out);
    BT_CUDA(cudaStreamSynchronize(s));  // the host copies outlive the uploads
    return st;
}

bt_status bt_save(const bt_tree *t, const char *path) {
    using namespace bt;
    if (!t || !path) return fail(BT_ERR_INVALID_ARGUMENT, "tree or path is NULL");
    ImageHeader h;
    std::memset(&h, 0, sizeof(h));
    std::memcpy(h.magic, kImageMagic, 8);
    h.version = kImageVersion;
    h.key_bytes = t->key_bytes;
    h.val_bytes = t->val_bytes;
    h.values_sorted = t->values_sorted;
    h.n = t->n;
    h.n_sectors = t->n_sectors;
    h.seps_elems = t->seps_elems;
    h.min_key = t->min_key;
    h.max_key = t->max_key;
    for (int l = 0; l < kMaxLevels; l++) {
        h.lvl_nodes[l] = t->lvl_nodes[l];
        h.lvl_entries[l] = t->lvl_entries[l];
        h.lvl_off[l] = t->dev.lvl_off[l];
    }
    h.nlevels = t->dev.nlevels;
    h.smem_level = t->dev.smem_level;
    h.smem_entries = t->dev.smem_entries;
    h.smem_bytes = t->dev.smem_bytes;
    h.leaf_bytes = t->n ? t->n_sectors * (uint64_t)leaf_stride(t->key_bytes, t->val_bytes) : 0;
    h.sep_bytes = t->n ? t->seps_elems * (uint64_t)t->key_bytes : 0;
    FILE *f = fopen(path, "wb");
    if (!f) return fail(BT_ERR_INVALID_ARGUMENT, std::string("tree image: cannot open ") + path);
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(t->device);
    bt_status st = fwrite(&h, sizeof(h), 1, f) == 1 ? BT_OK
                                                    : fail(BT_ERR_INVALID_ARGUMENT, "tree image: write failed");
    if (st == BT_OK && h.leaf_bytes) st = stream_file(f, t->d_leaves, h.leaf_bytes, true);
    if (st == BT_OK && h.sep_bytes) st = stream_file(f, t->d_seps, h.sep_bytes, true);
    cudaSetDevice(prev);
    if (fclose(f) != 0 && st == BT_OK) st = fail(BT_ERR_INVALID_ARGUMENT, "tree image: close failed");
    return st;
}

bt_status bt_load(const char *path, void *stream, bt_tree **out) {
    using namespace bt;
    (void)stream;
    if (!path || !out) return fail(BT_ERR_INVALID_ARGUMENT, "path or out is NULL");
    *out = nullptr;
    int dev = 0;
    BT_CUDA(cudaGetDevice(&dev));
    bt_status st = require_device(dev);
    if (st != BT_OK) return st;
    FILE *f = fopen(path, "rb");
    if (!f) return fail(BT_ERR_INVALID_ARGUMENT, std::string("tree image: cannot open ") + path);
    ImageHeader h;
    if (fread(&h, sizeof(h), 1, f) != 1 || std::memcmp(h.magic, kImageMagic, 8) != 0 ||
        h.version != kImageVersion || (h.key_bytes != 4 && h.key_bytes != 8) ||
        (h.val_bytes != 4 && h.val_bytes != 8) || h.nlevels < 0 || h.nlevels > kMaxLevels ||
        h.leaf_bytes != (h.n ? h.n_sectors * (uint64_t)leaf_stride(h.key_bytes, h.val_bytes) : 0) ||
        h.sep_bytes != (h.n ? h.seps_elems * (uint64_t)h.key_bytes : 0)) {
        fclose(f);
        return fail(BT_ERR_INVALID_ARGUMENT, "tree image: not a tree image of this version");
    }
    bt_tree *t = new bt_tree();
    std::memset(t, 0, sizeof(*t));
    t->device = dev;
    t->key_bytes = h.key_bytes;
    t->val_bytes = h.val_bytes;
    t->values_sorted = h.values_sorted;
    t->n = h.n;
    t->n_sectors = h.n_sectors;
    t->seps_elems = h.seps_elems;
    t->min_key = h.min_key;
    t->max_key = h.max_key;
    t->search_cfg = default_search_cfg(h.key_bytes);
    for (int l = 0; l < kMaxLevels; l++) {
        t->lvl_nodes[l] = h.lvl_nodes[l];
        t->lvl_entries[l] = h.lvl_entries[l];
        t->dev.lvl_off[l] = h.lvl_off[l];
    }
    cudaError_t e = cudaSuccess;
    if (h.leaf_bytes) e = cudaMalloc(&t->d_leaves, h.leaf_bytes);
    if (e == cudaSuccess && h.sep_bytes) e = cudaMalloc(&t->d_seps, h.sep_bytes);
    st = e == cudaSuccess ? BT_OK : cuda_fail(e, "tree image: device allocation");
    if (st == BT_OK && h.leaf_bytes) st = stream_file(f, t->d_leaves, h.leaf_bytes, false);
    if (st == BT_OK && h.sep_bytes) st = stream_file(f, t->d_seps, h.sep_bytes, false);
    fclose(f);
    if (st != BT_OK) {
        free_tree(t);
        return st;
    }
    DevTree &dt = t->dev;
    dt.leaves = t->d_leaves;
    dt.seps = t->d_seps;
    dt.n = t->n;
    dt.max_key = t->max_key;
    dt.n_sectors = t->n_sectors;
    dt.nlevels = h.nlevels;
    dt.smem_level = h.smem_level;
    dt.smem_entries = h.smem_entries;
    dt.smem_bytes = h.smem_bytes;
    *out = t;
    return BT_OK;
}

bt_status bt_destroy(bt_tree *tree) {
    if (!tree) return BT_OK;
    cudaDeviceSynchronize();
    bt::free_tree(tree);
    return BT_OK;
}

bt_status bt_set_search_config(bt_tree *t, int lanes_per_query, int rounds) {
    using namespace bt;
    if (!t) return fail(BT_ERR_INVALID_ARGUMENT, "tree is NULL");
    const int k = search_cfg_index(lanes_per_query, rounds);
    if (k < 0) return fail(BT_ERR_INVALID_ARGUMENT, "unsupported (lanes, rounds) search configuration");
    t->search_cfg = k;
    return BT_OK;
}

bt_status bt_get_info(const bt_tree *t, bt_info *info) {
    using namespace bt;
    if (!t || !info) return fail(BT_ERR_INVALID_ARGUMENT, "tree or info is NULL");
    std::memset(info, 0, sizeof(*info));
    info->num_keys = t->n;
    info->key_bytes = (uint32_t)t->key_bytes;
    info->value_bytes = (uint32_t)t->val_bytes;
    info->num_levels = (uint32_t)t->dev.nlevels;
    info->fanout = (uint32_t)(kLineBytes / t->key_bytes);
    info->leaf_keys = (uint32_t)(kSectorBytes / t->key_bytes);
    info->smem_levels = (uint32_t)(t->n ? t->dev.smem_level + 1 : 0);
    info->device_bytes = t->n_sectors * (uint64_t)leaf_stride(t->key_bytes, t->val_bytes) +
                         t->seps_elems * t->key_bytes;
    info->min_key = t->min_key;
    info->max_key = t->max_key;
    info->device = t->device;
    info->values_sorted = t->values_sorted;
    info->lanes_per_query = (uint32_t)search_cfg_lanes(t->search_cfg);
    info->rounds = (uint32_t)search_cfg_rounds(t->search_cfg);
    return BT_OK;
}

}  // extern "C"
