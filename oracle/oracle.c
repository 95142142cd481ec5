/*
 * CPU oracle for the B+tree index search path -- TEST INFRASTRUCTURE ONLY.
 * See oracle.h for the contract.  Only tests/, __graft_entry__.smoke() and
 * bench.py's CPU-baseline leg load this library, and only to check results or
 * as the timed CPU baseline.  The shipped engine never calls it.
 */
#include "oracle.h"

#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

static int orc_threads(int nthreads) {
#ifdef _OPENMP
    return nthreads > 0 ? nthreads : omp_get_max_threads();
#else
    (void)nthreads;
    return 1;
#endif
}

/* ------------------------------------------------------------------------ */
/* Ground truth: binary search over the sorted key array.                      */
/* ------------------------------------------------------------------------ */

/* first index i in [0, n) with keys[i] >= q (or > q when upper), else n */
#define DEFINE_BOUND(NAME, KT)                                                 \
    static inline uint64_t NAME(const KT *keys, uint64_t n, uint64_t q,        \
                                int upper) {                                   \
        uint64_t lo = 0, len = n;                                              \
        while (len > 0) {                                                      \
            uint64_t half = len >> 1;                                          \
            uint64_t k = (uint64_t)keys[lo + half];                            \
            int go_right = upper ? (k <= q) : (k < q);                         \
            if (go_right) {                                                    \
                lo += half + 1;                                                \
                len -= half + 1;                                               \
            } else {                                                           \
                len = half;                                                    \
            }                                                                  \
        }                                                                      \
        return lo;                                                             \
    }
DEFINE_BOUND(bound_u32, uint32_t)
DEFINE_BOUND(bound_u64, uint64_t)

static inline uint64_t key_at(const void *keys, int kb, uint64_t i) {
    return kb == 4 ? (uint64_t)((const uint32_t *)keys)[i]
                   : ((const uint64_t *)keys)[i];
}

static inline uint64_t bound_any(const void *keys, int kb, uint64_t n,
                                 uint64_t q, int upper) {
    return kb == 4 ? bound_u32((const uint32_t *)keys, n, q, upper)
                   : bound_u64((const uint64_t *)keys, n, q, upper);
}

static inline void store_val(void *out, int vb, uint64_t i, uint64_t v) {
    if (vb == 4)
        ((uint32_t *)out)[i] = (uint32_t)v;
    else
        ((uint64_t *)out)[i] = v;
}

static inline uint64_t val_at(const void *vals, int vb, uint64_t i) {
    return vb == 4 ? (uint64_t)((const uint32_t *)vals)[i]
                   : ((const uint64_t *)vals)[i];
}

static int widths_ok(int kb, int vb) {
    return (kb == 4 || kb == 8) && (vb == 4 || vb == 8);
}

int orc_point_search(const void *keys, const void *vals, uint64_t n,
                     int key_bytes, int val_bytes, const void *queries,
                     uint64_t nq, void *out, int nthreads) {
    if (!widths_ok(key_bytes, val_bytes)) return -1;
    const uint64_t miss = val_bytes == 4 ? 0xFFFFFFFFull : REFC_INVALID;
    const int nt = orc_threads(nthreads);
    int64_t i;
#pragma omp parallel for num_threads(nt) schedule(static)
    for (i = 0; i < (int64_t)nq; i++) {
        uint64_t q = key_at(queries, key_bytes, (uint64_t)i);
        uint64_t p = bound_any(keys, key_bytes, n, q, 0);
        uint64_t v = (p < n && key_at(keys, key_bytes, p) == q)
                         ? val_at(vals, val_bytes, p)
                         : miss;
        store_val(out, val_bytes, (uint64_t)i, v);
    }
    return 0;
}

int orc_bounds(const void *keys, uint64_t n, int key_bytes,
               const void *queries, uint64_t nq, int upper, uint64_t *pos,
               int nthreads) {
    if (key_bytes != 4 && key_bytes != 8) return -1;
    const int nt = orc_threads(nthreads);
    int64_t i;
#pragma omp parallel for num_threads(nt) schedule(static)
    for (i = 0; i < (int64_t)nq; i++)
        pos[i] = bound_any(keys, key_bytes, n,
                           key_at(queries, key_bytes, (uint64_t)i), upper);
    return 0;
}

int orc_range_count(const void *keys, uint64_t n, int key_bytes,
                    const void *lo, const void *hi, uint64_t nq,
                    uint64_t *counts, int nthreads) {
    if (key_bytes != 4 && key_bytes != 8) return -1;
    const int nt = orc_threads(nthreads);
    int64_t i;
#pragma omp parallel for num_threads(nt) schedule(static)
    for (i = 0; i < (int64_t)nq; i++) {
        uint64_t a = key_at(lo, key_bytes, (uint64_t)i);
        uint64_t b = key_at(hi, key_bytes, (uint64_t)i);
        if (a > b) {
            counts[i] = 0;
            continue;
        }
        uint64_t l = bound_any(keys, key_bytes, n, a, 0);
        uint64_t u = bound_any(keys, key_bytes, n, b, 1);
        counts[i] = u - l;
    }
    return 0;
}

static int cmp_u32(const void *a, const void *b) {
    uint32_t x = *(const uint32_t *)a, y = *(const uint32_t *)b;
    return (x > y) - (x < y);
}
static int cmp_u64(const void *a, const void *b) {
    uint64_t x = *(const uint64_t *)a, y = *(const uint64_t *)b;
    return (x > y) - (x < y);
}

int orc_range_ids(const void *keys, const void *vals, uint64_t n,
                  int key_bytes, int val_bytes, const void *lo,
                  const void *hi, uint64_t nq, const uint64_t *offsets,
                  void *ids, int nthreads) {
    if (!widths_ok(key_bytes, val_bytes)) return -1;
    const int nt = orc_threads(nthreads);
    int64_t i;
#pragma omp parallel for num_threads(nt) schedule(dynamic, 64)
    for (i = 0; i < (int64_t)nq; i++) {
        uint64_t a = key_at(lo, key_bytes, (uint64_t)i);
        uint64_t b = key_at(hi, key_bytes, (uint64_t)i);
        if (a > b) continue;
        uint64_t l = bound_any(keys, key_bytes, n, a, 0);
        uint64_t u = bound_any(keys, key_bytes, n, b, 1);
        uint64_t o = offsets[i];
        for (uint64_t p = l; p < u; p++)
            store_val(ids, val_bytes, o + (p - l), val_at(vals, val_bytes, p));
        if (u - l > 1) {
            if (val_bytes == 4)
                qsort((uint32_t *)ids + o, u - l, 4, cmp_u32);
            else
                qsort((uint64_t *)ids + o, u - l, 8, cmp_u64);
        }
    }
    return 0;
}

uint32_t orc_morton2_u16(uint16_t x, uint16_t y) {
    uint32_t z = 0;
    for (int b = 0; b < 16; b++) {
        z |= (uint32_t)((x >> b) & 1u) << (2 * b);
        z |= (uint32_t)((y >> b) & 1u) << (2 * b + 1);
    }
    return z;
}

static inline void morton_decode(uint32_t z, uint32_t *x, uint32_t *y) {
    uint32_t a = 0, b = 0;
    for (int i = 0; i < 16; i++) {
        a |= ((z >> (2 * i)) & 1u) << i;
        b |= ((z >> (2 * i + 1)) & 1u) << i;
    }
    *x = a;
    *y = b;
}

/* Every point inside [x0,x1]x[y0,y1] has a Morton code inside
 * [Z(x0,y0), Z(x1,y1)] (interleaving is monotone in each coordinate), so a
 * scan of that Z interval with an exact (x, y) filter finds all hits. */
int orc_rect_search(const uint32_t *z_sorted, const uint32_t *ids_sorted,
                    uint64_t n, const uint16_t *x0, const uint16_t *y0,
                    const uint16_t *x1, const uint16_t *y1, uint64_t nq,
                    uint64_t *counts, const uint64_t *offsets, uint32_t *ids,
                    int nthreads) {
    const int nt = orc_threads(nthreads);
    int64_t i;
#pragma omp parallel for num_threads(nt) schedule(dynamic, 16)
    for (i = 0; i < (int64_t)nq; i++) {
        uint32_t zlo = orc_morton2_u16(x0[i], y0[i]);
        uint32_t zhi = orc_morton2_u16(x1[i], y1[i]);
        uint64_t c = 0;
        if (x0[i] <= x1[i] && y0[i] <= y1[i]) {
            uint64_t p = bound_u32(z_sorted, n, zlo, 0);
            uint64_t o = offsets ? offsets[i] : 0;
            for (; p < n && z_sorted[p] <= zhi; p++) {
                uint32_t x, y;
                morton_decode(z_sorted[p], &x, &y);
                if (x >= x0[i] && x <= x1[i] && y >= y0[i] && y <= y1[i]) {
                    if (ids) ids[o + c] = ids_sorted[p];
                    c++;
                }
            }
            if (ids && c > 1) qsort(ids + o, c, 4, cmp_u32);
        }
        counts[i] = c;
    }
    return 0;
}

/* ------------------------------------------------------------------------ */
/* Literal restatement of the reference's page tree (BPTree.h:14-23).       */
/* ------------------------------------------------------------------------ */

typedef struct {
    uint64_t key[REFC_PAGESIZE];
    uint64_t data[REFC_PAGESIZE];
    int leafFlag;
    int size;
    uint64_t max;
    uint64_t min;
    int previous;
    int next;
} refc_page;

struct refc_tree {
    refc_page *pages;
    uint64_t npages;
    uint64_t root;
};

/* key[i] for i in [0, 2*PAGESIZE): the reference's AoS page puts data[]
 * right after key[], so key[PAGESIZE] reads data[0]
 * (BtreeRangeSearch.cu:359-363 can index key[size] of a full page). */
static inline uint64_t page_key(const refc_page *p, int64_t i) {
    return i < REFC_PAGESIZE ? p->key[i] : p->data[i - REFC_PAGESIZE];
}

/* data[PAGESIZE] of the reference's page reads the 8 bytes holding
 * `bool leafFlag` (offset 80000, padded) and `int size` (offset 80004),
 * BPTree.h:14-23; the pool is zeroed first (BPTree.cu:166). */
static inline uint64_t page_data(const refc_page *p, int64_t i) {
    if (i < REFC_PAGESIZE) return p->data[i];
    return (uint64_t)(p->leafFlag ? 1u : 0u) | ((uint64_t)(uint32_t)p->size << 32);
}

refc_tree *refc_build(const uint64_t *keys, const uint64_t *data, uint64_t n,
                      const uint64_t *leaf_sizes, uint64_t nleaves) {
    uint64_t L = leaf_sizes ? nleaves : (n + REFC_PAGESIZE - 1) / REFC_PAGESIZE;
    if (L == 0) return NULL;
    /* page count: leaves + every internal level down to a single root */
    uint64_t total = L, lvl = L;
    do {
        lvl = (lvl + REFC_PAGESIZE - 1) / REFC_PAGESIZE;
        total += lvl;
    } while (lvl > 1);
    refc_tree *t = (refc_tree *)calloc(1, sizeof(refc_tree));
    if (!t) return NULL;
    t->pages = (refc_page *)calloc(total, sizeof(refc_page)); /* pool memset 0, BPTree.cu:166 */
    if (!t->pages) {
        free(t);
        return NULL;
    }
    t->npages = total;
    /* leaves: assignDataToLeaf, BPTree.cu:73-125 */
    uint64_t prefix = 0;
    for (uint64_t g = 0; g < L; g++) {
        uint64_t cnt = leaf_sizes ? leaf_sizes[g]
                                  : ((g + 1) * REFC_PAGESIZE <= n ? REFC_PAGESIZE
                                                                  : n - g * REFC_PAGESIZE);
        refc_page *p = &t->pages[g];
        p->next = (g == L - 1) ? -1 : (int)(g + 1);
        p->previous = (g == 0) ? -1 : (int)(g - 1);
        p->size = (int)cnt;
        p->max = (prefix + cnt - 1 < n) ? keys[prefix + cnt - 1] : 0;
        p->min = (prefix < n) ? keys[prefix] : 0;
        p->leafFlag = 1;
        for (uint64_t h = 0; h < cnt; h++) {
            p->data[h] = (prefix + h < n) ? data[prefix + h] : 0;
            p->key[h] = (prefix + h < n) ? keys[prefix + h] : 0;
        }
        prefix += cnt;
    }
    /* internal levels: kernelMaxIntermidatePage, BPTree.cu:28-70, driven by
     * the host loop BPTree.cu:218-243 */
    uint64_t cur = L; /* next free page */
    uint64_t *child = (uint64_t *)malloc(L * sizeof(uint64_t));
    for (uint64_t g = 0; g < L; g++) child[g] = g;
    uint64_t prev = L;
    for (;;) {
        uint64_t up = (prev + REFC_PAGESIZE - 1) / REFC_PAGESIZE;
        int rem = (int)(prev % REFC_PAGESIZE);
        uint64_t *next_child = (uint64_t *)malloc(up * sizeof(uint64_t));
        for (uint64_t g = 0; g < up; g++) {
            int items = (g != up - 1) ? REFC_PAGESIZE : rem;
            if (items == 0 && g == up - 1) items = REFC_PAGESIZE;
            refc_page *w = &t->pages[cur + g];
            for (int k = 0; k < items; k++) {
                uint64_t c = child[g * REFC_PAGESIZE + (uint64_t)k];
                w->key[k] = t->pages[c].max;
                w->data[k] = c;
            }
            next_child[g] = cur + g;
            w->size = items;
            w->max = t->pages[w->data[items - 1]].max;
            w->min = t->pages[w->data[0]].min;
            w->next = -1;
            w->previous = -1;
            w->leafFlag = 0;
        }
        cur += up;
        free(child);
        child = next_child;
        if (up == 1) break;
        prev = up;
    }
    t->root = child[0];
    free(child);
    return t;
}

void refc_free(refc_tree *t) {
    if (!t) return;
    free(t->pages);
    free(t);
}

uint64_t refc_root(const refc_tree *t) { return t ? t->root : 0; }
uint64_t refc_num_pages(const refc_tree *t) { return t ? t->npages : 0; }

/* Exact-match binary search over v[0..size-1] as written in every reference
 * kernel (e.g. BPTreeExactSearch.cu:40-55).  Returns the matched index or
 * -1; *start_out receives the final `start`. */
static inline int64_t ref_bsearch(const uint64_t *v, int size, uint64_t q,
                                  int *start_out) {
    int start = 0, end = size - 1;
    while (start <= end) {
        int middle = start + (end - start) / 2;
        if (q == v[middle]) {
            *start_out = start;
            return middle;
        } else if (q < v[middle]) {
            end = middle - 1;
        } else {
            start = middle + 1;
        }
    }
    *start_out = start;
    return -1;
}

/* Descent to a leaf, BPTreeExactSearch.cu:36-68.  *parent receives the last
 * internal page visited (the range endpoint kernels compare against its size,
 * BtreeRangeSearch.cu:284). */
static inline uint64_t ref_descend(const refc_tree *t, uint64_t q,
                                   const refc_page **parent) {
    const refc_page *page = &t->pages[t->root];
    for (;;) {
        int start;
        int64_t f = ref_bsearch(page->key, page->size, q, &start);
        uint64_t foundAt = (f < 0) ? (uint64_t)start : (uint64_t)f;
        if (foundAt == (uint64_t)page->size) foundAt = (uint64_t)(start - 1);
        uint64_t c = page->data[foundAt];
        if (t->pages[c].leafFlag) {
            *parent = page;
            return c;
        }
        page = &t->pages[c];
    }
}

int refc_point_basic(const refc_tree *t, const uint64_t *q, uint64_t nq,
                     uint64_t *out, int nthreads) {
    const int nt = orc_threads(nthreads);
    int64_t i;
#pragma omp parallel for num_threads(nt) schedule(static)
    for (i = 0; i < (int64_t)nq; i++) {
        const refc_page *parent;
        uint64_t leaf = ref_descend(t, q[i], &parent);
        const refc_page *lp = &t->pages[leaf];
        int start;
        int64_t f = ref_bsearch(lp->key, lp->size, q[i], &start);
        out[i] = (f < 0) ? REFC_INVALID : lp->data[f];
    }
    return 0;
}

int refc_point_grouped(const refc_tree *t, const uint64_t *q, uint64_t nq,
                       uint64_t *out, int nthreads) {
    const int nt = orc_threads(nthreads);
    int64_t i;
#pragma omp parallel for num_threads(nt) schedule(static)
    for (i = 0; i < (int64_t)nq; i++) {
        const refc_page *parent;
        uint64_t leaf = ref_descend(t, q[i], &parent);
        const refc_page *lp = &t->pages[leaf];
        int start;
        /* BPTreeExactSearch.cu:269-276: the leaf search compares data[] */
        int64_t f = ref_bsearch(lp->data, lp->size, q[i], &start);
        out[i] = (f < 0) ? REFC_INVALID : lp->data[f];
    }
    return 0;
}

int refc_range_endpoint(const refc_tree *t, const uint64_t *q, uint64_t nq,
                        uint64_t *out, int nthreads) {
    const int nt = orc_threads(nthreads);
    int64_t i;
#pragma omp parallel for num_threads(nt) schedule(static)
    for (i = 0; i < (int64_t)nq; i++) {
        const refc_page *parent;
        uint64_t leaf = ref_descend(t, q[i], &parent);
        const refc_page *lp = &t->pages[leaf];
        int start;
        int64_t f = ref_bsearch(lp->key, lp->size, q[i], &start);
        uint64_t foundAt = (f < 0) ? (uint64_t)start : (uint64_t)f;
        /* BtreeRangeSearch.cu:284: compares with the parent page's size */
        if (foundAt == (uint64_t)parent->size) foundAt = (uint64_t)(start - 1);
        out[i] = (foundAt << 32) | leaf;
    }
    return 0;
}

int refc_range_count(const refc_tree *t, const uint64_t *lo, const uint64_t *hi,
                     const uint64_t *ep_lo, const uint64_t *ep_hi, uint64_t nq,
                     int grouped, uint64_t *counts, int nthreads) {
    const int nt = orc_threads(nthreads);
    int64_t i;
    int bad = 0;
#pragma omp parallel for num_threads(nt) schedule(dynamic, 64) reduction(| : bad)
    for (i = 0; i < (int64_t)nq; i++) {
        uint64_t a = lo[i], b = hi[i];
        uint64_t sPos = ep_lo[i] >> 32, sLeaf = ep_lo[i] & 0xffffffffull;
        uint64_t ePos = ep_hi[i] >> 32, eLeaf = ep_hi[i] & 0xffffffffull;
        uint64_t c = 0;
        /* BtreeRangeSearch.cu:297-374 (key[]) / :123-211 (data[]) */
#define REFC_V(p, k) (grouped ? (p)->data[k] : page_key((p), (k)))
        if (sLeaf != eLeaf) {
            const refc_page *p = &t->pages[sLeaf];
            for (int k = (int)sPos; k < p->size - 1; k++) {
                uint64_t v = REFC_V(p, k);
                if (v <= b && v >= a) c++;
            }
            uint64_t curLeaf = (uint64_t)(int64_t)t->pages[sLeaf].next;
            while (curLeaf != eLeaf) {
                if (curLeaf >= t->npages) { /* the reference walks off the list here */
                    bad = 1;
                    c = REFC_INVALID;
                    break;
                }
                const refc_page *m = &t->pages[curLeaf];
                for (int k = 0; k < m->size; k++) {
                    uint64_t v = REFC_V(m, k);
                    if (v <= b && v >= a) c++;
                }
                curLeaf = (uint64_t)(int64_t)m->next;
            }
            if (c != REFC_INVALID) {
                const refc_page *e = &t->pages[eLeaf];
                for (int k = 0; (uint64_t)k < ePos && k < e->size - 1; k++) {
                    uint64_t v = REFC_V(e, k);
                    if (v <= b && v >= a) c++;
                }
            }
        } else {
            const refc_page *e = &t->pages[eLeaf];
            for (int k = (int)sPos; (uint64_t)k <= ePos; k++) {
                uint64_t v = grouped ? page_data(e, k) : page_key(e, k);
                if (v >= a && v <= b) c++;
            }
        }
#undef REFC_V
        counts[i] = c;
    }
    return bad ? 1 : 0;
}

int refc_bucket(uint64_t v, int pass) {
    int maxPass = 64 / 8; /* grouping.cu:27 with BIT_PASS 8 */
    return (int)((v >> (8 * (maxPass - 1 - pass))) & 0xFF);
}

int refc_bucket2d(uint64_t a, uint64_t b, int pass) {
    int maxPass = 64 / 3 + ((64 % 3) > 0 ? 1 : 0); /* grouping2d.cu:26-27 */
    int n1 = (int)((a >> (3 * (maxPass - 1 - pass))) & 0xF);
    int n2 = (int)((b >> (3 * (maxPass - 1 - pass))) & 0xF);
    return n1 * n2;
}

static inline uint64_t spread32(uint64_t x) {
    x = (x | (x << 32)) & 0x00000000FFFFFFFFull;
    x = (x | (x << 16)) & 0x0000FFFF0000FFFFull;
    x = (x | (x << 8)) & 0x00FF00FF00FF00FFull;
    x = (x | (x << 4)) & 0x0F0F0F0F0F0F0F0Full;
    x = (x | (x << 2)) & 0x3333333333333333ull;
    x = (x | (x << 1)) & 0x5555555555555555ull;
    return x;
}

uint64_t refc_zorder(uint64_t a, uint64_t b, int ix, int iy) {
    /* zOrder2d.cu:29-35: the quotient is narrowed to int and widened back,
     * then the first mask keeps its low 32 bits. */
    int xg = (int)(uint32_t)(a / (uint64_t)(int64_t)ix);
    int yg = (int)(uint32_t)(b / (uint64_t)(int64_t)iy);
    uint64_t x = (uint64_t)(int64_t)xg;
    uint64_t y = (uint64_t)(int64_t)yg;
    return spread32(x) | (spread32(y) << 1);
}

int refc_zorder_interval(uint64_t max_value) {
    /* zOrder2d.cu:129: ceil((float)max / (float)2^32), in single precision */
    float f = (float)max_value / 4294967296.0f;
    int c = (int)f;
    if ((float)c < f) c++;
    return c;
}

/* ---- error-bounded segmentation (learned index) ------------------------ */

/* Points of a segment, relative to its first point: x = key - key[s] (exact
 * in 64 bits), y = rank - s +/- eps. */
typedef struct {
    uint64_t x;
    int64_t y;
} pla_pt;

/* Orientation of (o, a, b): > 0 when b lies above the directed line o -> a
 * (x increasing).  Exact: 128-bit products of 64-bit x and 34-bit y spans. */
static inline __int128 pla_cross(pla_pt o, pla_pt a, pla_pt b) {
    __int128 ax = (__int128)a.x - (__int128)o.x, bx = (__int128)b.x - (__int128)o.x;
    __int128 ay = (__int128)a.y - (__int128)o.y, by = (__int128)b.y - (__int128)o.y;
    return ax * by - ay * bx;
}

static inline double pla_line_at0(pla_pt a, pla_pt b, double *slope) {
    /* the line through a and b: slope and value at x = 0 (no contraction:
     * the file is built with -ffp-contract=off) */
    if (b.x == a.x) { /* duplicate keys: a flat line through the middle */
        *slope = 0.0;
        return ((double)a.y + (double)b.y) * 0.5;
    }
    double dx = (double)(b.x - a.x);
    double s = ((double)b.y - (double)a.y) / dx;
    *slope = s;
    return (double)a.y - s * (double)a.x;
}

uint64_t orc_pla_segments(const void *keys, uint64_t n, int key_bytes, uint32_t eps,
                          uint64_t chunk, int hull_cap, uint64_t *starts, double *slopes,
                          double *icpts, uint64_t max_out) {
    /* Greedy maximal segments with the optimal streaming fit (O'Rourke,
     * "An on-line algorithm for fitting straight lines between data ranges",
     * CACM 1981; the segmentation of the PGM-index, Ferragina & Vinciguerra,
     * VLDB 2020).  State of an open segment: the upper convex hull of the
     * lower points (x, y - eps), the lower convex hull of the upper points
     * (x, y + eps), the feasible line of largest slope M = (Ma, Mb) and of
     * smallest slope N = (Na, Nb).  A new point is feasible iff its lower
     * point is not above M and its upper point not below N. */
    if (hull_cap < 2) hull_cap = 2;
    pla_pt *lh = (pla_pt *)malloc(sizeof(pla_pt) * (size_t)hull_cap);
    pla_pt *uh = (pla_pt *)malloc(sizeof(pla_pt) * (size_t)hull_cap);
    const int64_t e = (int64_t)eps;
    uint64_t nseg = 0, i = 0;
    while (i < n) {
        const uint64_t s = i;
        uint64_t end = n;
        if (chunk) {
            const uint64_t ce = (s / chunk + 1) * chunk;
            if (ce < end) end = ce;
        }
        const uint64_t x0 = key_at(keys, key_bytes, s);
        int nl = 1, nu = 1;
        lh[0] = (pla_pt){0, -e};
        uh[0] = (pla_pt){0, e};
        pla_pt Ma = lh[0], Mb = uh[0], Na = uh[0], Nb = lh[0];
        uint64_t j = s + 1;
        if (j < end) {
            const pla_pt L = {key_at(keys, key_bytes, j) - x0, 1 - e};
            const pla_pt U = {L.x, 1 + e};
            Ma = lh[0];
            Mb = U;
            Na = uh[0];
            Nb = L;
            lh[nl++] = L;
            uh[nu++] = U;
            for (j = s + 2; j < end; j++) {
                const int64_t y = (int64_t)(j - s);
                const pla_pt L2 = {key_at(keys, key_bytes, j) - x0, y - e};
                const pla_pt U2 = {L2.x, y + e};
                if (pla_cross(Ma, Mb, L2) > 0 || pla_cross(Na, Nb, U2) < 0) break;
                int nl2 = nl, nu2 = nu;
                while (nl2 >= 2 && pla_cross(lh[nl2 - 2], lh[nl2 - 1], L2) >= 0) nl2--;
                while (nu2 >= 2 && pla_cross(uh[nu2 - 2], uh[nu2 - 1], U2) <= 0) nu2--;
                if (nl2 >= hull_cap || nu2 >= hull_cap) break;
                if (pla_cross(Ma, Mb, U2) < 0) { /* M pivots on U2: the lower point of least slope to it */
                    int b = 0;
                    for (int t = 1; t < nl; t++)
                        if (pla_cross(lh[b], U2, lh[t]) > 0) b = t;
                    Ma = lh[b];
                    Mb = U2;
                }
                if (pla_cross(Na, Nb, L2) > 0) { /* N pivots on L2: the upper point of most slope to it */
                    int b = 0;
                    for (int t = 1; t < nu; t++)
                        if (pla_cross(uh[b], L2, uh[t]) < 0) b = t;
                    Na = uh[b];
                    Nb = L2;
                }
                lh[nl2] = L2;
                nl = nl2 + 1;
                uh[nu2] = U2;
                nu = nu2 + 1;
            }
        }
        if (nseg < max_out) {
            if (starts) starts[nseg] = s;
            double sl = 0.0, ic = 0.0;
            if (j - s >= 2) {
                double sm, sn;
                const double m0 = pla_line_at0(Ma, Mb, &sm);
                const double n0 = pla_line_at0(Na, Nb, &sn);
                sl = (sm + sn) * 0.5;
                ic = (m0 + n0) * 0.5;
            }
            if (slopes) slopes[nseg] = sl;
            if (icpts) icpts[nseg] = ic;
        }
        nseg++;
        i = j;
    }
    free(lh);
    free(uh);
    return nseg;
}
