"""Seeded synthetic workloads for the benchmark configurations.

The reference ships no datasets (its runs read files at author paths,
run.sh:1, script.sh:5) and its generator cannot be built (randgen.cu:12
includes an absent third-party library), so every workload here is generated
from fixed seeds with numpy's PCG64:

  point_uniform  -- n unique uniform u32 keys (value = rank); queries: even
                    slots an existing key, odd slots uniform u32.
  point_zipf     -- n unique uniform u32 keys; queries: 90% keys whose rank
                    follows Zipf(0.99) through a random rank permutation,
                    10% uniform u32.
  zorder_points  -- (x, y) uniform u16 points keyed by their 32-bit Morton
                    code, value = point ID, sorted by (code, ID); rectangles
                    with a uniform corner and sides uniform in [1, 256].
  lognormal_keys -- u64 keys = cumulative sum of floor(lognormal(4, 2)) + 1.
  lognormal_point -- those keys (value = rank); queries 90% keys uniform over
                    the ranks, 10% uniform in [min, max].

Zipf sampling uses rejection-inversion (W. Hormann, G. Derflinger, "Rejection-
inversion to generate variates from monotone discrete distributions", ACM
TOMACS 6(3), 1996), vectorised.
"""
import numpy as np

KEY_SEED = 1


def rng(seed):
    return np.random.Generator(np.random.PCG64(seed))


def unique_sorted_u32(n, seed=KEY_SEED):
    """n distinct u32 values, uniform over [0, 2^32), sorted ascending."""
    if n > (1 << 31):
        raise ValueError("n too large for unique u32 keys")
    g = rng(seed)
    extra = max(1024, int(n * n / float(1 << 32)) * 2 + 4096)
    while True:
        v = np.unique(g.integers(0, 1 << 32, size=n + extra, dtype=np.uint64).astype(np.uint32))
        if len(v) >= n:
            break
        extra *= 2
    if len(v) > n:
        drop = g.choice(len(v), size=len(v) - n, replace=False)
        keep = np.ones(len(v), dtype=bool)
        keep[drop] = False
        v = v[keep]
    return v


def _h_integral(x, s):
    lx = np.log(x)
    t = (1.0 - s) * lx
    return np.where(np.abs(t) > 1e-8, np.expm1(t) / np.where(t == 0, 1, t), 1.0 + t / 2) * lx


def _h_integral_inv(x, s):
    t = x * (1.0 - s)
    t = np.maximum(t, -1.0 + 1e-16)
    f = np.where(np.abs(t) > 1e-8, np.log1p(t) / np.where(t == 0, 1, t), 1.0 - t / 2)
    return np.exp(f * x)


def zipf_ranks(num, n, s, g):
    """num draws from Zipf(s) over ranks 1..n (rejection-inversion)."""
    h = lambda x: np.exp(-s * np.log(x))
    hx1 = _h_integral(np.array(1.5), s) - 1.0
    hn = _h_integral(np.array(n + 0.5), s)
    ss = 2.0 - _h_integral_inv(_h_integral(np.array(2.5), s) - h(2.0), s)
    out = np.empty(num, dtype=np.int64)
    todo = np.arange(num)
    while len(todo):
        u = hn + g.random(len(todo)) * (hx1 - hn)
        x = _h_integral_inv(u, s)
        k = np.clip(np.floor(x + 0.5), 1, n)
        ok = (k - x <= ss) | (u >= _h_integral(k + 0.5, s) - h(k))
        out[todo[ok]] = k[ok].astype(np.int64)
        todo = todo[~ok]
    return out


def point_uniform(n_keys=1 << 20, n_queries=1 << 20, seed=KEY_SEED):
    """Plain point search workload: value = rank, 50% hits / 50% uniform."""
    keys = unique_sorted_u32(n_keys, seed)
    vals = np.arange(n_keys, dtype=np.uint32)
    g = rng(seed + 1)
    q = g.integers(0, 1 << 32, size=n_queries, dtype=np.uint64).astype(np.uint32)
    q[0::2] = keys[g.integers(0, n_keys, size=len(q[0::2]))]
    return keys, vals, q


def point_zipf(n_keys=1 << 26, n_queries=1 << 24, s=0.99, miss=0.10, seed=KEY_SEED):
    """Radix-grouped point search workload: Zipf(s) ranks over a random rank
    permutation, a `miss` fraction of uniform u32 queries."""
    keys = unique_sorted_u32(n_keys, seed)
    vals = np.arange(n_keys, dtype=np.uint32)
    g = rng(seed + 1)
    ranks = zipf_ranks(n_queries, n_keys, s, g) - 1
    perm = g.permutation(n_keys).astype(np.int64)
    q = keys[perm[ranks]]
    m = g.random(n_queries) < miss
    q[m] = g.integers(0, 1 << 32, size=int(m.sum()), dtype=np.uint64).astype(np.uint32)
    return keys, vals, q


def morton_u16(x, y):
    """32-bit Morton code: bits of x at even, bits of y at odd positions."""
    def spread(v):
        v = v.astype(np.uint32) & np.uint32(0xFFFF)
        v = (v | (v << np.uint32(8))) & np.uint32(0x00FF00FF)
        v = (v | (v << np.uint32(4))) & np.uint32(0x0F0F0F0F)
        v = (v | (v << np.uint32(2))) & np.uint32(0x33333333)
        v = (v | (v << np.uint32(1))) & np.uint32(0x55555555)
        return v
    return spread(x) | (spread(y) << np.uint32(1))


def compact_u16(z):
    """Inverse of the even-bit spread: the bits of z at even positions."""
    v = z.astype(np.uint32) & np.uint32(0x55555555)
    v = (v | (v >> np.uint32(1))) & np.uint32(0x33333333)
    v = (v | (v >> np.uint32(2))) & np.uint32(0x0F0F0F0F)
    v = (v | (v >> np.uint32(4))) & np.uint32(0x00FF00FF)
    v = (v | (v >> np.uint32(8))) & np.uint32(0x0000FFFF)
    return v


def zorder_points(n_points=1 << 24, n_rects=1 << 20, max_side=256, seed=KEY_SEED):
    """2-D points keyed by Morton code (duplicates allowed) and rectangles.
    Returns (z_sorted u32, ids u32 in the same order, x0, y0, x1, y1 u16)."""
    g = rng(seed)
    x = g.integers(0, 1 << 16, size=n_points, dtype=np.uint32)
    y = g.integers(0, 1 << 16, size=n_points, dtype=np.uint32)
    z = morton_u16(x, y)
    ids = np.arange(n_points, dtype=np.uint32)
    order = np.lexsort((ids, z))
    z, ids = z[order], ids[order]
    g2 = rng(seed + 1)
    x0 = g2.integers(0, 1 << 16, size=n_rects, dtype=np.uint32)
    y0 = g2.integers(0, 1 << 16, size=n_rects, dtype=np.uint32)
    w = g2.integers(1, max_side + 1, size=n_rects, dtype=np.uint32)
    h = g2.integers(1, max_side + 1, size=n_rects, dtype=np.uint32)
    x1 = np.minimum(x0 + w - 1, 0xFFFF)
    y1 = np.minimum(y0 + h - 1, 0xFFFF)
    u16 = np.uint16
    return z, ids, x0.astype(u16), y0.astype(u16), x1.astype(u16), y1.astype(u16)


def lognormal_keys(n_keys=1 << 28, mu=4.0, sigma=2.0, seed=KEY_SEED, chunk=1 << 24):
    """Unique ascending u64 keys: cumulative sum of floor(lognormal) + 1 gaps."""
    g = rng(seed)
    keys = np.empty(n_keys, dtype=np.uint64)
    acc = np.uint64(0)
    for i in range(0, n_keys, chunk):
        m = min(chunk, n_keys - i)
        gaps = np.floor(g.lognormal(mu, sigma, size=m)).astype(np.uint64) + np.uint64(1)
        c = np.cumsum(gaps, dtype=np.uint64) + acc
        keys[i:i + m] = c
        acc = c[-1]
    return keys


def lognormal_point(n_keys=1 << 28, n_queries=1 << 24, miss=0.10, seed=KEY_SEED, query_seed=None):
    """Learned-index workload: lognormal_keys (value = rank, u64); queries
    drawn uniformly over the ranks, a `miss` fraction uniform in [min, max]
    (mostly absent keys).  query_seed varies the batch, not the keys."""
    keys = lognormal_keys(n_keys, seed=seed)
    vals = np.arange(n_keys, dtype=np.uint64)
    g = rng((seed + 7) if query_seed is None else query_seed)
    q = keys[g.integers(0, n_keys, size=n_queries)]
    m = g.random(n_queries) < miss
    q[m] = g.integers(int(keys[0]), int(keys[-1]) + 1, size=int(m.sum()), dtype=np.uint64)
    return keys, vals, q


def forest(num_trees=4096, size_log2=(10, 20), batch_log2=(6, 16), hit=0.8, range_frac=0.01,
           max_width=1 << 12, seed=KEY_SEED):
    """Batched uneven forest: tree sizes round(2^U), U ~ uniform[size_log2];
    each tree's keys are a random walk with gaps uniform in [1, (2^32-1) // n]
    (strictly increasing u32, spanning about half the u32 range); value =
    rank.  Per tree round(2^U), U ~ uniform[batch_log2], point queries (`hit`
    of them existing keys, the rest uniform u32) and round(range_frac * that)
    range queries [key[r], key[min(r + w - 1, n - 1)]], w uniform in
    [1, max_width] (width in ranks).  Vectorised over all trees.  Returns
    keys, values, key offsets, queries, query offsets, lo, hi, range offsets."""
    g = rng(seed)
    u64 = np.uint64
    sizes = np.rint(2.0 ** g.uniform(*size_log2, size=num_trees)).astype(np.int64)
    batches = np.rint(2.0 ** g.uniform(*batch_log2, size=num_trees)).astype(np.int64)
    nr = np.rint(range_frac * batches).astype(np.int64)
    koff = np.concatenate([[0], np.cumsum(sizes)])
    qoff = np.concatenate([[0], np.cumsum(batches)])
    roff = np.concatenate([[0], np.cumsum(nr)])
    gmax = (0xFFFFFFFF // sizes).astype(np.float64)  # largest gap; n * gmax < 2^32
    keys = np.empty(koff[-1], dtype=np.uint32)
    step = 1 << 26
    t0 = 0
    while t0 < num_trees:  # trees in chunks of about 2^26 keys
        t1 = int(np.searchsorted(koff, koff[t0] + step, side="right"))
        t1 = min(max(t1 - 1, t0 + 1), num_trees)
        n = sizes[t0:t1]
        gaps = np.floor(g.random(int(n.sum())) * np.repeat(gmax[t0:t1], n)).astype(np.int64) + 1
        cs = np.cumsum(gaps)
        base = np.repeat(np.concatenate([[0], cs[np.cumsum(n)[:-1] - 1]]), n)
        keys[koff[t0]:koff[t1]] = (cs - base).astype(np.uint32)
        t0 = t1
    vals = (np.arange(koff[-1], dtype=np.int64) - np.repeat(koff[:-1], sizes)).astype(np.uint32)
    tq = np.repeat(np.arange(num_trees), batches)
    q = g.integers(0, 1 << 32, size=qoff[-1], dtype=np.uint64).astype(np.uint32)
    h = g.random(qoff[-1]) < hit
    pick = koff[tq[h]] + np.floor(g.random(int(h.sum())) * sizes[tq[h]]).astype(np.int64)
    q[h] = keys[pick]
    tr = np.repeat(np.arange(num_trees), nr)
    a = np.floor(g.random(roff[-1]) * sizes[tr]).astype(np.int64)
    w = g.integers(1, max_width + 1, size=roff[-1])
    lo = keys[koff[tr] + a]
    hi = keys[koff[tr] + np.minimum(a + w - 1, sizes[tr] - 1)]
    return keys, vals, koff.astype(u64), q, qoff.astype(u64), lo, hi, roff.astype(u64)


def reference_queries(kind, n, max_number, seed=KEY_SEED + 3):
    """Query families of the reference's generator (randomgenator/randgen.cu),
    seeded here where the original is seeded from the clock:

      uniform        -- integers uniform in [0, max_number] (randgen.cu:75-91);
      normal         -- normal around max_number / 2 with sigma 0.35 x that
                        mean, draws outside [0, max_number] replaced by the
                        mean (:104-128);
      normal_wide    -- the same with sigma 0.63 x the mean (:186-205);
      zipf           -- Zipf(1.0) ranks over 1..max_number used as keys
                        (:138-147; sampled here by rejection-inversion);
      multi_gaussian -- five equal parts, each a normal of sigma 0.1 around
                        its own uniform centre in [0, max_number], i.e. five
                        clusters of (nearly) one value each (:159-175).
    Returns u64."""
    g = rng(seed)
    mx = float(max_number)
    if kind == "uniform":
        return g.integers(0, int(max_number), size=n, dtype=np.uint64, endpoint=True)
    if kind in ("normal", "normal_wide"):
        mean = float(int(max_number) // 2)
        x = g.normal(mean, (0.35 if kind == "normal" else 0.63) * mean, size=n)
        x = np.where((x < 0) | (x > mx), mean, x)
        return np.floor(x).astype(np.uint64)
    if kind == "zipf":
        return zipf_ranks(n, int(max_number), 1.0, g).astype(np.uint64)
    if kind == "multi_gaussian":
        out = np.empty(n, dtype=np.uint64)
        part = n // 5
        for i in range(5):
            c = float(g.integers(0, int(max_number), endpoint=True))
            m = part if i < 4 else n - 4 * part
            x = g.normal(c, 0.1, size=m)
            x = np.where((x < 0) | (x > mx), c, x)
            out[i * part:i * part + m] = np.floor(x).astype(np.uint64)
        return out
    raise ValueError(f"unknown query family {kind!r}")


def range_queries(keys, n_queries, max_width_ranks, seed=KEY_SEED + 2):
    """Ranges [key[r], key[min(r + w - 1, n - 1)]] with w uniform in
    [1, max_width_ranks] (width in ranks), plus their exact counts."""
    g = rng(seed)
    n = len(keys)
    r = g.integers(0, n, size=n_queries)
    w = g.integers(1, max_width_ranks + 1, size=n_queries)
    e = np.minimum(r + w - 1, n - 1)
    return keys[r], keys[e]
