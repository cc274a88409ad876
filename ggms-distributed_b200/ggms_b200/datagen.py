"""Seeded synthetic inputs and k-sets for the benchmark and the tests.

Shapes follow the reference's generator table (DistributedSMOS/generateProblems.cu:
uniform/normal/half-normal/Cauchy/sorted generators at :43-440, k distributions
at :584-727), re-expressed with numpy's PCG64 so every input is reproducible
from its seed on any host.  None of the reference's data is used.
"""
from __future__ import annotations

import numpy as np


def rng(seed: int) -> np.random.Generator:
    return np.random.default_rng(seed)


# ------------------------------------------------------------------ values
def uniform_f32(n: int, seed: int) -> np.ndarray:
    return rng(seed).random(n, dtype=np.float32)


def normal_f32(n: int, seed: int) -> np.ndarray:
    return rng(seed).standard_normal(n, dtype=np.float32)


def normal_f64(n: int, seed: int) -> np.ndarray:
    return rng(seed).standard_normal(n, dtype=np.float64)


def uniform_u32(n: int, seed: int) -> np.ndarray:
    return rng(seed).integers(0, 2**32, size=n, dtype=np.uint32)


def half_normal_f32(n: int, seed: int) -> np.ndarray:
    return np.abs(rng(seed).standard_normal(n, dtype=np.float32))


def cauchy_f32(n: int, seed: int) -> np.ndarray:
    # location 0, scale 1: tan(pi (u - 1/2)) in double, rounded once to float
    u = rng(seed).random(n, dtype=np.float64)
    return np.tan(np.pi * (u - 0.5)).astype(np.float32)


def distinct256_f32(n: int, seed: int) -> np.ndarray:
    g = rng(seed)
    table = g.standard_normal(256, dtype=np.float32) * np.float32(100.0)
    return table[g.integers(0, 256, size=n, dtype=np.uint32)]


def sorted_desc_u32(n: int, seed: int) -> np.ndarray:
    """Sorted descending, spread over the whole uint32 range (O(n), no sort):
    ascending i*step + U[0, step), then reversed."""
    step = max(1, (1 << 32) // max(n, 1))
    a = np.arange(n, dtype=np.uint64) * np.uint64(step)
    a += rng(seed).integers(0, step, size=n, dtype=np.uint64)
    np.minimum(a, np.uint64(0xFFFFFFFF), out=a)
    return a.astype(np.uint32)[::-1].copy()


def mixture8_f32(n: int, seed: int) -> np.ndarray:
    """8 Gaussians: means U[-100,100], std log-uniform [0.01,10], weights Dirichlet(1)."""
    g = rng(seed)
    means = g.uniform(-100.0, 100.0, 8)
    stds = np.exp(g.uniform(np.log(0.01), np.log(10.0), 8))
    w = g.dirichlet(np.ones(8))
    comp = g.choice(8, size=n, p=w).astype(np.uint8)
    z = g.standard_normal(n, dtype=np.float32)
    return (means[comp].astype(np.float32) + stds[comp].astype(np.float32) * z).astype(np.float32)


def lognormal_f32(n: int, seed: int) -> np.ndarray:
    return np.exp(np.float32(2.0) * rng(seed).standard_normal(n, dtype=np.float32)).astype(np.float32)


VALUE_GENERATORS = {
    "uniform_f32": uniform_f32,
    "normal_f32": normal_f32,
    "normal_f64": normal_f64,
    "uniform_u32": uniform_u32,
    "half_normal_f32": half_normal_f32,
    "cauchy_f32": cauchy_f32,
    "distinct256_f32": distinct256_f32,
    "sorted_desc_u32": sorted_desc_u32,
    "mixture8_f32": mixture8_f32,
    "lognormal_f32": lognormal_f32,
}


# ------------------------------------------------------------------ k-sets (1-based k-th largest)
def ks_percentiles(n: int, count: int = 101) -> np.ndarray:
    """k = round(p (n-1)) + 1 for p = 0, 1/(count-1), ..., 1."""
    p = np.arange(count, dtype=np.float64) / (count - 1)
    return (np.round(p * (n - 1)) + 1).astype(np.uint32)


def ks_uniform_distinct(n: int, count: int, seed: int) -> np.ndarray:
    g = rng(seed)
    if count >= n:
        return g.permutation(np.arange(1, n + 1, dtype=np.uint64)).astype(np.uint32)
    ks = set()
    while len(ks) < count:
        ks.update(int(x) for x in g.integers(1, n + 1, size=count - len(ks)))
    arr = np.fromiter(ks, dtype=np.uint64)
    g.shuffle(arr)
    return arr.astype(np.uint32)


def ks_uniform(n: int, count: int, seed: int) -> np.ndarray:
    return rng(seed).integers(1, n + 1, size=count, dtype=np.uint64).astype(np.uint32)


def ks_top1pct(n: int, count: int, seed: int) -> np.ndarray:
    """count distinct ks among the top 1% of ranks, plus k = 1 and k = n."""
    top = max(2, n // 100)
    g = rng(seed)
    pool = np.arange(2, top + 1, dtype=np.uint64)
    pick = g.choice(pool, size=min(count, len(pool)), replace=False)
    ks = np.concatenate([pick, np.array([1, n], dtype=np.uint64)])
    g.shuffle(ks)
    return ks.astype(np.uint32)


# ------------------------------------------------------------------ batched segments
def segmented_batch(nseg: int, seed: int, lo_log2: int = 10, hi_log2: int = 24,
                    kmax: int = 512, dtype=np.float32, total_cap: int | None = None):
    """nseg segments with log-uniform lengths in [2^lo, 2^hi]; each gets 1..kmax
    random ks.  float32 segments alternate uniform / normal values."""
    g = rng(seed)
    lens = np.exp2(g.uniform(lo_log2, hi_log2, nseg)).astype(np.int64)
    if total_cap is not None and lens.sum() > total_cap:
        lens = np.maximum(1, (lens * (total_cap / lens.sum())).astype(np.int64))
    seg_off = np.zeros(nseg + 1, dtype=np.int64)
    seg_off[1:] = np.cumsum(lens)
    n = int(seg_off[-1])
    if np.dtype(dtype) == np.float32:
        vals = np.empty(n, dtype=np.float32)
        for s in range(nseg):
            a, b = seg_off[s], seg_off[s + 1]
            if s % 2 == 0:
                vals[a:b] = g.random(b - a, dtype=np.float32)
            else:
                vals[a:b] = g.standard_normal(b - a, dtype=np.float32)
    else:
        vals = g.integers(0, 2**32, size=n, dtype=np.uint32)
    nks = g.integers(1, kmax + 1, size=nseg)
    k_off = np.zeros(nseg + 1, dtype=np.int64)
    k_off[1:] = np.cumsum(nks)
    ks = np.empty(int(k_off[-1]), dtype=np.uint32)
    for s in range(nseg):
        ks[k_off[s]:k_off[s + 1]] = g.integers(1, lens[s] + 1, size=nks[s], dtype=np.uint64)
    return vals, seg_off, ks, k_off
