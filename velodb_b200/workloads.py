"""Seeded synthetic inputs for the oblivious operator workloads.

Every generator is a splitmix64 stream mapped to ranges with Lemire's
multiply-shift reduction ``(x * range) >> 64``, vectorised in numpy, so the
bytes are identical on every machine.  The shapes stand in for the TPC-H-like
tables the reference benchmarks (its dbgen data is not available):

* ``sort_kp``          -- 2^20 rows of (u64 key, u32 payload = row id)
* ``lineitem``         -- 6,001,215-row fact table for filter + group-by
* ``join_tables``      -- 1.5 M-row dimension + 6 M-row fact for the PK-FK join
* ``batch_instances``  -- 512 instances with log-uniform sizes 2^10..2^22
"""
from __future__ import annotations

import numpy as np

GAMMA = np.uint64(0x9E3779B97F4A7C15)
STREAM_STEP = np.uint64(0x632BE59BD9B4E019)

SEED_SORT = 0xB200000000000000
SEED_LINEITEM = 0xB200000000000001
SEED_JOIN = 0xB200000000000002
SEED_BATCH = 0xB200000000000003
SEED_SERVE = 0xB200000000000004


def splitmix64(seed: int, n: int, stream: int = 0, start: int = 0) -> np.ndarray:
    """Outputs start..start+n-1 of the splitmix64 generator started at
    seed + stream*STEP."""
    with np.errstate(over="ignore"):
        base = np.uint64(seed & 0xFFFFFFFFFFFFFFFF) + np.uint64(stream) * STREAM_STEP
        z = base + (np.arange(start + 1, start + n + 1, dtype=np.uint64) * GAMMA)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        return z ^ (z >> np.uint64(31))


def lemire(x: np.ndarray, rng: int) -> np.ndarray:
    """(x * rng) >> 64 for 0 < rng < 2^32, exact in 64-bit arithmetic."""
    assert 0 < rng < (1 << 32)
    r = np.uint64(rng)
    with np.errstate(over="ignore"):
        hi = x >> np.uint64(32)
        lo = x & np.uint64(0xFFFFFFFF)
        return (hi * r + ((lo * r) >> np.uint64(32))) >> np.uint64(32)


def uniform_int(seed: int, n: int, stream: int, lo: int, hi: int, dtype, start: int = 0) -> np.ndarray:
    """n integers uniform over [lo, hi] (inclusive), rows start..start+n-1."""
    return (lemire(splitmix64(seed, n, stream, start), hi - lo + 1).astype(np.int64) + lo).astype(dtype)


def permutation(seed: int, n: int, stream: int) -> np.ndarray:
    """A seeded permutation of 0..n-1 (stable argsort of a u64 stream)."""
    return np.argsort(splitmix64(seed, n, stream), kind="stable").astype(np.int64)


# --------------------------------------------------------------------------

def sort_kp(n: int = 1 << 20, seed: int = SEED_SORT):
    """Plain sort input: u64 keys from the stream, payload = row id."""
    return splitmix64(seed, n, 0), np.arange(n, dtype=np.uint32)


LINEITEM_ROWS = 6_001_215
# date range (~98 %) plus a discount band; the band is narrowed by quantity so
# that the combined selectivity is ~2 % (disc == 10 is 1/11, qty <= 11 is 22 %)
LINEITEM_PRED = dict(ship_lo=0, ship_hi=2504, disc_lo=10, disc_hi=10, qty_lo=1, qty_hi=11)
LINEITEM_GROUP_BOUND = 8


def lineitem(n: int = LINEITEM_ROWS, seed: int = SEED_LINEITEM, start: int = 0) -> dict:
    """Rows start..start+n-1 of the lineitem-shaped table of `seed`."""
    return dict(
        qty=uniform_int(seed, n, 0, 1, 50, np.int32, start),
        price=uniform_int(seed, n, 1, 90_000, 10_500_000, np.int64, start),
        disc=uniform_int(seed, n, 2, 0, 10, np.int32, start),
        tax=uniform_int(seed, n, 3, 0, 8, np.int32, start),
        shipdate=uniform_int(seed, n, 4, 0, 2556, np.int32, start),
        flag1=uniform_int(seed, n, 5, 0, 2, np.uint8, start),
        flag2=uniform_int(seed, n, 6, 0, 1, np.uint8, start),
    )


JOIN_DIM_ROWS = 1_500_000
JOIN_FACT_ROWS = 6_000_000
JOIN_PRED = dict(date_hi=1278, price_hi=5_295_000)
JOIN_TOPK = 10


def join_tables(n_dim: int = JOIN_DIM_ROWS, n_fact: int = JOIN_FACT_ROWS, seed: int = SEED_JOIN):
    dim = dict(
        key=(permutation(seed, n_dim, 0) + 1).astype(np.int32),
        date=uniform_int(seed, n_dim, 1, 0, 2556, np.int32),
    )
    fact = dict(
        fk=uniform_int(seed, n_fact, 2, 1, n_dim, np.int32),
        price=uniform_int(seed, n_fact, 3, 90_000, 10_500_000, np.int64),
    )
    return dim, fact


def batch_sizes(count: int = 512, lo_log2: float = 10.0, hi_log2: float = 22.0, seed: int = SEED_BATCH):
    """Instance sizes n_i = floor(2^u), u uniform over [lo_log2, hi_log2]."""
    u = splitmix64(seed, count, 0).astype(np.float64) / 2.0**64
    return np.floor(np.exp2(lo_log2 + u * (hi_log2 - lo_log2))).astype(np.int64)


def batch_instances(count: int = 512, seed: int = SEED_BATCH, max_log2: float = 22.0):
    """Instances: even index -> sort of (u64 key, u32 payload); odd -> compaction
    with Bernoulli(0.3) keep flags.  Returns a list of dicts."""
    sizes = batch_sizes(count, hi_log2=max_log2, seed=seed)
    out = []
    for i, n in enumerate(sizes):
        n = int(n)
        keys = splitmix64(seed, n, 1000 + i)
        pay = np.arange(n, dtype=np.uint32)
        inst = dict(kind="sort" if i % 2 == 0 else "compact", n=n, keys=keys, pay=pay)
        if i % 2 == 1:
            inst["marks"] = (lemire(splitmix64(seed, n, 5000 + i), 10) < 3).astype(np.uint8)
        out.append(inst)
    return out
