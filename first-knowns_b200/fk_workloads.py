"""The sweep workloads, as seeded synthetic interval sets.

Five shapes, each a list of ``Interval`` records:

  euler_plain    every p < 1e9, Euler runs >= 8, cap 64
  dickson_plain  k in [1, 2^34), m = 1..8, depth >= 6, sieve to 2^20
  ap_plain       p in [1e12, 1e12 + 2^40), difference 13#, chains >= 10,
                 cap 16
  mixed_batch    4096 intervals, engine uniform over {Euler, Dickson, AP},
                 length 2^U(20, 36), threshold uniform in 4..12, start
                 10^U(10, 18) (aligned to 30 for AP), seed 20261203
  served         Poisson arrivals of requests: length 2^U(16, 34),
                 threshold 6..14, start 10^U(18, 24)

Lengths and starts are in each engine's search variable (p for Euler and
AP, k for Dickson), which is also the unit "candidates swept" counts.
No public dataset is involved: these seeded draws are the whole workload.
"""

import dataclasses
import math

import numpy as np

EULER, DICKSON, AP = 0, 1, 2
KIND_NAMES = {EULER: "euler", DICKSON: "dickson", AP: "ap"}
SEED = 20261203
EULER_CEIL = 10 ** 24
K_FLOOR = 10 ** 4


@dataclasses.dataclass(frozen=True)
class Interval:
    kind: int          # EULER / DICKSON / AP
    n: int             # filter (sieve) parameter
    lo: int            # [lo, hi) in the search variable
    hi: int
    threshold: int     # keep depth >= threshold
    cap: int           # chain cap
    q2: int = 65536    # sieve depth
    d: int = 0         # AP difference (0: the n-th primorial)

    @property
    def length(self):
        return self.hi - self.lo


def primorial(n):
    d, k, q = 1, 0, 2
    while k < n:
        if all(q % p for p in range(2, int(q ** 0.5) + 1)):
            d *= q
            k += 1
        q += 1
    return d


def default_cap(kind, n):
    """The reference hunt defaults: Euler cap 100 (euler_gpu.py:1458),
    Dickson n + 8 (ladder_gpu.py:819), AP n (ap_search.py:160-194)."""
    return {EULER: 100, DICKSON: n + 8, AP: n}[kind]


def euler_plain():
    return [Interval(EULER, 8, 2, 10 ** 9, 8, 64)]


def dickson_plain():
    return [Interval(DICKSON, 6, 1, 2 ** 34, 6, 8, q2=1 << 20)]


def ap_plain(span=2 ** 40):
    lo = 10 ** 12
    return [Interval(AP, 10, lo, lo + span, 10, 16, d=30030)]


def mixed_batch(count=4096, seed=SEED):
    rng = np.random.default_rng(seed)
    kinds = rng.integers(0, 3, size=count)
    lens = np.exp2(rng.uniform(20, 36, size=count))
    thr = rng.integers(4, 13, size=count)
    starts = np.power(10.0, rng.uniform(10, 18, size=count))
    out = []
    for k, ln, t, s in zip(kinds.tolist(), lens.tolist(), thr.tolist(),
                           starts.tolist()):
        lo, length = int(s), max(int(ln), 1)
        if k == AP:
            lo -= lo % 30
            length = max(30, length - length % 30)
        out.append(Interval(k, t, lo, lo + length, t, default_cap(k, t)))
    return out


def served(count=2000, rate_hz=200.0, seed=SEED + 1):
    """(arrival time in s, Interval) pairs: Poisson arrivals at rate_hz."""
    rng = np.random.default_rng(seed)
    gaps = rng.exponential(1.0 / rate_hz, size=count)
    times = np.cumsum(gaps)
    kinds = rng.integers(0, 3, size=count)
    lens = np.exp2(rng.uniform(16, 34, size=count))
    thr = rng.integers(6, 15, size=count)
    starts = np.power(10.0, rng.uniform(18, 24, size=count))
    out = []
    for tm, k, ln, t, s in zip(times.tolist(), kinds.tolist(), lens.tolist(),
                               thr.tolist(), starts.tolist()):
        lo, length = int(s), max(int(ln), 1)
        if k == EULER:
            lo = min(lo, EULER_CEIL - length)
        if k == AP:
            lo -= lo % 30
            length = max(30, length - length % 30)
        out.append((tm, Interval(k, t, lo, lo + length, t,
                                 default_cap(k, t))))
    return out


def shard(intervals, rank, world):
    """The intervals rank `rank` of `world` sweeps: a round-robin split of
    the list, disjoint across ranks and covering it (no interval is cut,
    so no survivor is shared and no collective is needed)."""
    return [iv for i, iv in enumerate(intervals) if i % world == rank]


def total_length(intervals):
    return sum(iv.length for iv in intervals)


def describe(intervals):
    by = {}
    for iv in intervals:
        by.setdefault(KIND_NAMES[iv.kind], []).append(iv.length)
    return {k: {"count": len(v), "candidates": float(sum(v)),
                "log2_mean_len": float(np.mean(np.log2(v)))}
            for k, v in by.items()}


def engine_key(iv):
    return (iv.kind, iv.n, iv.q2, iv.d)


def line_range(iv, W=1):
    """The interval in the engine's device line variable: p for Euler and
    AP, j = k / W for Dickson (k in [lo, hi) <=> j in [ceil(lo/W),
    ceil(hi/W)))."""
    if iv.kind == DICKSON:
        return -(-iv.lo // W), -(-iv.hi // W)
    return iv.lo, iv.hi


def rows_to_results(iv, offsets, depths, W=1):
    """Device results -> [(x, depth)] in the search variable."""
    jlo, _ = line_range(iv, W)
    if iv.kind == DICKSON:
        return [((jlo + int(o)) * W, int(dd))
                for o, dd in zip(offsets.tolist(), depths.tolist())]
    return [(iv.lo + int(o), int(dd))
            for o, dd in zip(offsets.tolist(), depths.tolist())]


def log_uniform_mean(a, b):
    return (2 ** b - 2 ** a) / ((b - a) * math.log(2))
