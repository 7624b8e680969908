"""The 13#-difference AP line, whole, on the GPU.

Workload: terms p + i*30030 (difference 13#), p over [1e12, 1e12 + 2^40),
chains of at least 10 terms, chain cap 16, sieve to 65536.  The line is
1.1e12 candidates: the device sweeps all of it in one batch, and

  * every chain it reports is re-proved by the oracle: its depth by the
    reference's two-pass chain_depth (primorial-ap/ap_search.py:160-194),
    each of its terms by mr_is_prime (huntlib/primes.py:23-47), and the
    term after the chain composite or past the cap;
  * 16 seeded sub-windows of 2^28 spread over the line are swept by the
    oracle in a process pool: their pre-primality streams, their chains of
    at least 5 terms, and the whole-line chains falling inside them are
    all bit-identical to the device's.

The oracle here is the reference's AP engine with the difference
overridden and its forbidden sets rebuilt by its own formula
(primorial-ap/ap_search.py:99-106), pinned by tests/golden/ap.json.
"""

import concurrent.futures as cf
import multiprocessing as mp
import os
import random
import time

import pytest

from oracle import ap as oap
from oracle import primes as opr

pytestmark = pytest.mark.gpu

LO = 10 ** 12
SPAN = 2 ** 40
D = 30030
N = 10
CAP = 16
SUB = 2 ** 28


def _sub_windows(count=16, seed=20261204):
    """Seeded windows of SUB, one in each of `count` equal slices of the
    line, starts aligned to 30 (the mod-30 wheel's period)."""
    rng = random.Random(seed)
    out = []
    step = SPAN // count
    for i in range(count):
        a = LO + i * step + rng.randrange(0, step - SUB)
        a -= a % 30
        out.append((a, a + SUB))
    return out


def _oracle_window(job):
    lo, hi = job
    eng = oap.CpuEngine(N, 65536, d=D)
    s = eng.survivors(lo, hi - lo).tolist()
    # the hunt of ap_search.py:196-207 on the stream just computed
    h = [(lo + o, dep) for o in s
         for dep in [eng.chain_depth(lo + o, CAP)] if dep >= 5]
    return s, h


@pytest.fixture(scope="module")
def whole_line():
    import fk_workloads as W
    from fk_batch import BatchEngine
    ivs = W.ap_plain()
    assert ivs[0].lo == LO and ivs[0].length == SPAN and ivs[0].d == D
    be = BatchEngine(ivs)
    be.run_arrays(ivs[:1], graph=False)             # warm: tables, buffers
    t0 = time.perf_counter()
    hits = be.run(ivs, graph=False)[0]
    wall = time.perf_counter() - t0
    st = be.stats()
    print(f"13#-difference AP line, 2^40 candidates: {len(hits)} chains "
          f">= 10, device {st['total_ms']:.0f} ms "
          f"({SPAN / (st['total_ms'] * 1e-3):.3g} candidates/s), wall "
          f"{wall:.2f} s, {st['candidates']} pre-primality survivors")
    return be, hits


def test_whole_line_chains_are_reproved(whole_line):
    _, hits = whole_line
    assert len(hits) > 1000
    ps = [p for p, _ in hits]
    assert ps == sorted(ps) and len(set(ps)) == len(ps)
    assert all(LO <= p < LO + SPAN for p in ps)
    for p, dep in hits:
        assert dep >= N
        assert oap.chain_depth_two_pass(p, D, CAP) == dep
        assert all(opr.mr_is_prime(p + j * D) for j in range(dep))
        assert dep == CAP or not opr.mr_is_prime(p + dep * D)


def test_sub_windows_match_the_oracle(whole_line):
    import fk_abi
    be, hits = whole_line
    wins = _sub_windows()
    with cf.ProcessPoolExecutor(max_workers=min(16, os.cpu_count() or 1),
                                mp_context=mp.get_context("spawn")) as pool:
        want = list(pool.map(_oracle_window, wins))
    eng = fk_abi.Engine(fk_abi.AP, N, q2=65536, d=D)
    n_surv = n_hits = 0
    for (a, b), (surv, h5) in zip(wins, want):
        assert eng.sieve(a, b).tolist() == surv
        off, dep = eng.hunt(a, b, 5, CAP)
        assert [(a + int(o), int(d)) for o, d in zip(off, dep)] == h5
        assert [(p, d) for p, d in hits if a <= p < b] == \
            [(p, d) for p, d in h5 if d >= N]
        n_surv += len(surv)
        n_hits += len(h5)
    assert n_surv > 200 and n_hits > 0
