"""GPU parity past u64: the Dickson deep zone and the served workload.

The served workload starts requests at 1e18..1e24, so Dickson requests put
j = k / W past 2^64 (about 5e21 at n = 6) and their chain values near
2^165 (three 64-bit limbs).  These tests compare the device with

  * golden fixtures made by the reference itself past 2^64 (its
    CpuEngine.survives and run_length, exact at any j:
    tests/golden/dickson_deep.json), every survivor with its chain depth;
  * the oracle's deep-zone sieve (oracle/dickson.py survivors_j_deep) on
    wider windows at n = 6, 10, 14;
  * the oracle's per-interval hunt (oracle/sweep.py hunt_interval) on
    requests drawn from the served workload, through the batch engine and
    the serving loop, and -- hunted at threshold 0 -- every survivor of
    those requests with its chain depth.

Everything is integer and bit-exact.
"""

import concurrent.futures as cf
import multiprocessing as mp
import os

import pytest

from golden_util import ints, load
from oracle import ap as oap
from oracle import dickson as odk
from oracle import euler as oeu
from oracle import sweep as osw

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def pool():
    # the oracle runs in spawned workers (never forked from a process that
    # has a CUDA context)
    with cf.ProcessPoolExecutor(max_workers=min(16, os.cpu_count() or 1),
                                mp_context=mp.get_context("spawn")) as p:
        yield p


@pytest.fixture(params=["rounds", "mark"])
def sieve(request):
    return request.param


def _dickson(n, q2, sieve, p0=6):
    import fk_abi
    return fk_abi.Engine(fk_abi.DICKSON, n, q2=q2, p0=p0, sieve=sieve)


# ------------------------------------------------ reference fixtures ---

@pytest.mark.parametrize("p0", [6, 9])
@pytest.mark.parametrize("case",
                         range(len(load("dickson_deep")["cases"])))
def test_deep_zone_matches_reference_fixtures(case, sieve, p0):
    c = load("dickson_deep")["cases"][case]
    lo, hi = int(c["j_lo"]), int(c["j_hi"])
    want = ints(c["survivors"])
    eng = _dickson(c["n"], c["q2"], sieve, p0)
    got = [lo + int(o) for o in eng.sieve(lo, hi).tolist()]
    assert got == want
    # threshold 0: every survivor comes back with its exact chain depth
    off, dep = eng.hunt(lo, hi, 0, c["cap"])
    assert [lo + int(o) for o in off.tolist()] == want
    assert dep.tolist() == c["runs"]


def test_deep_zone_through_the_mirror():
    """ladder_gpu.GpuEngine.survivors_j_deep returns the fixtures' Python
    ints up to its reach J_REACH = P * J_CEIL, and refuses past it, as the
    reference's does (dickson-ladders/ladder_gpu.py:783-804)."""
    import ladder_gpu
    for c in load("dickson_deep")["cases"]:
        lo, hi = int(c["j_lo"]), int(c["j_hi"])
        eng = ladder_gpu.GpuEngine(c["n"], q2=c["q2"])
        if hi <= eng.J_REACH:
            assert eng.survivors_j_deep(lo, hi) == ints(c["survivors"])
        else:
            with pytest.raises(ValueError):
                eng.survivors_j_deep(lo, hi)
        with pytest.raises(ValueError):        # u64 API: refuses past 2^62
            eng.survivors_j(lo, hi)


# ------------------------------------------- oracle, wider windows ---

# (n, q2, j_lo, log2 span): wide enough that each window holds survivors
DEEP_WINDOWS = [(6, 65536, 2 ** 64 - 2 ** 21, 22), (6, 65536, 3 * 10 ** 20, 22),
                (6, 65536, 5 * 10 ** 21, 22), (10, 4096, 2 ** 64 + 99, 22),
                (10, 4096, 10 ** 21, 22), (14, 2048, 7 * 10 ** 19, 24),
                (14, 2048, 3 * 10 ** 20, 24)]


def _oracle_deep(job):
    n, q2, lo, hi, cap = job
    eng = odk.CpuEngine(n, q2)
    s = eng.survivors_j_deep(lo, hi)
    return s, [odk.run_length(j * eng.W, cap) for j in s]


@pytest.mark.parametrize("n,q2,lo,lspan", DEEP_WINDOWS)
def test_deep_windows_match_the_oracle(n, q2, lo, lspan, sieve, pool):
    span = 1 << lspan
    cap = n + 8
    parts = [(n, q2, lo + i * (span // 8), lo + (i + 1) * (span // 8), cap)
             for i in range(8)]
    res = list(pool.map(_oracle_deep, parts))
    want = [j for s, _ in res for j in s]
    runs = [r for _, rr in res for r in rr]
    assert want, "vacuous window"
    eng = _dickson(n, q2, sieve)
    got = [lo + int(o) for o in eng.sieve(lo, lo + span).tolist()]
    assert got == want
    off, dep = eng.hunt(lo, lo + span, 0, cap)
    assert [lo + int(o) for o in off.tolist()] == want
    assert dep.tolist() == runs


# ---------------------------------------------- the served workload ---

def _served(count, clip=1 << 20):
    """Requests of the served workload (starts 1e18..1e24), each clipped to
    `clip` units of its engine's line variable (p; j = k / W)."""
    import fk_workloads as W
    out = []
    for _, iv in W.served(count=count, rate_hz=400.0):
        if iv.kind == W.DICKSON:
            w = odk.wheel_modulus(iv.n)
            hi = min(iv.hi, iv.lo + clip * w)
        elif iv.kind == W.AP:
            hi = iv.lo + max(30, (min(iv.hi, iv.lo + clip) - iv.lo) // 30 * 30)
        else:
            hi = min(iv.hi, iv.lo + clip)
        out.append(W.Interval(iv.kind, iv.n, iv.lo, hi, iv.threshold, iv.cap))
    return out


def _oracle_hunt(iv):
    return osw.hunt_interval(iv.kind, iv.n, iv.lo, iv.hi, iv.threshold,
                             iv.cap, iv.q2, iv.d)


def _oracle_depths(job):
    """Every pre-primality survivor of one request, as a line-variable
    offset, with its chain depth by the reference's definition for the
    engine (Euler mr_run_length, Dickson run_length of k = W*j, AP the
    two-pass chain_depth)."""
    kind, n, lo, hi, cap, q2, d = job
    if kind == 0:
        wheel = oeu.WHEEL_PRIMES if n <= 8 else oeu.WHEEL_PRIMES_29
        s = oeu.CpuEngine(n, wheel).survivors_pre_mr(lo, hi)
        return [(p - lo, oeu.mr_run_length(p, cap)) for p in s]
    if kind == 1:
        eng = odk.CpuEngine(n, q2)
        return [(j - lo, odk.run_length(j * eng.W, cap))
                for j in eng.survivors_j_deep(lo, hi)]
    eng = oap.CpuEngine(n, q2, d=d or None)
    return [(o, eng.chain_depth(lo + o, cap))
            for o in eng.survivors(lo, hi - lo).tolist()]


def test_served_requests_match_the_oracle(pool):
    """Requests drawn from the served workload (values to 2^165), through
    the batch engine and the serving loop: identical to the oracle's hunt
    per request."""
    from fk_batch import BatchEngine
    from fk_serve import ServeLoop
    ivs = _served(72)
    want = list(pool.map(_oracle_hunt, ivs))
    be = BatchEngine(ivs)
    assert be.run(ivs) == want
    loop = ServeLoop(engset=be.engset, slots=2, max_items=8)
    res, lat, st = loop.run([(0.002 * i, iv) for i, iv in enumerate(ivs)])
    assert st["requests"] == len(ivs) and st["batches"] > 2
    for iv, (off, dep), w in zip(ivs, res, want):
        from fk_workloads import rows_to_results
        e = be.engset.get(be.engset.key_for(iv))
        assert rows_to_results(iv, off, dep,
                               e.W if iv.kind == 1 else 1) == w


def test_served_requests_depths_match_the_oracle(pool):
    """Served-workload requests clipped to 2^22, hunted at threshold 0 so
    that every pre-primality survivor comes back with its chain depth --
    the three-limb Dickson chains and the 80-bit Euler values included,
    hits or not -- against the oracle's survivors and depth functions."""
    import fk_abi
    from fk_batch import EngineSet
    from fk_workloads import line_range
    ivs = _served(72, clip=1 << 22)
    es = EngineSet()
    specs, jobs = [], []
    for iv in ivs:
        key = es.key_for(iv)
        e = es.get(key)
        lo, hi = line_range(iv, e.W if iv.kind == 1 else 1)
        specs.append((es.index(key), fk_abi.MODE_HUNT, 0, iv.cap, lo, hi))
        jobs.append((iv.kind, iv.n, lo, hi, iv.cap, iv.q2, iv.d))
    want = list(pool.map(_oracle_depths, jobs))
    rows = fk_abi.Batch(es.engines()).run(specs)
    total = deep = 0
    for iv, (off, dep), w in zip(ivs, rows, want):
        assert list(zip(off.tolist(), dep.tolist())) == w
        total += len(w)
        deep += sum(1 for _, r in w if r > 0) if iv.kind == 1 else 0
    assert total > 800 and deep > 0
