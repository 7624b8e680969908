"""GPU parity against the CPU oracle on seeded windows and edge cases.

Bit-exact: every survivor stream and every depth must equal the oracle's
(tests/test_oracle_golden.py pins the oracle against the reference).
Each window runs through both sieve kernels (per-candidate compaction
rounds and the marking sieve).
"""

import random

import numpy as np
import pytest

from oracle import ap as oap
from oracle import dickson as odk
from oracle import euler as oeu
from oracle import sweep as osw

pytestmark = pytest.mark.gpu


@pytest.fixture(params=["rounds", "mark"])
def sieve(request):
    return request.param


@pytest.fixture(params=[6, 7])
def p0(request):
    """The 13# wheel (pattern primes from 17) and the 17# wheel."""
    return request.param


def _engine(kind, n, q2=65536, d=None, sieve="auto", p0=6):
    import fk_abi
    return fk_abi.Engine(kind, n, q2=q2, p0=p0, d=d, sieve=sieve)


EULER_CASES = [(4, 10 ** 7, 2 * 10 ** 6), (6, 10 ** 12, 3 * 10 ** 7),
               (9, 10 ** 16, 10 ** 9), (11, 10 ** 20, 6 * 10 ** 9),
               (7, 10 ** 24 - 10 ** 8, 10 ** 8)]


@pytest.mark.parametrize("n,lo,span", EULER_CASES)
def test_euler_windows(n, lo, span, sieve, p0):
    eng = _engine(0, n, sieve=sieve, p0=p0)
    got = (eng.sieve(lo, lo + span) + np.uint64(0)).tolist()
    want = oeu.CpuEngine(n, oeu.WHEEL_PRIMES).survivors_pre_mr(lo, lo + span)
    assert [lo + o for o in got] == want
    assert len(want) > 0
    off, dep = eng.hunt(lo, lo + span, n, 100)
    hw = oeu.CpuEngine(n, oeu.WHEEL_PRIMES).hunt(lo, lo + span, cap=100)
    assert [(lo + int(o), int(d)) for o, d in zip(off, dep)] == hw


DICKSON_CASES = [(4, 4096, 10 ** 9, 1 << 20), (7, 65536, 10 ** 13, 1 << 22),
                 (10, 2048, 10 ** 17, 1 << 22),
                 (5, 1 << 18, 3 * 10 ** 18, 1 << 18)]


@pytest.mark.parametrize("n,q2,jlo,span", DICKSON_CASES)
def test_dickson_windows(n, q2, jlo, span, sieve, p0):
    eng = _engine(1, n, q2=q2, sieve=sieve, p0=p0)
    got = (eng.sieve(jlo, jlo + span) + np.uint64(jlo)).tolist()
    want = odk.CpuEngine(n, q2).survivors_j(jlo, jlo + span).tolist()
    assert got == want and len(want) > 0


AP_CASES = [(5, 2048, None, 10 ** 8 + 10, 30 * (1 << 18)),
            (9, 4096, None, 7 * 10 ** 15 + 11, 30 * (1 << 20)),
            (12, 65536, None, 10 ** 18 - 10 ** 9, 30 * (1 << 22)),
            (10, 65536, 30030, 10 ** 12 + 2 ** 35, 30 * (1 << 22)),
            (16, 2048, None, 10 ** 25 + 7, 30 * (1 << 20))]


@pytest.mark.parametrize("n,q2,d,base,span", AP_CASES)
def test_ap_windows(n, q2, d, base, span, sieve, p0):
    eng = _engine(2, n, q2=q2, d=d, sieve=sieve, p0=p0)
    got = eng.sieve(base, base + span).tolist()
    want = oap.CpuEngine(n, q2, d=d).survivors(base, span).tolist()
    assert got == want and len(want) > 0
    cap = 16 if d else n
    off, dep = eng.hunt(base, base + span, 4, cap)
    hw = oap.CpuEngine(n, q2, d=d).hunt(base, span, min_depth=4, cap=cap)
    assert [(base + int(o), int(x)) for o, x in zip(off, dep)] == hw


def test_edge_ranges(sieve):
    """Empty, one-element, period-straddling and unaligned ranges."""
    eng = _engine(2, 8, q2=4096, sieve=sieve)
    ref = oap.CpuEngine(8, 4096)
    base = 4 * 10 ** 13 + 17
    assert eng.sieve(base, base).size == 0
    rng = random.Random(5)
    full = ref.survivors(base, 3 * 10 ** 6).tolist()
    for _ in range(40):
        a = rng.randrange(0, 3 * 10 ** 6)
        w = rng.choice([1, 2, 29, 30, 31, 30029, 30030, 30031, 70000])
        b = min(a + w, 3 * 10 ** 6)
        got = (eng.sieve(base + a, base + b) + np.uint64(a)).tolist()
        assert got == [o for o in full if a <= o < b]
    # one survivor exactly: a one-element range on it and beside it
    o = full[len(full) // 2]
    assert eng.sieve(base + o, base + o + 1).tolist() == [0]
    assert eng.sieve(base + o + 1, base + o + 2).size == 0


def test_depths_of_known_chains():
    """Chain depths of the reference's knowns and campaign finds, including
    values past the deterministic bound (strong-probable-prime chains),
    against the oracle's chain functions."""
    from golden_util import load
    kn = load("known")
    e = _engine(0, 8)
    ps = [int(v) for v in kn["euler_known"].values()] + [
        int(kn["euler_a21_upper"]), 348284517256411907,
        8461068614861832371, 3744101869688673856367]
    got = e.depths(ps, 100).tolist()
    assert got == [oeu.mr_run_length(p, cap=100) for p in ps]
    d = _engine(1, 13)
    ks = [int(v) for v in kn["dickson_known"].values()] + [
        9328409578841430, 433871469806557860, 55119263286518170740,
        12094123415384869458600]
    got = d.depths(ks, 20).tolist()
    assert got == [odk.run_length(k, cap=20) for k in ks]
    for n, p in ((16, 116781362669989), (17, 2097209048106247),
                 (18, 14042451608819603), (15, 158317270283)):
        a = _engine(2, n)
        assert a.depths([p], n + 3).tolist() == [
            oap.chain_depth_two_pass(p, oap.difference(n), n + 3)]


def test_values_past_192_bits_are_refused():
    e = _engine(1, 6)
    with pytest.raises(ValueError):
        e.hunt(10 ** 30, 10 ** 30 + 100, 6, 14)


def test_interval_api_matches_oracle_sweep():
    """oracle.sweep.hunt_interval == the plain engine on clipped mixed
    intervals of every kind."""
    import fk_workloads as W
    from fk_batch import PlainEngine
    ivs = []
    for iv in W.mixed_batch(60, W.SEED + 9):
        hi = min(iv.hi, iv.lo + (1 << 22))
        if iv.kind == W.AP:
            hi = iv.lo + max(30, (hi - iv.lo) // 30 * 30)
        ivs.append(W.Interval(iv.kind, iv.n, iv.lo, hi, iv.threshold,
                              iv.cap))
    got = PlainEngine().run(ivs)
    for iv, g in zip(ivs, got):
        assert g == osw.hunt_interval(iv.kind, iv.n, iv.lo, iv.hi,
                                      iv.threshold, iv.cap, iv.q2, iv.d)


@pytest.mark.parametrize("sieve_mode,span", [("rounds", 3_400_000_000_000_000),
                                             ("mark", 100_000_000_000_000)])
def test_widest_family_matches_the_23_wheel(sieve_mode, span):
    """The 31# line (p0 = 11: 37 and up as pattern primes) gives the same
    survivor stream as the 23# line (p0 = 9), which the windows above pin
    against the oracle; the long window's lanes are 266 words, so it runs
    one warp per lane; unaligned ends."""
    wide = _engine(0, 17, sieve=sieve_mode, p0=11)
    mid = _engine(0, 17, sieve=sieve_mode, p0=9)
    assert wide.M == 200560490130 and wide.L == 29937600
    lo = 611 * 10 ** 18 + 12345
    got = wide.sieve(lo, lo + span).tolist()
    want = mid.sieve(lo, lo + span).tolist()
    assert got == want and len(want) > 0
    off, dep = wide.hunt(lo, lo + span, 3, 100)
    o2, d2 = mid.hunt(lo, lo + span, 3, 100)
    assert off.tolist() == o2.tolist() and dep.tolist() == d2.tolist()
