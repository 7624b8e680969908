"""The CPU oracle against the reference's own outputs (no GPU).

The golden fixtures were produced by importing the reference's CPU
engines and huntlib.primes (tests/golden/make_golden.py).  The oracle is
a restatement of that code; these tests pin it bit for bit before it is
trusted as the checker of the CUDA engine.  Windows the numpy oracle
cannot finish in seconds are checked on seeded sub-windows: the golden
stream restricted to the sub-window must equal the oracle's sweep of it.
"""

import random

import numpy as np
import pytest

from golden_util import ints, load
from oracle import ap as oap
from oracle import dickson as odk
from oracle import euler as oeu
from oracle import primes as opr


def test_mr_verdicts_match_reference():
    g = load("mr")
    vals = ints(g["values"])
    assert [opr.mr_is_prime(v) for v in vals] == g["mr_is_prime"]
    assert [opr.sprp_base2(v) for v in vals] == g["sprp_base2"]


def _subwindows(lo, hi, width, count, seed, around=()):
    """Seeded sub-windows of [lo, hi); when golden survivors are given,
    each window is placed over one of them, so no check is vacuous."""
    rng = random.Random(seed)
    if hi - lo <= width:
        return [(lo, hi)]
    out = []
    for _ in range(count):
        if around:
            s = rng.choice(list(around))
            a = min(max(lo, s - rng.randrange(0, width)), hi - width)
        else:
            a = rng.randrange(lo, hi - width)
        out.append((a, a + width))
    return out


# ------------------------------------------------------------------ Euler --

@pytest.mark.parametrize("case", range(len(load("euler")["surv"])))
def test_euler_survivors(case):
    c = load("euler")["surv"][case]
    lo, hi, n = int(c["lo"]), int(c["hi"]), c["n"]
    wheel = oeu.WHEEL_PRIMES if c["wheel_top"] == 23 else oeu.WHEEL_PRIMES_29
    eng = oeu.CpuEngine(n, wheel)
    want = ints(c["survivors"])
    width = 2 * eng.M if hi - lo > 4 * eng.M else hi - lo
    for a, b in _subwindows(lo, hi, width, 2, case, want):
        got = eng.survivors_pre_mr(a, b)
        assert got == [p for p in want if a <= p < b]


@pytest.mark.parametrize("case", [0, 1, 2, 3])
def test_euler_hunt(case):
    c = load("euler")["hunt"][case]
    lo, hi = int(c["lo"]), int(c["hi"])
    wheel = oeu.WHEEL_PRIMES if c["wheel_top"] == 23 else oeu.WHEEL_PRIMES_29
    eng = oeu.CpuEngine(c["n"], wheel)
    want = [(int(p), r) for p, r in c["hits"]]
    a, b = lo, min(hi, lo + 2 * 10 ** 8)
    assert eng.hunt(a, b, cap=c["cap"]) == [h for h in want if a <= h[0] < b]


def test_euler_low_pass():
    want = [(p, r) for p, r in load("euler")["low_pass_cap64"]]
    assert oeu.low_pass(4, cap=64) == want


def test_euler_knowns():
    for n in (8, 9, 10):
        assert oeu.mr_run_length(oeu.KNOWN[n], cap=64) == n


# ---------------------------------------------------------------- Dickson --

@pytest.mark.parametrize("case", range(len(load("dickson")["surv"])))
def test_dickson_survivors(case):
    c = load("dickson")["surv"][case]
    lo, hi = int(c["j_lo"]), int(c["j_hi"])
    eng = odk.CpuEngine(c["n"], c["q2"])
    want = ints(c["survivors"])
    for a, b in _subwindows(lo, hi, 1 << 20, 1, case, want):
        got = eng.survivors_j(a, b).tolist()
        assert got == [j for j in want if a <= j < b]


def test_dickson_hunt_first_occurrence():
    c = next(h for h in load("dickson")["hunt"] if h["n"] == 7)
    eng = odk.CpuEngine(7, 65536)
    hits = eng.hunt(odk.K_FLOOR, odk.KNOWN[7], cap=None)
    assert hits == [(int(k), r) for k, r in c["hits"]]
    assert min(k for k, r in hits if r >= 7) == odk.KNOWN[7]


def test_dickson_low_pass():
    want = [(k, r) for k, r in load("dickson")["low_pass_cap12"]]
    assert odk.low_pass(1, 12) == want


@pytest.mark.parametrize("case", range(len(load("dickson_deep")["cases"])))
def test_dickson_deep_zone(case):
    """Past u64 j (up to j ~ 5e21, k ~ 1e24): the oracle's deep sieve and
    run lengths equal the reference's survives() and run_length on the
    same window, and every survivor passes the divisibility definition."""
    c = load("dickson_deep")["cases"][case]
    lo, hi = int(c["j_lo"]), int(c["j_hi"])
    assert lo >= 1 << 64
    eng = odk.CpuEngine(c["n"], c["q2"])
    want = ints(c["survivors"])
    for a, b in _subwindows(lo, hi, 1 << 22, 2, case, want):
        got = eng.survivors_j_deep(a, b)
        assert got == [j for j in want if a <= j < b]
    runs = dict(zip(want, c["runs"]))
    for j in want:
        assert eng.divisor(j * eng.W) is None
        assert odk.run_length(j * eng.W, cap=c["cap"]) == runs[j]
    if c["n"] == 6:
        assert len(want) > 100 and max(c["runs"]) >= 2


# --------------------------------------------------------------------- AP --

@pytest.mark.parametrize("case", range(len(load("ap")["surv"])))
def test_ap_survivors(case):
    c = load("ap")["surv"][case]
    base, span = int(c["base"]), int(c["span"])
    d = int(c["d"]) if c["d"] else None
    eng = oap.CpuEngine(c["n"], c["q2"], d=d)
    want = ints(c["offsets"])
    width = min(span, 30 * (1 << 19))
    rng = random.Random(case)
    if want and span > width:
        o = rng.choice(want)
        start = max(0, min(o - rng.randrange(0, width), span - width))
        start -= start % 30
    else:
        start = 0
    got = eng.survivors(base + start, width).tolist()
    assert [start + o for o in got] == [o for o in want
                                        if start <= o < start + width]


def test_ap_hunt_fixed_difference():
    c = next(h for h in load("ap")["hunt"]
             if h["d"] and h["min_depth"] == 6)
    base, span = int(c["base"]), int(c["span"])
    eng = oap.CpuEngine(c["n"], c["q2"], d=int(c["d"]))
    width = 30 * (1 << 20)
    got = eng.hunt(base, width, min_depth=c["min_depth"], cap=c["cap"])
    want = [(int(p), r) for p, r in c["hits"] if int(p) < base + width]
    assert got == want


def test_ap_knowns():
    for n in (7, 8, 9, 10):
        p = oap.KNOWN[n]
        assert oap.chain_depth_two_pass(p, oap.difference(n), n) == n


# ------------------------------------------------------------ drills -----

def test_comparator_catches_a_planted_mistake():
    """The parity comparison must fail on a corrupted stream: a survivor
    planted into, and one dropped from, the ORACLE's output (the CPU
    side) both break equality with the golden stream."""
    c = load("ap")["surv"][0]
    base, span = int(c["base"]), int(c["span"])
    eng = oap.CpuEngine(c["n"], c["q2"])
    width = 30 * (1 << 16)
    got = eng.survivors(base, width)
    want = np.array([o for o in ints(c["offsets"]) if o < width],
                    dtype=np.uint64)
    assert np.array_equal(got, want) and got.size > 4
    planted = np.sort(np.append(got, got[1] + 30))
    dropped = np.delete(got, 2)
    assert not np.array_equal(planted, want)
    assert not np.array_equal(dropped, want)
