"""The reference's score harness, run against the mirrors.

Each project's score.py (euler-prime-runs/score.py:80-108,
dickson-ladders/score.py:62-96, primorial-ap/score.py:67-83) prints a SCORE
only if its gates are green and its frozen benchmark shapes reproduce their
work fingerprints: huntlib/scoring.py:24-56 runs the gates, then times
``runs`` = 3 sweeps of each shape after a warm-up on the same window and
takes the median rate, checking the survivor count and the xor checksum.
``fingerprint_benchmark`` below restates that rule; the gates here are the
oracle parity checks these mirrors answer to (the reference's own gate
functions drive CuPy kernels and cannot run on this engine); the shapes
and fingerprints are the reference's, frozen in tests/golden/known.json.
"""

import statistics
import time

import numpy as np
import pytest

from golden_util import load

pytestmark = pytest.mark.gpu


def run_gates(gates):
    """huntlib/scoring.py:24-31: every gate runs; all must pass."""
    ok = True
    for g in gates:
        good, msg = g()
        print(("PASS " if good else "FAIL ") + msg)
        ok = ok and good
    return ok


def fingerprint_benchmark(work_fn, span, count_expect, checksum_expect,
                          runs=3):
    """huntlib/scoring.py:34-56: the median rate of `runs` calls, and
    whether the last result's count and xor checksum are the frozen ones.
    Returns (rate, ok, count, checksum)."""
    import torch
    rates, out = [], None
    for _ in range(runs):
        t0 = time.perf_counter()
        out = work_fn()
        torch.cuda.synchronize()
        rates.append(span / max(time.perf_counter() - t0, 1e-9))
    arr = np.asarray([int(x) for x in out], dtype=object)
    count = len(arr)
    checksum = 0
    for x in arr:
        checksum ^= int(x)
    ok = count == count_expect and checksum == checksum_expect
    return statistics.median(rates), ok, count, checksum


def _gate_euler():
    from euler_gpu import GpuEngine
    from oracle import euler as oeu
    lo, hi = 10 ** 12, 10 ** 12 + 3 * 10 ** 8
    ok = GpuEngine(9).survivors_pre_mr(lo, hi) == \
        oeu.CpuEngine(9, oeu.WHEEL_PRIMES_29).survivors_pre_mr(lo, hi)
    return ok, "euler stream == oracle on [1e12, +3e8), n = 9"


def _gate_dickson():
    from ladder_gpu import GpuEngine
    from oracle import dickson as odk
    j0 = 10 ** 12
    ok = GpuEngine(10).survivors_j(j0, j0 + 2 ** 22).tolist() == \
        odk.CpuEngine(10).survivors_j(j0, j0 + 2 ** 22).tolist()
    return ok, "dickson stream == oracle on j in [1e12, +2^22), n = 10"


def _gate_ap():
    from ap_gpu import GpuEngine
    from oracle import ap as oap
    base, span = 4 * 10 ** 13 - (4 * 10 ** 13) % 30, 30 * 2 ** 20
    got = np.concatenate(list(GpuEngine(8, 4096).survivors(base, span)))
    ok = got.tolist() == oap.CpuEngine(8, 4096).survivors(base, span).tolist()
    return ok, "ap stream == oracle on [4e13, +30*2^20), n = 8"


def test_euler_scores():
    """euler-prime-runs/score.py: three shapes of the n = 17 stream, each
    warmed on its own window, timed as the median of three sweeps."""
    from euler_gpu import GpuEngine
    assert run_gates([_gate_euler])
    fp = load("known")["fingerprints"]
    for label in ("euler_score", "euler_score128", "euler_score_wide"):
        f = fp[label]
        lo, hi = int(f["lo"]), int(f["hi"])
        eng = GpuEngine(17)
        eng.survivors_pre_mr(lo, hi)                     # warm on the window
        rate, ok, c, x = fingerprint_benchmark(
            lambda: eng.survivors_pre_mr(lo, hi), hi - lo, f["count"],
            int(f["xor"]))
        assert ok, (label, c, x)
        print(f"{label} {rate / 1e6:,.0f} Mp/s")


def test_dickson_scores():
    """dickson-ladders/score.py: SCORE, SCORE12, SCORE13 on the j line;
    the printed rate is in k = W*j."""
    from ladder_gpu import GpuEngine
    assert run_gates([_gate_dickson])
    fp = load("known")["fingerprints"]
    for label in ("dickson_score", "dickson_score12", "dickson_score13"):
        f = fp[label]
        j0, span = int(f["j_lo"]), int(f["span"])
        eng = GpuEngine(f["n"], q2=f["q2"])
        eng.survivors_j(j0, j0 + span)                   # warm on the window
        rate, ok, c, x = fingerprint_benchmark(
            lambda: eng.survivors_j(j0, j0 + span), span, f["count"],
            int(f["xor"]))
        assert ok, (label, c, x)
        print(f"{label} {rate * eng.W / 1e6:,.0f} Mk/s")


def test_ap_score():
    """primorial-ap/score.py: every timed call builds its GpuEngine and
    concatenates the per-launch survivor arrays, as the reference's _work
    does; one warm-up call first."""
    from ap_gpu import GpuEngine
    assert run_gates([_gate_ap])
    f = load("known")["fingerprints"]["ap_score"]
    base, span = int(f["base"]), int(f["span"])

    def work():
        eng = GpuEngine(f["n"], f["q2"], launch_u=1 << 25)
        parts = list(eng.survivors(base, span))
        return np.concatenate(parts) if parts else np.zeros(0, np.uint64)

    work()
    rate, ok, c, x = fingerprint_benchmark(work, span, f["count"],
                                           int(f["xor"]))
    assert ok, (c, x)
    print(f"SCORE {rate / 1e6:,.0f} Mp/s")
