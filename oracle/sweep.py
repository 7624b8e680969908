"""One interval of any engine kind, through the CPU oracle (oracle).

TEST INFRASTRUCTURE ONLY (see oracle/__init__.py): the checker for the
interval-level API and the timed CPU baseline of the benchmark.

``hunt_interval`` restates what the reference's per-project ``hunt`` calls
return for one interval, in the search variable of the project:

  Euler    [lo, hi) in p: euler_search.CpuEngine(n).hunt(lo, hi, cap),
           with the launcher's low pass below P_FLOOR
  Dickson  [lo, hi) in k: ladder_search.CpuEngine(n, q2).hunt(lo, hi-1,
           cap), with the low pass below K_FLOOR, and the deep-zone sieve
           (dickson.CpuEngine.hunt_deep) once j = k / W leaves J_CEIL
  AP       [lo, hi) in p: ap_search.CpuEngine(n, q2).hunt with the
           difference d (0: P(n)), chain cap ``cap``
"""

import functools

from . import ap, dickson, euler

EULER, DICKSON, AP = 0, 1, 2


@functools.lru_cache(maxsize=16)
def _euler(n):
    # the survivor set does not depend on the wheel (euler_search.py:1-20);
    # the 23# table keeps small n affordable (29# has 3.5e7 offsets at n=4)
    wheel = euler.WHEEL_PRIMES if n <= 8 else euler.WHEEL_PRIMES_29
    return euler.CpuEngine(n, wheel)


@functools.lru_cache(maxsize=16)
def _dickson(n, q2):
    return dickson.CpuEngine(n, q2)


@functools.lru_cache(maxsize=16)
def _ap(n, q2, d):
    return ap.CpuEngine(n, q2, d=d or None)


def hunt_interval(kind, n, lo, hi, threshold, cap, q2=65536, d=0):
    """[(x, depth)] ascending with depth >= threshold over [lo, hi)."""
    lo, hi = int(lo), int(hi)
    if hi <= lo:
        return []
    out = []
    if kind == EULER:
        if lo < euler.P_FLOOR:
            out.extend(euler.low_pass(threshold, cap=cap, lo=lo,
                                      hi=min(hi, euler.P_FLOOR)))
            lo = euler.P_FLOOR
        if hi > lo:
            eng = _euler(n)
            for p, r in eng.hunt(lo, hi, cap=cap):
                out.append((p, r))
        return [(p, r) for p, r in out
                if (p >= euler.P_FLOOR or r >= threshold)]
    if kind == DICKSON:
        if lo < dickson.K_FLOOR:
            out.extend(dickson.low_pass(threshold, cap, lo=max(1, lo),
                                        hi=min(hi, dickson.K_FLOOR)))
            lo = dickson.K_FLOOR
        if hi > lo:
            eng = _dickson(n, q2)
            if (hi - 1) // eng.W + 1 > dickson.J_CEIL:
                out.extend(eng.hunt_deep(lo, hi - 1, cap=cap))
            else:
                out.extend(eng.hunt(lo, hi - 1, cap=cap))
        return out
    eng = _ap(n, q2, d)
    return eng.hunt(lo, hi - lo, min_depth=threshold, cap=cap)


def run_job(job):
    """Pool worker: job = (kind, n, lo, hi, threshold, cap, q2, d)."""
    return hunt_interval(*job)
