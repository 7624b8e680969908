"""Drop-in for euler-prime-runs/euler_gpu.py's GpuEngine, on libfk.

Same constructor, attributes and sweep methods as the reference class
(euler-prime-runs/euler_gpu.py:897-1464), so euler-prime-runs/launch.py
and score.py take it unchanged once this directory is first on sys.path:

    GpuEngine(n, wheel_primes=None)
    .n, .M, .wheel_primes                  checkpoint cursor units
    survivors_pre_mr(lo, hi, periods_per_launch=None) -> sorted [int]
    hunt(lo, hi, cap=100, periods_per_launch=None)     -> [(p, run)]

``.M`` and ``.wheel_primes`` report the wheel the reference would pick
for these arguments (euler_search.best_wheel, euler_search.py:200-212),
because the launcher's checkpoint cursor counts periods of that M
(euler-prime-runs/launch.py:191-218).  The device sieves its own line
(fk_params.p0), which changes nothing about the survivor stream: the
stream is the set of p with no prime q < 65536 dividing any x^2+x+p,
x < n, whatever the wheel.

Unlike the reference, ``hunt`` classifies on the device: the strong
probable-prime chain (huntlib mr_is_prime, 7 bases) runs in the same
launch as the sieve.
"""

import functools

from fk_abi import EULER, MODE_SIEVE, Batch, Engine

WHEEL_PRIMES = [2, 3, 5, 7, 11, 13, 17, 19, 23]
WHEEL_PRIMES_29 = WHEEL_PRIMES + [29]
WHEEL_PRIMES_31 = WHEEL_PRIMES_29 + [31]
WHEEL_PRIMES_37 = WHEEL_PRIMES_31 + [37]
Q2 = 65536
P_FLOOR = 100_000
P_CEIL = 10 ** 24
WHEEL_BUDGET_OFFS = 50_000_000
FACTORED_FROM = 37


def _forbidden(q, n):
    return {(-(x * x + x)) % q for x in range(n)}


def wheel_offset_count(n, wheel_primes):
    """Admissible residues of p mod prod(wheel_primes) (euler_search.py:
    90-95)."""
    c = 1
    for q in wheel_primes:
        c *= q - len(_forbidden(q, n))
    return c


def wheel_base(wheel_primes):
    """euler_search.py:98-110: the materialized part of a factored wheel."""
    wp = list(wheel_primes)
    return wp[:-1] if wp[-1] >= FACTORED_FROM else wp


def best_wheel(n, budget=WHEEL_BUDGET_OFFS):
    """euler_search.py:200-212: the largest wheel whose table fits."""
    for wp in (WHEEL_PRIMES_37, WHEEL_PRIMES_31, WHEEL_PRIMES_29,
               WHEEL_PRIMES):
        if wheel_offset_count(n, wheel_base(wp)) <= budget:
            return wp
    return WHEEL_PRIMES


@functools.lru_cache(maxsize=None)
def _device_engine(n, p0):
    return Engine(EULER, n, q2=Q2, p0=p0)


class GpuEngine:
    """The Euler-form sieve + SPRP engine (reference API)."""

    def __init__(self, n, wheel_primes=None):
        self.n = int(n)
        self.wheel_primes = list(wheel_primes or best_wheel(self.n))
        M = 1
        for q in self.wheel_primes:
            M *= q
        self.M = M
        # the device lines: the widest wheel whose lane table stays within
        # 2^26 entries (31#, else 23#), 23# for mid-length windows, 13#
        # for short ones
        self._p0_wide = 9 if self.n >= 3 else 6
        if wheel_offset_count(self.n, WHEEL_PRIMES_31) <= 1 << 26:
            self._p0_wide = 11
        self._wide = _device_engine(self.n, self._p0_wide)
        self._mid = (_device_engine(self.n, 9) if self._p0_wide == 11
                     else None)
        self._narrow = _device_engine(self.n, 6)
        self._batches = {}

    def _eng_for(self, lo, hi):
        # a window shorter than a few wide-wheel words wastes most lanes
        if hi - lo >= 64 * 4 * self._wide.M:
            return self._wide
        if self._mid is not None and hi - lo >= 64 * 4 * self._mid.M:
            return self._mid
        return self._narrow

    def _check(self, lo, hi):
        lo, hi = int(lo), int(hi)
        if lo < P_FLOOR:
            raise ValueError("GPU engine floor is %d" % P_FLOOR)
        if hi > P_CEIL:
            raise ValueError("GPU engine ceiling is %d" % P_CEIL)
        return lo, hi

    def survivors_pre_mr(self, lo, hi, periods_per_launch=None):
        """Sorted list of exact survivor p (Python ints) in [lo, hi).

        With ``periods_per_launch`` the range is swept in launches of that
        many periods of .M, as the reference's launches are
        (euler-prime-runs/euler_gpu.py:1335-1456): each launch window is
        one device item of a batch run, 256 launches per device call at
        most.  The stream is the same either way."""
        lo, hi = self._check(lo, hi)
        if hi <= lo:
            return []
        eng = self._eng_for(lo, hi)
        if not periods_per_launch:
            off = eng.sieve(lo, hi)
            return [lo + int(o) for o in off.tolist()]
        step = int(periods_per_launch) * self.M
        if step <= 0:
            raise ValueError("periods_per_launch must be positive")
        if id(eng) not in self._batches:
            self._batches[id(eng)] = Batch([eng])
        b = self._batches[id(eng)]
        starts = list(range(lo - lo % step, hi, step))
        out = []
        for g in range(0, len(starts), 256):
            specs = [(0, MODE_SIEVE, 0, 0, max(lo, a), min(hi, a + step))
                     for a in starts[g:g + 256]]
            for (a, _m, _t, _c, wlo, _whi), (off, _d) in zip(
                    specs, b.run(specs, graph=False)):
                out.extend(wlo + int(o) for o in off.tolist())
        return out

    def hunt(self, lo, hi, cap=100, periods_per_launch=None):
        """Ascending [(p, exact_run)] with run >= n in [lo, hi)."""
        lo, hi = self._check(lo, hi)
        if hi <= lo:
            return []
        off, dep = self._eng_for(lo, hi).hunt(lo, hi, self.n, int(cap))
        return [(lo + int(o), int(d)) for o, d in zip(off.tolist(),
                                                       dep.tolist())]


def low_pass(n, cap=100, lo=2, hi=P_FLOOR):
    """Every p in [lo, hi) below the engine floor with run >= n, classified
    on the device with no sieve (euler-prime-runs/launch.py:410-420)."""
    eng = _device_engine(int(n), 6)
    off, dep = eng.dense(lo, hi, int(n), int(cap))
    return [(lo + int(o), int(d)) for o, d in zip(off.tolist(),
                                                   dep.tolist())]


def sweep(lo, hi, n, cap=100):
    """(p, run >= n) over [lo, hi) from any lo >= 2: the low pass below
    the floor, then the engine."""
    out = []
    if lo < P_FLOOR:
        out.extend(low_pass(n, cap, lo, min(hi, P_FLOOR)))
        lo = P_FLOOR
    if hi > lo:
        out.extend(GpuEngine(n).hunt(lo, hi, cap=cap))
    return out
