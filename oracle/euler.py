"""Euler-form runs x^2 + x + p: CPU restatement of the reference (oracle).

TEST INFRASTRUCTURE ONLY (see oracle/__init__.py).

Restates euler-prime-runs/euler_search.py (wheel mathematics and the
numpy ``CpuEngine``) and euler-prime-runs/euler_reference.py (the run
definition), plus the launcher's low pass below the engine floor
(euler-prime-runs/launch.py:410-424).

Survivor definition (euler_search.py:1-20, 284-359): p in [lo, hi) such
that no prime q < Q2 divides any of the n values x^2 + x + p, x < n.  The
wheel only decides which primes are removed by enumeration rather than by
sieving; the survivor set does not depend on it.
"""

import numpy as np

from .primes import mr_is_prime, primes_below

# euler_search.py:51-60
WHEEL_PRIMES = [2, 3, 5, 7, 11, 13, 17, 19, 23]
WHEEL_PRIMES_29 = WHEEL_PRIMES + [29]
Q1 = 1024
Q2 = 65536
P_FLOOR = 100_000
# euler_search.py:276
P_CEIL = 10 ** 24

# euler_reference.py:22-40 (OEIS A164926 data frozen by the reference)
KNOWN = {1: 2, 2: 3, 3: 107, 4: 5, 5: 347, 6: 1607, 7: 1277, 8: 21557,
         9: 51867197, 10: 11, 11: 180078317, 12: 1761702947,
         13: 8776320587, 14: 27649987598537, 15: 291598227841757,
         16: 17, 40: 41}
# euler_reference.py:45 and launch.py:121-128 (campaign finds)
A21_UPPER = 234505015943235329417


def forbidden(q, n):
    """euler_search.py:85-87: residues r of p mod q for which q divides
    x^2 + x + p for some x < n."""
    return {(-(x * x + x)) % q for x in range(n)}


def build_wheel(n, wheel_primes):
    """euler_search.py:215-250 ``build_wheel``: the admissible residues of
    p modulo prod(wheel_primes), sorted, and that product.

    Built by CRT lifting one prime at a time: a residue r mod m lifts to
    r + t*m mod m*q for t in [0, q), keeping the lifts whose residue mod q
    is admissible.
    """
    offs = np.zeros(1, dtype=np.uint64)
    m = 1
    for q in wheel_primes:
        bad = np.array(sorted(forbidden(q, n)), dtype=np.int64)
        t = np.arange(q, dtype=np.uint64)
        lift = (offs[None, :] + t[:, None] * np.uint64(m)).ravel()
        keep = ~np.isin((lift % np.uint64(q)).astype(np.int64), bad)
        offs = lift[keep]
        m *= q
    offs.sort()
    return offs, m


def wheel_offset_count(n, wheel_primes):
    """euler_search.py:90-95."""
    c = 1
    for q in wheel_primes:
        c *= q - len(forbidden(q, n))
    return c


def mr_run_length(p, cap=100):
    """euler_search.py:258-262: consecutive x >= 0 with x^2+x+p passing
    mr_is_prime, capped at ``cap``."""
    x = 0
    while x < cap and mr_is_prime(x * x + x + p):
        x += 1
    return x


class CpuEngine:
    """euler_search.py:284-359 ``CpuEngine`` restated: survivors of the
    sieve as exact Python ints, computed with numpy ``%`` on (k, off)
    pairs, p = k*M + off."""

    def __init__(self, n, wheel_primes=None):
        self.n = int(n)
        self.wheel_primes = list(wheel_primes or WHEEL_PRIMES_29)
        self.offs, self.M = build_wheel(self.n, self.wheel_primes)
        top = self.wheel_primes[-1]
        self.primes = primes_below(Q2, start=top + 1)
        self.xx = [x * x + x for x in range(self.n)]
        self.lut = {}
        for q in self.primes:
            t = np.zeros(q, dtype=bool)
            t[sorted(forbidden(q, self.n))] = True
            self.lut[q] = t

    def survivors_pre_mr(self, lo, hi, periods_per_chunk=16):
        """Sorted survivor p in [lo, hi) (euler_search.py:301-347)."""
        lo, hi = int(lo), int(hi)
        if lo < P_FLOOR:
            raise ValueError("engine floor is %d" % P_FLOOR)
        if hi > P_CEIL:
            raise ValueError("engine ceiling is %d" % P_CEIL)
        M = int(self.M)
        out = []
        k_first, k_last = lo // M, (hi - 1) // M
        for kc in range(k_first, k_last + 1, periods_per_chunk):
            ks = np.arange(kc, min(kc + periods_per_chunk, k_last + 1),
                           dtype=np.uint64)
            K = np.repeat(ks, self.offs.size)
            O = np.tile(self.offs, ks.size)
            # window test on exact ints would be slow; do it in (k, off):
            # p >= lo  <=> k > lo//M or off >= lo%M, and likewise for hi
            keep = ((K > np.uint64(lo // M)) | (O >= np.uint64(lo % M))) & \
                   ((K < np.uint64((hi - 1) // M)) |
                    (O <= np.uint64((hi - 1) % M)))
            K, O = K[keep], O[keep]
            for q in self.primes:
                if K.size == 0:
                    break
                qq = np.uint64(q)
                r = ((K % qq) * np.uint64(M % q) + O % qq) % qq
                alive = ~self.lut[q][r.astype(np.int64)]
                K, O = K[alive], O[alive]
            out.extend(sorted(int(k) * M + int(o)
                              for k, o in zip(K.tolist(), O.tolist())))
        return out

    def hunt(self, lo, hi, cap=100):
        """euler_search.py:349-356: (p, run) with all n values prime."""
        res = []
        for p in self.survivors_pre_mr(lo, hi):
            if all(mr_is_prime(p + v) for v in self.xx):
                res.append((p, mr_run_length(p, cap=cap)))
        return res


def low_pass(n, cap=100, lo=2, hi=P_FLOOR):
    """euler-prime-runs/launch.py:410-420: every p in [lo, hi) below the
    engine floor with run >= n, by direct classification.  The reference
    uses sympy's isprime here; mr_is_prime is exact at these sizes."""
    return [(p, r) for p in range(lo, hi)
            for r in [mr_run_length(p, cap=cap)] if r >= n]


def sweep(lo, hi, n, cap=100, wheel_primes=None):
    """Whole-line (p, run >= n) over [lo, hi), low pass included: the
    oracle's restatement of what a campaign segment reports."""
    out = []
    if lo < P_FLOOR:
        out.extend(low_pass(n, cap=cap, lo=lo, hi=min(hi, P_FLOOR)))
        lo = P_FLOOR
    if hi > lo:
        out.extend(CpuEngine(n, wheel_primes).hunt(lo, hi, cap=cap))
    return out
