"""Primorial-step progressions p + j*d: CPU restatement (oracle).

TEST INFRASTRUCTURE ONLY (see oracle/__init__.py).

Restates primorial-ap/ap_search.py (the flat numpy ``CpuEngine`` with its
two-pass ``chain_depth``) and primorial-ap/ap_reference.py (difference,
KNOWN, floor).  The difference may be overridden (``d=``): that is the
adapter for a fixed difference such as 13# = 30030 with chains counted to
a threshold, built from the reference's own residue formula
(ap_search.py:99-106) with the override in place of P(n).

Survivor definition (ap_search.py:92-141): p in [base, base + span),
coprime to 30, such that no prime 7 <= q < q2 divides p + j*d for any
j < n.
"""

import numpy as np

from .primes import mr_is_prime, primes_below, sprp_base2

# ap_reference.py:61-75, 89-93
KNOWN = {1: 2, 2: 5, 3: 7, 4: 13, 5: 37, 6: 73, 7: 7937, 8: 7703,
         9: 272809, 10: 640943, 11: 5378959, 12: 116137159,
         13: 3708797237, 14: 114649314209, 15: 158317270283}
P_FLOOR = 10 ** 4
W0 = 30
W0_RESIDUES = (1, 7, 11, 13, 17, 19, 23, 29)
# ap_search.py:65-67, 80-86
Q2_DEFAULT = 1 << 16
P_CEIL = 10 ** 26
DEPTH_EXACT_FROM = 6


def difference(n):
    """ap_reference.py:99-110: the n-th primorial P(n)."""
    d = 1
    for q in primes_below(10 ** 4)[:n]:
        d *= q
    return d


def chain_depth_two_pass(p, d, cap):
    """ap_search.py:160-194: base-2 chain from j = 0; if it is below
    DEPTH_EXACT_FROM it is returned, else the 7-base chain."""
    j = 0
    while j < cap and sprp_base2(p + j * d):
        j += 1
    if j < DEPTH_EXACT_FROM:
        return j
    j = 0
    while j < cap and mr_is_prime(p + j * d):
        j += 1
    return j


_WHEEL30 = np.array([all(r % q for q in (2, 3, 5)) for r in range(W0)],
                    dtype=bool)


class CpuEngine:
    """ap_search.py:92-207 ``CpuEngine`` restated, with an optional
    difference override for fixed-difference sweeps."""

    def __init__(self, n, q2=Q2_DEFAULT, d=None):
        self.n = int(n)
        self.q2 = int(q2)
        self.d = int(d) if d is not None else difference(self.n)
        self.primes = primes_below(self.q2, start=7)
        self.forb = {q: sorted({(-j * self.d) % q for j in range(self.n)})
                     for q in self.primes}
        self.forbset = {q: frozenset(v) for q, v in self.forb.items()}
        self.floor = max(P_FLOOR, self.q2)

    def survivors(self, base, span, block=1 << 23):
        """ap_search.py:109-141: sorted u64 offsets o with base + o
        surviving, over [base, base + span)."""
        base, span = int(base), int(span)
        if base < self.floor:
            raise ValueError("below the engine floor")
        if base + span > P_CEIL:
            raise ValueError("past the enforced ceiling")
        parts = []
        off = 0
        while off < span:
            size = min(block, span - off)
            b = base + off
            ph = b % W0
            alive = np.tile(_WHEEL30, size // W0 + 2)[ph:ph + size].copy()
            for q in self.primes:
                bm = b % q
                for f in self.forb[q]:
                    s = (f - bm) % q
                    if s < size:
                        alive[s::q] = False
            idx = np.nonzero(alive)[0]
            if idx.size:
                parts.append((idx + off).astype(np.uint64))
            off += size
        if not parts:
            return np.empty(0, dtype=np.uint64)
        return np.concatenate(parts)

    def survives(self, p):
        """ap_search.py:143-157."""
        p = int(p)
        if p % 2 == 0 or p % 3 == 0 or p % 5 == 0:
            return False
        return all(p % q not in self.forbset[q] for q in self.primes)

    def chain_depth(self, p, cap=None):
        cap = self.n if cap is None else int(cap)
        return chain_depth_two_pass(int(p), self.d, cap)

    def hunt(self, base, span, min_depth=None, cap=None):
        """ap_search.py:196-207: (p, depth) for survivors reaching
        min_depth (default n); ``cap`` is chain_depth's cap (default n)."""
        want = self.n if min_depth is None else int(min_depth)
        out = []
        for o in self.survivors(base, span).tolist():
            p = int(base) + int(o)
            dep = self.chain_depth(p, cap)
            if dep >= want:
                out.append((p, dep))
        return out


def first_p(n, lo=2, hi=None, d=None, cap=None):
    """ap_reference.py:130-143 (wheel=False form, with the two-pass depth
    the engines report): least p in [lo, hi] whose chain reaches n."""
    dd = difference(n) if d is None else int(d)
    cap = n if cap is None else cap
    p = int(lo)
    while hi is None or p <= hi:
        if chain_depth_two_pass(p, dd, cap) >= n:
            return p
        p += 1
    return None
