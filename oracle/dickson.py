"""Dickson ladders m*k^2 + 1: CPU restatement of the reference (oracle).

TEST INFRASTRUCTURE ONLY (see oracle/__init__.py).

Restates dickson-ladders/ladder_search.py (the segmented numpy
``CpuEngine`` over j with k = W*j), dickson-ladders/ladder_reference.py
(wheel modulus, run definition, K_FLOOR) and the launcher's low pass and
two-pass ``sprp_run`` (dickson-ladders/launch.py:310-343, 653-669).

Survivor definition (ladder_search.py:56-112): j in [j_lo, j_hi) such that
no prime q with n+2 <= q < q2 divides m*(W*j)^2 + 1 for any m = 1..n.
"""

import numpy as np

from .primes import mr_is_prime, primes_below, sprp_base2

# ladder_reference.py:37-45, 57
KNOWN = {1: 1, 2: 1, 3: 6, 4: 3240, 5: 113730, 6: 30473520,
         7: 3776600100, 8: 16341921960, 9: 3332396388090}
K_FLOOR = 10 ** 4
# ladder_search.py:52-53
Q2_DEFAULT = 65536
J_CEIL = 4 * 10 ** 18
# dickson-ladders/launch.py:308
SPRP_EXACT_FROM = 5


def wheel_modulus(n):
    """ladder_reference.py:60-66: product of the primes <= n+1."""
    w = 1
    for q in primes_below(n + 2):
        w *= q
    return w


def _sqrt_mod_prime(a, q):
    """All square roots of a modulo the odd prime q (Tonelli-Shanks)."""
    a %= q
    if a == 0:
        return [0]
    if pow(a, (q - 1) // 2, q) != 1:
        return []
    if q % 4 == 3:
        r = pow(a, (q + 1) // 4, q)
    else:
        s, t = 0, q - 1
        while t % 2 == 0:
            t //= 2
            s += 1
        z = 2
        while pow(z, (q - 1) // 2, q) != q - 1:
            z += 1
        c, r, tt, mm = pow(z, t, q), pow(a, (t + 1) // 2, q), pow(a, t, q), s
        while tt != 1:
            i, t2 = 0, tt
            while t2 != 1:
                t2 = t2 * t2 % q
                i += 1
            b = pow(c, 1 << (mm - i - 1), q)
            r, c = r * b % q, b * b % q
            tt, mm = tt * c % q, i
    return sorted({r, q - r})


def forbidden_j(q, n, W):
    """ladder_search.py:71-89: killed residues of j mod q.  k^2 == -1/m
    (mod q) for some m <= n, with j = k * W^-1."""
    winv = pow(W % q, q - 2, q)
    out = set()
    for m in range(1, n + 1):
        for root in _sqrt_mod_prime(-pow(m, q - 2, q), q):
            out.add(root * winv % q)
    return np.array(sorted(out), dtype=np.int64)


def run_length(k, cap=64):
    """ladder_search.py:143-148: largest r <= cap with m*k^2+1 passing
    mr_is_prime for every m = 1..r."""
    r = 0
    while r < cap and mr_is_prime((r + 1) * k * k + 1):
        r += 1
    return r


def sprp_run(k, cap):
    """dickson-ladders/launch.py:310-343: base-2 chain first; below
    SPRP_EXACT_FROM it is returned as is, else the 7-base chain."""
    kk = k * k
    r = 0
    while r < cap and sprp_base2((r + 1) * kk + 1):
        r += 1
    if r < SPRP_EXACT_FROM:
        return r
    r = 0
    while r < cap and mr_is_prime((r + 1) * kk + 1):
        r += 1
    return r


class CpuEngine:
    """ladder_search.py:56-162 ``CpuEngine`` restated."""

    def __init__(self, n, q2=Q2_DEFAULT):
        self.n = int(n)
        self.q2 = int(q2)
        self.W = wheel_modulus(self.n)
        self.primes = primes_below(self.q2, start=self.n + 2)
        self.table = {q: forbidden_j(q, self.n, self.W) for q in self.primes}
        self._sets = None

    def survivors_j(self, j_lo, j_hi, block=1 << 22):
        """ladder_search.py:92-112: sorted u64 survivors in [j_lo, j_hi)."""
        if j_hi > J_CEIL:
            raise ValueError("j past the enforced ceiling")
        if j_lo * self.W < K_FLOOR:
            raise ValueError("engines refuse to run below K_FLOOR")
        parts = []
        j0 = int(j_lo)
        while j0 < j_hi:
            j1 = min(j0 + block, int(j_hi))
            alive = np.ones(j1 - j0, dtype=bool)
            for q in self.primes:
                s = j0 % q
                for r in self.table[q]:
                    first = int((int(r) - s) % q)
                    if first < alive.size:
                        alive[first::q] = False
            idx = np.nonzero(alive)[0]
            if idx.size:
                parts.append((j0 + idx).astype(np.uint64))
            j0 = j1
        if not parts:
            return np.empty(0, dtype=np.uint64)
        return np.concatenate(parts)

    def survivors_j_deep(self, j_lo, j_hi, block=1 << 22):
        """Sorted surviving j in [j_lo, j_hi) as Python ints, at any depth.

        The same strided marking as survivors_j with the segment base kept
        as a Python int, so j may leave u64: the restatement of the deep
        zone the reference's GPU engine reaches through survivors_j_deep
        (dickson-ladders/ladder_gpu.py:783-804) and that its gate G17
        checks against big-integer divisibility of the values themselves
        (dickson-ladders/ladder_gpu.py:1206-1280; ``divisor`` below).  The
        reference's CPU engine refuses j past J_CEIL only to keep its u64
        output arrays exact (ladder_search.py:121-140 says so); nothing of
        the mathematics changes there."""
        j_lo, j_hi = int(j_lo), int(j_hi)
        if j_lo * self.W < K_FLOOR:
            raise ValueError("engines refuse to run below K_FLOOR")
        out = []
        j0 = j_lo
        while j0 < j_hi:
            j1 = min(j0 + block, j_hi)
            alive = np.ones(j1 - j0, dtype=bool)
            for q in self.primes:
                s = j0 % q
                for r in self.table[q]:
                    first = int((int(r) - s) % q)
                    if first < alive.size:
                        alive[first::q] = False
            out.extend(j0 + int(i) for i in np.nonzero(alive)[0].tolist())
            j0 = j1
        return out

    def divisor(self, k):
        """The first sieve prime dividing one of the values m*k^2 + 1,
        m = 1..n, or None: the survivor definition itself, on Python ints,
        as the reference's G17 evaluates it past u64 j
        (dickson-ladders/ladder_gpu.py:1248-1255)."""
        k = int(k)
        for q in self.primes:
            t = (k % q) * (k % q) % q
            for m in range(1, self.n + 1):
                if (m * t + 1) % q == 0:
                    return q
        return None

    def hunt_deep(self, k_lo, k_hi, cap=None, min_run=None):
        """hunt over [k_lo, k_hi] (inclusive) through survivors_j_deep, for
        k past the u64 j ceiling; ``min_run`` (default n) is the least run
        kept (ladder_search.py:150-162 keeps run >= n)."""
        cap = cap or self.n + 8
        want = self.n if min_run is None else int(min_run)
        j_lo = max(1, -(-int(k_lo) // self.W))
        j_hi = int(k_hi) // self.W + 1
        out = []
        for j in self.survivors_j_deep(j_lo, j_hi):
            k = j * self.W
            if k < k_lo or k > k_hi:
                continue
            r = run_length(k, cap=cap)
            if r >= want:
                out.append((k, r))
        return out

    def survivors_pre_mr(self, k_lo, k_hi):
        """ladder_search.py:114-119: the stream on the k line, both ends
        inclusive."""
        j_lo = max(1, -(-int(k_lo) // self.W))
        j_hi = int(k_hi) // self.W + 1
        return self.survivors_j(j_lo, j_hi)

    def survives(self, j):
        """ladder_search.py:121-140: one-candidate membership, any j."""
        j = int(j)
        if self._sets is None:
            self._sets = {q: frozenset(int(r) for r in t)
                          for q, t in self.table.items()}
        return all(j % q not in self._sets[q] for q in self.primes)

    def run_length(self, k, cap=64):
        return run_length(k, cap)

    def hunt(self, k_lo, k_hi, cap=None):
        """ladder_search.py:150-162: (k, run) with run >= n, k in
        [k_lo, k_hi] (inclusive), cap defaulting to n + 8."""
        cap = cap or self.n + 8
        out = []
        for j in self.survivors_pre_mr(k_lo, k_hi).tolist():
            k = int(j) * self.W
            if k < k_lo or k > k_hi:
                continue
            r = run_length(k, cap=cap)
            if r >= self.n:
                out.append((k, r))
        return out


def low_pass(n, cap, lo=1, hi=K_FLOOR):
    """dickson-ladders/launch.py:653-669 restated for one filter n: every
    k in [lo, hi) below the floor with run >= n, classified directly with
    no wheel (the exception zone of the wheel argument lives here)."""
    return [(k, r) for k in range(lo, hi)
            for r in [run_length(k, cap)] if r >= n]


def sweep(k_lo, k_hi, n, cap=None, q2=Q2_DEFAULT):
    """Whole-line (k, run >= n) over [k_lo, k_hi) half-open, low pass
    included."""
    cap = cap or n + 8
    out = []
    if k_lo < K_FLOOR:
        out.extend(low_pass(n, cap, lo=max(1, k_lo), hi=min(k_hi, K_FLOOR)))
        k_lo = K_FLOOR
    if k_hi > k_lo:
        out.extend(CpuEngine(n, q2).hunt(k_lo, k_hi - 1, cap=cap))
    return out
