"""Drop-in for dickson-ladders/ladder_gpu.py's GpuEngine, on libfk.

Same constructor, attributes and sweep methods as the reference class
(dickson-ladders/ladder_gpu.py:424-829):

    GpuEngine(n, q2=65536, ns=None, T=None, ratio=2.0, launch=2**34,
              warp_pop=2**16, vote=1, fold="auto")
    .n, .q2, .W, .P, .offs, .J_REACH        read by launch.py / cursors
    survivors_j(j_lo, j_hi, launch=None)    -> sorted np.uint64
    survivors_j_deep(j_lo, j_hi, launch=None) -> sorted [int]
    survivors_pre_mr(k_lo, k_hi, launch=None) (k range, both ends inclusive)
    run_length(k, cap=64), hunt(k_lo, k_hi, cap=None) -> [(k, run)]

The reference's tuning knobs (ns, T, ratio, launch, warp_pop, vote) are
accepted and validated as the reference validates them; they do not
change the stream, and the device engine takes its own geometry.  The
fold prime P keeps its reference meaning (``J_REACH = P * J_CEIL`` and the
API refusals built on it); the device line folds every sieve prime below
its first pattern prime into its wheel instead.
"""

import functools

import numpy as np

from fk_abi import DICKSON, Engine

Q2_DEFAULT = 65536
Q2_MAX = 1 << 30
J_CEIL = 4 * 10 ** 18
K_FLOOR = 10 ** 4


def _primes(lo, hi):
    out = []
    for q in range(max(2, lo), hi):
        if all(q % d for d in range(2, int(q ** 0.5) + 1)):
            out.append(q)
    return out


def wheel_modulus(n):
    """ladder_reference.py:60-66: product of the primes <= n + 1."""
    w = 1
    for q in _primes(2, n + 2):
        w *= q
    return w


@functools.lru_cache(maxsize=None)
def _device_engine(n, q2, two_pass=False):
    try:
        return Engine(DICKSON, n, q2=q2, p0=9, two_pass=two_pass)
    except ValueError:
        return Engine(DICKSON, n, q2=q2, p0=6, two_pass=two_pass)


class GpuEngine:
    """The Dickson-ladder sieve + SPRP engine (reference API)."""

    def __init__(self, n, q2=Q2_DEFAULT, ns=None, T=None, ratio=2.0,
                 launch=2 ** 34, warp_pop=2 ** 16, vote=1, fold="auto"):
        if not (2 < q2 <= Q2_MAX):
            raise ValueError(f"q2 {q2} is outside the range this engine's "
                             f"arithmetic is exact for (2, {Q2_MAX}]")
        if (T is not None and T < 1) or launch < 64 or vote < 1:
            raise ValueError("bad tuning constants")
        self.n = int(n)
        self.q2 = int(q2)
        self.W = wheel_modulus(self.n)
        self.LAUNCH = int(launch)
        # the first sieve prime above the wheel, computed from the square
        # roots directly (the reference's fold offsets, ladder_gpu.py:
        # 596-614, are the j residues the fold prime does not kill)
        first = None
        q = self.n + 2
        while first is None:
            if all(q % d for d in range(2, int(q ** 0.5) + 1)):
                first = q
            q += 1
        nxt = q
        while not all(nxt % d for d in range(2, int(nxt ** 0.5) + 1)):
            nxt += 1
        allp_gt1 = nxt < self.q2 and first < self.q2
        if fold == "auto":
            fold = first if allp_gt1 else None
        if fold:
            fold = int(fold)
            if fold < self.n + 2 or fold >= self.q2 or \
                    not all(fold % d for d in range(2, int(fold ** .5) + 1)):
                raise ValueError(f"fold prime {fold} is not a sieve prime "
                                 f"at n={n}, q2={q2}")
        self.P = int(fold) if fold else 1
        self.offs = self._fold_offsets(self.P) if fold else [0]
        self.J_REACH = self.P * J_CEIL
        self._dev = _device_engine(self.n, self.q2)

    def _fold_offsets(self, P):
        wm = self.W % P
        offs = []
        for s in range(P):
            t = (wm * s) * (wm * s) % P
            if all((m * t + 1) % P for m in range(1, self.n + 1)):
                offs.append(s)
        return offs

    def _sweep_j(self, j_lo, j_hi):
        if j_hi <= j_lo:
            return []
        off = self._dev.sieve(j_lo, j_hi)
        return off

    def survivors_j(self, j_lo, j_hi, launch=None):
        """Sorted u64 array of surviving j in [j_lo, j_hi)."""
        reach = min(self.J_REACH, 1 << 62)
        if j_hi > reach:
            raise ValueError(f"j {j_hi} past this API's reach {reach}; the "
                             f"deep zone is survivors_j_deep's")
        if j_lo * self.W < K_FLOOR:
            raise ValueError("engines refuse to run below K_FLOOR")
        j_lo, j_hi = int(j_lo), int(j_hi)
        off = self._sweep_j(j_lo, j_hi)
        if len(off) == 0:
            return np.empty(0, dtype=np.uint64)
        return off + np.uint64(j_lo)

    def survivors_j_deep(self, j_lo, j_hi, launch=None):
        """Sorted list of surviving j in [j_lo, j_hi) as Python ints."""
        j_lo, j_hi = int(j_lo), int(j_hi)
        if j_hi > self.J_REACH:
            raise ValueError(f"j {j_hi} past the enforced reach "
                             f"{self.J_REACH} (= fold {self.P} x J_CEIL)")
        if j_lo * self.W < K_FLOOR:
            raise ValueError("engines refuse to run below K_FLOOR")
        off = self._sweep_j(j_lo, j_hi)
        return [j_lo + int(o) for o in np.asarray(off).tolist()]

    def survivors_pre_mr(self, k_lo, k_hi, launch=None):
        """The same stream on the k line (both ends inclusive)."""
        j_lo = max(1, -(-int(k_lo) // self.W))
        j_hi = int(k_hi) // self.W + 1
        return self.survivors_j(j_lo, j_hi, launch)

    def run_length(self, k, cap=64):
        """Largest r <= cap with m*k^2+1 a strong probable prime for all
        m = 1..r, on the device (ladder_gpu.py:813-817)."""
        return int(self._dev.depths([int(k)], int(cap))[0])

    def hunt(self, k_lo, k_hi, cap=None):
        """[(k, run)] for k in [k_lo, k_hi] whose run reaches n."""
        cap = cap or self.n + 8
        j_lo = max(1, -(-int(k_lo) // self.W))
        j_hi = int(k_hi) // self.W + 1
        if j_hi > min(self.J_REACH, 1 << 62):
            raise ValueError("j past this API's reach")
        if j_lo * self.W < K_FLOOR:
            raise ValueError("engines refuse to run below K_FLOOR")
        if j_hi <= j_lo:
            return []
        off, dep = self._dev.hunt(j_lo, j_hi, self.n, int(cap))
        W = self.W
        return [((j_lo + int(o)) * W, int(d))
                for o, d in zip(off.tolist(), dep.tolist())]


def low_pass(n, cap, lo=1, hi=K_FLOOR, q2=Q2_DEFAULT):
    """Every k in [lo, hi) below the floor with run >= n, classified on the
    device with no wheel (dickson-ladders/launch.py:653-669)."""
    eng = _device_engine(int(n), int(q2))
    off, dep = eng.dense(lo, hi, int(n), int(cap))
    return [(lo + int(o), int(d)) for o, d in zip(off.tolist(),
                                                   dep.tolist())]


def sweep(k_lo, k_hi, n, cap=None, q2=Q2_DEFAULT):
    """(k, run >= n) over [k_lo, k_hi) half-open, low pass included."""
    cap = cap or n + 8
    out = []
    if k_lo < K_FLOOR:
        out.extend(low_pass(n, cap, max(1, k_lo), min(k_hi, K_FLOOR), q2))
        k_lo = K_FLOOR
    if k_hi > k_lo:
        out.extend(GpuEngine(n, q2=q2).hunt(k_lo, k_hi - 1, cap=cap))
    return out
