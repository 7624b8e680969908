"""Drop-in for primorial-ap/ap_gpu.py's GpuEngine, on libfk.

Same constructor, attributes and methods as the reference class
(primorial-ap/ap_gpu.py:398-670):

    GpuEngine(n, q2=65536, launch_u=2**27)
    .n, .q2, .d, .primes, .floor, .launch_u, nbytes()
    survivors(base, span, launch_u=None)  yields ascending u64 offset
                                          arrays, one per launch
    hunt(base, span, min_depth=None)      -> [(p, depth)]
    survives(p)                           -> bool (verification legs)
    chain_depth(p, cap=None)              two-pass depth (base 2 first)

An optional ``d=`` overrides the difference P(n) for fixed-difference
sweeps (e.g. 13# with chains counted to a threshold); the residue sets
are then {-j*d mod q : j < n}, the reference's own formula
(primorial-ap/ap_search.py:99-106) with the override in place of P(n).
"""

import functools

import numpy as np

from fk_abi import AP, MODE_SIEVE, Batch, Engine

Q2_DEFAULT = 1 << 16
Q2_MAX = 1 << 30
LAUNCH_U = 1 << 27
# launches swept per device call by survivors(): each launch is one item
# of a single batch run, so the host holds at most this many launches'
# survivors at once
LAUNCHES_PER_CALL = 256
P_FLOOR = 10 ** 4
P_CEIL = 10 ** 26
W0 = 30


def _primes(lo, hi):
    out = []
    for q in range(max(2, lo), hi):
        if all(q % d for d in range(2, int(q ** 0.5) + 1)):
            out.append(q)
    return out


def difference(n):
    """ap_reference.py:99-110: the n-th primorial."""
    d, k, q = 1, 0, 2
    while k < n:
        if all(q % p for p in range(2, int(q ** 0.5) + 1)):
            d *= q
            k += 1
        q += 1
    return d


@functools.lru_cache(maxsize=None)
def _device_engine(n, q2, d):
    return Engine(AP, n, q2=q2, p0=6, d=d)


@functools.lru_cache(maxsize=None)
def _device_batch(n, q2, d):
    """One batch per device engine, shared by every GpuEngine of these
    parameters (its buffers grow once and stay)."""
    return Batch([_device_engine(n, q2, d)])


class GpuEngine:
    """The primorial-step AP sieve + SPRP engine (reference API)."""

    def __init__(self, n, q2=Q2_DEFAULT, launch_u=LAUNCH_U, d=None):
        if not 7 <= q2 <= Q2_MAX:
            raise ValueError(f"q2 {q2} outside [7, {Q2_MAX}]")
        self.n = int(n)
        self.q2 = int(q2)
        self._fixed_d = d is not None
        self.d = int(d) if d is not None else difference(self.n)
        self.launch_u = int(launch_u)
        self.floor = max(P_FLOOR, self.q2)
        self._dev = _device_engine(self.n, self.q2, self.d)
        self._primes = None

    @property
    def primes(self):
        if self._primes is None:
            self._primes = _primes(7, self.q2)
        return self._primes

    def nbytes(self):
        return int(self._dev.device_bytes)

    def _check(self, base, span):
        base, span = int(base), int(span)
        # the reference GPU API takes whole wheel periods; a fixed-difference
        # sweep follows the CPU engine's contract (ap_search.py:109-141),
        # which takes any base
        if not self._fixed_d and (base % W0 or span % W0):
            raise ValueError(f"base and span must be multiples of {W0}")
        if base < self.floor:
            raise ValueError(f"the engine refuses to sieve below {self.floor}")
        if base + span > P_CEIL:
            raise ValueError(f"p {base + span} is past the enforced ceiling "
                             f"{P_CEIL}")
        return base, span

    def survivors(self, base, span, launch_u=None):
        """Yield uint64 arrays of offsets o with base + o surviving,
        ascending, one array per launch of launch_u wheel periods (empty
        launches yield nothing), as the reference's generator does
        (primorial-ap/ap_gpu.py:555-635).  Each launch window is one item
        of a batch run, up to LAUNCHES_PER_CALL of them per device call, so
        a campaign-length segment never sits on the host whole."""
        base, span = self._check(base, span)
        if span <= 0:
            return
        step = W0 * int(launch_u or self.launch_u)
        batch = _device_batch(self.n, self.q2, self.d)
        starts = list(range(0, span, step))
        for g in range(0, len(starts), LAUNCHES_PER_CALL):
            group = starts[g:g + LAUNCHES_PER_CALL]
            specs = [(0, MODE_SIEVE, 0, 0, base + a, base + min(span, a + step))
                     for a in group]
            rows = batch.run(specs, graph=False)
            for a, (off, _dep) in zip(group, rows):
                if off.size:
                    yield off + np.uint64(a)

    def hunt(self, base, span, min_depth=None):
        """[(p, depth)] for every survivor whose chain reaches min_depth."""
        base, span = self._check(base, span)
        want = self.n if min_depth is None else int(min_depth)
        if span <= 0:
            return []
        off, dep = self._dev.hunt(base, base + span, want, self.n)
        return [(base + int(o), int(dd)) for o, dd in zip(off.tolist(),
                                                           dep.tolist())]

    def hunt_cap(self, base, span, min_depth, cap):
        """hunt with an explicit chain cap (fixed-difference sweeps count
        chains past n)."""
        base, span = self._check(base, span)
        off, dep = self._dev.hunt(base, base + span, int(min_depth), int(cap))
        return [(base + int(o), int(dd)) for o, dd in zip(off.tolist(),
                                                           dep.tolist())]

    def survives(self, p):
        """One-candidate membership: the device sieve over [p, p + 1)."""
        p = int(p)
        if p % 2 == 0 or p % 3 == 0 or p % 5 == 0:
            return False
        return self._dev.sieve(p, p + 1).size == 1

    def chain_depth(self, p, cap=None):
        """Two-pass chain depth of p (ap_search.py:160-194), on the
        device."""
        cap = self.n if cap is None else int(cap)
        return int(self._dev.depths([int(p)], cap)[0])
