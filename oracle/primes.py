"""Strong-probable-prime tests, restated from huntlib/primes.py (oracle).

TEST INFRASTRUCTURE ONLY (see oracle/__init__.py).

The device SPRP stage must reproduce these verdicts bit for bit,
including the two details that matter below the deterministic bound:
trial division by the primes to 37 returns ``m == sp`` (so the small
primes themselves are prime), and every base is reduced ``a %= m`` with
a zero base skipped.
"""

# huntlib/primes.py:17-18: the Sorenson-Webster 7-base set, deterministic
# below 3.317e24.
MR_BASES = (2, 325, 9375, 28178, 450775, 9780504, 1795265022)
MR_VALID_BELOW = 3_317_044_064_679_887_385_961_981

# huntlib/primes.py:20: trial-division primes.
SMALL_PRIMES = (2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37)


def _split_odd(m):
    """(d, s) with m - 1 = d * 2^s, d odd."""
    d, s = m - 1, 0
    while not d & 1:
        d >>= 1
        s += 1
    return d, s


def _strong_witness_passes(a, d, s, m):
    """True iff m passes the strong test to base a (a already in [1, m))."""
    x = pow(a, d, m)
    if x == 1 or x == m - 1:
        return True
    for _ in range(s - 1):
        x = x * x % m
        if x == m - 1:
            return True
    return False


def mr_is_prime(m):
    """huntlib/primes.py:23-47 ``mr_is_prime``: trial division by 2..37
    (returning ``m == sp`` on a hit), then the strong test to every base in
    MR_BASES after ``a %= m`` (a zero base is skipped)."""
    m = int(m)
    if m < 2:
        return False
    for sp in SMALL_PRIMES:
        if m % sp == 0:
            return m == sp
    d, s = _split_odd(m)
    for a in MR_BASES:
        a %= m
        if a == 0:
            continue
        if not _strong_witness_passes(a, d, s, m):
            return False
    return True


def sprp_base2(m):
    """huntlib/primes.py:50-80 ``sprp_base2``: the same trial division,
    then the strong test to base 2 alone."""
    m = int(m)
    if m < 2:
        return False
    for sp in SMALL_PRIMES:
        if m % sp == 0:
            return m == sp
    d, s = _split_odd(m)
    return _strong_witness_passes(2, d, s, m)


def primes_below(limit, start=2):
    """All primes p with start <= p < limit (simple sieve of Eratosthenes)."""
    import numpy as np
    limit = int(limit)
    if limit <= 2:
        return []
    flags = np.ones(limit, dtype=bool)
    flags[:2] = False
    for i in range(2, int(limit ** 0.5) + 1):
        if flags[i]:
            flags[i * i::i] = False
    return [int(q) for q in np.nonzero(flags)[0] if q >= start]
