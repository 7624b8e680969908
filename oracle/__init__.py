"""CPU oracle for the sieve + strong-probable-prime hot path.

TEST INFRASTRUCTURE ONLY.  This package is a plain-Python/numpy
restatement of the reference CPU engines of jhg023/first-knowns, kept so
that the CUDA engine can be checked against an independent
implementation on identical inputs.  Only ``tests/``,
``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline / reference
arm may import it, and only as the checker or as the timed CPU baseline.
The product path (``first-knowns_b200/``) never imports it and has no
CPU fallback.

Every function cites the reference ``file:line`` it restates.  The
restatement is pinned by ``tests/test_oracle_golden.py`` against golden
vectors that ``tests/golden/make_golden.py`` produced by importing the
reference itself (its ``CpuEngine`` classes and ``huntlib.primes``), and
against the literature tables and score fingerprints that the reference
freezes in its own source.

Modules:
  primes  -- mr_is_prime / sprp_base2 (huntlib/primes.py)
  euler   -- Euler-form runs x^2+x+p (euler-prime-runs/)
  dickson -- Dickson ladders m*k^2+1 (dickson-ladders/)
  ap      -- primorial-step progressions p + j*d (primorial-ap/)
"""
