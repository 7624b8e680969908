"""Fixed small sweeps for profiling one kernel at a time (ncu).

    python first-knowns_b200/fk_profile.py --case NAME [--runs 2]

Each case runs the same batch ``runs`` times (the first is a warm-up), so
an ncu capture can skip the first launch of a kernel (``-s 1 -c 1``) and
measure a warm one.  The cases keep device memory to a few hundred MB:

  mark_ap6      8 AP intervals (n = 6) of 2^32: the marking sieve (k_mark)
  rounds_ap10   8 AP intervals (n = 10) of 2^33: per-candidate rounds
                (k_sieve)
  sprp_euler4   8 Euler intervals (n = 4) of 2^34: the SPRP chains
                (k_classify)
  mixed         256 intervals of the mixed workload, clipped to 2^28
"""

import argparse
import pathlib
import sys
import time

HERE = pathlib.Path(__file__).resolve().parent
sys.path.insert(0, str(HERE))

import fk_workloads as W  # noqa: E402
from fk_batch import BatchEngine  # noqa: E402


def case(name):
    if name == "mark_ap6":
        return [W.Interval(W.AP, 6, 10 ** 14 + i * 2 ** 33,
                           10 ** 14 + i * 2 ** 33 + 2 ** 32 - 2 ** 32 % 30,
                           6, 6) for i in range(8)]
    if name == "rounds_ap10":
        return [W.Interval(W.AP, 10, 10 ** 15 + i * 2 ** 34,
                           10 ** 15 + i * 2 ** 34 + 2 ** 33 - 2 ** 33 % 30,
                           10, 10) for i in range(8)]
    if name == "sprp_euler4":
        return [W.Interval(W.EULER, 4, 10 ** 16 + i * 2 ** 35,
                           10 ** 16 + i * 2 ** 35 + 2 ** 34, 4, 100)
                for i in range(8)]
    if name == "mixed":
        out = []
        for iv in W.mixed_batch(256):
            hi = min(iv.hi, iv.lo + (1 << 28))
            if iv.kind == W.AP:
                hi = iv.lo + max(30, (hi - iv.lo) // 30 * 30)
            out.append(W.Interval(iv.kind, iv.n, iv.lo, hi, iv.threshold,
                                  iv.cap))
        return out
    raise SystemExit(f"unknown case {name}")


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--case", required=True)
    ap.add_argument("--runs", type=int, default=2)
    args = ap.parse_args()
    ivs = case(args.case)
    be = BatchEngine(ivs)
    for r in range(args.runs):
        t0 = time.perf_counter()
        rows = be.run_arrays(ivs, graph=False)
        dt = time.perf_counter() - t0
        st = be.stats()
        print(f"{args.case} run {r}: {dt * 1e3:.1f} ms wall, sieve "
              f"{st['sieve_ms']:.1f} ms, classify {st['classify_ms']:.1f} ms,"
              f" {sum(x[0].size for x in rows)} hits, {st['launches']} "
              f"launches, candidates {st['candidates']}, s1_words "
              f"{st['s1_words']}, s2_tests {st['s2_tests']}, marks "
              f"{st['marks']}, sprp_values {st['sprp_values']}", flush=True)


if __name__ == "__main__":
    main()
