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
  sprp_dickson6 8 Dickson intervals (n = 6) of 2^34 at k = 1e18: SPRP
                chains on 122-bit values (four 32-bit limbs)
  mixed         256 intervals of the mixed workload, clipped to 2^28
  euler_wide17  the Euler n = 17 pre-primality stream over [6.11e20,
                +2e15) through the reference-API mirror (31# wheel, the
                pattern sieve of the SCORE_WIDE window at a tenth of its
                length)
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
    if name == "sprp_dickson6":
        return [W.Interval(W.DICKSON, 6, 10 ** 18 + i * 2 ** 36,
                           10 ** 18 + i * 2 ** 36 + 2 ** 34, 6, 14)
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


def euler_wide(runs, warp_lane_words=0):
    from euler_gpu import GpuEngine
    eng = GpuEngine(17)
    lo, span = 611 * 10 ** 18, 2 * 10 ** 15
    if warp_lane_words:
        eng._eng_for(lo, lo + span).set_tuning(
            warp_lane_words=warp_lane_words)
    for r in range(runs):
        t0 = time.perf_counter()
        s = eng.survivors_pre_mr(lo, lo + span)
        dt = time.perf_counter() - t0
        st = eng._eng_for(lo, lo + span).stats()
        print(f"euler_wide17 run {r}: {dt * 1e3:.1f} ms wall, sieve "
              f"{st['sieve_ms']:.1f} ms, {len(s)} survivors, s1_words "
              f"{st['s1_words']}, s2_tests {st['s2_tests']}", flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--case", required=True)
    ap.add_argument("--runs", type=int, default=2)
    ap.add_argument("--warp-lane-words", type=int, default=0,
                    help="euler_wide17: lanes from this many words go one "
                         "warp per lane (0: the engine default)")
    args = ap.parse_args()
    if args.case == "euler_wide17":
        return euler_wide(args.runs, args.warp_lane_words)
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
