"""Autotuner for the batch pipeline's kernel shape.

The search space is fk_tuning (include/fk.h): CTAs per SM of the three
persistent grids (pattern sieve + rounds, marking sieve, SPRP), chains per
SM when lanes are cut into chains, the compaction cadence (a warp's queue
shorter than ``warp_queue`` goes one candidate per warp), the marking task
length in segments, the lane length from which a warp sweeps one lane,
the lane length from which eight threads sweep one lane
(``group_lane_words``), the marking sieve's prime bound (primes below
``mark_limit`` are marked, the rest tested per candidate), the bias
between marking and compaction rounds, the survival at which a
compaction round is cut (``round_cut``: lower means fewer, longer rounds),
and three kernel-variant choices: the marking segment length in bytes
(``mark_segment``: 16, 32 or 64 KiB of shared byte map) and the pattern
primes each CTA stages in shared memory, per sieve kernel
(``pattern_primes``, ``mark_pattern_primes``: 24, 32 or 40), and the
blocks of chains per CTA task of the rounds kernel (``warp_tasks``).
None of them can change a result; they only move time.

``tune`` runs coordinate descent: starting from the current setting it
tries every value of one parameter at a time on a sample of the workload,
keeps the fastest (median device time of ``repeats`` runs, CUDA events on
the pipeline's stream), and sweeps the parameters until a pass improves
nothing or the time budget is spent.  The best setting can be saved as
JSON and loaded by any later BatchEngine.
"""

import json
import pathlib
import statistics
import time

SPACE = {
    "mark_bias": [0.5, 0.7, 1.4, 2.0],
    "mark_limit": [49152, 65536],
    "seg_per_task": [2, 4, 8, 16],
    "chains_per_sm": [1024, 2048, 4096, 8192],
    "warp_queue": [8, 16, 64, 128],
    "sieve_ctas_per_sm": [2, 3],
    "mark_ctas_per_sm": [2, 3],
    "classify_ctas_per_sm": [4, 8, 16],
    "warp_lane_words": [64, 1024, 1 << 30],
    "round_cut": [0.3, 0.7, 0.85],
    "group_lane_words": [16, 64, 1 << 30],
    "pattern_primes": [24, 40],
    "mark_pattern_primes": [24, 40],
    "mark_segment": [16384, 65536],
    "warp_tasks": [16, 32],
}

DEFAULT_PATH = pathlib.Path(__file__).resolve().parent / "tuning.json"


def measure(engine, intervals, repeats=2, give_up_ms=None):
    """Median device time (ms) of the batch pipeline on the intervals.  A
    first run slower than ``give_up_ms`` is returned alone: a setting that
    far behind is not timed again."""
    times = []
    for _ in range(repeats):
        engine.run_arrays(intervals, graph=False)
        times.append(engine.stats()["total_ms"])
        if give_up_ms is not None and times[0] > give_up_ms:
            return times[0]
    return statistics.median(times)


def tune(engine, intervals, repeats=2, max_passes=2, budget_s=120.0,
         log=None, space=SPACE):
    """Coordinate descent over ``space``; applies and returns the best.

    A candidate replaces the incumbent only when it is at least 1% faster,
    so run-to-run noise (repeated trials of one setting agree within about
    0.3% of device time) does not wander the setting."""
    engine.run_arrays(intervals, graph=False)          # warm: tables, buffers
    best = engine.tuning()
    best_ms = measure(engine, intervals, repeats)
    t0 = time.time()
    trials = [{"setting": dict(best), "ms": best_ms}]
    for _ in range(max_passes):
        improved = False
        for key, values in space.items():
            for v in values:
                if time.time() - t0 > budget_s:
                    break
                if v == best[key]:
                    continue
                cand = dict(best)
                cand[key] = v
                engine.set_tuning(**cand)
                ms = measure(engine, intervals, repeats,
                             give_up_ms=1.5 * best_ms)
                trials.append({"setting": cand, "ms": ms})
                if log:
                    log(f"tune {key}={v}: {ms:.1f} ms (best {best_ms:.1f})")
                if ms < best_ms * 0.99:
                    best, best_ms, improved = cand, ms, True
            engine.set_tuning(**best)
        if not improved or time.time() - t0 > budget_s:
            break
    engine.set_tuning(**best)
    return {"best": best, "best_ms": best_ms, "trials": trials,
            "seconds": time.time() - t0}


def save(result, path=DEFAULT_PATH):
    pathlib.Path(path).write_text(json.dumps(result["best"], indent=1))


def load(engine, path=DEFAULT_PATH):
    """Apply a saved setting to a BatchEngine (or PlainEngine); False when
    there is none."""
    p = pathlib.Path(path)
    if not p.exists():
        return False
    engine.set_tuning(**json.loads(p.read_text()))
    return True
