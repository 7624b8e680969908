"""The batched and served engines: identical to the plain engine.

One persistent launch over many intervals of mixed engine type must give,
for every interval, exactly the stream the plain per-interval call gives,
whether replayed from a captured CUDA graph or launched eagerly, and
whether the interval runs alone or in a mix; the serving loop must return
the same results for requests that overlap on the device.
"""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _clipped(count, seed, clip=1 << 26):
    import fk_workloads as W
    out = []
    for iv in W.mixed_batch(count, seed):
        hi = min(iv.hi, iv.lo + clip)
        if iv.kind == W.AP:
            hi = iv.lo + max(30, (hi - iv.lo) // 30 * 30)
        out.append(W.Interval(iv.kind, iv.n, iv.lo, hi, iv.threshold, iv.cap))
    return out


def _same(a, b):
    return len(a) == len(b) and all(
        np.array_equal(x[0], y[0]) and np.array_equal(x[1], y[1])
        for x, y in zip(a, b))


def test_batch_equals_plain_graph_and_eager():
    from fk_batch import BatchEngine, PlainEngine
    ivs = _clipped(300, 77)
    be = BatchEngine(ivs)
    g1 = be.run_arrays(ivs, graph=True)
    g2 = be.run_arrays(ivs, graph=True)          # graph replay
    e1 = be.run_arrays(ivs, graph=False)
    p = PlainEngine(be.engset).run_arrays(ivs)
    assert _same(g1, g2) and _same(g1, e1) and _same(g1, p)
    assert sum(x[0].size for x in g1) > 100


def test_alone_equals_in_the_mix():
    from fk_batch import BatchEngine
    ivs = _clipped(120, 78)
    be = BatchEngine(ivs)
    mix = be.run(ivs)
    for i in (0, 7, 33, 119):
        assert be.run([ivs[i]])[0] == mix[i]


def test_batch_equals_oracle_on_a_sample():
    from fk_batch import BatchEngine
    from oracle import sweep
    ivs = _clipped(24, 79, clip=1 << 21)
    got = BatchEngine(ivs).run(ivs)
    for iv, g in zip(ivs, got):
        assert g == sweep.hunt_interval(iv.kind, iv.n, iv.lo, iv.hi,
                                        iv.threshold, iv.cap, iv.q2, iv.d)


def test_full_length_intervals_through_the_marking_sieve():
    """Unclipped long intervals (the marking kernel's territory) agree
    between the batch and the plain engine, and the batch stats show the
    marking sieve ran."""
    import fk_workloads as W
    from fk_batch import BatchEngine, PlainEngine
    ivs = [iv for iv in W.mixed_batch(200, 80) if iv.length > 2 ** 33][:6]
    be = BatchEngine(ivs)
    got = be.run_arrays(ivs)
    assert be.stats()["marks"] > 0
    assert _same(got, PlainEngine(be.engset).run_arrays(ivs))


def test_serving_loop_matches_plain_results():
    import fk_workloads as W
    from fk_batch import PlainEngine
    from fk_serve import ServeLoop
    reqs = []
    for t, iv in W.served(count=150, rate_hz=400.0):
        hi = min(iv.hi, iv.lo + (1 << 24))
        if iv.kind == W.AP:
            hi = iv.lo + max(30, (hi - iv.lo) // 30 * 30)
        reqs.append((t, W.Interval(iv.kind, iv.n, iv.lo, hi, iv.threshold,
                                   iv.cap)))
    loop = ServeLoop(slots=2, max_items=32)
    res, lat, st = loop.run(reqs)
    assert st["requests"] == len(reqs) and st["batches"] > 1
    assert np.all(lat >= 0)
    plain = PlainEngine(loop.engset).run_arrays([iv for _, iv in reqs])
    assert _same(res, plain)


def test_serving_loop_chunks_long_requests():
    """Requests cut into many chunks (1/16 of their line each, spread over
    several batches of a small work budget) come back identical to the
    plain engine's single call on the whole request, Dickson (k = W*j)
    included."""
    import fk_workloads as W
    from fk_batch import PlainEngine
    from fk_serve import ServeLoop
    reqs = []
    for t, iv in W.served(count=40, rate_hz=2000.0, seed=W.SEED + 5):
        hi = min(iv.hi, iv.lo + (1 << 26))
        if iv.kind == W.AP:
            hi = iv.lo + max(30, (hi - iv.lo) // 30 * 30)
        reqs.append((t, W.Interval(iv.kind, iv.n, iv.lo, hi, 0, iv.cap)))
    loop = ServeLoop(slots=2, chunk=1 << 22, batch_work=1 << 24)
    pieces = [len(loop.chunks(iv)) for _, iv in reqs]
    assert max(pieces) >= 8
    res, lat, st = loop.run(reqs)
    assert st["requests"] == len(reqs) and st["batches"] >= sum(pieces) // 8
    plain = PlainEngine(loop.engset).run_arrays([iv for _, iv in reqs])
    assert _same(res, plain)
    assert sum(x[0].size for x in plain) > 1000


def test_submit_ready_wait():
    import fk_abi
    from fk_batch import BatchEngine
    ivs = _clipped(40, 81)
    be = BatchEngine(ivs)
    want = be.run_arrays(ivs, graph=False)
    be.submit(ivs)
    import time
    t0 = time.time()
    while not be._batch.ready():
        assert time.time() - t0 < 60
        time.sleep(0.001)
    assert _same(be.wait_arrays(), want)
    st = be.stats()
    assert st["launches"] >= 5 and st["total_ms"] > 0
    assert fk_abi.peak("imad") > 1e12


def test_tuning_changes_no_result():
    """Every fk_tuning knob only moves time: the batch stream is identical
    under each setting, and the plain engine agrees under another one."""
    from fk_batch import BatchEngine, PlainEngine
    ivs = _clipped(200, 81, clip=1 << 30)
    be = BatchEngine(ivs)
    ref = be.run_arrays(ivs, graph=False)
    assert sum(x[0].size for x in ref) > 50
    settings = [dict(mark_limit=8192), dict(mark_limit=2048, mark_bias=2.0),
                dict(seg_per_task=1, mark_bias=4.0),
                dict(warp_lane_words=32, mark_limit=4096),
                dict(warp_lane_words=1 << 30),
                dict(warp_queue=4, chains_per_sm=512),
                dict(warp_queue=512, mark_bias=0.25),
                dict(sieve_ctas_per_sm=1, mark_ctas_per_sm=1,
                     classify_ctas_per_sm=2),
                dict(group_lane_words=1 << 30),
                dict(group_lane_words=8, warp_lane_words=1 << 30),
                dict(round_cut=0.7), dict(round_cut=0.2, warp_queue=64),
                dict(round_cut=0.95, mark_bias=0.5),
                # kernel variants: pattern primes per CTA x marking segment
                dict(pattern_primes=24, mark_pattern_primes=24,
                     mark_segment=16384, mark_bias=4.0),
                dict(pattern_primes=40, mark_pattern_primes=40,
                     mark_segment=65536, mark_bias=4.0),
                dict(pattern_primes=24, mark_pattern_primes=40,
                     mark_segment=16384, mark_limit=4096, seg_per_task=3),
                dict(pattern_primes=40, mark_pattern_primes=24,
                     mark_segment=65536, mark_bias=0.25),
                dict(pattern_primes=32, mark_pattern_primes=32,
                     mark_segment=65536, seg_per_task=1, mark_bias=2.0),
                dict(warp_tasks=16, warp_lane_words=32),
                dict(warp_tasks=32, group_lane_words=8, chains_per_sm=8192),
                dict(sieve_ctas_per_sm=3, mark_ctas_per_sm=3,
                     classify_ctas_per_sm=8, mark_limit=65536,
                     seg_per_task=8, warp_queue=32, mark_bias=1.0,
                     chains_per_sm=2048, warp_lane_words=256,
                     round_cut=0.5, group_lane_words=32,
                     pattern_primes=32, mark_pattern_primes=32,
                     mark_segment=32768, warp_tasks=8)]
    for kw in settings:
        be.set_tuning(**kw)
        assert _same(be.run_arrays(ivs, graph=True), ref), kw
    pe = PlainEngine(be.engset)
    pe.set_tuning(mark_limit=16384, seg_per_task=3)
    assert _same(pe.run_arrays(ivs), ref)
    with pytest.raises(ValueError):
        be.set_tuning(mark_ctas_per_sm=9)
    with pytest.raises(ValueError):
        be.set_tuning(round_cut=0.99)
    with pytest.raises(ValueError):
        be.set_tuning(mark_segment=20000)
    with pytest.raises(ValueError):
        be.set_tuning(pattern_primes=33)
    with pytest.raises(ValueError):
        be.set_tuning(mark_pattern_primes=16)
    with pytest.raises(ValueError):
        be.set_tuning(warp_tasks=12)


def test_overflow_grows_the_buffers_and_reruns():
    """First buffers sized far below the survival estimate overflow; the
    pipeline grows them and reruns, and the rerun's stream is bit-identical
    to a run that never overflowed: in fk_batch_run (graph and eager), in
    fk_batch_submit / fk_batch_wait, and in the plain engine's fk_hunt."""
    import fk_abi
    from fk_batch import BatchEngine
    ivs = _clipped(200, 83)
    ref_be = BatchEngine(ivs)
    ref = ref_be.run_arrays(ivs)
    assert ref_be.stats()["reruns"] == 0
    assert ref_be.stats()["candidates"] > 20000   # past the 4096 floor
    for graph in (True, False):
        small = BatchEngine(engset=ref_be.engset)
        small.set_tuning(capacity_scale=1e-4)
        assert _same(small.run_arrays(ivs, graph=graph), ref)
        assert small.stats()["reruns"] >= 1
        assert _same(small.run_arrays(ivs, graph=graph), ref)
        assert small.stats()["reruns"] == 0       # grown buffers are kept
    sw = BatchEngine(engset=ref_be.engset)
    sw.set_tuning(capacity_scale=1e-4)
    sw.submit(ivs)
    assert _same(sw.wait_arrays(), ref)
    assert sw.stats()["reruns"] >= 1
    # the plain per-interval call on its own engine (Euler n = 2: about
    # 57,000 survivors in 2^24, far past the 4096-entry floor)
    lo, hi = 10 ** 12, 10 ** 12 + (1 << 24)
    eng = fk_abi.Engine(fk_abi.EULER, 2, p0=6)
    eng.set_tuning(capacity_scale=1e-4)
    off, dep = eng.hunt(lo, hi, 0, 100)
    assert eng.stats()["candidates"] > 8192 and eng.stats()["reruns"] >= 1
    ref_eng = fk_abi.Engine(fk_abi.EULER, 2, p0=6)
    roff, rdep = ref_eng.hunt(lo, hi, 0, 100)
    assert ref_eng.stats()["reruns"] == 0
    assert np.array_equal(off, roff) and np.array_equal(dep, rdep)


def test_wide_wheel_intervals_match_the_narrow_wheel():
    """Long intervals run on the 17# wheel; the streams equal those of the
    13# wheel on the same intervals, in a mix with short ones."""
    import fk_workloads as W
    from fk_batch import BatchEngine, EngineSet
    long_ivs = [W.Interval(k, n, lo, lo + (1 << 35), n, W.default_cap(k, n))
                for k, n, lo in ((W.EULER, 5, 10 ** 15),
                                 (W.DICKSON, 6, 10 ** 13),
                                 (W.AP, 7, 3 * 10 ** 16))]
    ivs = long_ivs + _clipped(40, 82)
    wide = BatchEngine(ivs)
    assert all(wide.engset.key_for(iv)[-1] == 7 for iv in long_ivs)
    narrow = BatchEngine(ivs, engset=EngineSet(wide=False))
    a = wide.run_arrays(ivs)
    assert _same(a, narrow.run_arrays(ivs))
    assert sum(x[0].size for x in a[:3]) > 100


def test_engines_added_to_a_batch_keep_its_results():
    """A batch that meets new engines is extended in place
    (fk_batch_add_engines): its later runs, graph and eager, over the old
    and the new engines equal those of a batch built with all of them."""
    from fk_batch import BatchEngine
    ivs = _clipped(60, 91)
    be = BatchEngine(ivs[:3])
    n0 = len(be.engset.engines())
    be.run_arrays(ivs[:3], graph=True)         # buffers and a graph
    b0 = be._batch
    got_g = be.run_arrays(ivs, graph=True)     # new engines: extended
    assert len(be.engset.engines()) > n0 and be._batch is b0
    got_e = be.run_arrays(ivs, graph=False)
    want = BatchEngine(ivs).run_arrays(ivs, graph=False)
    assert _same(got_g, want) and _same(got_e, want)
