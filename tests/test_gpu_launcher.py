"""The reference's launcher segment loops, restated over the mirrors.

The launchers sweep the line one checkpoint segment at a time
(euler-prime-runs/launch.py:649-700, dickson-ladders/launch.py:1077-1098,
primorial-ap/launch.py:586-640): the cursor names the next segment in the
engine's own units (Euler: periods of the wheel M; Dickson: j, k = W*j;
AP: periods of 30 from the engine floor), the engine sweeps the segment,
and the cursor advances only once the segment is fully classified
(CONVENTIONS.md:278-295: a checkpoint holds the last segment boundary, so
an interrupted run redoes exactly the segment in flight).  Each loop below
is that loop with the device's fused depth stream (``hunt``) in place of
the host classification pool, and the tests check

  * split == whole: the concatenated segment streams equal one sweep of
    the whole range and the reference's golden hunt on it;
  * ordering: each segment's stream is ascending and inside its segment,
    so the concatenation is strictly ascending across boundaries;
  * interrupt and resume at a segment boundary (the cursor written with
    an atomic replace, read back under the key check of
    huntlib/checkpoint.py:114-165) give the straight run, no double count;
  * the cursor units and keys are the reference's own
    (tests/golden/cursor.json, from euler_search.best_wheel,
    ladder_reference.wheel_modulus and ap_search's engine floor);
  * the AP verification leg's one-candidate ``survives`` agrees with the
    reference's survivor stream (primorial-ap/launch.py:372-410).  The
    Dickson leg uses the host CpuEngine.survives
    (dickson-ladders/launch.py:404-462), so it needs no device path.
"""

import json
import os
import random

import pytest

from golden_util import ints, load

pytestmark = pytest.mark.gpu

EULER_KEY = ("euler-prime-runs/v4/n={n}/wheel={wheel}#"
             "/Q1=1024/Q2=65536/ceil=1e24")       # euler launch.py:107-108
DICKSON_KEY = "dickson-ladders/v2/q2={q2}/jceil=4e18"   # launch.py:91
AP_KEY = "primorial-ap/v1/q2={q2}/pceil=1e26"            # launch.py:95


class CursorRefused(RuntimeError):
    pass


def save_cursor(path, state):
    """Atomic write: the file is either the old cursor or the new one."""
    tmp = str(path) + ".tmp"
    with open(tmp, "w") as f:
        json.dump(state, f)
        f.flush()
        os.fsync(f.fileno())
    os.replace(tmp, path)


def load_cursor(path, expect_key):
    """huntlib/checkpoint.py:114-165 restated: a cursor whose key this
    configuration cannot read is a refusal, never a silent fresh start."""
    with open(path) as f:
        state = json.load(f)
    if state.get("key") != expect_key:
        raise CursorRefused(f"stored key {state.get('key')!r}, wanted "
                            f"{expect_key!r}")
    return state


def _check_segment(hits, lo, hi):
    xs = [x for x, _ in hits]
    assert xs == sorted(xs) and len(set(xs)) == len(xs)
    assert all(lo <= x < hi for x in xs)


# ---------------------------------------------------------------- Euler --

def euler_loop(eng, c, p_cap, seg, stop_after=None, cap=64):
    """euler-prime-runs/launch.py:649-700 with the fused depth stream."""
    import euler_gpu
    M = eng.M
    k_cap = -(-p_cap // M)
    out, done = [], 0
    while c["next_k"] < k_cap:
        k0 = c["next_k"]
        k1 = min(k0 + seg, k_cap)
        lo = max(euler_gpu.P_FLOOR, k0 * M)
        hi = min(p_cap, k1 * M)
        if lo >= hi:
            c["next_k"] = k1
            continue
        hits = eng.hunt(lo, hi, cap=cap)
        _check_segment(hits, lo, hi)
        out.extend(hits)
        c["next_k"] = k1                       # the segment boundary
        c["hits"] += len(hits)
        done += 1
        if stop_after is not None and done == stop_after:
            break
    return out


def test_euler_segment_loop(tmp_path):
    import euler_gpu
    g = next(h for h in load("euler")["hunt"]
             if h["n"] == 8 and int(h["hi"]) == 10 ** 9)
    want = [(int(p), r) for p, r in g["hits"]]
    # the 23# wheel: [1e5, 1e9) is five periods, so segments cut it
    eng = euler_gpu.GpuEngine(8, wheel_primes=euler_gpu.WHEEL_PRIMES)
    key = EULER_KEY.format(n=8, wheel=eng.wheel_primes[-1])
    whole = eng.hunt(10 ** 5, 10 ** 9, cap=64)
    assert whole == want and len(want) > 5
    # launches of one wheel period: the same stream as one sweep
    assert eng.survivors_pre_mr(10 ** 5, 10 ** 9, periods_per_launch=1) == \
        eng.survivors_pre_mr(10 ** 5, 10 ** 9)
    for seg in (1, 2, 7):
        c = {"key": key, "M": eng.M, "next_k": 0, "hits": 0}
        assert euler_loop(eng, c, 10 ** 9, seg) == want
        assert c["hits"] == len(want)
    # interrupt after two segments, resume from the saved boundary
    path = tmp_path / "euler.json"
    c = {"key": key, "M": eng.M, "next_k": 0, "hits": 0}
    first = euler_loop(eng, c, 10 ** 9, 1, stop_after=2)
    save_cursor(path, c)
    eng2 = euler_gpu.GpuEngine(8, wheel_primes=euler_gpu.WHEEL_PRIMES)
    c2 = load_cursor(path, EULER_KEY.format(n=8, wheel=eng2.wheel_primes[-1]))
    assert c2["M"] == eng2.M
    rest = euler_loop(eng2, c2, 10 ** 9, 1)
    assert first + rest == want and c2["hits"] == len(want)
    # a cursor written for another wheel is refused, not reinterpreted
    other = euler_gpu.GpuEngine(8)
    with pytest.raises(CursorRefused):
        load_cursor(path, EULER_KEY.format(n=8, wheel=other.wheel_primes[-1]))


def test_euler_cursor_units_are_the_reference_wheel():
    import euler_gpu
    ref = load("cursor")["euler"]
    for n in (1, 4, 8, 9, 12, 17, 20):
        eng = euler_gpu.GpuEngine(n)
        assert eng.wheel_primes == ref[str(n)]["wheel_primes"]
        assert eng.M == int(ref[str(n)]["M"])


def test_euler_loop_on_a_long_range_splits_like_the_whole():
    """Seven segments of 11 periods over 77 periods of 23#, at 1e13."""
    import euler_gpu
    eng = euler_gpu.GpuEngine(6, wheel_primes=euler_gpu.WHEEL_PRIMES)
    k0 = 10 ** 13 // eng.M
    p_cap = (k0 + 77) * eng.M
    whole = eng.hunt(k0 * eng.M, p_cap, cap=100)
    c = {"next_k": k0, "hits": 0}
    assert euler_loop(eng, c, p_cap, 11, cap=100) == whole
    assert len(whole) > 10


# -------------------------------------------------------------- Dickson --

def dickson_loop(eng, c, j_cap, seg, stop_after=None, cap=None):
    """dickson-ladders/launch.py:1077-1098 with the fused depth stream:
    the segment [j0, j1) is k in [j0*W, j1*W - 1] (hunt takes k, both ends
    inclusive, dickson-ladders/ladder_gpu.py:819-829)."""
    W = eng.W
    out, done = [], 0
    while c["next_j"] < j_cap:
        j0, j1 = c["next_j"], min(c["next_j"] + seg, j_cap)
        hits = eng.hunt(j0 * W, j1 * W - 1, cap=cap)
        _check_segment(hits, j0 * W, j1 * W)
        out.extend(hits)
        c["next_j"] = j1
        c["hits"] += len(hits)
        done += 1
        if stop_after is not None and done == stop_after:
            break
    return out


def test_dickson_segment_loop(tmp_path):
    import ladder_gpu
    g = next(h for h in load("dickson")["hunt"] if h["n"] == 6)
    want = [(int(k), r) for k, r in g["hits"]]
    eng = ladder_gpu.GpuEngine(6, q2=g["q2"])
    W = eng.W
    assert W == int(load("cursor")["dickson"]["6"]["W"])
    k_hi = int(g["k_hi"])                          # inclusive
    j_cap = k_hi // W + 1
    fresh = {"key": DICKSON_KEY.format(q2=eng.q2), "n": 6, "W": W,
             "next_j": max(1, -(-ladder_gpu.K_FLOOR // W)), "hits": 0}
    for seg in (1 << 23, 10 ** 7 + 3):
        c = dict(fresh)
        assert dickson_loop(eng, c, j_cap, seg, cap=g["cap"]) == want
    path = tmp_path / "dickson.json"
    c = dict(fresh)
    first = dickson_loop(eng, c, j_cap, 1 << 23, stop_after=3, cap=g["cap"])
    save_cursor(path, c)
    c2 = load_cursor(path, DICKSON_KEY.format(q2=eng.q2))
    # check_cursor (dickson-ladders/launch.py:604-610): next_j counts
    # multiples of this very wheel
    assert c2["W"] == eng.W == ladder_gpu.wheel_modulus(c2["n"])
    rest = dickson_loop(eng, c2, j_cap, 1 << 23, cap=g["cap"])
    assert first + rest == want and c2["hits"] == len(want)
    with pytest.raises(CursorRefused):
        load_cursor(path, DICKSON_KEY.format(q2=65536))


# ------------------------------------------------------------------- AP --

def ap_loop(eng, c, p_end, seg, stop_after=None, min_depth=None):
    """primorial-ap/launch.py:586-640 with the fused depth stream: the
    segment is `seg` (a multiple of 30) from base = next_u * 30."""
    out, done = [], 0
    while c["next_u"] * 30 < p_end:
        base = c["next_u"] * 30
        span = min(seg, p_end - base)
        span -= span % 30
        hits = eng.hunt(base, span, min_depth=min_depth)
        _check_segment(hits, base, base + span)
        # the same segment's pre-primality stream, one array per launch
        chunks = list(eng.survivors(base, span))
        step = 30 * eng.launch_u
        for i, ch in enumerate(chunks):
            assert ch.size and list(ch) == sorted(ch)
        flat = [int(o) for ch in chunks for o in ch.tolist()]
        assert flat == sorted(set(flat)) and all(0 <= o < span for o in flat)
        # a launch never spills into the next launch's window
        for ch in chunks:
            assert int(ch[0]) // step == int(ch[-1]) // step
        out.extend(hits)
        c["next_u"] += span // 30
        c["hits"] += len(hits)
        done += 1
        if stop_after is not None and done == stop_after:
            break
    return out


def test_ap_segment_loop(tmp_path):
    import ap_gpu
    g = next(h for h in load("ap")["hunt"] if h["n"] == 8)
    want = [(int(p), d) for p, d in g["hits"]]
    base, span = int(g["base"]), int(g["span"])
    eng = ap_gpu.GpuEngine(8, q2=g["q2"], launch_u=1 << 17)
    assert eng.floor == int(load("cursor")["ap_floor"][str(g["q2"])])
    key = AP_KEY.format(q2=eng.q2)
    for seg in (30 * (1 << 19), 30 * 1234567):
        c = {"key": key, "n": 8, "next_u": base // 30, "hits": 0}
        assert ap_loop(eng, c, base + span, seg, min_depth=4) == want
    path = tmp_path / "ap.json"
    c = {"key": key, "n": 8, "next_u": base // 30, "hits": 0}
    first = ap_loop(eng, c, base + span, 30 * (1 << 19), stop_after=3,
                    min_depth=4)
    save_cursor(path, c)
    c2 = load_cursor(path, key)
    rest = ap_loop(eng, c2, base + span, 30 * (1 << 19), min_depth=4)
    assert first + rest == want and c2["hits"] == len(want)
    # a fresh cursor starts at the engine floor, in periods of 30
    assert -(-eng.floor // 30) * 30 >= eng.floor


def test_ap_survives_matches_the_reference_stream():
    """The verification leg's one-candidate test (primorial-ap/launch.py:
    372-410 re-sieves a reported p alone) against the reference's own
    survivor stream on the same window: sampled survivors and non-
    survivors, coprime to 30 or not."""
    import ap_gpu
    g = next(s for s in load("ap")["surv"]
             if s["n"] == 8 and s["q2"] == 4096)
    base, span = int(g["base"]), int(g["span"])
    surv = set(ints(g["offsets"]))
    eng = ap_gpu.GpuEngine(8, q2=4096)
    rng = random.Random(5)
    alive = rng.sample(sorted(surv), 60)
    dead = [o for o in rng.sample(range(span), 400) if o not in surv][:120]
    for o in alive:
        assert eng.survives(base + o)
    for o in dead:
        assert not eng.survives(base + o)
