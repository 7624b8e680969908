"""Generate the golden fixtures in tests/golden/ from the reference itself.

Run in a checkout that has jhg023/first-knowns available read-only (the
path is the first argument, default /root/reference).  It imports the
reference's own CPU engines and ``huntlib.primes`` -- the reference's
parity oracle for its GPU engines -- and freezes their outputs on the
windows below as JSON.  The reference does not travel to the GPU host;
these fixtures do.

    python tests/golden/make_golden.py [/path/to/first-knowns] [--extras-only]

Big integers are stored as decimal strings.  Sub-windows are swept in a
process pool (``spawn``), and the result is the concatenation in window
order, exactly as the reference's own G6 gate assembles its CPU side.
"""

import json
import multiprocessing as mp
import os
import pathlib
import random
import sys
import time

HERE = pathlib.Path(__file__).resolve().parent


def _setup(ref):
    for sub in ("", "euler-prime-runs", "dickson-ladders", "primorial-ap"):
        p = os.path.join(ref, sub)
        if p not in sys.path:
            sys.path.insert(0, p)
    sys.dont_write_bytecode = True


# ------------------------------------------------------------- workers ---

def _euler_surv(job):
    ref, n, wheel, lo, hi = job
    _setup(ref)
    import euler_search as es
    wp = {23: es.WHEEL_PRIMES, 29: es.WHEEL_PRIMES_29}[wheel]
    eng = es.CpuEngine(n, wheel_primes=wp)
    return [p for chunk in eng.survivors_pre_mr(lo, hi) for p in chunk]


def _euler_hunt(job):
    ref, n, wheel, lo, hi, cap = job
    _setup(ref)
    import euler_search as es
    wp = {23: es.WHEEL_PRIMES, 29: es.WHEEL_PRIMES_29}[wheel]
    return es.CpuEngine(n, wheel_primes=wp).hunt(lo, hi, cap=cap)


def _dickson_surv(job):
    ref, n, q2, j_lo, j_hi = job
    _setup(ref)
    import ladder_search as ls
    eng = ls.CpuEngine(n, q2=q2)
    out = []
    for chunk in eng.survivors_j(j_lo, j_hi):
        out.extend(int(v) for v in chunk.tolist())
    return out


def _dickson_hunt(job):
    ref, n, q2, k_lo, k_hi, cap = job
    _setup(ref)
    import ladder_search as ls
    return ls.CpuEngine(n, q2=q2).hunt(k_lo, k_hi, cap=cap)


def _ap_engine(ref, n, q2, d):
    _setup(ref)
    import ap_search as aps
    eng = aps.CpuEngine(n, q2)
    if d is not None:
        # fixed-difference adapter: the reference's own residue formula
        # (ap_search.py:99-106) with the difference overridden
        eng.d = d
        eng.forb = {q: sorted({(-j * eng.d) % q for j in range(eng.n)})
                    for q in eng.primes}
        eng.forbset = {q: frozenset(v) for q, v in eng.forb.items()}
    return eng


def _ap_surv(job):
    ref, n, q2, d, base, span = job
    eng = _ap_engine(ref, n, q2, d)
    out = []
    for chunk in eng.survivors(base, span):
        out.extend(int(v) for v in chunk.tolist())
    return out


def _ap_hunt(job):
    ref, n, q2, d, base, span, min_depth, cap = job
    eng = _ap_engine(ref, n, q2, d)
    out = []
    for chunk in eng.survivors(base, span):
        for o in chunk.tolist():
            p = base + int(o)
            dep = eng.chain_depth(p, cap)
            if dep >= min_depth:
                out.append((p, dep))
    return out


def _dickson_deep(job):
    """Survivors of a window past u64 j by the reference's one-candidate
    membership test (ladder_search.py:121-140 ``survives``, exact at any
    j), with the reference's run length of each (ladder_search.py:
    143-148) -- so every survivor's chain depth is frozen, hits or not."""
    ref, n, q2, j_lo, j_hi, cap = job
    _setup(ref)
    import numpy as np
    import ladder_search as ls
    eng = ls.CpuEngine(n, q2=q2)
    # candidates the reference's own residue table leaves for its primes
    # below 2000 (strided, the way survivors_j marks); survives() then
    # decides every one of them over all primes
    alive = np.ones(j_hi - j_lo, dtype=bool)
    for q in eng.primes:
        if q >= 2000:
            break
        for r in eng.table[q]:
            alive[int((int(r) - j_lo) % q)::q] = False
    out = []
    for t in np.nonzero(alive)[0].tolist():
        j = j_lo + int(t)
        if eng.survives(j):
            out.append((j, eng.run_length(j * eng.W, cap=cap)))
    return out


# (n, q2, j_lo, span): the deep zone past u64 j, where the reference's
# G17 gate checks its GPU stream against big-integer divisibility
# (dickson-ladders/ladder_gpu.py:1206-1280), out to the served workload's
# k ~ 1e24 (j = k / W up to about 5e21 at n = 6)
DEEP_CASES = [(6, 65536, 2 ** 64 + 12345, 2 ** 20),
              (6, 65536, 10 ** 21, 2 ** 20),
              (6, 65536, 5 * 10 ** 21 - 2 ** 20, 2 ** 20),
              (10, 65536, 2 ** 64, 2 ** 26),
              (10, 4096, 5 * 10 ** 19, 2 ** 22),
              (14, 4096, 2 ** 64 + 1, 2 ** 22),
              (14, 2048, 3 * 10 ** 19, 2 ** 25),
              (13, 2048, 17 * 4 * 10 ** 18 - 2 ** 22, 2 ** 22)]


def dickson_deep(ref, pool):
    out = {"cases": [], "source": "dickson-ladders/ladder_search.py:121-148 "
                                  "survives and run_length of the reference"}
    for n, q2, j_lo, span in DEEP_CASES:
        parts = _split(j_lo, j_lo + span, 64)
        cap = n + 8
        res = pool.map(_dickson_deep, [(ref, n, q2, a, b, cap)
                                       for a, b in parts])
        rows = [r for rr in res for r in rr]
        out["cases"].append({"n": n, "q2": q2, "j_lo": _s(j_lo),
                             "j_hi": _s(j_lo + span), "cap": cap,
                             "survivors": [_s(j) for j, _ in rows],
                             "runs": [r for _, r in rows]})
        print(f"dickson deep n={n} j={j_lo:.3g}: {len(rows)} survivors, "
              f"max run {max((r for _, r in rows), default=0)}", flush=True)
    (HERE / "dickson_deep.json").write_text(json.dumps(out))


def cursor_units(ref):
    """The values the launchers' checkpoint cursors are denominated in,
    computed by the reference's own functions: the Euler wheel its engines
    pick by default (euler_search.py:200-212 best_wheel; cursor key
    euler-prime-runs/launch.py:191-200) and its period M, the Dickson wheel
    modulus W (ladder_reference.py:60-66; next_j counts multiples of it,
    dickson-ladders/launch.py:491-497, 604-610), and the AP engine floor
    (ap_search.py:106; next_u starts at ceil(floor / 30),
    primorial-ap/launch.py:262-273)."""
    _setup(ref)
    import ap_search as aps
    import euler_search as es
    import ladder_reference as lr
    out = {"euler": {}, "dickson": {}, "ap_floor": {}}
    for n in range(1, 21):
        wp = list(es.best_wheel(n))
        m = 1
        for q in wp:
            m *= q
        out["euler"][str(n)] = {"wheel_primes": wp, "M": _s(m)}
        out["dickson"][str(n)] = {"W": _s(lr.wheel_modulus(n))}
    for q2 in (2048, 4096, 65536, 1 << 18):
        out["ap_floor"][str(q2)] = _s(aps.CpuEngine(8, q2).floor)
    out["source"] = ("euler_search.best_wheel, ladder_reference."
                     "wheel_modulus, ap_search.CpuEngine.floor")
    (HERE / "cursor.json").write_text(json.dumps(out, indent=1))
    print("cursor units written", flush=True)


def _split(lo, hi, parts, align=1):
    step = max(align, (hi - lo) // parts // align * align)
    cuts = list(range(lo, hi, step)) + [hi]
    cuts = sorted(set(cuts))
    return list(zip(cuts, cuts[1:]))


def _s(v):
    return str(int(v))


def main(ref):
    _setup(ref)
    from huntlib import primes as hp
    import euler_reference as er
    import ladder_reference as lr
    import ap_reference as ar
    import euler_search as es
    import ladder_search as ls

    ctx = mp.get_context("spawn")
    pool = ctx.Pool(os.cpu_count() or 4)
    t0 = time.time()

    # ------------------------------------------------------------ MR ---
    rng = random.Random(20261203)
    vals = list(range(0, 3001))
    # base-2 strong pseudoprimes below 2e6, found by the reference's own
    # functions (composite yet passing sprp_base2)
    for m in range(3001, 2_000_000, 2):
        if hp.sprp_base2(m) and not hp.mr_is_prime(m):
            vals.append(m)
    for a in hp.MR_BASES:
        for dv in range(-40, 41):
            if a + dv >= 0:
                vals.append(a + dv)
        vals.extend([a * 3, a * 7 + 1, 2 * a + 1])
    for bits in (20, 31, 32, 33, 40, 50, 62, 63, 64, 65, 70, 80, 96, 100,
                 127, 128, 129, 150, 170, 180, 190, 191, 192):
        for _ in range(40):
            vals.append(rng.getrandbits(bits) | (1 << (bits - 1)) | 1)
    from sympy import nextprime, prevprime
    for bits in (31, 32, 62, 63, 64, 65, 80, 96, 127, 128, 129, 160, 191):
        for _ in range(6):
            p = int(nextprime(rng.getrandbits(bits) | (1 << (bits - 1))))
            q = int(nextprime(rng.getrandbits(bits // 2 + 1) | 1))
            vals.extend([p, p * q, p * p, p + 2])
    for e in (32, 64, 96, 128, 160, 192):
        vals.append(int(prevprime(1 << e)))
        vals.append((1 << e) - 1)
        vals.append((1 << e) + 1)
    # Carmichael numbers (6k+1)(12k+1)(18k+1) with all three factors prime
    for k in range(1, 4000):
        a, b, c = 6 * k + 1, 12 * k + 1, 18 * k + 1
        if hp.mr_is_prime(a) and hp.mr_is_prime(b) and hp.mr_is_prime(c):
            vals.append(a * b * c)
    # chain values the engines classify: Euler, Dickson and AP knowns
    for p in (er.KNOWN[15], er.A21_UPPER, 3744101869688673856367):
        vals.extend(p + x * x + x for x in range(25))
    for k in (lr.KNOWN[9], 12094123415384869458600):
        vals.extend(m * k * k + 1 for m in range(1, 16))
    d16 = ar.difference(16)
    vals.extend(14042451608819603 + j * ar.difference(18) for j in range(19))
    vals.extend(ar.KNOWN[15] + j * ar.difference(15) for j in range(16))
    vals.extend(116781362669989 + j * d16 for j in range(17))
    vals = sorted(set(vals))
    mr = {"values": [_s(v) for v in vals],
          "mr_is_prime": [bool(hp.mr_is_prime(v)) for v in vals],
          "sprp_base2": [bool(hp.sprp_base2(v)) for v in vals],
          "source": "huntlib/primes.py:23-80 of the reference"}
    (HERE / "mr.json").write_text(json.dumps(mr))
    print(f"mr: {len(vals)} values ({time.time()-t0:.0f}s)", flush=True)

    # --------------------------------------------------------- Euler ---
    # (n, wheel top, lo, hi): the reference's G6 windows that the CPU
    # engine finishes in seconds (euler_gpu.py:1493-1499) plus the
    # whole-line plain case [1e5, 1e9) at n = 8.
    ecases = [(5, 29, 10**5, 4 * 10**5), (9, 29, 10**6, 6 * 10**7),
              (13, 29, 10**5, 8_900_000_000),
              (8, 29, 10**5, 10**9),
              (17, 29, 10**15, 10**15 + 3 * 10**12),
              (17, 29, er.A21_UPPER - 10**10, er.A21_UPPER + 10**10),
              (17, 29, es.P_CEIL - 10**13, es.P_CEIL),
              (12, 23, 10**14, 10**14 + 10**11)]
    euler = {"surv": [], "hunt": []}
    for n, wt, lo, hi in ecases:
        M = 6469693230
        parts = _split(lo, hi, 64 if hi - lo > 64 * M else 8)
        res = pool.map(_euler_surv, [(ref, n, wt, a, b) for a, b in parts])
        s = [p for r in res for p in r]
        euler["surv"].append({"n": n, "wheel_top": wt, "lo": _s(lo),
                              "hi": _s(hi), "survivors": [_s(p) for p in s]})
        print(f"euler surv n={n} [{lo:.3g},{hi:.3g}): {len(s)} "
              f"({time.time()-t0:.0f}s)", flush=True)
    hcases = [(8, 29, 10**5, 10**9, 64), (10, 23, 10**5, 2 * 10**8, 100),
              (11, 29, 10**5, 200_000_000, 100), (5, 29, 10**5, 4 * 10**5, 3),
              (14, 29, er.KNOWN[14] - 10**10, er.KNOWN[14] + 10**9, 100),
              (17, 29, er.A21_UPPER - 10**10, er.A21_UPPER + 10**10, 100)]
    for n, wt, lo, hi, cap in hcases:
        parts = _split(lo, hi, 32)
        res = pool.map(_euler_hunt, [(ref, n, wt, a, b, cap)
                                     for a, b in parts])
        h = [(p, r) for rr in res for p, r in rr]
        euler["hunt"].append({"n": n, "wheel_top": wt, "lo": _s(lo),
                              "hi": _s(hi), "cap": cap,
                              "hits": [[_s(p), r] for p, r in h]})
        print(f"euler hunt n={n}: {len(h)} hits ({time.time()-t0:.0f}s)",
              flush=True)
    # low pass below the engine floor (launch.py:410-420), cap 64
    low = [(p, er.run_length(p, cap=64)) for p in range(2, es.P_FLOOR)]
    euler["low_pass_cap64"] = [[p, r] for p, r in low if r >= 4]
    (HERE / "euler.json").write_text(json.dumps(euler))

    # ------------------------------------------------------- Dickson ---
    # (n, q2, j_lo, j_hi): the reference's G6 windows
    # (ladder_gpu.py:955-959) plus config-shaped windows at n = 6.
    dcases = [(10, 65536, 10**6, 10**6 + 4 * 10**7),
              (10, 65536, 4 * 10**9, 4 * 10**9 + 4 * 10**7),
              (10, 65536, 10**12, 10**12 + 4 * 10**7),
              (12, 2048, 6 * 10**11, 6 * 10**11 + 2 * 10**6),
              (13, 2048, ls.J_CEIL - 4 * 10**6, ls.J_CEIL),
              (6, 1 << 20, 48, 48 + 2 ** 22),
              (6, 1 << 20, 7 * 10**7, 7 * 10**7 + 2 ** 22),
              (4, 4096, 10**15, 10**15 + 10**6)]
    dick = {"surv": [], "hunt": []}
    for n, q2, a, b in dcases:
        parts = _split(a, b, 16)
        res = pool.map(_dickson_surv, [(ref, n, q2, x, y) for x, y in parts])
        s = [v for r in res for v in r]
        dick["surv"].append({"n": n, "q2": q2, "j_lo": _s(a), "j_hi": _s(b),
                             "survivors": [_s(v) for v in s]})
        print(f"dickson surv n={n} q2={q2}: {len(s)} "
              f"({time.time()-t0:.0f}s)", flush=True)
    # hunt: k ranges inclusive, as ladder_search.hunt takes them
    dh = [(6, 1 << 20, lr.K_FLOOR, 2 ** 34 - 1, 8),
          (7, 65536, lr.K_FLOOR, lr.KNOWN[7], None),
          (8, 65536, lr.KNOWN[8] - 10**9, lr.KNOWN[8] + 10**9, None),
          (4, 4096, 10**12, 10**12 + 10**9, 12)]
    for n, q2, k_lo, k_hi, cap in dh:
        W = lr.wheel_modulus(n)
        j_lo, j_hi = -(-k_lo // W), k_hi // W + 1
        cuts = _split(j_lo, j_hi, 64)
        jobs = [(ref, n, q2, max(k_lo, x * W), min(k_hi, y * W - 1), cap)
                for x, y in cuts]
        res = pool.map(_dickson_hunt, jobs)
        h = sorted({(k, r) for rr in res for k, r in rr})
        dick["hunt"].append({"n": n, "q2": q2, "k_lo": _s(k_lo),
                             "k_hi": _s(k_hi), "cap": cap,
                             "hits": [[_s(k), r] for k, r in h]})
        print(f"dickson hunt n={n}: {len(h)} hits ({time.time()-t0:.0f}s)",
              flush=True)
    low = []
    for k in range(1, lr.K_FLOOR):
        r = lr.run_length(k, cap=12)
        if r >= 1:
            low.append([k, r])
    dick["low_pass_cap12"] = low
    (HERE / "dickson.json").write_text(json.dumps(dick))

    # ------------------------------------------------------------ AP ---
    def down(p):
        return int(p) - int(p) % 30
    acases = [(13, 2048, None, down(10**6), down(2 * 10**7)),
              (16, 2048, None, down(10**9), down(5 * 10**7)),
              (8, 4096, None, down(4 * 10**13), down(3 * 10**6)),
              (5, 2048, None, down(10**26 - 3 * 10**6), down(10**6)),
              (5, 1 << 18, None, down(4 * 10**13), down(2 * 10**6)),
              (16, 65536, None, down(4 * 10**13), 30 * 2 ** 22),
              (10, 65536, 30030, 10**12, 30 * 2 ** 24),
              (10, 65536, 30030, 10**12 + 2 ** 39, 30 * 2 ** 24)]
    ap = {"surv": [], "hunt": []}
    for n, q2, d, base, span in acases:
        parts = _split(base, base + span, 16, align=30)
        res = pool.map(_ap_surv, [(ref, n, q2, d, x, y - x)
                                  for x, y in parts])
        s = []
        for (x, _y), r in zip(parts, res):
            s.extend(x - base + v for v in r)
        ap["surv"].append({"n": n, "q2": q2, "d": d and _s(d),
                           "base": _s(base), "span": _s(span),
                           "offsets": [_s(v) for v in s]})
        print(f"ap surv n={n} q2={q2} d={d}: {len(s)} "
              f"({time.time()-t0:.0f}s)", flush=True)
    ah = [(13, 4096, None, 65550, down(ar.KNOWN[13] + 30) - 65550, 13, 13),
          (8, 4096, None, down(4 * 10**13), 30 * 2 ** 22, 4, 8),
          (10, 65536, 30030, 10**12, 30 * 2 ** 26, 10, 16),
          (10, 65536, 30030, 10**12, 30 * 2 ** 23, 6, 16)]
    for n, q2, d, base, span, md, cap in ah:
        parts = _split(base, base + span, 64, align=30)
        res = pool.map(_ap_hunt, [(ref, n, q2, d, x, y - x, md, cap)
                                  for x, y in parts])
        h = [(p, dd) for rr in res for p, dd in rr]
        ap["hunt"].append({"n": n, "q2": q2, "d": d and _s(d),
                           "base": _s(base), "span": _s(span),
                           "min_depth": md, "cap": cap,
                           "hits": [[_s(p), dd] for p, dd in h]})
        print(f"ap hunt n={n} d={d}: {len(h)} hits ({time.time()-t0:.0f}s)",
              flush=True)
    (HERE / "ap.json").write_text(json.dumps(ap))

    # ------------------------------------------------------- knowns ---
    known = {
        "euler_known": {str(k): _s(v) for k, v in er.KNOWN.items()},
        "euler_a21_upper": _s(er.A21_UPPER),
        "dickson_known": {str(k): _s(v) for k, v in lr.KNOWN.items()},
        "ap_known": {str(k): _s(v) for k, v in ar.KNOWN.items()},
        # score fingerprints frozen in the reference's score.py files
        "fingerprints": {
            "euler_score": {"n": 17, "lo": _s(10**16),
                            "hi": _s(10**16 + 5 * 10**14), "count": 178,
                            "xor": _s(120489734542316),
                            "source": "euler-prime-runs/score.py:57-60"},
            "euler_score128": {"n": 17, "lo": _s(230 * 10**18),
                               "hi": _s(230 * 10**18 + 5 * 10**14),
                               "count": 178, "xor": _s(133625321009290),
                               "source": "euler-prime-runs/score.py:65-68"},
            "euler_score_wide": {"n": 17, "lo": _s(611 * 10**18),
                                 "hi": _s(611 * 10**18 + 2 * 10**16),
                                 "count": 6996, "xor": _s(71330844491704598),
                                 "source": "euler-prime-runs/score.py:74-77"},
            "dickson_score": {"n": 10, "q2": 65536, "j_lo": _s(10**12),
                              "span": _s(2**32), "count": 1213,
                              "xor": _s(1003170806905),
                              "source": "dickson-ladders/score.py:56"},
            "dickson_score12": {"n": 12, "q2": 65536, "j_lo": _s(6 * 10**11),
                                "span": _s(2**32), "count": 292,
                                "xor": _s(2752794123),
                                "source": "dickson-ladders/score.py:57"},
            "dickson_score13": {"n": 13, "q2": 65536, "j_lo": _s(7 * 10**16),
                                "span": _s(2**38), "count": 2739,
                                "xor": _s(70000110051605722),
                                "source": "dickson-ladders/score.py:58"},
            "ap_score": {"n": 16, "q2": 65536,
                         "base": _s((4 * 10**13 // 30) * 30),
                         "span": _s(30 * 2**25 * 16), "count": 192,
                         "xor": _s(4046714554),
                         "source": "primorial-ap/score.py:42-50"},
        },
    }
    (HERE / "known.json").write_text(json.dumps(known, indent=1))
    dickson_deep(ref, pool)
    cursor_units(ref)
    pool.close()
    print(f"done in {time.time()-t0:.0f}s")


if __name__ == "__main__":
    args = [a for a in sys.argv[1:] if not a.startswith("--")]
    ref_root = args[0] if args else "/root/reference"
    if "--extras-only" in sys.argv:
        # the deep-zone Dickson and cursor-unit fixtures alone
        # (dickson_deep.json, cursor.json)
        _setup(ref_root)
        with mp.get_context("spawn").Pool(os.cpu_count() or 4) as pl:
            dickson_deep(ref_root, pl)
        cursor_units(ref_root)
    else:
        main(ref_root)
