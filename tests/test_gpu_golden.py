"""GPU parity against the golden fixtures produced by the reference itself.

Every assertion is bit-exact: the survivor streams, the depths and the
SPRP verdicts are integer results and must equal the reference CPU
engines' output on the same windows (tests/golden/make_golden.py), and the
fingerprinted score windows must reproduce the reference's frozen count
and xor checksum.
"""

import os

import numpy as np
import pytest

from golden_util import ints, load, xor_all

pytestmark = pytest.mark.gpu


@pytest.fixture(autouse=True, params=["auto", "rounds", "mark"])
def sieve_kernel(request, monkeypatch):
    """Every golden case through each sieve kernel: the cost-model choice,
    the per-candidate compaction rounds only, and the marking sieve for
    every item."""
    import ap_gpu
    import euler_gpu
    import ladder_gpu
    monkeypatch.setenv("FK_SIEVE", request.param)
    for m in (euler_gpu, ladder_gpu, ap_gpu):
        m._device_engine.cache_clear()
    yield request.param
    for m in (euler_gpu, ladder_gpu, ap_gpu):
        m._device_engine.cache_clear()


# ---------------------------------------------------------------- SPRP ---

def test_sprp_rejects_values_past_192_bits():
    import fk_abi
    with pytest.raises(ValueError):
        fk_abi.sprp([1 << 192])


def test_sprp_matches_reference_verdicts():
    import fk_abi
    g = load("mr")
    keep = [i for i, v in enumerate(ints(g["values"])) if v < 1 << 192]
    assert len(keep) > 4800
    vals = [int(g["values"][i]) for i in keep]
    mr = [g["mr_is_prime"][i] for i in keep]
    b2 = [g["sprp_base2"][i] for i in keep]
    got = fk_abi.sprp(vals).tolist()
    bad = [v for v, a, b in zip(vals, got, mr) if a != b]
    assert not bad, f"mr_is_prime mismatch at {bad[:5]}"
    got2 = fk_abi.sprp(vals, base2_only=True).tolist()
    bad = [v for v, a, b in zip(vals, got2, b2) if a != b]
    assert not bad, f"sprp_base2 mismatch at {bad[:5]}"


# --------------------------------------------------------------- Euler ---

@pytest.mark.parametrize("case", range(len(load("euler")["surv"])))
def test_euler_survivors(case):
    from euler_gpu import GpuEngine
    c = load("euler")["surv"][case]
    lo, hi = int(c["lo"]), int(c["hi"])
    got = GpuEngine(c["n"]).survivors_pre_mr(lo, hi)
    assert got == ints(c["survivors"])


@pytest.mark.parametrize("case", range(len(load("euler")["hunt"])))
def test_euler_hunt(case):
    from euler_gpu import GpuEngine
    c = load("euler")["hunt"][case]
    got = GpuEngine(c["n"]).hunt(int(c["lo"]), int(c["hi"]), cap=c["cap"])
    assert got == [(int(p), r) for p, r in c["hits"]]


def test_euler_low_pass():
    import euler_gpu
    want = [(p, r) for p, r in load("euler")["low_pass_cap64"]]
    got = euler_gpu.low_pass(4, cap=64)
    assert got == want


def test_euler_plain_config_whole_line():
    """p < 1e9, run >= 8, cap 64: the low pass plus the engine, and the
    least p for each run length (KNOWN a(8), a(9), a(10), a(11))."""
    import euler_gpu
    e = load("euler")
    want = [(p, r) for p, r in e["low_pass_cap64"] if r >= 8]
    want += [(int(p), r) for p, r in
             next(h for h in e["hunt"] if h["n"] == 8 and h["cap"] == 64)
             ["hits"]]
    got = euler_gpu.sweep(2, 10 ** 9, 8, cap=64)
    assert got == want
    least = {}
    for p, r in got:
        least.setdefault(r, p)
    known = {int(k): int(v) for k, v in load("known")["euler_known"].items()}
    for n in (8, 9, 10, 11):
        assert least[n] == known[n]


@pytest.mark.parametrize("name", ["euler_score", "euler_score128"])
def test_euler_score_fingerprint(name):
    from euler_gpu import GpuEngine
    f = load("known")["fingerprints"][name]
    got = GpuEngine(f["n"]).survivors_pre_mr(int(f["lo"]), int(f["hi"]))
    assert len(got) == f["count"]
    assert xor_all(got) == int(f["xor"])


@pytest.mark.slow
def test_euler_score_wide_fingerprint():
    from euler_gpu import GpuEngine
    f = load("known")["fingerprints"]["euler_score_wide"]
    got = GpuEngine(f["n"]).survivors_pre_mr(int(f["lo"]), int(f["hi"]))
    assert len(got) == f["count"]
    assert xor_all(got) == int(f["xor"])


# ------------------------------------------------------------- Dickson ---

@pytest.mark.parametrize("case", range(len(load("dickson")["surv"])))
def test_dickson_survivors(case):
    from ladder_gpu import GpuEngine
    c = load("dickson")["surv"][case]
    got = GpuEngine(c["n"], q2=c["q2"]).survivors_j(int(c["j_lo"]),
                                                    int(c["j_hi"]))
    assert got.dtype == np.uint64
    assert got.tolist() == ints(c["survivors"])


@pytest.mark.parametrize("case", range(len(load("dickson")["hunt"])))
def test_dickson_hunt(case):
    from ladder_gpu import GpuEngine
    c = load("dickson")["hunt"][case]
    got = GpuEngine(c["n"], q2=c["q2"]).hunt(int(c["k_lo"]), int(c["k_hi"]),
                                             cap=c["cap"])
    assert got == [(int(k), r) for k, r in c["hits"]]


def test_dickson_low_pass():
    import ladder_gpu
    want = [(k, r) for k, r in load("dickson")["low_pass_cap12"]]
    got = ladder_gpu.low_pass(1, 12)
    assert got == want


def test_dickson_plain_config_whole_line():
    """k in [1, 2^34), m = 1..8, depth >= 6, sieve to 2^20."""
    import ladder_gpu
    d = load("dickson")
    low = [(k, min(r, 8)) for k, r in d["low_pass_cap12"] if min(r, 8) >= 6]
    main = next(h for h in d["hunt"] if h["n"] == 6 and h["q2"] == 1 << 20)
    want = low + [(int(k), r) for k, r in main["hits"]]
    got = ladder_gpu.sweep(1, 2 ** 34, 6, cap=8, q2=1 << 20)
    assert got == want
    known = {int(k): int(v) for k, v in load("known")["dickson_known"].items()}
    first6 = min(k for k, r in got if r >= 6)
    assert first6 == known[6]


@pytest.mark.parametrize("name", ["dickson_score", "dickson_score12"])
def test_dickson_score_fingerprint(name):
    from ladder_gpu import GpuEngine
    f = load("known")["fingerprints"][name]
    j0 = int(f["j_lo"])
    got = GpuEngine(f["n"], q2=f["q2"]).survivors_j(j0, j0 + int(f["span"]))
    assert got.size == f["count"]
    assert int(np.bitwise_xor.reduce(got)) == int(f["xor"])


@pytest.mark.slow
def test_dickson_score13_fingerprint():
    from ladder_gpu import GpuEngine
    f = load("known")["fingerprints"]["dickson_score13"]
    j0 = int(f["j_lo"])
    got = GpuEngine(f["n"], q2=f["q2"]).survivors_j(j0, j0 + int(f["span"]))
    assert got.size == f["count"]
    assert int(np.bitwise_xor.reduce(got)) == int(f["xor"])


# ------------------------------------------------------------------ AP ---

@pytest.mark.parametrize("case", range(len(load("ap")["surv"])))
def test_ap_survivors(case):
    from ap_gpu import GpuEngine
    c = load("ap")["surv"][case]
    d = int(c["d"]) if c["d"] else None
    eng = GpuEngine(c["n"], c["q2"], launch_u=1 << 16, d=d)
    parts = list(eng.survivors(int(c["base"]), int(c["span"])))
    got = np.concatenate(parts) if parts else np.empty(0, dtype=np.uint64)
    assert got.tolist() == ints(c["offsets"])


@pytest.mark.parametrize("case", range(len(load("ap")["hunt"])))
def test_ap_hunt(case):
    from ap_gpu import GpuEngine
    c = load("ap")["hunt"][case]
    d = int(c["d"]) if c["d"] else None
    eng = GpuEngine(c["n"], c["q2"], d=d)
    got = eng.hunt_cap(int(c["base"]), int(c["span"]), c["min_depth"],
                       c["cap"])
    assert got == [(int(p), r) for p, r in c["hits"]]


def test_ap_score_fingerprint():
    from ap_gpu import GpuEngine
    f = load("known")["fingerprints"]["ap_score"]
    eng = GpuEngine(f["n"], f["q2"], launch_u=1 << 25)
    parts = list(eng.survivors(int(f["base"]), int(f["span"])))
    got = np.concatenate(parts)
    assert got.size == f["count"]
    assert int(np.bitwise_xor.reduce(got)) == int(f["xor"])


def test_ap_rediscovers_a13_first():
    """a(13) = 3708797237 as the FIRST full chain from the floor
    (primorial-ap/ap_gpu.py:754-775, at q2 = 4096)."""
    from ap_gpu import GpuEngine
    known = {int(k): int(v) for k, v in load("known")["ap_known"].items()}
    eng = GpuEngine(13, q2=1 << 12)
    base = -(-eng.floor // 30) * 30
    span = -(-(known[13] + 1) // 30) * 30 - base
    hits = eng.hunt(base, span)
    assert min(p for p, dd in hits if dd >= 13) == known[13]
