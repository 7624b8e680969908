"""C-ABI exports and host logic, no GPU needed.

The library must load and export every symbol include/fk.h declares,
with a ctypes binding for each; constructing an engine without a CUDA
device must raise (there is no CPU fallback).  The workload generators
must be deterministic and match their stated distributions, and the
mirrors' host-side arithmetic must match the reference's rules.
"""

import ctypes
import pathlib
import re

import numpy as np
import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]


def _declared():
    txt = (ROOT / "include" / "fk.h").read_text()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return set(re.findall(r"\b(fk_[a-z0-9_]+)\s*\(", txt))


def _lib():
    import build as fkbuild
    fkbuild.build()
    import fk_abi
    return fk_abi, fk_abi.load()


def test_library_exports_every_declared_symbol():
    fk_abi, lib = _lib()
    names = _declared()
    assert len(names) >= 20
    for n in sorted(names):
        assert hasattr(lib, n), f"{n} declared in fk.h but not exported"
    assert names == set(fk_abi.SIGNATURES), \
        "ctypes bindings and fk.h disagree"


def test_version_and_error_calls_need_no_device():
    fk_abi, lib = _lib()
    assert b"sm_100a" in lib.fk_version()
    assert isinstance(lib.fk_last_error(), bytes)


def test_engine_without_a_device_fails_loudly():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    fk_abi, _ = _lib()
    with pytest.raises(RuntimeError):
        fk_abi.Engine(fk_abi.EULER, 8)


def test_u128_limbs():
    fk_abi, _ = _lib()
    x = (7 << 64) + 12345
    v = fk_abi.u128(x)
    assert (v[0], v[1]) == (12345, 7)
    with pytest.raises(ValueError):
        fk_abi.u128(1 << 128)


def test_mixed_batch_is_deterministic_and_as_stated():
    import fk_workloads as W
    a = W.mixed_batch(4096)
    b = W.mixed_batch(4096)
    assert a == b
    assert a != W.mixed_batch(4096, W.SEED + 1)
    kinds = np.array([iv.kind for iv in a])
    assert all(abs((kinds == k).mean() - 1 / 3) < 0.03 for k in range(3))
    for iv in a:
        assert 4 <= iv.threshold <= 12 and iv.n == iv.threshold
        assert 2 ** 20 - 30 <= iv.length <= 2 ** 36
        assert 10 ** 10 - 30 <= iv.lo <= 10 ** 18
        if iv.kind == W.AP:
            assert iv.lo % 30 == 0 and iv.length % 30 == 0
        assert iv.cap == W.default_cap(iv.kind, iv.n)


def test_served_requests():
    import fk_workloads as W
    reqs = W.served(count=500)
    times = [t for t, _ in reqs]
    assert times == sorted(times)
    for _, iv in reqs:
        assert 6 <= iv.threshold <= 14
        if iv.kind == W.EULER:
            assert iv.hi <= W.EULER_CEIL


def test_dickson_line_range_covers_the_k_interval_exactly():
    import fk_workloads as W
    for lo, hi, Wm in ((10 ** 10 + 7, 10 ** 10 + 10 ** 6, 2310),
                       (30030 * 5, 30030 * 9, 30030)):
        iv = W.Interval(W.DICKSON, 10, lo, hi, 10, 18)
        jlo, jhi = W.line_range(iv, Wm)
        ks = [j * Wm for j in range(jlo, jhi)]
        want = [k for k in range(lo - lo % Wm, hi + Wm, Wm) if lo <= k < hi]
        assert ks == want


def test_euler_mirror_wheel_attributes_follow_the_reference_rule():
    import euler_gpu as E
    # euler_search.best_wheel: 37# is reachable at n = 17 because only its
    # 31# base table is materialized (2.99e7 offsets <= 5e7)
    assert E.best_wheel(17) == E.WHEEL_PRIMES_37
    assert E.wheel_offset_count(17, E.WHEEL_PRIMES_31) == 29937600
    assert E.best_wheel(5) in (E.WHEEL_PRIMES, E.WHEEL_PRIMES_29)


def test_generated_montgomery_header_is_current(tmp_path, monkeypatch):
    """fk_mont32.cuh is what gen_mont32.py writes (no hand edits)."""
    import importlib.util
    csrc = ROOT / "first-knowns_b200" / "csrc"
    spec = importlib.util.spec_from_file_location("gen_mont32",
                                                  csrc / "gen_mont32.py")
    gen = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(gen)
    monkeypatch.setattr(gen, "HERE", tmp_path)
    gen.main()
    assert (tmp_path / "fk_mont32.cuh").read_text() == \
        (csrc / "fk_mont32.cuh").read_text()


def test_noalloc_device_rule_rejects_a_foreign_device(tmp_path):
    """fk_sieve_noalloc refuses to launch with an engine whose tables live
    on another GPU than the current one (FK_ERR_DEVICE before any launch):
    the check it calls, compiled host-only with g++ and driven on the CPU,
    since a one-GPU machine cannot make the devices differ."""
    import subprocess
    import fk_abi
    exe = tmp_path / "device_check"
    src = ROOT / "tests" / "native" / "device_check.cpp"
    subprocess.run(["g++", "-std=c++17", "-O1", "-o", str(exe), str(src)],
                   check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True,
                         text=True).stdout.splitlines()
    rows = [line.split(" ", 3) for line in out]
    got = {(int(r[0]), int(r[1])): (int(r[2]), r[3] if len(r) > 3 else "")
           for r in rows}
    assert got[(0, 0)] == (fk_abi.FK_OK, "")
    assert got[(7, 7)] == (fk_abi.FK_OK, "")
    st, msg = got[(0, 1)]
    assert st == fk_abi.FK_ERR_DEVICE and "device 0" in msg \
        and "device 1 is current" in msg
    assert got[(3, 2)][0] == fk_abi.FK_ERR_DEVICE
