"""fk_sieve_noalloc: the allocation-free sieve entry point, on the GPU.

Callers that cannot allocate device memory while they sweep (a fixed
memory budget, an allocator of their own, no implicit synchronisation
allowed) call fk_sieve_noalloc with output buffers they own; its scratch
is a fixed device array inside libfk.  These tests call it through the C
ABI and require its result to equal the allocating entry point's
(fk_sieve) exactly -- the streams are integer survivor offsets, so the
tolerance is zero -- on two calls in a row, so the second call also shows
that the shared array is reset between calls.  Every pattern family (p0)
runs, and one case runs on a stream the caller created.

This file is named to be collected last: if it fails, a run that stops
at the first failure has already run every other test.
"""

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CAP = 1 << 18


def _bind():
    import fk_abi
    lib = fk_abi.load()
    f = lib.fk_sieve_noalloc
    f.restype = ctypes.c_int32
    f.argtypes = [ctypes.c_void_p, ctypes.POINTER(ctypes.c_uint64),
                  ctypes.POINTER(ctypes.c_uint64), ctypes.c_void_p,
                  ctypes.c_uint64, ctypes.c_void_p, ctypes.c_void_p]
    return fk_abi, f


def _call(f, fk_abi, eng, lo, hi, out, cnt, cap=CAP, stream=None):
    import torch
    handle = stream.cuda_stream if stream is not None else None
    st = f(eng.handle, fk_abi.u128(lo), fk_abi.u128(hi), out.data_ptr(),
           cap, cnt.data_ptr(), handle)
    if stream is not None:
        stream.synchronize()
    torch.cuda.synchronize()
    return st


def _cases(p0):
    import fk_abi
    ap_lo = 4 * 10 ** 13 - (4 * 10 ** 13) % 30
    if p0 == 11:
        # the 31# wheel fits n = 17 only (30 million lanes): the reference's
        # SCORE window [1e16, 1e16 + 5e14), 178 survivors
        return [(fk_abi.Engine(fk_abi.EULER, 17, p0=11), 10 ** 16,
                 10 ** 16 + 5 * 10 ** 14)]
    out = [(fk_abi.Engine(fk_abi.EULER, 8, p0=p0), 10 ** 5, 10 ** 9)]
    if p0 <= 9:
        out += [(fk_abi.Engine(fk_abi.AP, 8, q2=4096, p0=p0), ap_lo,
                 ap_lo + 3 * 10 ** 6),
                (fk_abi.Engine(fk_abi.DICKSON, 6, q2=4096, p0=p0), 10 ** 6,
                 10 ** 6 + 2 ** 20)]
    return out


@pytest.mark.parametrize("p0", [6, 7, 9, 11])
def test_noalloc_equals_fk_sieve_on_two_calls_in_a_row(p0):
    import torch
    fk_abi, f = _bind()
    out = torch.zeros(CAP, dtype=torch.int64, device="cuda")
    cnt = torch.zeros(1, dtype=torch.int64, device="cuda")
    for eng, lo, hi in _cases(p0):
        want = eng.sieve(lo, hi)
        assert want.size > 50
        for _ in range(2):                     # two calls in a row
            out.fill_(-1)
            cnt.fill_(-1)
            assert _call(f, fk_abi, eng, lo, hi, out, cnt) == 0
            n = int(cnt.item())
            got = out[:n].cpu().numpy().view(np.uint64)
            assert n == want.size
            assert np.array_equal(got, want)


def test_noalloc_on_a_caller_stream_near_the_survivor_limit():
    """A call on a stream the caller created, with about 236,000
    survivors (the array holds 262,144), timed with CUDA events on that
    stream: the result equals fk_sieve's on two calls in a row."""
    import torch
    fk_abi, f = _bind()
    eng = fk_abi.Engine(fk_abi.EULER, 2, p0=6)
    lo, hi = 10 ** 12, 10 ** 12 + 7 * 10 ** 7
    want = eng.sieve(lo, hi)
    assert 150_000 < want.size < CAP
    s = torch.cuda.Stream()
    out = torch.zeros(CAP, dtype=torch.int64, device="cuda")
    cnt = torch.zeros(1, dtype=torch.int64, device="cuda")
    times = []
    for _ in range(2):
        with torch.cuda.stream(s):
            out.fill_(-1)
            cnt.fill_(-1)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(s)
        assert _call(f, fk_abi, eng, lo, hi, out, cnt, stream=s) == 0
        e1.record(s)
        e1.synchronize()
        times.append(e0.elapsed_time(e1))
        n = int(cnt.item())
        assert n == want.size
        assert np.array_equal(out[:n].cpu().numpy().view(np.uint64), want)
    print(f"fk_sieve_noalloc, {want.size} survivors: "
          f"{min(times):.2f} ms per call")


def test_noalloc_rejects_what_does_not_fit():
    import torch
    fk_abi, f = _bind()
    out = torch.zeros(16, dtype=torch.int64, device="cuda")
    cnt = torch.zeros(1, dtype=torch.int64, device="cuda")
    deep = fk_abi.Engine(fk_abi.DICKSON, 6, q2=1 << 20, p0=6)
    assert _call(f, fk_abi, deep, 10 ** 6, 10 ** 6 + 1000, out, cnt) == \
        fk_abi.FK_ERR_DOMAIN                   # 82,000 primes: too many
    assert b"65536 sieve primes" in fk_abi.load().fk_last_error()
    eng = fk_abi.Engine(fk_abi.EULER, 8, p0=6)
    assert _call(f, fk_abi, eng, 10 ** 5, 10 ** 5, out, cnt) == \
        fk_abi.FK_ERR_DOMAIN                   # empty interval
    assert _call(f, fk_abi, eng, 10 ** 5, 10 ** 5 + 2 ** 63, out, cnt) == \
        fk_abi.FK_ERR_DOMAIN                   # wider than fk_sieve takes
    # more survivors than the caller's capacity: count reports UINT64_MAX
    # (UINT64_MAX - 1 would mean a device wait gave up)
    assert _call(f, fk_abi, eng, 10 ** 5, 10 ** 9, out, cnt, cap=16) == 0
    assert int(cnt.item()) == -1


def test_noalloc_short_sub_period_and_empty_results():
    """Survivors are ordered by bucketing their offsets from lo over the
    interval's length (2048 buckets, each sorted by one CTA): intervals
    shorter than the bucket count (one offset per bucket, then two), one
    that sits inside a single period of the 23# wheel, and one with no
    survivors at all give fk_sieve's stream exactly."""
    import torch
    fk_abi, f = _bind()
    out = torch.zeros(CAP, dtype=torch.int64, device="cuda")
    cnt = torch.zeros(1, dtype=torch.int64, device="cuda")
    e2 = fk_abi.Engine(fk_abi.EULER, 2, p0=6)
    e8 = fk_abi.Engine(fk_abi.EULER, 8, p0=9)
    e17 = fk_abi.Engine(fk_abi.EULER, 17, p0=11)
    M23 = 223092870
    base = 25 * M23
    # survivor counts (a numpy sieve to 65536): 12, 17, 8 and 0
    cases = [(e2, 10 ** 12 + 7, 10 ** 12 + 7 + 2047, 10),
             (e2, 10 ** 12, 10 ** 12 + 4095, 15),
             (e8, base + 12345, base + 12345 + 2 * 10 ** 8, 5),
             (e17, 10 ** 16, 10 ** 16 + 10 ** 6, 0)]
    for eng, lo, hi, least in cases:
        want = eng.sieve(lo, hi)
        assert want.size >= least
        if least == 0:
            assert want.size == 0
        out.fill_(-1)
        cnt.fill_(-1)
        assert _call(f, fk_abi, eng, lo, hi, out, cnt) == 0
        n = int(cnt.item())
        assert n == want.size
        assert np.array_equal(out[:n].cpu().numpy().view(np.uint64), want)
