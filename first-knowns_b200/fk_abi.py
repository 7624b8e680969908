"""ctypes binding of libfk.so (include/fk.h).

This is the thin C-ABI layer the reference-API mirrors (euler_gpu.py,
ladder_gpu.py, ap_gpu.py) and the batch / serving engines call.  There is
no CPU fallback: if the library is missing or no CUDA device is present,
every entry point raises.

Status codes map to the reference's exception types: a domain violation
is ValueError (the reference engines raise ValueError for bad ranges and
parameters), a capacity overflow, device fault or bounded-wait timeout is
RuntimeError (the reference raises RuntimeError on queue overflow).
"""

import ctypes
import os
import pathlib

import numpy as np

HERE = pathlib.Path(__file__).resolve().parent
LIB_PATH = HERE / "libfk.so"

FK_OK, FK_ERR_DOMAIN, FK_ERR_OVERFLOW, FK_ERR_DEVICE, FK_ERR_TIMEOUT, \
    FK_ERR_ARG = range(6)
EULER, DICKSON, AP = 0, 1, 2
MODE_SIEVE, MODE_HUNT, MODE_DENSE = 0, 1, 2

_u64 = ctypes.c_uint64
_u32 = ctypes.c_uint32


class Params(ctypes.Structure):
    _fields_ = [("kind", _u32), ("n", _u32), ("q2", _u32), ("p0", _u32),
                ("d_lo", _u64), ("d_hi", _u64), ("two_pass", _u32),
                ("sieve", _u32)]


class Info(ctypes.Structure):
    _fields_ = [("M", _u64), ("W", _u64), ("L", _u32), ("NP", _u32),
                ("first_prime", _u32), ("nrounds", _u32),
                ("device_bytes", _u64), ("use_mark", _u32),
                ("marked_primes", _u32), ("survival", ctypes.c_double)]


class Result(ctypes.Structure):
    _fields_ = [("count", _u64), ("offset", ctypes.POINTER(_u64)),
                ("depth", ctypes.POINTER(ctypes.c_uint8))]


class Item(ctypes.Structure):
    _fields_ = [("engine", _u32), ("mode", _u32), ("threshold", _u32),
                ("cap", _u32), ("lo", _u64 * 2), ("hi", _u64 * 2)]


class Stats(ctypes.Structure):
    _fields_ = [("launches", _u64), ("items", _u64), ("candidates", _u64),
                ("outputs", _u64), ("s1_words", _u64), ("s2_tests", _u64),
                ("imad_alg", _u64), ("sprp_values", _u64),
                ("marks", _u64), ("h2d_bytes", _u64), ("d2h_bytes", _u64),
                ("sieve_ms", ctypes.c_float), ("classify_ms", ctypes.c_float),
                ("total_ms", ctypes.c_float), ("mark_ms", ctypes.c_float),
                ("rounds_ms", ctypes.c_float), ("reruns", _u32)]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


class Tuning(ctypes.Structure):
    _fields_ = [("sieve_ctas_per_sm", _u32), ("mark_ctas_per_sm", _u32),
                ("chains_per_sm", _u32), ("warp_queue", _u32),
                ("seg_per_task", _u32), ("classify_ctas_per_sm", _u32),
                ("mark_limit", _u32), ("mark_bias", ctypes.c_float),
                ("warp_lane_words", _u32),
                ("capacity_scale", ctypes.c_float),
                ("round_cut", ctypes.c_float), ("group_lane_words", _u32),
                ("mark_segment", _u32), ("pattern_primes", _u32),
                ("mark_pattern_primes", _u32), ("warp_tasks", _u32)]

    def as_dict(self):
        return {f: getattr(self, f) for f, _ in self._fields_}


TUNING_FIELDS = [f for f, _ in Tuning._fields_]


class BatchResult(ctypes.Structure):
    _fields_ = [("nitems", _u64), ("item_start", ctypes.POINTER(_u64)),
                ("offset", ctypes.POINTER(_u64)),
                ("depth", ctypes.POINTER(ctypes.c_uint8))]


_lib = None

# every symbol include/fk.h declares, with its ctypes signature
SIGNATURES = {
    "fk_engine_create": (ctypes.c_int32, [ctypes.POINTER(Params),
                                          ctypes.POINTER(ctypes.c_void_p)]),
    "fk_engine_destroy": (None, [ctypes.c_void_p]),
    "fk_engine_info": (ctypes.c_int32, [ctypes.c_void_p,
                                        ctypes.POINTER(Info)]),
    "fk_sieve": (ctypes.c_int32, [ctypes.c_void_p, ctypes.POINTER(_u64),
                                  ctypes.POINTER(_u64),
                                  ctypes.POINTER(Result)]),
    "fk_hunt": (ctypes.c_int32, [ctypes.c_void_p, ctypes.POINTER(_u64),
                                 ctypes.POINTER(_u64), _u32, _u32,
                                 ctypes.POINTER(Result)]),
    "fk_dense": (ctypes.c_int32, [ctypes.c_void_p, ctypes.POINTER(_u64),
                                  ctypes.POINTER(_u64), _u32, _u32,
                                  ctypes.POINTER(Result)]),
    "fk_depths": (ctypes.c_int32, [ctypes.c_void_p, ctypes.POINTER(_u64),
                                   _u64, _u32,
                                   ctypes.POINTER(ctypes.c_uint8)]),
    "fk_batch_create": (ctypes.c_int32, [ctypes.POINTER(ctypes.c_void_p),
                                         _u32,
                                         ctypes.POINTER(ctypes.c_void_p)]),
    "fk_batch_destroy": (None, [ctypes.c_void_p]),
    "fk_batch_add_engines": (ctypes.c_int32, [ctypes.c_void_p,
                                              ctypes.POINTER(ctypes.c_void_p),
                                              ctypes.c_uint32]),
    "fk_batch_run": (ctypes.c_int32, [ctypes.c_void_p, ctypes.POINTER(Item),
                                      _u64, ctypes.c_int,
                                      ctypes.POINTER(BatchResult)]),
    "fk_batch_submit": (ctypes.c_int32, [ctypes.c_void_p,
                                         ctypes.POINTER(Item), _u64,
                                         ctypes.c_int]),
    "fk_batch_wait": (ctypes.c_int32, [ctypes.c_void_p,
                                       ctypes.POINTER(BatchResult)]),
    "fk_batch_ready": (ctypes.c_int32, [ctypes.c_void_p,
                                        ctypes.POINTER(ctypes.c_int)]),
    "fk_batch_last_ms": (ctypes.c_int32, [ctypes.c_void_p,
                                          ctypes.POINTER(ctypes.c_float),
                                          ctypes.POINTER(ctypes.c_float),
                                          ctypes.POINTER(ctypes.c_float)]),
    "fk_batch_stats": (ctypes.c_int32, [ctypes.c_void_p,
                                        ctypes.POINTER(Stats)]),
    "fk_engine_stats": (ctypes.c_int32, [ctypes.c_void_p,
                                         ctypes.POINTER(Stats)]),
    "fk_batch_set_tuning": (ctypes.c_int32, [ctypes.c_void_p,
                                             ctypes.POINTER(Tuning)]),
    "fk_batch_get_tuning": (ctypes.c_int32, [ctypes.c_void_p,
                                             ctypes.POINTER(Tuning)]),
    "fk_engine_set_tuning": (ctypes.c_int32, [ctypes.c_void_p,
                                              ctypes.POINTER(Tuning)]),
    "fk_set_device": (ctypes.c_int32, [ctypes.c_int]),
    "fk_peak": (ctypes.c_int32, [ctypes.c_int,
                                 ctypes.POINTER(ctypes.c_double)]),
    "fk_last_error": (ctypes.c_char_p, []),
    "fk_sprp": (ctypes.c_int32, [ctypes.POINTER(_u64), _u64, ctypes.c_int,
                                 ctypes.POINTER(ctypes.c_uint8)]),
    "fk_version": (ctypes.c_char_p, []),
    "fk_sieve_noalloc": (ctypes.c_int32, [ctypes.c_void_p,
                                          ctypes.POINTER(_u64),
                                          ctypes.POINTER(_u64),
                                          ctypes.c_void_p, _u64,
                                          ctypes.c_void_p, ctypes.c_void_p]),
}


def load(path=None):
    """Load libfk.so (once) and bind every declared entry point."""
    global _lib
    if _lib is not None:
        return _lib
    p = pathlib.Path(path) if path else LIB_PATH
    if not p.exists():
        raise RuntimeError(
            f"{p} is missing: build it with "
            f"`python first-knowns_b200/build.py` (nvcc, sm_100a)")
    lib = ctypes.CDLL(str(p))
    for name, (res, args) in SIGNATURES.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


def _check(st):
    if st == FK_OK:
        return
    msg = _lib.fk_last_error().decode(errors="replace")
    if st in (FK_ERR_DOMAIN, FK_ERR_ARG):
        raise ValueError(msg)
    raise RuntimeError(f"libfk status {st}: {msg}")


def u128(x):
    """A Python int in [0, 2^128) as two little-endian u64 limbs."""
    x = int(x)
    if x < 0 or x >> 128:
        raise ValueError(f"{x} does not fit 128 bits")
    return (_u64 * 2)(x & (2 ** 64 - 1), x >> 64)


def _arrays(res):
    n = int(res.count)
    if n == 0:
        return (np.empty(0, dtype=np.uint64), np.empty(0, dtype=np.uint8))
    off = np.ctypeslib.as_array(res.offset, shape=(n,)).copy()
    dep = np.ctypeslib.as_array(res.depth, shape=(n,)).copy()
    return off, dep


class Engine:
    """One device engine: wheel, pattern tables, kill tests, rounds."""

    def __init__(self, kind, n, q2=65536, p0=0, d=None, two_pass=False,
                 sieve=None):
        lib = load()
        p = Params()
        if sieve is None:
            sieve = os.environ.get("FK_SIEVE", "auto")
        p.sieve = {"auto": 0, "rounds": 1, "mark": 2}[sieve]
        p.kind, p.n, p.q2, p.p0 = int(kind), int(n), int(q2), int(p0)
        dd = int(d or 0)
        p.d_lo, p.d_hi = dd & (2 ** 64 - 1), dd >> 64
        p.two_pass = 1 if two_pass else 0
        h = ctypes.c_void_p()
        _check(lib.fk_engine_create(ctypes.byref(p), ctypes.byref(h)))
        self._h = h
        self._lib = lib
        self.kind, self.n, self.q2 = int(kind), int(n), int(q2)
        inf = Info()
        _check(lib.fk_engine_info(h, ctypes.byref(inf)))
        self.M, self.W, self.L = int(inf.M), int(inf.W), int(inf.L)
        self.NP, self.first_prime = int(inf.NP), int(inf.first_prime)
        self.nrounds = int(inf.nrounds)
        self.device_bytes = int(inf.device_bytes)
        self.use_mark = bool(inf.use_mark)
        self.marked_primes = int(inf.marked_primes)
        self.survival = float(inf.survival)

    def close(self):
        if getattr(self, "_h", None):
            self._lib.fk_engine_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self):
        return self._h

    def sieve(self, lo, hi):
        """Ascending pre-primality survivors of [lo, hi) as offsets x - lo."""
        r = Result()
        _check(self._lib.fk_sieve(self._h, u128(lo), u128(hi),
                                  ctypes.byref(r)))
        return _arrays(r)[0]

    def hunt(self, lo, hi, threshold, cap):
        """(offsets x - lo, depths) of survivors with depth >= threshold."""
        r = Result()
        _check(self._lib.fk_hunt(self._h, u128(lo), u128(hi), int(threshold),
                                 int(cap), ctypes.byref(r)))
        return _arrays(r)

    def dense(self, lo, hi, threshold, cap):
        """Every x in [lo, hi) classified directly (no sieve)."""
        r = Result()
        _check(self._lib.fk_dense(self._h, u128(lo), u128(hi),
                                  int(threshold), int(cap), ctypes.byref(r)))
        return _arrays(r)

    def stats(self):
        st = Stats()
        _check(self._lib.fk_engine_stats(self._h, ctypes.byref(st)))
        return st.as_dict()

    def set_tuning(self, **kw):
        """Kernel shape of this engine's plain calls (fk_tuning fields;
        unnamed fields keep their values)."""
        _check(self._lib.fk_engine_set_tuning(self._h,
                                              ctypes.byref(_tuning(kw))))

    def depths(self, xs, cap):
        """Chain depth of each explicit chain start in xs."""
        xs = [int(x) for x in xs]
        n = len(xs)
        if n == 0:
            return np.empty(0, dtype=np.uint8)
        limbs = np.empty(2 * n, dtype=np.uint64)
        for i, x in enumerate(xs):
            if x < 0 or x >> 128:
                raise ValueError(f"{x} does not fit 128 bits")
            limbs[2 * i] = x & (2 ** 64 - 1)
            limbs[2 * i + 1] = x >> 64
        out = np.empty(n, dtype=np.uint8)
        _check(self._lib.fk_depths(
            self._h, limbs.ctypes.data_as(ctypes.POINTER(_u64)), n, int(cap),
            out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8))))
        return out


class Batch:
    """Many intervals over several engines in one persistent launch."""

    def __init__(self, engines):
        lib = load()
        self._engines = list(engines)
        arr = (ctypes.c_void_p * len(self._engines))(
            *[e.handle for e in self._engines])
        h = ctypes.c_void_p()
        _check(lib.fk_batch_create(arr, len(self._engines), ctypes.byref(h)))
        self._h, self._lib = h, lib

    def add_engines(self, engines):
        """Append engines (indexed after the existing ones); the batch's
        buffers are kept."""
        new = list(engines)
        if not new:
            return
        arr = (ctypes.c_void_p * len(new))(*[e.handle for e in new])
        _check(self._lib.fk_batch_add_engines(self._h, arr, len(new)))
        self._engines.extend(new)

    def close(self):
        if getattr(self, "_h", None):
            self._lib.fk_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @staticmethod
    def items(specs):
        """[(engine_index, mode, threshold, cap, lo, hi)] -> ctypes array."""
        arr = (Item * max(len(specs), 1))()
        for i, (e, m, t, c, lo, hi) in enumerate(specs):
            it = arr[i]
            it.engine, it.mode, it.threshold, it.cap = int(e), int(m), \
                int(t), int(c)
            it.lo[:] = list(u128(lo))
            it.hi[:] = list(u128(hi))
        return arr

    def _unpack(self, br):
        ni = int(br.nitems)
        if ni == 0:
            return []
        start = np.ctypeslib.as_array(br.item_start, shape=(ni + 1,)).copy()
        tot = int(start[-1])
        if tot:
            off = np.ctypeslib.as_array(br.offset, shape=(tot,)).copy()
            dep = np.ctypeslib.as_array(br.depth, shape=(tot,)).copy()
        else:
            off = np.empty(0, dtype=np.uint64)
            dep = np.empty(0, dtype=np.uint8)
        return [(off[start[i]:start[i + 1]], dep[start[i]:start[i + 1]])
                for i in range(ni)]

    def run(self, specs, graph=True):
        """Run all items; per item (offsets x - lo, depths), ascending."""
        arr = self.items(specs)
        br = BatchResult()
        _check(self._lib.fk_batch_run(self._h, arr, len(specs),
                                      1 if graph else 0, ctypes.byref(br)))
        return self._unpack(br)

    def submit(self, specs, graph=False):
        arr = self.items(specs)
        self._pending_arr = arr
        _check(self._lib.fk_batch_submit(self._h, arr, len(specs),
                                         1 if graph else 0))

    def ready(self):
        r = ctypes.c_int()
        _check(self._lib.fk_batch_ready(self._h, ctypes.byref(r)))
        return bool(r.value)

    def wait(self):
        br = BatchResult()
        _check(self._lib.fk_batch_wait(self._h, ctypes.byref(br)))
        return self._unpack(br)

    def stats(self):
        st = Stats()
        _check(self._lib.fk_batch_stats(self._h, ctypes.byref(st)))
        return st.as_dict()

    def get_tuning(self):
        t = Tuning()
        _check(self._lib.fk_batch_get_tuning(self._h, ctypes.byref(t)))
        return t.as_dict()

    def set_tuning(self, **kw):
        """Set fk_tuning fields by name; unnamed fields keep their values."""
        _check(self._lib.fk_batch_set_tuning(self._h,
                                             ctypes.byref(_tuning(kw))))

    def last_ms(self):
        a, c, t = ctypes.c_float(), ctypes.c_float(), ctypes.c_float()
        _check(self._lib.fk_batch_last_ms(self._h, ctypes.byref(a),
                                          ctypes.byref(c), ctypes.byref(t)))
        return float(a.value), float(c.value), float(t.value)


_FLOAT_FIELDS = ("mark_bias", "capacity_scale", "round_cut")


def _tuning(kw):
    t = Tuning()
    for k, v in kw.items():
        if k not in TUNING_FIELDS:
            raise ValueError(f"unknown tuning field {k}")
        setattr(t, k, float(v) if k in _FLOAT_FIELDS else int(v))
    return t


def sprp(values, base2_only=False):
    """Device verdicts of huntlib's mr_is_prime (or sprp_base2) for values
    below 2^192."""
    lib = load()
    vals = [int(v) for v in values]
    n = len(vals)
    if n == 0:
        return np.empty(0, dtype=bool)
    limbs = np.empty(3 * n, dtype=np.uint64)
    for i, v in enumerate(vals):
        if v < 0 or v >> 192:
            raise ValueError(f"{v} does not fit 192 bits")
        limbs[3 * i] = v & (2 ** 64 - 1)
        limbs[3 * i + 1] = (v >> 64) & (2 ** 64 - 1)
        limbs[3 * i + 2] = v >> 128
    out = np.empty(n, dtype=np.uint8)
    _check(lib.fk_sprp(limbs.ctypes.data_as(ctypes.POINTER(_u64)), n,
                       1 if base2_only else 0,
                       out.ctypes.data_as(ctypes.POINTER(ctypes.c_uint8))))
    return out.astype(bool)


def version():
    return load().fk_version().decode()


def set_device(device):
    """Point libfk's runtime at a CUDA device for this host thread."""
    _check(load().fk_set_device(int(device)))


PEAKS = {"imad": 0, "smem": 1, "smem_st": 2, "imad_lo": 3, "imad_hi": 4,
         "mul64hi": 5, "smem_or": 6}


def peak(which):
    """Measured peak: 'imad' -> 32-bit multiply-adds/s (mad.lo and mad.hi
    alternating), 'imad_lo' / 'imad_hi' -> each half alone, 'mul64hi' ->
    high halves of 64 x 64-bit products/s, 'smem' -> shared load bytes/s,
    'smem_st' -> shared byte stores/s, 'smem_or' -> shared bit marks
    (red.shared.or.b32)/s."""
    out = ctypes.c_double()
    _check(load().fk_peak(PEAKS[which], ctypes.byref(out)))
    return float(out.value)


def device_count():
    """CUDA devices visible to libfk's runtime (0 when none)."""
    try:
        import torch
        return torch.cuda.device_count()
    except Exception:
        return 0


if os.environ.get("FK_PRELOAD") == "1":
    load()
