"""The persistent batched engine and its plain per-interval counterpart.

``BatchEngine`` keeps one device engine per (kind, n, q2, d) -- wheel,
pattern, prime and kill-test tables stay resident across runs -- and
sweeps any number of intervals of mixed engine type in ONE pipeline: a
persistent sieve grid pulls (interval, chain block) tasks from a device
counter, the SPRP stage classifies every survivor, and the stream comes
back ordered per interval.  With ``graph=True`` the pipeline is a
captured CUDA graph, replayed while the batch shape is unchanged.

``PlainEngine`` runs the same intervals one at a time through each
engine's own per-interval call (fk_hunt): the baseline the batch is
measured against.  Both return identical results by construction; the
tests check it.
"""

import fk_abi
from fk_workloads import (AP, DICKSON, EULER, engine_key, line_range,
                          rows_to_results)


# Pattern families (fk_params.p0): 6 puts 2..13 in the wheel and starts
# the pattern primes at 17; 7 also folds 17 into the wheel, which drops
# every position 17 kills (a fraction f/17 of them, f = 17's forbidden
# residues) at the price of 17x fewer periods per lane.  The wider wheel
# pays when lanes stay long: at least LONG_PERIODS periods, one segment of
# the marking sieve, so each lane's per-prime setup is still spread thin.
P0_NARROW, P0_WIDE = 6, 7
LONG_PERIODS = 1 << 15


class EngineSet:
    """Device engines keyed by (kind, n, q2, d, p0), created on first use."""

    def __init__(self, wide=True):
        self._engines = {}
        self._order = []
        self.wide = wide

    def get(self, key):
        if len(key) == 4:
            key = key + (P0_NARROW,)
        if key not in self._engines:
            kind, n, q2, d, p0 = key
            self._engines[key] = fk_abi.Engine(kind, n, q2=q2, p0=p0,
                                               d=d or None)
            self._order.append(key)
        return self._engines[key]

    def key_for(self, iv):
        """The engine an interval runs on: the 17# wheel when its lanes
        stay at least LONG_PERIODS periods long, else the 13# wheel."""
        base = engine_key(iv) + (P0_NARROW,)
        if not self.wide:
            return base
        e = self.get(base)
        lo, hi = line_range(iv, e.W if iv.kind == DICKSON else 1)
        if hi - lo >= LONG_PERIODS * 17 * e.M:
            wide = engine_key(iv) + (P0_WIDE,)
            if hi - lo >= LONG_PERIODS * self.get(wide).M:
                return wide
        return base

    def index(self, key):
        self.get(key)
        return self._order.index(key)

    def engines(self):
        return [self._engines[k] for k in self._order]

    def device_bytes(self):
        return sum(e.device_bytes for e in self._engines.values())


def item_specs(engset, intervals):
    """fk_item specs (engine index, mode, threshold, cap, lo, hi)."""
    specs = []
    for iv in intervals:
        key = engset.key_for(iv)
        e = engset.get(key)
        lo, hi = line_range(iv, e.W if iv.kind == DICKSON else 1)
        specs.append((engset.index(key), fk_abi.MODE_HUNT, iv.threshold,
                      iv.cap, lo, hi))
    return specs


class BatchEngine:
    """Sweep many intervals in one persistent launch."""

    def __init__(self, intervals=(), engset=None):
        self.engset = engset or EngineSet()
        for iv in intervals:
            self.engset.get(self.engset.key_for(iv))
        self._batch = None
        self._nengines = -1

    def _ensure(self):
        engines = self.engset.engines()
        if self._batch is None:
            self._batch = fk_abi.Batch(engines)
            self._nengines = len(engines)
            if getattr(self, "_tuning", None):
                self._batch.set_tuning(**self._tuning)
        elif len(engines) != self._nengines:
            # engines are only ever appended to the set: extend the batch
            # in place, keeping its buffers
            self._batch.add_engines(engines[self._nengines:])
            self._nengines = len(engines)
        return self._batch

    def run_arrays(self, intervals, graph=True):
        """Per interval, (offsets, depths) as numpy arrays, ascending, in
        the engine's device line variable: x = lo + offset for Euler and
        AP, k = W * (ceil(lo / W) + offset) for Dickson.  No per-hit
        Python objects: the form to use at high hit rates."""
        specs = item_specs(self.engset, intervals)
        return self._ensure().run(specs, graph=graph)

    def run(self, intervals, graph=True):
        """[(x, depth)] per interval, ascending, depth >= threshold."""
        specs = item_specs(self.engset, intervals)
        b = self._ensure()
        rows = b.run(specs, graph=graph)
        out = []
        for iv, (off, dep) in zip(intervals, rows):
            e = self.engset.get(self.engset.key_for(iv))
            out.append(rows_to_results(iv, off, dep,
                                       e.W if iv.kind == DICKSON else 1))
        return out

    def submit(self, intervals, graph=False):
        specs = item_specs(self.engset, intervals)
        self._pending = list(intervals)
        self._ensure().submit(specs, graph=graph)

    def wait_arrays(self):
        """The submitted run's per-interval (offsets, depths) arrays."""
        return self._batch.wait()

    def wait(self):
        rows = self._batch.wait()
        out = []
        for iv, (off, dep) in zip(self._pending, rows):
            e = self.engset.get(self.engset.key_for(iv))
            out.append(rows_to_results(iv, off, dep,
                                       e.W if iv.kind == DICKSON else 1))
        return out

    def last_ms(self):
        """(sieve, classify, whole pipeline) device ms of the last run."""
        return self._batch.last_ms()

    def stats(self):
        """Device work counters and event times of the last run."""
        return self._batch.stats()

    def tuning(self):
        """The batch's kernel shape (fk_tuning fields)."""
        return self._ensure().get_tuning()

    def set_tuning(self, **kw):
        """Set fk_tuning fields (the autotuner's knobs) by name."""
        self._tuning = dict(getattr(self, "_tuning", {}), **kw)
        self._ensure().set_tuning(**kw)


class PlainEngine:
    """The same intervals, one fk_hunt call each."""

    def __init__(self, engset=None):
        self.engset = engset or EngineSet()

    def set_tuning(self, **kw):
        """Apply fk_tuning fields to every engine's plain calls, and to
        engines created later."""
        self._tuning = dict(getattr(self, "_tuning", {}), **kw)
        self._tuned = set()
        for e in self.engset.engines():
            e.set_tuning(**self._tuning)
            self._tuned.add(id(e))

    def _engine(self, iv):
        e = self.engset.get(self.engset.key_for(iv))
        if getattr(self, "_tuning", None) and id(e) not in self._tuned:
            e.set_tuning(**self._tuning)
            self._tuned.add(id(e))
        return e

    def run_arrays(self, intervals):
        """Per interval (offsets, depths) as BatchEngine.run_arrays."""
        out = []
        for iv in intervals:
            e = self._engine(iv)
            lo, hi = line_range(iv, e.W if iv.kind == DICKSON else 1)
            out.append(e.hunt(lo, hi, iv.threshold, iv.cap))
        return out

    def run(self, intervals):
        out = []
        for iv in intervals:
            e = self._engine(iv)
            W = e.W if iv.kind == DICKSON else 1
            lo, hi = line_range(iv, W)
            off, dep = e.hunt(lo, hi, iv.threshold, iv.cap)
            out.append(rows_to_results(iv, off, dep, W))
        return out


__all__ = ["BatchEngine", "PlainEngine", "EngineSet", "EULER", "DICKSON",
           "AP"]
