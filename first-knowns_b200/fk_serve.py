"""Continuous-batching sweep server.

Requests (engine kind, interval, threshold) arrive over time.  The loop
keeps every device table resident (one ``EngineSet`` shared by all slots)
and runs ``slots`` batch pipelines, each on its own CUDA stream, so two
batches overlap on the device while the host collects one and fills the
other.

Requests are cut into chunks of at most ``chunk`` units of their engine's
line variable (p, or j = k / W for Dickson), and of at most a quarter of
the HBM budget's predicted footprint, and queued chunk by chunk in
arrival order.  Whenever a slot is free it takes queued chunks, oldest
first, while the batch stays under a work budget (``batch_work`` line
units) and an HBM budget, and submits them as one persistent launch; a
request is answered when its last chunk comes back, its chunks' streams
concatenated in order.  A long request therefore never holds a slot for
long: short requests that arrive behind it join the next batch, and the
device never idles while work is queued.

Admission by footprint: a chunk is charged the device bytes its run needs
-- the base-residue table of its engine (4 bytes per sieve prime) plus
candidate and output slots for twice the survivors the engine's density
predicts (``fk_info.survival``, the product of 1 - f_q/q over the wheel and
sieve primes) -- and a batch admits chunks while the sum stays under
``hbm_budget``.

Results are bit-identical to sweeping each request alone with the plain
engine: every chunk is an independent interval, and a request's chunks
tile it (the tests check alone == in the mix == plain).

While the loop runs, everything the process built before it (engine
tables, the caller's objects, imported modules) is moved out of the
cyclic garbage collector's reach (``gc.freeze``), so a full collection
triggered by the loop's own small allocations does not rescan that heap
between two batches: in a process that imports torch such a pass stalls
the loop for tens to hundreds of milliseconds.
"""

import collections
import gc
import time

import numpy as np

from fk_batch import BatchEngine, EngineSet
from fk_workloads import DICKSON, Interval, line_range

# device bytes per candidate slot: key + item, output record, ordered copy,
# ordering scratch
ENTRY_BYTES = 8 + 4 + 16 + 8 + 16


class ServeLoop:
    def __init__(self, engset=None, slots=2, max_items=256,
                 hbm_budget=2 << 30, chunk=1 << 30, batch_work=1 << 34):
        self.engset = engset or EngineSet()
        self.slots = [BatchEngine(engset=self.engset) for _ in range(slots)]
        self.max_items = int(max_items)
        self.hbm_budget = int(hbm_budget)
        self.chunk = int(chunk)
        self.batch_work = int(batch_work)

    def _engine(self, iv):
        return self.engset.get(self.engset.key_for(iv))

    def footprint(self, iv):
        """Device bytes a chunk's run needs (see the module docstring)."""
        e = self._engine(iv)
        lo, hi = line_range(iv, e.W if iv.kind == DICKSON else 1)
        expect = (hi - lo) * e.survival + 64
        return 4 * e.NP + int(2 * expect) * ENTRY_BYTES + 256

    def chunk_units(self, iv):
        """Line units per chunk of this request: at most `chunk`, and at
        most what keeps one chunk's predicted footprint within a quarter of
        the HBM budget, so no single chunk -- always admitted, even alone
        over the budget -- grows a slot's buffers past what batches of the
        budget need (a growth reallocates gigabytes while requests wait)."""
        e = self._engine(iv)
        per_unit = 2 * e.survival * ENTRY_BYTES
        cap = int(self.hbm_budget / 4 / per_unit) if per_unit > 0 else self.chunk
        return min(self.chunk, max(1 << 20, cap))

    def chunks(self, iv):
        """The request as intervals of at most `chunk_units` line units,
        in order; each is an Interval of the same engine and threshold."""
        W = self._engine(iv).W if iv.kind == DICKSON else 1
        lo, hi = line_range(iv, W)
        step = self.chunk_units(iv)
        out = []
        a = lo
        while a < hi:
            b = min(hi, a + step)
            if iv.kind == DICKSON:   # back to k: [a*W, b*W) covers j in [a, b)
                klo = iv.lo if a == lo else a * W
                khi = iv.hi if b == hi else b * W
                out.append(Interval(iv.kind, iv.n, klo, khi, iv.threshold,
                                    iv.cap, iv.q2, iv.d))
            else:
                out.append(Interval(iv.kind, iv.n, a, b, iv.threshold,
                                    iv.cap, iv.q2, iv.d))
            a = b
        return out or [iv]

    def run(self, requests, time_limit=None):
        """requests: [(arrival_s, Interval)] sorted by arrival.  Returns
        (per request (offsets, depths) as the batch engine gives them for
        the whole request, latency_s per request, stats)."""
        # tables resident up front: every engine a chunk will run on (the
        # wheel follows an interval's length, so a chunk can run on another
        # engine than its whole request), so none is built while requests
        # wait
        for _, iv in requests:
            for c in self.chunks(iv):
                self._engine(c)
        for s in self.slots:
            s._ensure()
        self._prime(requests)
        gc.collect()
        gc.freeze()
        try:
            return self._run(requests, time_limit)
        finally:
            gc.unfreeze()

    def _prime(self, requests):
        """Run, on every slot and before the clock starts, one batch of
        the requests' largest-footprint chunks that fits the budgets, so
        the slots' device and pinned buffers already have the size a batch
        can need (a slot whose engine set grew starts with none, and
        growing them under load reallocates while requests wait)."""
        cs = [(self.footprint(c), i, c) for i, c in enumerate(
            c for _, iv in requests for c in self.chunks(iv))]
        cs.sort(key=lambda x: (-x[0], x[1]))
        take, foot, work = [], 0, 0
        for f, _, c in cs:
            e = self._engine(c)
            lo, hi = line_range(c, e.W if c.kind == DICKSON else 1)
            if take and (foot + f > self.hbm_budget or
                         work + (hi - lo) > self.batch_work or
                         len(take) >= self.max_items):
                continue
            take.append(c)
            foot += f
            work += hi - lo
        if take:
            for s in self.slots:
                s.submit(take)
                s.wait_arrays()

    def _run(self, requests, time_limit):
        n = len(requests)
        parts = [None] * n                      # per request: chunk results
        left = [0] * n                          # chunks still out
        results = [None] * n
        latency = np.full(n, np.nan)
        queue = collections.deque()             # (request, chunk index, iv)
        inflight = {}                           # slot -> [(request, chunk, iv)]
        nxt = 0
        t0 = time.perf_counter()
        busy_s = 0.0
        inflight_s = 0.0                        # wall time with a batch out
        last = 0.0
        batches = 0
        work_done = 0
        host_calls = []                         # (host s, kind, t, chunks)
        while nxt < n or queue or inflight:
            now = time.perf_counter() - t0
            if inflight:
                inflight_s += now - last
            last = now
            if time_limit is not None and now > time_limit and not inflight:
                break
            while nxt < n and requests[nxt][0] <= now:
                cs = self.chunks(requests[nxt][1])
                parts[nxt] = [None] * len(cs)
                left[nxt] = len(cs)
                for ci, c in enumerate(cs):
                    queue.append((nxt, ci, c))
                nxt += 1
            # collect finished slots
            for si in list(inflight):
                if not self.slots[si]._batch.ready():
                    continue
                done = inflight.pop(si)
                tw = time.perf_counter()
                rows = self.slots[si].wait_arrays()
                host_calls.append((time.perf_counter() - tw, "wait",
                                   tw - t0, len(done)))
                st = self.slots[si].stats()
                busy_s += st["total_ms"] * 1e-3
                t_done = time.perf_counter() - t0
                for (rid, ci, civ), row in zip(done, rows):
                    parts[rid][ci] = (civ, row)
                    left[rid] -= 1
                    if left[rid] == 0:
                        results[rid] = self._join(requests[rid][1],
                                                  parts[rid])
                        parts[rid] = None
                        latency[rid] = t_done - requests[rid][0]
            # fill free slots, oldest chunks first
            for si in range(len(self.slots)):
                if si in inflight or not queue:
                    continue
                if time_limit is not None and now > time_limit:
                    break
                take, foot, work = [], 0, 0
                while queue and len(take) < self.max_items:
                    rid, ci, civ = queue[0]
                    f = self.footprint(civ)
                    e = self._engine(civ)
                    lo, hi = line_range(civ, e.W if civ.kind == DICKSON
                                        else 1)
                    if take and (foot + f > self.hbm_budget or
                                 work + (hi - lo) > self.batch_work):
                        break
                    take.append(queue.popleft())
                    foot += f
                    work += hi - lo
                ts = time.perf_counter()
                self.slots[si].submit([c for _, _, c in take])
                host_calls.append((time.perf_counter() - ts, "submit",
                                   ts - t0, len(take)))
                inflight[si] = take
                batches += 1
                work_done += work
            if not queue and nxt < n and not inflight:
                delay = requests[nxt][0] - (time.perf_counter() - t0)
                if delay > 0:
                    time.sleep(min(delay, 0.005))
            elif inflight:
                time.sleep(0.0001)
        wall = time.perf_counter() - t0
        served = ~np.isnan(latency)
        host_calls.sort(reverse=True)
        stats = {"requests": int(served.sum()), "batches": batches,
                 "wall_s": wall, "device_busy_s": busy_s,
                 "inflight_s": inflight_s, "line_units": work_done,
                 # the five longest submit / wait calls on the host: a
                 # stall there holds every queued request
                 "slowest_host_calls": [
                     {"ms": round(d * 1e3, 2), "call": k,
                      "at_s": round(t, 3), "chunks": n}
                     for d, k, t, n in host_calls[:5]]}
        return results, latency, stats

    def _join(self, iv, parts):
        """A request's (offsets, depths) from its chunks' rows: offsets are
        relative to each chunk's start in the line variable, so they are
        shifted to the request's start and concatenated in order."""
        if len(parts) == 1:
            return parts[0][1]
        e = self._engine(iv)
        W = e.W if iv.kind == DICKSON else 1
        lo0, _ = line_range(iv, W)
        offs, deps = [], []
        for civ, (off, dep) in parts:
            clo, _ = line_range(civ, W)
            offs.append(off + np.uint64(clo - lo0))
            deps.append(dep)
        return (np.concatenate(offs).astype(np.uint64),
                np.concatenate(deps).astype(np.uint8))
