"""Continuous-batching sweep server.

Requests (engine kind, interval, threshold) arrive over time.  The loop
keeps every device table resident (one ``EngineSet`` shared by all
slots), and runs ``slots`` batch pipelines, each on its own CUDA stream:
whenever a slot is free and requests are waiting, it admits as many as
fit the slot's HBM budget and item limit and submits them, so requests
that arrive while others are on the GPU start as soon as a slot frees up,
and two batches overlap on the device.  A request's latency is the wall
time from its arrival to its results being on the host.

Admission by footprint: a request is charged the bytes its run needs on
the device -- the base-residue table of its engine (4 bytes per sieve
prime) plus candidate and output slots sized by the engine's survival
estimate -- and a batch admits requests while the sum stays under
``hbm_budget``.  Results are bit-identical to running each request alone
(the pipeline computes every interval independently); the tests check
it.
"""

import collections
import time

import numpy as np

from fk_batch import BatchEngine, EngineSet

ENTRY_BYTES = 8 + 4 + 16 + 8 + 16   # candidate key/item, out rec, sorted, scratch


class ServeLoop:
    def __init__(self, engset=None, slots=2, max_items=256,
                 hbm_budget=2 << 30):
        self.engset = engset or EngineSet()
        self.slots = [BatchEngine(engset=self.engset) for _ in range(slots)]
        self.max_items = int(max_items)
        self.hbm_budget = int(hbm_budget)

    def footprint(self, iv):
        e = self.engset.get(self.engset.key_for(iv))
        span = iv.length // (e.W if iv.kind == 1 else 1) + 1
        # wheel density x survival estimate, with the pipeline's headroom
        expect = span * e.L / max(e.M, 1) * 0.05 + 64
        return 4 * e.NP + int(expect * 2) * ENTRY_BYTES + 256

    def run(self, requests, time_limit=None):
        """requests: [(arrival_s, Interval)] sorted by arrival.  Returns
        (results per request, latency_s per request, stats)."""
        for _, iv in requests:
            self.engset.get(self.engset.key_for(iv))   # tables resident up front
        for s in self.slots:
            s._ensure()
        n = len(requests)
        results = [None] * n
        latency = np.full(n, np.nan)
        waiting = collections.deque()
        inflight = {}                          # slot index -> [request ids]
        nxt = 0
        t0 = time.perf_counter()
        busy_s = 0.0
        batches = 0
        while nxt < n or waiting or inflight:
            now = time.perf_counter() - t0
            if time_limit is not None and now > time_limit and not inflight:
                break
            while nxt < n and requests[nxt][0] <= now:
                waiting.append(nxt)
                nxt += 1
            # collect finished slots
            for si in list(inflight):
                if self.slots[si]._batch.ready():
                    ids = inflight.pop(si)
                    rows = self.slots[si].wait_arrays()
                    done = time.perf_counter() - t0
                    st = self.slots[si].stats()
                    busy_s += st["total_ms"] * 1e-3
                    for rid, r in zip(ids, rows):
                        results[rid] = r
                        latency[rid] = done - requests[rid][0]
            # admit into free slots
            for si in range(len(self.slots)):
                if si in inflight or not waiting:
                    continue
                if time_limit is not None and now > time_limit:
                    break
                ids, foot = [], 0
                while waiting and len(ids) < self.max_items:
                    f = self.footprint(requests[waiting[0]][1])
                    if ids and foot + f > self.hbm_budget:
                        break
                    ids.append(waiting.popleft())
                    foot += f
                self.slots[si].submit([requests[i][1] for i in ids])
                inflight[si] = ids
                batches += 1
            if not waiting and nxt < n and not inflight:
                # idle until the next arrival
                delay = requests[nxt][0] - (time.perf_counter() - t0)
                if delay > 0:
                    time.sleep(min(delay, 0.01))
            elif inflight:
                time.sleep(0.0002)
        wall = time.perf_counter() - t0
        served = ~np.isnan(latency)
        stats = {"requests": int(served.sum()), "batches": batches,
                 "wall_s": wall, "device_busy_s": busy_s}
        return results, latency, stats
