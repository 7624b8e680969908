"""Host logic of the autotuner and of the batch's wheel choice (no GPU).

The coordinate descent must find the best setting of a known cost
surface, apply it and keep to its time budget; the saved setting must
load back; the ctypes mirrors of fk_tuning and fk_stats must list the
header's fields in the header's order; and the batch must put exactly
the intervals whose lanes stay long on the 17# wheel.
"""

import json
import re

import pytest

import fk_workloads as W


class FakeBatch:
    """Stands in for BatchEngine: total_ms is a known function of the
    setting (best at mark_bias 1.4, mark_limit 49152, seg_per_task 4)."""

    def __init__(self):
        import fk_tune
        self.setting = {k: v[0] for k, v in fk_tune.SPACE.items()}
        self.setting.update(mark_bias=1.0, mark_limit=65536, seg_per_task=8)
        self.runs = 0

    def tuning(self):
        return dict(self.setting)

    def set_tuning(self, **kw):
        self.setting.update(kw)

    def run_arrays(self, intervals, graph=True):
        self.runs += 1
        return []

    def stats(self):
        s = self.setting
        ms = 100.0
        ms += 40 * abs(s["mark_bias"] - 1.4)
        ms += 0.001 * abs(s["mark_limit"] - 49152)
        ms += 5 * abs(s["seg_per_task"] - 4)
        return {"total_ms": ms}


def test_coordinate_descent_finds_the_minimum():
    import fk_tune
    fb = FakeBatch()
    res = fk_tune.tune(fb, [], repeats=1, max_passes=3, budget_s=60)
    best = res["best"]
    assert best["mark_bias"] == 1.4
    assert best["mark_limit"] == 49152
    assert best["seg_per_task"] == 4
    assert fb.setting == best                   # applied
    assert res["best_ms"] == pytest.approx(100.0)
    assert len(res["trials"]) > 1


def test_a_far_slower_setting_is_timed_once():
    """A candidate whose first run is over 1.5x the incumbent is not run
    again: the budget goes to settings that can win."""
    import fk_tune
    fb = FakeBatch()
    fb.setting.update(mark_bias=50.0)            # 2000 ms slower
    ms = fk_tune.measure(fb, [], repeats=3, give_up_ms=150.0)
    assert fb.runs == 1 and ms > 150.0
    fb.runs = 0
    fb.setting.update(mark_bias=1.4)
    fk_tune.measure(fb, [], repeats=3, give_up_ms=150.0)
    assert fb.runs == 3


def test_tuner_keeps_to_its_budget():
    import fk_tune
    fb = FakeBatch()
    res = fk_tune.tune(fb, [], repeats=1, max_passes=3, budget_s=0.0)
    assert len(res["trials"]) == 1              # only the starting point
    assert fb.setting == res["best"]


def test_saved_setting_loads_back(tmp_path):
    import fk_tune
    fb = FakeBatch()
    res = fk_tune.tune(fb, [], repeats=1, budget_s=60)
    path = tmp_path / "tuning.json"
    fk_tune.save(res, path)
    assert json.loads(path.read_text()) == res["best"]
    other = FakeBatch()
    assert fk_tune.load(other, path)
    assert other.setting == res["best"]
    assert not fk_tune.load(other, tmp_path / "missing.json")


def _header_fields(struct):
    import pathlib
    txt = (pathlib.Path(__file__).resolve().parents[1] / "include" /
           "fk.h").read_text()
    body = re.search(r"typedef struct %s \{(.*?)\} %s;" % (struct, struct),
                     txt, re.S).group(1)
    body = re.sub(r"/\*.*?\*/", "", body, flags=re.S)
    names = []
    for decl in body.split(";"):
        decl = decl.strip()
        if not decl:
            continue
        _, rest = decl.split(None, 1)
        names += [n.strip().lstrip("*") for n in rest.split(",")]
    return names


def test_ctypes_structs_follow_the_header():
    import fk_abi
    assert [f for f, _ in fk_abi.Tuning._fields_] == _header_fields(
        "fk_tuning")
    assert [f for f, _ in fk_abi.Stats._fields_] == _header_fields(
        "fk_stats")
    assert [f for f, _ in fk_abi.Info._fields_] == _header_fields("fk_info")
    assert [f for f, _ in fk_abi.Params._fields_] == _header_fields(
        "fk_params")
    assert set(fk_abi.TUNING_FIELDS) >= set(__import__("fk_tune").SPACE)


class FakeEngine:
    def __init__(self, kind, n, q2=65536, p0=6, d=None):
        self.kind, self.n, self.p0 = kind, n, p0
        self.W = 210 if kind == W.DICKSON else 1
        # the line's wheel period: 13# for p0 = 6, 17# for p0 = 7
        self.M = 30030 if p0 == 6 else 510510

    def set_tuning(self, **kw):
        pass


def test_long_intervals_take_the_wider_wheel(monkeypatch):
    import fk_abi
    import fk_batch
    monkeypatch.setattr(fk_abi, "Engine", FakeEngine)
    es = fk_batch.EngineSet()
    need = fk_batch.LONG_PERIODS * 17 * 30030
    short = W.Interval(W.EULER, 8, 10 ** 12, 10 ** 12 + need - 1, 8, 100)
    long_ = W.Interval(W.EULER, 8, 10 ** 12, 10 ** 12 + need, 8, 100)
    assert es.key_for(short)[-1] == fk_batch.P0_NARROW
    assert es.key_for(long_)[-1] == fk_batch.P0_WIDE
    assert es.get(es.key_for(long_)).p0 == 7
    # Dickson lengths count in k; the line is j = k / W
    dk = W.Interval(W.DICKSON, 6, 10 ** 12, 10 ** 12 + need * 210, 6, 14)
    assert es.key_for(dk)[-1] == fk_batch.P0_WIDE
    narrow = fk_batch.EngineSet(wide=False)
    assert narrow.key_for(long_)[-1] == fk_batch.P0_NARROW


def test_serving_chunks_keep_their_footprint_within_the_budget():
    """A chunk's predicted footprint (twice the survival estimate's
    survivors, ENTRY_BYTES each) stays within a quarter of the HBM budget;
    the line-unit cap still applies, and the chunks tile the request."""
    import types
    import fk_serve
    import fk_workloads as W
    loop = fk_serve.ServeLoop.__new__(fk_serve.ServeLoop)
    loop.chunk, loop.hbm_budget = 1 << 30, 1 << 30
    eng = types.SimpleNamespace(survival=1e-2, W=1, NP=6542, M=30030)
    loop._engine = lambda iv: eng
    iv = W.Interval(W.EULER, 6, 10 ** 12, 10 ** 12 + (1 << 34), 6, 64)
    units = loop.chunk_units(iv)
    assert 2 * eng.survival * units * fk_serve.ENTRY_BYTES <= loop.hbm_budget / 4
    cs = loop.chunks(iv)
    assert cs[0].lo == iv.lo and cs[-1].hi == iv.hi
    assert all(a.hi == b.lo for a, b in zip(cs, cs[1:]))
    assert all(c.hi - c.lo <= units for c in cs)
    eng.survival = 1e-9                         # the line-unit cap binds
    assert loop.chunk_units(iv) == loop.chunk
