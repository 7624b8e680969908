"""The multi-rank path on CPU: two gloo ranks, as bench.py runs N GPUs.

Each rank sweeps its own shard with no data-path collective; the only
cross-rank traffic is the barrier and the max over ranks of the timed
region.  Here two processes (world size 2, gloo) take disjoint shards of
one interval list, sweep clipped pieces of them with the CPU oracle, and
check that the shards cover the list exactly once, that the union of the
per-rank results equals the single-process result, and that the max-over-
ranks reduction returns the slower rank's time.
"""

import os
import pathlib
import sys

import pytest

ROOT = pathlib.Path(__file__).resolve().parents[1]


def _rank_main(rank, world, port, out_dir):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port),
                      RANK=str(rank), WORLD_SIZE=str(world),
                      LOCAL_RANK=str(rank))
    for p in (str(ROOT), str(ROOT / "first-knowns_b200")):
        sys.path.insert(0, p)
    import json
    import bench
    import fk_workloads as W
    from oracle import sweep
    dist = bench.Dist(world, rank, backend="gloo")
    ivs = W.mixed_batch(24, W.SEED)
    mine = W.shard(ivs, rank, world)
    res = []
    for iv in mine:
        hi = min(iv.hi, iv.lo + (1 << 16))
        if iv.kind == W.AP:
            hi = iv.lo + max(30, (hi - iv.lo) // 30 * 30)
        res.append([ivs.index(iv), sweep.hunt_interval(
            iv.kind, iv.n, iv.lo, hi, iv.threshold, iv.cap, iv.q2, iv.d)])
    dist.barrier()
    mx = dist.max(1.0 + rank)
    with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as f:
        json.dump({"ids": [i for i, _ in res], "res": res, "max": mx}, f)
    dist.close()


def test_two_gloo_ranks_shard_and_reduce(tmp_path):
    import socket
    import torch.multiprocessing as tmp
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    tmp.start_processes(_rank_main, args=(2, port, str(tmp_path)), nprocs=2,
                        join=True, start_method="spawn")
    import json
    sys.path.insert(0, str(ROOT / "first-knowns_b200"))
    import fk_workloads as W
    from oracle import sweep
    r0 = json.loads((tmp_path / "rank0.json").read_text())
    r1 = json.loads((tmp_path / "rank1.json").read_text())
    assert set(r0["ids"]).isdisjoint(r1["ids"])
    assert sorted(r0["ids"] + r1["ids"]) == list(range(24))
    assert r0["max"] == r1["max"] == 2.0
    ivs = W.mixed_batch(24, W.SEED)
    got = {i: [tuple(h) for h in r] for i, r in r0["res"] + r1["res"]}
    for i in (0, 5, 11):
        iv = ivs[i]
        hi = min(iv.hi, iv.lo + (1 << 16))
        if iv.kind == W.AP:
            hi = iv.lo + max(30, (hi - iv.lo) // 30 * 30)
        want = sweep.hunt_interval(iv.kind, iv.n, iv.lo, hi, iv.threshold,
                                   iv.cap, iv.q2, iv.d)
        assert got[i] == [tuple(h) for h in want]
