"""World-size-2 test of the sharded-count host logic on CPU (gloo): each rank
counts its slice of the first-vertex range with the oracle's reference-engine
restatement, the ranks combine with graphautotune_b200.dist.reduce_shards,
and the result equals the single-process count.  Also checks the shard
arithmetic covers the work queue exactly once."""
import os
import sys
from pathlib import Path

import pytest
import torch.multiprocessing as mp

ROOT = Path(__file__).resolve().parents[1]


def test_shard_bounds_partition():
    from graphautotune_b200.dist import shard_bounds

    for total in (0, 1, 7, 1000, 15700152):
        for world in (1, 2, 3, 8):
            spans = [shard_bounds(total, r, world) for r in range(world)]
            assert spans[0][0] == 0 and spans[-1][1] == total
            assert all(a[1] == b[0] for a, b in zip(spans, spans[1:]))
    with pytest.raises(ValueError):
        shard_bounds(10, 2, 2)


def _worker(rank, world, port, out_path):
    sys.path.insert(0, str(ROOT))
    sys.path.insert(0, str(ROOT / "oracle"))
    import json

    import torch.distributed as dist

    import graphautotune_b200 as g
    import pyoracle
    from graphautotune_b200.dist import reduce_shards, shard_bounds

    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        sched = {}
        for line in (ROOT / "tests/golden/ref_schedules.jsonl").read_text().splitlines():
            d = json.loads(line)
            sched[d["pattern"]] = d
        gr = g.Graph.load(str(ROOT / "tests/golden/graphs/er200.bin"))
        off, adj = gr.csr()
        V = len(off) - 1
        pats = ["011101110", "0101101001011010", "0100110110010110110010100"]
        lo, hi = shard_bounds(V, rank, world)
        raws = []
        for p in pats:
            st, raw, _ = pyoracle.ref_engine(off, adj, sched[p], roots=(lo, hi), threads=1)
            assert st == 0
            raws.append(raw)
        counts, ms = reduce_shards(raws, [1] * len(pats), float(rank + 1))
        if rank == 0:
            whole = [pyoracle.ref_engine(off, adj, sched[p], threads=1)[1] for p in pats]
            Path(out_path).write_text(json.dumps({"counts": counts, "whole": whole, "ms": ms}))
    finally:
        dist.destroy_process_group()


def test_two_rank_gloo_shards_sum_to_whole(tmp_path):
    import json
    import socket

    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    out = tmp_path / "result.json"
    mp.start_processes(_worker, args=(2, port, str(out)), nprocs=2, join=True,
                       start_method="spawn")
    r = json.loads(out.read_text())
    assert r["counts"] == r["whole"] and r["ms"] == 2.0
