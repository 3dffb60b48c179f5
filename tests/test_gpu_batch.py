"""Batched persistent launches: every job's count equals the single-job
count, for several launch shapes, with and without CUDA-graph replay, and on
repeated runs of the same prepared batch."""
import json
from pathlib import Path

import pytest

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden" / "graphs"


def test_batch_equals_single_counts(gat):
    graphs = [gat.Graph.load(str(GOLDEN / f"{n}.bin")) for n in ("er60", "ba60", "rmat6", "k7")]
    graphs.append(gat.Graph.rmat(10, 8000, 0.57, 0.19, 0.19, 31))
    hubby = gat.Graph.barabasi_albert(3000, 4, 77)
    hubby.upload(degree_order=True, hub_min_degree=8, hub_max_bytes=1 << 26)
    graphs.append(hubby)
    jobs = [(p, "exact") for p in gat.enumerate_patterns(4)]
    jobs += [(p, "exact") for p in ("0100110110010110110010100", "0111110111110111110111110",
                                    "0000100001000010000111110")]
    jobs += [("0111101111011110", "ref"), ("0100110110010110110010100", "ref")]
    ex = gat.Executor()
    b = gat.Batch()
    want = []
    for g in graphs:
        for p, mode in jobs:
            s = gat.Schedule(p, mode)
            b.add(g, s)
            want.append(ex.count(g, s).count)
    assert len(b) == len(want)
    shapes = [dict(), dict(threads_per_warp=8, threads_per_block=128, chunk=1),
              dict(threads_per_warp=1, threads_per_block=64, chunk=32, num_blocks=40)]
    for shape in shapes:
        cfg = gat.Config.engine_default()
        for k, v in shape.items():
            setattr(cfg, k, v)
        for cuda_graph in (True, False):
            b.prepare(cfg, cuda_graph=cuda_graph)
            for _ in range(2):
                r = b.run()
                assert r.kernel_ms > 0 and r.tile == (shape.get("threads_per_warp") or 32)
                assert b.counts() == want, (shape, cuda_graph)


def test_sliced_jobs_sum_to_whole(gat):
    """Jobs added as slices of their work queue (the autotuner's sample
    batches) report raw totals that add up, over all slices, to the whole
    job's raw total; the executor's shard counts agree slice by slice."""
    graphs = [gat.Graph.rmat(11, 1 << 14, 0.57, 0.19, 0.19, 31),
              gat.Graph.barabasi_albert(3000, 9, 32)]
    pats = ["0111101111011110", "0100110110010110110010100", "0110010101100111010101110"]
    P = 5
    b = gat.Batch()
    for gr in graphs:
        for p in pats:
            s = gat.Schedule(p, "exact")
            for k in range(P):
                b.add_shard(gr, s, k, P)
    b.prepare(gat.Config.engine_default(), cuda_graph=True)
    b.run()
    raw = b.counts()
    ex = gat.Executor(gat.Config.engine_default())
    i = 0
    for gr in graphs:
        for p in pats:
            s = gat.Schedule(p, "exact")
            whole = ex.count(gr, s)
            parts = raw[i:i + P]
            assert parts == [ex.count_shard(gr, s, k, P)[0] for k in range(P)]
            assert sum(parts) == whole.raw_sum
            assert sum(parts) // whole.divisor == whole.count
            i += P


def test_tune_count_measures_points_and_keeps_the_count(gat, tmp_path):
    """tuner.tune_count: the default point and proposals, each measured by
    the count's device time, all giving the same count; record.json and
    best_config.json are written beside each other."""
    from graphautotune_b200 import tuner

    g = gat.Graph.rmat(12, 1 << 15, 0.57, 0.19, 0.19, 4)
    s = gat.Schedule("0100110110010110110010100", "exact")  # the house: plan interpreter
    rec = tmp_path / "tuning_results" / "record.json"
    cfg, hist, counts = tuner.tune_count(g, s, budget=6, record=str(rec))
    assert len(hist) == 6 and len(set(counts.values())) == 1
    assert hist[0][0] == tuner.fingerprint(tuner.default_point())
    best = json.loads((rec.parent / "best_config.json").read_text())
    assert best[1] == min(y for _, y in hist)
    assert gat.Executor(cfg).count(g, s).count == next(iter(counts.values()))
