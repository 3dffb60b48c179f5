"""Slow planner sweep (set GAT_SLOW_TESTS=1): every exact plan variant of
every connected 5- and 6-vertex pattern, interpreted on the CPU, gives the
oracle's count on er60, and the default plans do on ba60 (about 1,600 plans;
a few minutes)."""
import os

import pytest

import plan_model

pytestmark = pytest.mark.skipif(os.environ.get("GAT_SLOW_TESTS") != "1",
                                reason="slow sweep; set GAT_SLOW_TESTS=1")


@pytest.mark.parametrize("graph,max_variants", [("er60", 16), ("ba60", 1)])
def test_all_plan_variants_exact(gat, oracle, golden_graphs, graph, max_variants):
    off, adj = golden_graphs[graph].csr()
    for p in gat.enumerate_patterns(5) + gat.enumerate_patterns(6):
        want = oracle.exact_count(off, adj, p)
        for v in range(min(max_variants, gat.Schedule.variants(p))):
            P = plan_model.parse(gat.Schedule(p, "exact", variant=v).plan_bytes())
            raw, div = plan_model.run(P, off, adj)
            assert raw % div == 0 and raw // div == want, (graph, p, v)
