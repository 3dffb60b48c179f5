"""GPU parity: libgat counts through the C ABI against the oracle and the
reference's own answers.

  * exact mode == naive_pm Answer / |Aut| (reference binary, golden file)
  * ref mode   == the reference engine's per-unit rules (oracle restatement),
                  and GAT_ERR_UNDEFINED exactly where the reference reads
                  uninitialised state or crashes
  * every launch shape (tile width, search type, chunk) gives the same count
"""
import pytest

from graphautotune_b200._lib import GAT_ERR_UNDEFINED, GatError

pytestmark = pytest.mark.gpu

CONFIGS = [
    dict(threads_per_warp=32, threads_per_block=256, num_blocks=0, set_search_type=0, chunk=8),
    dict(threads_per_warp=8, threads_per_block=128, num_blocks=0, set_search_type=0, chunk=3),
    dict(threads_per_warp=4, threads_per_block=64, num_blocks=7, set_search_type=16, chunk=1),
    # the reference's generated default_config.hpp
    dict(threads_per_warp=1, threads_per_block=128, num_blocks=256, set_search_type=64, chunk=16),
]


def _executor(gat, **kw):
    c = gat.Config.engine_default()
    for k, v in kw.items():
        setattr(c, k, v)
    return gat.Executor(c)


@pytest.fixture(scope="module")
def executors(gat):
    return [_executor(gat, **c) for c in CONFIGS]


def test_exact_matches_naive_matcher(gat, oracle, golden_naive, golden_graphs, executors):
    checked = 0
    for e in golden_naive:
        g = golden_graphs[e["graph"]]
        s = gat.Schedule(e["adj"], "exact")
        aut = oracle.automorphisms(e["adj"])
        assert e["naive_answer"] % aut == 0
        want = e["naive_answer"] // aut
        for ex in executors:
            got = ex.count(g, s).count
            assert got == want, (e["graph"], e["pattern"], got, want)
        checked += 1
    assert checked > 300


def test_ref_mode_matches_reference_engine_rules(gat, oracle, golden_schedules, golden_naive,
                                                  golden_graphs, executors):
    checked = undefined = 0
    seen = set()
    for e in golden_naive:
        key = (e["graph"], e["adj"])
        if key in seen:
            continue
        seen.add(key)
        sd = golden_schedules[e["adj"]]
        g = golden_graphs[e["graph"]]
        off, adj = g.csr()
        if sd.get("crash"):
            with pytest.raises(GatError) as ei:
                executors[0].count(g, gat.Schedule(e["adj"], "ref"))
            assert ei.value.status == GAT_ERR_UNDEFINED
            undefined += 1
            continue
        st, want, _ = oracle.ref_engine(off, adj, sd)
        s = gat.Schedule(e["adj"], "ref")
        if st in oracle.REF_UNDEFINED:
            with pytest.raises(GatError) as ei:
                executors[0].count(g, s)
            assert ei.value.status == GAT_ERR_UNDEFINED
            undefined += 1
            continue
        assert st == 0
        for ex in executors:
            got = ex.count(g, s).count
            assert got == want, (e["graph"], e["pattern"], got, want)
        checked += 1
    assert checked > 200 and undefined > 0


# Sized so the exhaustive CPU enumeration finishes in seconds.
MEDIUM = [
    ("er", (2000, 10.0), 5),
    ("rmat", (9, 3072), 6),
    ("ba", (2000, 3), 7),
]
NAMED = ["011101110", "0111101111011110", "0101101001011010",
         "0100110110010110110010100", "0111110111110111110111110"]


def _graph(gat, kind, params, seed):
    if kind == "er":
        return gat.Graph.erdos_renyi(*params, seed)
    if kind == "rmat":
        return gat.Graph.rmat(params[0], params[1], 0.57, 0.19, 0.19, seed)
    return gat.Graph.barabasi_albert(*params, seed)


@pytest.mark.parametrize("kind,params,seed", MEDIUM)
def test_medium_graphs_exact_and_ref(gat, oracle, golden_schedules, kind, params, seed,
                                     executors):
    g = _graph(gat, kind, params, seed)
    off, adj = g.csr()
    pats = NAMED + gat.enumerate_patterns(5)
    for p in pats:
        want = oracle.exact_count(off, adj, p)
        s = gat.Schedule(p, "exact")
        for ex in executors[:2]:
            assert ex.count(g, s).count == want, (kind, p)
        sd = golden_schedules.get(p)
        if sd is None or sd.get("crash"):
            continue
        st, ref_want, _ = oracle.ref_engine(off, adj, sd)
        if st != 0:
            continue
        assert executors[0].count(g, gat.Schedule(p, "ref")).count == ref_want, (kind, p)


def test_ref_mode_larger_rmat(gat, oracle, golden_schedules, executors):
    """Reference-engine rules on a power-law graph with hubs (R-MAT scale 12)."""
    g = gat.Graph.rmat(12, 1 << 15, 0.57, 0.19, 0.19, 9)
    off, adj = g.csr()
    for p in NAMED:
        st, want, _ = oracle.ref_engine(off, adj, golden_schedules[p])
        assert st == 0
        for ex in executors[:3]:
            assert ex.count(g, gat.Schedule(p, "ref")).count == want, p


def test_hub_bitmap_path(gat, oracle, golden_schedules, executors):
    """Hub bitmaps built for every vertex of degree >= 4 (most of the graph):
    exact and reference-mode counts still equal the oracle's, with and
    without bitmaps, on both device copies."""
    no_bm = _executor(gat, **{**CONFIGS[0], "hub_bitmaps": 0})
    for kind, params, seed in MEDIUM:
        g = _graph(gat, kind, params, seed)
        g.upload(degree_order=True, hub_min_degree=4, hub_max_bytes=1 << 28)
        assert g.hubs(True) > 0 and g.hubs(False) > 0
        off, adj = g.csr()
        for p in NAMED + ["0101110101010101010011000"]:
            want = oracle.exact_count(off, adj, p)
            s = gat.Schedule(p, "exact")
            for ex in (executors[0], executors[1], executors[3], no_bm):
                assert ex.count(g, s).count == want, (kind, p)
            sd = golden_schedules.get(p)
            if sd is None or sd.get("crash"):
                continue
            st, ref_want, _ = oracle.ref_engine(off, adj, sd)
            if st != 0:
                continue
            for ex in (executors[0], executors[2], no_bm):
                assert ex.count(g, gat.Schedule(p, "ref")).count == ref_want, (kind, p)


def test_four_cycle_wedge_kernel_equals_plan(gat, oracle, golden_graphs):
    """The exact 4-cycle count has a dedicated wedge-aggregation kernel; it
    must equal the oracle and the generic plan (special_kernels=0), for
    whole graphs, root ranges and shards, and on repeated calls (its counter
    rows must come back zeroed)."""
    c4 = "0101101001011010"
    s = gat.Schedule(c4, "exact")
    wedge = [_executor(gat, threads_per_warp=t, threads_per_block=b, chunk=c)
             for t, b, c in ((32, 256, 8), (8, 128, 1), (4, 64, 32))]
    plan = _executor(gat, special_kernels=0)
    graphs = list(golden_graphs.values()) + [gat.Graph.rmat(12, 1 << 15, 0.57, 0.19, 0.19, 5),
                                             gat.Graph.barabasi_albert(4000, 6, 8)]
    for g in graphs:
        off, adj = g.csr()
        want = oracle.exact_count(off, adj, c4) if len(off) < 5000 else plan.count(g, s).count
        assert plan.count(g, s).count == want
        for ex in wedge:
            for _ in range(2):
                assert ex.count(g, s).count == want
        V = len(off) - 1
        bounds = [0, V // 5, V // 2, V]
        assert sum(wedge[0].count_range(g, s, a, b)[0] for a, b in zip(bounds, bounds[1:])) \
            == want
        assert sum(wedge[1].count_shard(g, s, r, 3)[0] for r in range(3)) == want


def test_relabelling_and_sharding_invariance(gat, executors):
    """Size-independent properties: the exact count does not depend on the
    vertex ids (degree-ordered vs given ids), and root-range shards sum to
    the whole."""
    g1 = gat.Graph.rmat(13, 1 << 16, 0.57, 0.19, 0.19, 21)
    g2 = gat.Graph.rmat(13, 1 << 16, 0.57, 0.19, 0.19, 21)
    g1.upload(degree_order=True)
    g2.upload(degree_order=False)
    V = g1.v_cnt()
    for p in NAMED:
        s = gat.Schedule(p, "exact")
        a = executors[0].count(g1, s)
        b = executors[1].count(g2, s)
        assert a.count == b.count, p
        bounds = [0, 1, 17, V // 3, V // 2, V - 5, V]
        raw = sum(executors[0].count_range(g1, s, lo, hi)[0]
                  for lo, hi in zip(bounds, bounds[1:]))
        assert raw == a.raw_sum and raw // a.divisor == a.count, p


def test_lane_last_level_equals_tile_path(gat, oracle, golden_schedules):
    """The one-candidate-per-lane last level (special_kernels=2: the lane
    path without the dedicated 4-cycle and clique kernels) gives the same
    counts and the same algorithmic byte totals as the tile-cooperative path
    (special_kernels=0), on every tile width, with and without hub bitmaps,
    in both modes."""
    shapes = ((32, 256, 8), (8, 128, 1), (1, 128, 16))
    lanes = [_executor(gat, threads_per_warp=t, threads_per_block=b, chunk=c,
                       special_kernels=2) for t, b, c in shapes]
    tiles = [_executor(gat, threads_per_warp=t, threads_per_block=b, chunk=c,
                       special_kernels=0) for t, b, c in shapes]
    pats = NAMED + gat.enumerate_patterns(5)
    graphs = [_graph(gat, *m) for m in MEDIUM]
    hubby = gat.Graph.rmat(12, 1 << 15, 0.57, 0.19, 0.19, 9)
    hubby.upload(degree_order=True, hub_min_degree=8, hub_max_bytes=1 << 28)
    graphs.append(hubby)
    for g in graphs:
        off, adj = g.csr()
        for p in pats:
            for mode in ("exact", "ref"):
                s = gat.Schedule(p, mode)
                if mode == "ref":
                    sd = golden_schedules.get(p)
                    if sd is None or sd.get("crash") or oracle.ref_engine(off, adj, sd)[0] != 0:
                        continue
                want = None
                for a, b in zip(lanes, tiles):
                    ra, rb = a.count(g, s, balg=True), b.count(g, s, balg=True)
                    assert ra.count == rb.count, (p, mode)
                    assert ra.balg_bytes == rb.balg_bytes, (p, mode)
                    want = ra.count if want is None else want
                    assert ra.count == want, (p, mode)
                if mode == "exact" and len(off) <= 2001:
                    assert want == oracle.exact_count(off, adj, p), p


def test_ref_mode_equals_reference_binary(gat, golden_graphs, golden_ref_engine, executors):
    """GPU reference-compatible counts equal the reference engine's own
    answers (its CUDA build run on a B200) on the golden graphs."""
    for e in golden_ref_engine:
        g = golden_graphs[e["graph"]]
        s = gat.Schedule(e["adj"], "ref")
        for ex in executors:
            assert ex.count(g, s).count == e["ref_engine_answer"], (e["graph"], e["pattern"])


def _bipartite_with_ring(gat, n: int):
    """K_{2,n} (vertices 0 and 1 joined to 2 .. n+1) plus a ring through the
    n leaves: vertices 0 and 1 share n >= 2^16 neighbours."""
    import numpy as np

    leaves = np.arange(2, n + 2, dtype=np.int64)
    u = np.concatenate([np.zeros(n, np.int64), np.ones(n, np.int64), leaves])
    v = np.concatenate([leaves, leaves, np.roll(leaves, -1)])
    V = n + 2
    key = np.unique(np.concatenate([u * V + v, v * V + u]))
    off = np.zeros(V + 1, np.int64)
    np.cumsum(np.bincount(key // V, minlength=V), out=off[1:])
    return gat.Graph.from_csr(off, (key % V).astype(np.int32))


def test_four_cycle_kernel_paths(gat, oracle):
    """The 4-cycle kernels' paths: warp tables for light roots, roots
    deferred to the CTA table, CTA windows over the ids (one window on a
    dense graph, several when V exceeds a window), the tail of a root's
    wedges through the CTA table, roots with more upper neighbours than a
    CTA has threads (up to 15,544 on the scale-17 R-MAT), 32-bit window
    counters when a pair of vertices shares 2^16 or more neighbours, odd V;
    repeated calls with one executor across graphs, and shards.  Each count equals the host oracle's count at each
    cycle's largest vertex and the schedule plan's."""
    c4 = "0101101001011010"
    s = gat.Schedule(c4, "exact")
    plan = _executor(gat, special_kernels=0)
    cases = [gat.Graph.erdos_renyi(600, 300.0, 11),
             gat.Graph.barabasi_albert(120000, 12, 12),
             gat.Graph.rmat(14, 1 << 17, 0.57, 0.19, 0.19, 13),
             gat.Graph.barabasi_albert(3001, 8, 21),
             _bipartite_with_ring(gat, 70000),
             gat.Graph.rmat(17, 1 << 21, 0.57, 0.19, 0.19, 17)]
    assert cases[1].info()[2] > 1024 and cases[4].info()[2] >= 1 << 16
    wants = []
    for g in cases:
        off, adj = g.csr()
        want = oracle.c4_rooted(off, adj, at_largest=True)
        assert plan.count(g, s).count == want
        wants.append(want)
    assert wants[4] >= 70000 * 69999 // 2
    shared = _executor(gat)
    for _ in range(2):
        for g, want in zip(cases, wants):
            assert shared.count(g, s).count == want
    for tile, block in ((32, 256), (8, 128)):
        ex = _executor(gat, threads_per_warp=tile, threads_per_block=block)
        for g, want in zip(cases, wants):
            assert ex.count(g, s).count == want
    for g, want in zip(cases, wants):
        assert sum(shared.count_shard(g, s, k, 5)[0] for k in range(5)) == want


def test_full_size_workload_graph_against_oracle(gat):
    """The bench's graph at full size (R-MAT 2^20, 2^24 samples, seed 2):
    GPU reference-compatible 4-clique = the oracle's restatement of the
    reference engine over the whole graph (tests/golden/c2_oracle.json,
    made on the host by make_c2_oracle.py) = 4 x the GPU exact count; GPU
    exact 4-cycle = the host's whole-graph count by another rooting."""
    import json
    from pathlib import Path

    pins = json.loads((Path(__file__).parent / "golden" / "c2_oracle.json").read_text())
    gspec = pins["graph"]
    g = gat.Graph.rmat(gspec["scale"], gspec["samples"], *gspec["abc"], gspec["seed"])
    assert g.info()[:2] == (gspec["V"], gspec["E"])
    ex = gat.Executor(gat.Config.engine_default())
    k4 = pins["k4"]
    exact = ex.count(g, gat.Schedule(k4["pattern"], "exact")).count
    ref = ex.count(g, gat.Schedule(k4["pattern"], "ref")).count
    assert ref == k4["ref_engine_oracle"]
    assert ref == 4 * exact
    # The 4-cycle: the wedge kernels (cycles rooted at their smallest vertex
    # of the degree-ordered copy) and the plan path against the host count
    # rooted at each cycle's largest vertex on the graph's own ids.
    c4 = pins["c4"]
    s = gat.Schedule(c4["pattern"], "exact")
    assert ex.count(g, s).count == c4["exact_at_largest_vertex"]
    plain = gat.Config.engine_default()
    plain.special_kernels = 0
    assert gat.Executor(plain).count(g, s).count == c4["exact_at_largest_vertex"]


def test_schedule_variants_count_the_same(gat, oracle):
    """Every exact plan variant gives the same count on the GPU (and the
    oracle's on a small graph); the slice-timed pick returns one of them."""
    from graphautotune_b200 import tuner

    ex = _executor(gat, **CONFIGS[0])
    small = gat.Graph.barabasi_albert(800, 4, 17)
    big = gat.Graph.rmat(13, 1 << 16, 0.57, 0.19, 0.19, 18)
    off, adj = small.csr()
    for p in ("0100110110010110110010100", "0001100101010101010011000",
              "011000101100110011000110001010001100"):
        n = gat.Schedule.variants(p)
        want_small = oracle.exact_count(off, adj, p)
        counts = set()
        for v in range(n):
            s = gat.Schedule(p, "exact", variant=v)
            assert ex.count(small, s).count == want_small, (p, v)
            counts.add(ex.count(big, s).count)
        assert len(counts) == 1, (p, counts)
        best, timings = tuner.pick_schedule(ex, big, p, parts=16, slices=2)
        assert len(timings) == n and ex.count(big, best).count in counts


def test_config5_patterns_on_small_graphs(gat, oracle, golden_graphs):
    """The learned-cost-model workload's patterns (6-clique, 6-cycle with a
    chord, 7-vertex triangle + path) counted by the engine on small graphs:
    exact counts equal the oracle's, with the dedicated kernels and with the
    plan interpreter, on the default launch shape and five random points of
    the tuner's space."""
    import random

    from graphautotune_b200 import tuner
    from graphautotune_b200.experiments import C5_PATTERNS

    rng = random.Random(5)
    shapes = [tuner.default_point()] + [tuner.random_point(rng) for _ in range(5)]
    exs = [gat.Executor(tuner.to_config(d)) for d in shapes]
    plain = _executor(gat, special_kernels=0)
    graphs = [golden_graphs["er60"], golden_graphs["ba60"], golden_graphs["k7"],
              golden_graphs["rmat6"], gat.Graph.barabasi_albert(400, 3, 11)]
    for g in graphs:
        off, adj = g.csr()
        for name, p in C5_PATTERNS.items():
            want = oracle.exact_count(off, adj, p)
            s = gat.Schedule(p, "exact")
            assert plain.count(g, s).count == want, (name, "plan")
            for ex in exs:
                assert ex.count(g, s).count == want, (name, ex)
