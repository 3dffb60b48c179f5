"""Pins the CPU oracle to the reference's own answers (no GPU).

  * oracle naive matcher == reference naive_pm binary Answer (golden file)
  * oracle backtracking counter == the same
  * the reference's only numeric unit test: |{1..30} n {2,4,..,60}| = 15
    (tests/test_vertex_set.cu:44-48,76)
  * |Aut| == the reference Schedule's multiplicity
  * reference-engine restatement: triangle/K4/K5 count 3x/4x/5x the
    subgraphs and the house (P2 labelling) exactly once
    (core/schedule.hpp:827-831 keeps only restrictions inside the basic
    vertices; scripts/run_pattern_matching.sh:16-17 for P2)
"""
import numpy as np
import pytest


def test_intersection_pin(oracle):
    a = np.arange(1, 31, dtype=np.int32)
    b = np.arange(2, 61, 2, dtype=np.int32)
    assert oracle.intersect_size(a, b) == 15


def test_naive_and_backtrack_match_reference_binary(oracle, golden_naive, golden_graphs):
    assert len(golden_naive) > 300
    for e in golden_naive:
        off, adj = golden_graphs[e["graph"]].csr()
        want = e["naive_answer"]
        if e["graph"] in ("er60", "k5", "k7", "rmat6", "ba60") and len(e["adj"]) <= 25:
            assert oracle.naive_labelled(off, adj, e["adj"]) == want, e
        assert oracle.backtrack_labelled(off, adj, e["adj"]) == want, e


def test_automorphisms_match_reference(oracle, golden_schedules):
    for p, sd in golden_schedules.items():
        if sd.get("crash"):
            continue
        assert oracle.automorphisms(p) == sd["aut"], p


@pytest.mark.parametrize("name,factor", [("triangle", 3), ("k4", 4), ("k5", 5), ("house_p2", 1)])
def test_ref_engine_known_multiples(oracle, golden_naive, golden_schedules, golden_graphs,
                                    name, factor):
    seen = 0
    for e in golden_naive:
        if e["pattern"] != name:
            continue
        off, adj = golden_graphs[e["graph"]].csr()
        st, tot, _ = oracle.ref_engine(off, adj, golden_schedules[e["adj"]])
        assert st == 0
        exact = e["naive_answer"] // oracle.automorphisms(e["adj"])
        assert tot == factor * exact, (e["graph"], tot, exact)
        seen += 1
    assert seen >= 5


def test_ref_engine_root_ranges_add_up(oracle, golden_schedules, golden_graphs):
    off, adj = golden_graphs["er200"].csr()
    V = len(off) - 1
    for p in ("011101110", "0101101001011010", "0100110110010110110010100"):
        sd = golden_schedules[p]
        st, whole, balg = oracle.ref_engine(off, adj, sd)
        parts = [oracle.ref_engine(off, adj, sd, roots=(lo, hi))[1]
                 for lo, hi in ((0, 7), (7, 100), (100, V))]
        assert st == 0 and sum(parts) == whole and balg > 0


def test_ref_engine_flags_undefined_schedules(oracle, golden_schedules, golden_graphs):
    off, adj = golden_graphs["k7"].csr()
    flagged = 0
    for p, sd in golden_schedules.items():
        if sd.get("crash"):
            continue
        st, _, _ = oracle.ref_engine(off, adj, sd)
        if sd["ub_read"]:
            flagged += st in oracle.REF_UNDEFINED
    assert flagged > 0


def test_oracle_ref_engine_equals_reference_binary(oracle, golden_schedules, golden_graphs,
                                                   golden_ref_engine):
    """The CPU restatement of the reference engine's per-unit rules gives the
    reference engine's own answers (its CUDA build, run on a B200), for every
    pattern up to 5 vertices on er60, k7 and rmat6 and the triangle on the
    config-1 graph."""
    checked = 0
    for e in golden_ref_engine:
        sd = golden_schedules[e["adj"]]
        assert not sd.get("crash")
        off, adj = golden_graphs[e["graph"]].csr()
        st, got, _ = oracle.ref_engine(off, adj, sd)
        assert st == 0, (e["graph"], e["pattern"])
        assert got == e["ref_engine_answer"], (e["graph"], e["pattern"], got)
        checked += 1
    assert checked >= 140


def test_restricted_counts_of_exact_plans_match_reference_binary(gat, oracle, golden_naive,
                                                                 golden_graphs):
    """The full-size pins rest on this: for every exact plan, labelled
    embeddings of the plan's vertex order under its order conditions, summed
    over all roots and divided by the plan's divisor, give the reference
    naive matcher's Answer / |Aut| on every golden graph."""
    checked = 0
    plans = {}
    for e in golden_naive:
        n = int(round(len(e["adj"]) ** 0.5))
        if n < 3 or e["graph"] == "c1_er10000" and n > 3:
            continue
        if e["adj"] not in plans:
            try:
                d = gat.Schedule(e["adj"], "exact").dump()
            except gat.GatError:
                continue  # disconnected patterns have no exact plan
            plans[e["adj"]] = (*oracle.plan_conditions(d), d["divisor"])
        q, less, div = plans[e["adj"]]
        off, adj = golden_graphs[e["graph"]].csr()
        raw = oracle.restricted_labelled(off, adj, q, less)
        assert raw % div == 0 and raw // div == e["naive_answer"] // oracle.automorphisms(e["adj"]), e
        checked += 1
    assert checked > 250


def test_c4_rooted_counts_match_reference_binary(oracle, golden_naive, golden_graphs):
    """4-cycles counted at their smallest and at their largest vertex both
    give naive_pm's Answer / 8, and root ranges add up."""
    seen = 0
    for e in golden_naive:
        if e["adj"] != "0101101001011010":
            continue
        off, adj = golden_graphs[e["graph"]].csr()
        want = e["naive_answer"] // 8
        assert oracle.c4_rooted(off, adj) == want
        assert oracle.c4_rooted(off, adj, at_largest=True) == want
        V = len(off) - 1
        cuts = [0, V // 3, V // 2, V]
        assert sum(oracle.c4_rooted(off, adj, roots=(a, b))
                   for a, b in zip(cuts, cuts[1:])) == want
        seen += 1
    assert seen >= 5


def test_degree_order_restatement(gat, oracle, golden_graphs):
    """The oracle's relabel (decreasing degree, ties by id) is a relabelling:
    same degree sequence sorted, same counts."""
    off, adj = golden_graphs["ba60"].csr()
    no, na = oracle.degree_order(off, adj)
    deg = np.diff(off)
    assert (np.diff(no) == np.sort(deg)[::-1]).all()
    for p in ("011101110", "0101101001011010", "0100110110010110110010100"):
        assert oracle.exact_count(no, na, p) == oracle.exact_count(off, adj, p)
