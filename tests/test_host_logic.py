"""Host-side logic without a GPU: the C ABI loads and exports every declared
symbol, config parsing follows the tuner's formats, graph I/O follows the
reference layouts, generators are deterministic, and both planners give the
oracle's counts when their plans are interpreted on the CPU (plan_model)."""
import json
import re
from pathlib import Path

import numpy as np
import pytest

import plan_model

ROOT = Path(__file__).resolve().parents[1]


def test_library_exports_every_declared_symbol(gat):
    from graphautotune_b200 import _lib

    l = _lib.lib()
    header = (ROOT / "include" / "gat.h").read_text()
    declared = set(re.findall(r"\b(gat_[a-z0-9_]+)\s*\(", header))
    assert len(declared) > 25
    for name in declared:
        assert hasattr(l, name), name
    assert set(_lib.exported_names()) <= declared
    assert "sm_100a" in _lib.version()


def test_config_defaults_and_formats(gat):
    ref = gat.Config.reference_default()
    # include/generated/default_config.hpp:5
    assert (ref.set_search_type, ref.num_blocks, ref.threads_per_block, ref.threads_per_warp,
            ref.max_regs) == (64, 256, 128, 1, 32)
    text = ref.format()
    assert text.startswith("{.vertex_set_config = {.set_search_type = 64")
    ref_fields = Config_fields = ("set_search_type", "set_intersection_type",
                                  "vertex_store_type", "graph_backend_type", "num_blocks",
                                  "threads_per_block", "threads_per_warp", "max_regs")

    def same(a, b):
        return all(getattr(a, f) == getattr(b, f) for f in Config_fields)

    assert same(gat.Config.engine_default().parse(text), ref)
    # the generated header file form (tuning/tuning/common/const.py:15-21)
    hdr = ("#pragma once\n#include \"configs/config.hpp\"\n\nconstexpr Config default_config"
           + text + ";\n")
    assert same(gat.Config.engine_default().parse(hdr), ref) and ref_fields
    # config.json value dict (tuning/tuning/role/driver.py:50-51)
    d = {"vertex_set_config.set_search_type": 2147483647,
         "vertex_set_config.set_intersection_type": "Parallel",
         "vertex_set_config.vertex_store_type": "Array",
         "infra_config.graph_backend_type": "InMemory",
         "engine_config.launch_config.num_blocks": 512,
         "engine_config.launch_config.threads_per_block": 64,
         "engine_config.launch_config.threads_per_warp": 16,
         "engine_config.launch_config.max_regs": 96}
    c = ref.parse(json.dumps(d))
    assert (c.set_search_type, c.num_blocks, c.threads_per_block, c.threads_per_warp,
            c.max_regs) == (2**31 - 1, 512, 64, 16, 96)
    with pytest.raises(gat.GatError):
        ref.parse("{.num_blocks = banana}")


def test_graph_binary_roundtrip_and_text_loader(gat, tmp_path):
    g = gat.Graph.rmat(8, 1500, 0.57, 0.19, 0.19, 3)
    p = tmp_path / "g.bin"
    g.save(str(p))
    h = gat.Graph.load(str(p))
    o1, a1 = g.csr()
    o2, a2 = h.csr()
    assert np.array_equal(o1, o2) and np.array_equal(a1, a2)
    raw = p.read_bytes()
    V = int(np.frombuffer(raw[:4], np.int32)[0])
    E = int(np.frombuffer(raw[4:12], np.int64)[0])
    assert V == len(o1) - 1 and E == len(a1) and len(raw) == 12 + 8 * (V + 1) + 4 * E
    # text layout with sparse ids, a self loop and a duplicate
    # (graph_backend.cuh:23-89 renumbers by increasing id)
    t = tmp_path / "g.txt"
    t.write_text("5 6\n10 20\n20 30\n30 10\n10 10\n20 10\n40 50\n")
    tg = gat.Graph.load(str(t), binary=False)
    off, adj = tg.csr()
    assert off.tolist() == [0, 2, 4, 6, 7, 8]
    assert adj.tolist() == [1, 2, 0, 2, 0, 1, 4, 3]
    with pytest.raises(gat.GatError):
        gat.Graph.load(str(tmp_path / "missing.bin"))
    (tmp_path / "trunc.bin").write_bytes(raw[:40])
    with pytest.raises(gat.GatError):
        gat.Graph.load(str(tmp_path / "trunc.bin"))


def test_from_csr_validates(gat):
    off = np.array([0, 1, 2], np.int64)
    with pytest.raises(gat.GatError):
        gat.Graph.from_csr(off, np.array([1, 1], np.int32))  # self loop at 1
    with pytest.raises(gat.GatError):
        gat.Graph.from_csr(np.array([0, 1, 1], np.int64), np.array([1], np.int32))  # asym.
    g = gat.Graph.from_csr(off, np.array([1, 0], np.int32))
    assert g.info() == (2, 2, 1)


def test_generators_deterministic(gat):
    for mk in (lambda: gat.Graph.erdos_renyi(3000, 12.0, 9),
               lambda: gat.Graph.rmat(12, 40000, 0.57, 0.19, 0.19, 9),
               lambda: gat.Graph.barabasi_albert(3000, 5, 9)):
        a, b = mk(), mk()
        oa, aa = a.csr()
        ob, ab = b.csr()
        assert np.array_equal(oa, ob) and np.array_equal(aa, ab)
    er = gat.Graph.erdos_renyi(10000, 16.0, 1)
    V, E, _ = er.info()
    assert V == 10000 and abs(E / V - 16.0) < 0.5
    ba = gat.Graph.barabasi_albert(1000, 4, 1)
    assert ba.info()[1] == 2 * (10 + (1000 - 5) * 4)


def test_pattern_errors(gat):
    for bad in ("", "0", "01", "0120", "01" * 50 + "1"):
        with pytest.raises(gat.GatError):
            gat.Pattern(bad)
    with pytest.raises(gat.GatError):
        gat.Schedule("0000", "exact")  # two isolated vertices
    assert gat.Pattern("0111101111011110").automorphisms() == 24


def test_planners_on_cpu_model(gat, oracle, golden_naive, golden_schedules, golden_graphs):
    """Interpreting each plan on the CPU gives the oracle's counts."""
    done = 0
    for e in golden_naive:
        if e["graph"] not in ("er60", "k7", "ba60") or len(e["adj"]) > 36:
            continue
        off, adj = golden_graphs[e["graph"]].csr()
        want = e["naive_answer"] // oracle.automorphisms(e["adj"])
        P = plan_model.parse(gat.Schedule(e["adj"], "exact").plan_bytes())
        raw, div = plan_model.run(P, off, adj)
        assert raw % div == 0 and raw // div == want, (e["graph"], e["pattern"])
        sd = golden_schedules[e["adj"]]
        if sd.get("crash"):
            continue
        st, ref_want, _ = oracle.ref_engine(off, adj, sd)
        s = gat.Schedule(e["adj"], "ref")
        if st != 0:
            with pytest.raises(gat.GatError):
                s.plan_bytes()
            continue
        raw, _ = plan_model.run(plan_model.parse(s.plan_bytes()), off, adj)
        assert raw == ref_want, (e["graph"], e["pattern"])
        done += 1
    assert done > 100


def test_lane_last_flag(gat):
    """The lane-per-candidate last level is flagged exactly on plans whose
    last enumerated level stores nothing: each of its sets (at most 8) is a
    count with a father or the candidate's own list, with at most 8 IEP
    slots."""
    named = {"011101110": 1, "0111101111011110": 1, "0111110111110111110111110": 1}
    for p, want in named.items():
        for mode in ("exact", "ref"):
            assert plan_model.parse(gat.Schedule(p, mode).plan_bytes()).lane_last == want
    flagged = 0
    for p in gat.enumerate_patterns(5) + gat.enumerate_patterns(6):
        P = plan_model.parse(gat.Schedule(p, "exact").plan_bytes())
        k = P.basic - 1
        lvl = range(P.l_pbegin[k], P.l_pbegin[k + 1])
        ok = (P.basic >= 2 and 1 <= P.iep_num <= 8 and len(lvl) <= 8
              and all((P.p_kind[q] == plan_model.COUNT and P.p_father[q] >= 0)
                      or P.p_kind[q] == plan_model.ALIAS for q in lvl))
        assert P.lane_last == int(ok), p
        flagged += P.lane_last
    assert flagged > 20


def test_every_schedule_variant_is_exact(gat, oracle, golden_graphs):
    """Data-aware schedule choice may run any of the distinct exact plans of
    the best-ranked vertex orders: each of them, interpreted on the CPU,
    gives the oracle's count."""
    pats = ["0100110110010110110010100", "0001100101010101010011000",
            "0110010101100111010101110", "0001100111010111110111110",
            "011000101100110011000110001010001100"]
    checked = 0
    for name in ("er60", "ba60"):
        off, adj = golden_graphs[name].csr()
        for p in pats:
            n = gat.Schedule.variants(p)
            assert 1 <= n <= 16
            want = oracle.exact_count(off, adj, p)
            plans = set()
            for v in range(n):
                raw_plan = gat.Schedule(p, "exact", variant=v).plan_bytes()
                plans.add(raw_plan)
                raw, div = plan_model.run(plan_model.parse(raw_plan), off, adj)
                assert raw % div == 0 and raw // div == want, (name, p, v)
                checked += 1
            assert len(plans) == n  # variants are distinct plans
            with pytest.raises(gat.GatError):
                gat.Schedule(p, "exact", variant=n)
    assert checked > 20


def test_pm_cli_rejects_unknown_schedule_variant():
    """The pm-compatible CLI builds the schedule before touching the GPU; an
    exact plan variant that does not exist fails with a non-zero exit (which
    the reference's driver reads as an infinite time)."""
    import subprocess

    pm = ROOT / "graphautotune_b200" / "bin" / "pm"
    graph = ROOT / "tests" / "golden" / "graphs" / "er60.bin"
    r = subprocess.run([str(pm), str(graph), "0100110110010110110010100", "--mode", "exact",
                        "--variant", "99"], capture_output=True, text=True, timeout=60)
    assert r.returncode != 0
    assert "schedule variant out of range" in r.stderr
    r = subprocess.run([str(pm)], capture_output=True, text=True, timeout=60)
    assert r.returncode == 2 and "--variant" in r.stderr


def test_config5_patterns_exact_on_cpu_model(gat, oracle, golden_graphs):
    """The learned-cost-model workload's patterns (6-clique, 6-cycle with a
    chord, 7-vertex triangle + path): the first exact plan variants,
    interpreted on the CPU, give the oracle's count."""
    from graphautotune_b200.experiments import C5_PATTERNS

    for name in ("er60",):
        off, adj = golden_graphs[name].csr()
        for pname, p in C5_PATTERNS.items():
            want = oracle.exact_count(off, adj, p)
            for v in range(min(4, gat.Schedule.variants(p))):
                raw, div = plan_model.run(
                    plan_model.parse(gat.Schedule(p, "exact", variant=v).plan_bytes()), off, adj)
                assert raw % div == 0 and raw // div == want, (name, pname, v)
