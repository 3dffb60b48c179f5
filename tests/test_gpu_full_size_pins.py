"""Parity at the benchmark configurations' full sizes.

Exact counts are sums over roots.  tests/golden/full_size_pins.json (made on
the host by make_full_size_pins.py) holds, for every configuration pattern,
root ranges spread over the degree order (hub roots included) and the CPU
oracle's count on each: labelled embeddings of the plan's vertex order under
its order conditions, by plain backtracking.  Here the engine counts the same
roots of the same graph with count_range and must give exactly those totals,
on the default path and with the dedicated kernels switched off.  The
4-cycle's wedge kernels are also checked against the oracle's count of the
cycles whose smallest vertex lies in each range.

The device's degree-ordered copy must have the oracle relabel's checksum, so
both sides count on the same ids.
"""
import hashlib
import json
from pathlib import Path

import pytest

pytestmark = pytest.mark.gpu

PINS = json.loads((Path(__file__).parent / "golden" / "full_size_pins.json").read_text())
ABC = (0.57, 0.19, 0.19)


def _graph(gat, spec):
    # built on the device (identical to the host generators' graphs; the
    # digest check below compares the result with the oracle's copy)
    if spec["kind"] == "rmat":
        return gat.Graph.rmat(spec["scale"], spec["samples"], *ABC, spec["seed"], device=True)
    return gat.Graph.barabasi_albert(spec["n"], spec["m"], spec["seed"], device=True)


def _digest(off, adj) -> str:
    h = hashlib.blake2b(digest_size=16)
    h.update(memoryview(off).cast("B"))
    h.update(memoryview(adj).cast("B"))
    return h.hexdigest()


@pytest.mark.parametrize("workload", sorted(PINS))
def test_full_size_root_ranges_match_oracle(gat, workload):
    w = PINS[workload]
    g = _graph(gat, w["graph"])
    V, E, _ = g.info()
    assert (V, E) == (w["V"], w["E"])
    g.upload(degree_order=True)
    assert _digest(*g.ordered_csr()) == w["ordered_digest"]
    ex = gat.Executor(gat.Config.engine_default())
    plain = gat.Config.engine_default()
    plain.special_kernels = 0
    ex_plain = gat.Executor(plain)
    checked = 0
    for name, p in w["patterns"].items():
        s = gat.Schedule(p["adj"], "exact", stats_graph=g)
        d = s.dump()
        assert (d["perm"], d["restrictions"], d["divisor"]) == \
            (p["perm"], p["restrictions"], p["divisor"]), name
        for b, e, want in p["plan_ranges"]:
            got, _ = ex_plain.count_range(g, s, b, e)
            assert got == want, (workload, name, b, e, "plan", got, want)
            if "c4_ranges" not in p:
                got, _ = ex.count_range(g, s, b, e)
                assert got == want, (workload, name, b, e, got, want)
            checked += 1
        for b, e, want in p.get("c4_ranges", []):
            got, _ = ex.count_range(g, s, b, e)
            assert got == want, (workload, name, b, e, "wedge kernels", got, want)
            checked += 1
    assert checked >= 8
