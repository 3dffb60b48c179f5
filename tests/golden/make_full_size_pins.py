"""Full-size parity pins for every benchmark configuration's patterns,
computed on the host by the CPU oracle and written to
tests/golden/full_size_pins.json.

An exact count is a sum over roots, so a GPU count over a root range can be
checked at full size on root ranges the CPU can afford.  For each workload
graph (generated by libgat's seeded generators) and each pattern:

  * the graph is relabelled by decreasing degree by the oracle's own
    restatement (oracle_degree_order); the GPU test compares a checksum of
    the device's degree-ordered copy with the one stored here, so both sides
    count on the same ids;
  * the exact schedule the engine builds for that graph is recorded (vertex
    order, order conditions, divisor), and for root ranges spread over the
    degree order - always including the hub roots [0, h) - the oracle counts
    the labelled embeddings of the plan's vertex order that satisfy its
    conditions (oracle_restricted_labelled: plain backtracking, nothing of
    the engine's prefix sets or inclusion-exclusion).  The GPU's
    count_range over the same roots must give exactly this undivided total;
  * for the 4-cycle, whose dedicated kernels root each cycle at its smallest
    vertex, the oracle's oracle_c4_rooted over the same ranges as well.

Each range grows (x4) from one root until the oracle needs about --budget
seconds on it; a root whose search alone is beyond that moves the range's
start on (some hub roots of the 5- to 7-vertex patterns).

    python tests/golden/make_full_size_pins.py [--only c2,c3,...] [--budget 4]
"""
from __future__ import annotations

import argparse
import hashlib
import json
import os
import sys
import time
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "oracle"))

ABC = [0.57, 0.19, 0.19]


def _edges(n, pairs):
    s = ["0"] * (n * n)
    for u, v in pairs:
        s[u * n + v] = s[v * n + u] = "1"
    return "".join(s)


K4 = "0111101111011110"
C4 = "0101101001011010"
HOUSE_P2 = "0100110110010110110010100"
K5 = "0111110111110111110111110"
K6 = _edges(6, [(i, j) for i in range(6) for j in range(i + 1, 6)])
C6_CHORD = _edges(6, [(0, 1), (1, 2), (2, 3), (3, 4), (4, 5), (5, 0), (0, 3)])
TRI_PATH_7V = _edges(7, [(0, 1), (1, 2), (0, 2), (2, 3), (3, 4), (4, 5), (5, 6)])

# Root-range starts as fractions of V (ids are degree-ordered: the hubs come
# first); 0 is the hub range.
STARTS = (0.0, 1e-4, 1e-3, 1e-2, 0.05, 0.2, 0.5, 0.9)
STARTS_C4 = (0.0, 1e-3, 0.05, 0.5)


def workloads() -> dict:
    from graphautotune_b200.experiments import c4_graph_spec

    out = {
        "c2": {"graph": {"kind": "rmat", "scale": 20, "samples": 1 << 24, "seed": 2},
               "patterns": {"k4": K4, "c4": C4}, "starts": STARTS},
        "c3": {"graph": {"kind": "rmat", "scale": 22, "samples": 1 << 26, "seed": 3},
               "patterns": {"house": HOUSE_P2, "k5": K5}, "starts": STARTS},
        "c5": {"graph": {"kind": "rmat", "scale": 24, "samples": 12 << 24, "seed": 4},
               "patterns": {"k6": K6, "c6_chord": C6_CHORD, "tri_path_7v": TRI_PATH_7V},
               "starts": STARTS},
    }
    for seed in (150, 155):  # config 4's largest R-MAT and largest Barabasi-Albert graph
        # patterns None: the 21 connected 5-vertex patterns
        out[f"c4_seed{seed}"] = {"graph": c4_graph_spec(seed), "patterns": None,
                                 "starts": STARTS_C4}
    return out


def make_graph(gat, spec: dict):
    if spec["kind"] == "rmat":
        return gat.Graph.rmat(spec["scale"], spec["samples"], *ABC, spec["seed"])
    return gat.Graph.barabasi_albert(spec["n"], spec["m"], spec["seed"])


def csr_digest(off, adj) -> str:
    h = hashlib.blake2b(digest_size=16)
    h.update(memoryview(off).cast("B"))
    h.update(memoryview(adj).cast("B"))
    return h.hexdigest()


def grow(fn, V: int, start: int, budget: float, limit: int, max_width: int = 1 << 16):
    """[start, start + w) with w grown x4 from 1 while fn takes under
    budget / 4 seconds; returns (begin, end, value, seconds), or None.  fn
    returns None when it gives up (work cap): a wider range then keeps the
    previous width, and a single root over the cap moves the start on by 1,
    2, 4, ... roots, never to `limit` or beyond (the next range's start): hub
    roots whose search alone exceeds the host budget are skipped."""
    s0, step, w, best = start, 1, 1, None
    while start < min(V, limit):
        e = min(V, start + w)
        t0 = time.time()
        val = fn(start, e)
        dt = time.time() - t0
        if val is None:
            if best is not None:
                return best
            start = s0 + step
            step *= 2
            continue
        best = (start, e, int(val), dt)
        if dt >= budget / 4 or w >= max_width or e >= V:
            return best
        w *= 4
    return best


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--only", default="")
    ap.add_argument("--budget", type=float, default=4.0)
    ap.add_argument("--threads", type=int, default=os.cpu_count() or 1)
    a = ap.parse_args()
    import graphautotune_b200 as gat
    import pyoracle as O

    out_path = HERE / "full_size_pins.json"
    out = json.loads(out_path.read_text()) if out_path.exists() else {}
    wl = workloads()
    only = [x for x in a.only.split(",") if x] or list(wl)
    for name in only:
        w = wl[name]
        pats = w["patterns"] or {f"p5_{i}": p for i, p in
                                 enumerate(gat.enumerate_patterns(5))}
        t0 = time.time()
        g = make_graph(gat, w["graph"])
        off, adj = g.csr()
        V = len(off) - 1
        oo, oa = O.degree_order(off, adj)
        rec = {"graph": w["graph"], "V": V, "E": int(len(adj)),
               "ordered_digest": csr_digest(oo, oa), "patterns": {}}
        print(name, "V", V, "E", len(adj), f"setup {time.time() - t0:.1f}s", flush=True)
        for pname, p in pats.items():
            d = gat.Schedule(p, "exact", stats_graph=g).dump()
            q, less = O.plan_conditions(d)
            prec = {"adj": p, "perm": d["perm"], "restrictions": d["restrictions"],
                    "divisor": d["divisor"], "plan_ranges": []}
            secs = 0.0
            # about 1.5e8 candidates per second on 8 threads
            cap = int(1.5e8 * a.budget * a.threads / 8)
            starts = [int(V * f) for f in w["starts"]] + [V]
            for s0, s1 in zip(starts, starts[1:]):
                r = grow(lambda lo, hi: O.restricted_labelled_capped(
                    oo, oa, q, less, (lo, hi), cap, threads=a.threads), V, s0, a.budget, s1)
                if r is None:
                    continue
                b, e, raw, dt = r
                prec["plan_ranges"].append([b, e, raw])
                secs += dt
            if p == C4:
                prec["c4_ranges"] = []
                for s0, s1 in zip(starts, starts[1:]):
                    b, e, c, dt = grow(lambda lo, hi: O.c4_rooted(
                        oo, oa, roots=(lo, hi), threads=a.threads), V, s0, a.budget, s1)
                    prec["c4_ranges"].append([b, e, c])
                    secs += dt
            prec["oracle_seconds"] = round(secs, 1)
            rec["patterns"][pname] = prec
            print(" ", pname, prec["plan_ranges"], prec.get("c4_ranges", ""),
                  f"{secs:.1f}s", flush=True)
        out[name] = rec
        out_path.write_text(json.dumps(out, indent=1) + "\n")


if __name__ == "__main__":
    main()
