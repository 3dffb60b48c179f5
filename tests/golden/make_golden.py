"""Regenerates the golden fixtures in tests/golden/ from the reference itself.

Needs the reference sources where oracle/Makefile finds them (its REF, or
$GAT_REFERENCE) to build oracle/_ref/ (target `ref`).  Writes:

  graphs/*.bin            small seeded graphs in the reference binary layout
  ref_schedules.jsonl     the reference's Core::Schedule for every pattern in
                          PATTERNS (oracle/_ref/schedule_dump)
  naive_counts.json       the reference naive matcher's Answer
                          (oracle/_ref/naive_pm, target/naive_pm.cu) for every
                          (graph, pattern) pair whose count fits its int
  patterns.json           the pattern list with its provenance

The graphs are generated by libgat's seeded generators once and then frozen
as files, so the fixtures do not move if a generator changes.

    python tests/golden/make_golden.py [--jobs N]
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import json
import os
import random
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT))

REF = Path(subprocess.run(["make", "-s", "-C", str(ROOT / "oracle"), "print-ref"],
                          capture_output=True, text=True, check=True).stdout.strip())

# Pattern strings named in the reference's scripts and in the benchmark
# configurations (scripts/run_pattern_matching.sh:14-21).
def from_edges(n: int, edges: list[tuple[int, int]]) -> str:
    s = ["0"] * (n * n)
    for u, v in edges:
        s[u * n + v] = s[v * n + u] = "1"
    return "".join(s)


NAMED = {
    "triangle": "011101110",
    "k4": "0111101111011110",
    "c4": "0101101001011010",
    "house_p2": "0100110110010110110010100",
    "k5": "0111110111110111110111110",
    "p3_6v": "011011101110110101011000110000101000",
    "k6": from_edges(6, [(i, j) for i in range(6) for j in range(i + 1, 6)]),
    # 6-cycle with one chord between opposite vertices
    "c6_chord": from_edges(6, [(0, 1), (1, 2), (2, 3), (3, 4), (4, 5), (5, 0), (0, 3)]),
    # triangle with a 4-edge path hanging off one corner (7 vertices)
    "tri_path_7v": from_edges(7, [(0, 1), (1, 2), (0, 2), (2, 3), (3, 4), (4, 5), (5, 6)]),
    "p4_7v": "0111111101111111011101110100111100011100001100000",
}

GRAPHS = {
    # name: (generator kind, params, seed)
    "er60": ("er", (60, 8.0), 11),
    "er200": ("er", (200, 6.0), 12),
    "rmat6": ("rmat", (6, 256), 13),
    "ba60": ("ba", (60, 3), 14),
    "k5": ("complete", (5,), 0),
    "k7": ("complete", (7,), 0),
    # configuration 1 at full size: G(n=10,000, avg degree 16), seed 1
    "c1_er10000": ("er", (10000, 16.0), 1),
}
# Full-size graphs get only the configuration's own pattern.
ONLY = {"c1_er10000": {"triangle"}}
NAIVE_TIMEOUT_S = 600


def connected_order(p: str) -> str:
    """The same pattern relabelled so every vertex after the first has an
    earlier neighbour (BFS from vertex 0).  The naive matcher's labelled
    count does not depend on the labelling, but its running time does: it
    scans all V vertices for every pattern vertex without an earlier
    neighbour."""
    n = int(round(len(p) ** 0.5))
    adj = [[p[i * n + j] == "1" or p[j * n + i] == "1" for j in range(n)] for i in range(n)]
    order, seen = [0], {0}
    while len(order) < n:
        nxt = next((v for v in range(n) if v not in seen and any(adj[v][u] for u in order)),
                   None)
        if nxt is None:
            nxt = next(v for v in range(n) if v not in seen)
        order.append(nxt)
        seen.add(nxt)
    pos = {v: i for i, v in enumerate(order)}
    s = ["0"] * (n * n)
    for i in range(n):
        for j in range(n):
            if adj[i][j]:
                s[pos[i] * n + pos[j]] = "1"
    return "".join(s)


def relabel(p: str, rng: random.Random) -> str:
    n = int(round(len(p) ** 0.5))
    perm = list(range(n))
    rng.shuffle(perm)
    s = ["0"] * (n * n)
    for i in range(n):
        for j in range(n):
            if p[i * n + j] == "1":
                s[perm[i] * n + perm[j]] = "1"
    return "".join(s)


def pattern_list() -> list[tuple[str, str]]:
    import graphautotune_b200 as g

    out = [(k, v) for k, v in NAMED.items()]
    for n in (3, 4, 5):
        out += [(f"conn{n}_{i}", p) for i, p in enumerate(g.enumerate_patterns(n))]
    six = g.enumerate_patterns(6)
    rng = random.Random(2024)
    out += [(f"conn6_{i}", six[i]) for i in sorted(rng.sample(range(len(six)), 16))]
    base = [p for _, p in out if len(p) <= 25]
    out += [(f"relabel_{i}", relabel(p, rng)) for i, p in enumerate(rng.sample(base, 24))]
    seen, uniq = set(), []
    for name, p in out:
        if p not in seen:
            seen.add(p)
            uniq.append((name, p))
    return uniq


def make_graphs() -> dict[str, Path]:
    import numpy as np

    import graphautotune_b200 as g

    gdir = HERE / "graphs"
    gdir.mkdir(exist_ok=True)
    paths = {}
    for name, (kind, params, seed) in GRAPHS.items():
        path = gdir / f"{name}.bin"
        if kind == "er":
            gr = g.Graph.erdos_renyi(params[0], params[1], seed)
        elif kind == "rmat":
            gr = g.Graph.rmat(params[0], params[1], 0.57, 0.19, 0.19, seed)
        elif kind == "ba":
            gr = g.Graph.barabasi_albert(params[0], params[1], seed)
        else:
            n = params[0]
            off = np.arange(0, n * (n - 1) + 1, n - 1, dtype=np.int64)
            adj = np.array([u for v in range(n) for u in range(n) if u != v], np.int32)
            gr = g.Graph.from_csr(off, adj)
        if not path.exists():
            gr.save(str(path))
        paths[name] = path
    return paths


def run_naive(args):
    graph_path, pattern = args
    try:
        r = subprocess.run([str(ROOT / "oracle/_ref/naive_pm"), str(graph_path),
                            connected_order(pattern)],
                           capture_output=True, text=True, timeout=NAIVE_TIMEOUT_S)
    except subprocess.TimeoutExpired:
        return None
    for line in r.stdout.splitlines():
        if line.startswith("Answer:"):
            return int(line.split()[1])
    raise RuntimeError(f"naive_pm failed: {r.stdout} {r.stderr}")


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--jobs", type=int, default=os.cpu_count() or 4)
    a = ap.parse_args()
    if not REF.exists():
        sys.exit(f"reference sources not found at {REF}")
    subprocess.run(["make", "-C", str(ROOT / "oracle"), f"REF={REF}", "ref", "all"], check=True)
    pats = pattern_list()
    (HERE / "patterns.json").write_text(json.dumps([{"name": n, "adj": p} for n, p in pats],
                                                   indent=0))
    # One process per pattern: the reference's Schedule dereferences
    # restrictions[0] of an empty list for patterns without symmetry
    # (core/schedule.hpp:836-842) and dies; that outcome is recorded.
    def dump_one(p: str) -> str:
        r = subprocess.run([str(ROOT / "oracle/_ref/schedule_dump")], input=p + "\n",
                           capture_output=True, text=True)
        if r.returncode != 0:
            return json.dumps({"pattern": p, "crash": True, "returncode": r.returncode})
        return r.stdout.strip()

    with cf.ThreadPoolExecutor(a.jobs) as ex:
        lines = list(ex.map(dump_one, [p for _, p in pats]))
    (HERE / "ref_schedules.jsonl").write_text("\n".join(lines) + "\n")
    graphs = make_graphs()
    # naive counts: all patterns up to 5 vertices on every graph; the larger
    # named patterns only on the small graphs.
    jobs = []
    for gname, gpath in graphs.items():
        for pname, p in pats:
            n = int(round(len(p) ** 0.5))
            if gname in ONLY:
                if pname in ONLY[gname]:
                    jobs.append((gname, pname, gpath, p))
                continue
            if n >= 6 and gname not in ("er60", "k7", "k5"):
                continue
            if n >= 5 and gname == "er200":
                continue
            jobs.append((gname, pname, gpath, p))
    with cf.ThreadPoolExecutor(a.jobs) as ex:
        res = list(ex.map(run_naive, [(gp, p) for _, _, gp, p in jobs]))
    counts = [{"graph": gn, "pattern": pn, "adj": p, "naive_answer": r}
              for (gn, pn, _, p), r in zip(jobs, res) if r is not None]
    skipped = [f"{gn}/{pn}" for (gn, pn, _, _), r in zip(jobs, res) if r is None]
    if skipped:
        print(f"naive_pm over {NAIVE_TIMEOUT_S}s, not recorded: {skipped}")
    (HERE / "naive_counts.json").write_text(json.dumps(counts, indent=0))
    print(f"{len(pats)} patterns, {len(counts)} naive counts")


if __name__ == "__main__":
    main()
