"""Runs the reference engine itself (oracle/_ref/pm: target/pm.cu built from
the reference sources for sm_100a by `make -C oracle ref_gpu`) on the golden
graphs and writes its answers to tests/golden/ref_engine_counts.json.

Needs a GPU, so it runs on a B200 box (oracle/_ref/ travels with the
repository snapshot; the reference sources are not needed there).  Only
(graph, pattern) pairs whose reference result is defined are run: patterns
on which the reference's Schedule crashes or reads uninitialised state are
skipped (libgat refuses them with GAT_ERR_UNDEFINED).

    python tests/golden/make_ref_engine_golden.py [--timeout 120]
"""
from __future__ import annotations

import argparse
import json
import re
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT))


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--timeout", type=float, default=120)
    ap.add_argument("--out", default=str(HERE / "ref_engine_counts.json"))
    # Every run of the reference binary allocates most of the device memory
    # (engine/engine.cuh:171-175) and pays a context start, so the default
    # set is bounded: all patterns up to 5 vertices on these graphs.
    ap.add_argument("--graphs", default="er60,k7,rmat6,c1_er10000")
    ap.add_argument("--max-n", type=int, default=5)
    a = ap.parse_args()
    wanted = set(a.graphs.split(","))
    import graphautotune_b200 as g

    pm = ROOT / "oracle/_ref/pm"
    if not pm.exists():
        sys.exit("oracle/_ref/pm missing: make -C oracle ref_gpu")
    naive = json.loads((HERE / "naive_counts.json").read_text())
    seen, out = set(), []
    for e in naive:
        key = (e["graph"], e["adj"])
        if key in seen or e["graph"] not in wanted or len(e["adj"]) > a.max_n ** 2:
            continue
        seen.add(key)
        try:
            g.Schedule(e["adj"], "ref").plan_bytes()
        except g.GatError:
            continue  # undefined in the reference
        graph = (HERE / "graphs" / f"{e['graph']}.bin").resolve()
        try:
            r = subprocess.run([str(pm), str(graph), e["adj"]], capture_output=True, text=True,
                               timeout=a.timeout)
        except subprocess.TimeoutExpired:
            print(f"timeout {e['graph']} {e['pattern']}", flush=True)
            continue
        m = re.search(r"^Answer: (-?\d+)$", r.stdout, re.M)
        t = re.search(r"^Time: (\d+) us", r.stdout, re.M)
        if r.returncode != 0 or not m:
            print(f"failed {e['graph']} {e['pattern']} rc={r.returncode}", flush=True)
            continue
        out.append({"graph": e["graph"], "pattern": e["pattern"], "adj": e["adj"],
                    "ref_engine_answer": int(m.group(1)),
                    "ref_engine_us": int(t.group(1)) if t else None})
    Path(a.out).write_text(json.dumps(out, indent=0))
    print(f"{len(out)} reference-engine answers -> {a.out}")


if __name__ == "__main__":
    main()
