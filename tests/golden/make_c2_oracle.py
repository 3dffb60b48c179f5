"""Full-size pins for the 4-clique / 4-cycle workload graph (R-MAT 2^20,
2^24 samples, (a,b,c) = (.57,.19,.19), seed 2), computed on the host and
written to tests/golden/c2_oracle.json:

  k4      the oracle's restatement of the reference engine (oracle/oracle.cpp,
          OpenMP) over the whole graph, root range by root range (about 45
          minutes on 8 threads);
  c4      the exact 4-cycle count by another route than the GPU's: wedges on
          the graph's own ids, each cycle counted at its LARGEST vertex
          (oracle_c4_rooted, at_largest = 1).  The GPU kernels count each
          cycle at its smallest vertex of the degree-ordered copy, so the two
          share neither the rooting nor the vertex ids.

    python tests/golden/make_c2_oracle.py [--threads 8] [--patterns k4,c4]
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "oracle"))

PATTERNS = {"k4": "0111101111011110", "c4": "0101101001011010"}


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--threads", type=int, default=os.cpu_count() or 1)
    ap.add_argument("--patterns", default="k4,c4")
    ap.add_argument("--parts", type=int, default=64)
    a = ap.parse_args()
    import graphautotune_b200 as gat
    import pyoracle as O

    sched = {}
    for line in (HERE / "ref_schedules.jsonl").read_text().splitlines():
        if line.strip():
            d = json.loads(line)
            sched[d["pattern"]] = d
    g = gat.Graph.rmat(20, 1 << 24, 0.57, 0.19, 0.19, 2)
    off, adj = g.csr()
    V = len(off) - 1
    out_path = HERE / "c2_oracle.json"
    out = json.loads(out_path.read_text()) if out_path.exists() else {}
    out["graph"] = {"kind": "rmat", "scale": 20, "samples": 1 << 24, "abc": [0.57, 0.19, 0.19],
                    "seed": 2, "V": V, "E": int(len(adj))}
    for name in a.patterns.split(","):
        p = PATTERNS[name]
        t0 = time.time()
        if name == "c4":
            tot = O.c4_rooted(off, adj, at_largest=True, threads=a.threads)
            out[name] = {"pattern": p, "exact_at_largest_vertex": tot,
                         "seconds": time.time() - t0, "threads": a.threads}
            out_path.write_text(json.dumps(out, indent=1) + "\n")
            print(name, tot, flush=True)
            continue
        tot = 0
        for i in range(a.parts):
            st, c, _ = O.ref_engine(off, adj, sched[p], roots=(V * i // a.parts,
                                                              V * (i + 1) // a.parts),
                                    threads=a.threads)
            assert st == 0
            tot += c
        out[name] = {"pattern": p, "ref_engine_oracle": tot, "seconds": time.time() - t0,
                     "threads": a.threads}
        out_path.write_text(json.dumps(out, indent=1) + "\n")
        print(name, tot, flush=True)


if __name__ == "__main__":
    main()
