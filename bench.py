"""Benchmark: exact 4-clique and 4-cycle counts on an R-MAT graph with 2^20
vertices (2^24 edge samples, a=0.57 b=0.19 c=0.19, seed 2), on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

A step is one count of every workload pattern over the whole graph (exact
subgraph counts, uint64).  `value` is matches/s = (sum of the step's exact
counts, over all ranks) / (device time of the step's search launches, max over
ranks), graph resident in HBM.  `e2e` is the same metric through the public C
ABI from host CSR buffers: graph creation from pinned host arrays, upload
(including the degree-ordered copy), the counts, and the results back on the
host, every step.  Multi-GPU runs split the work queue into equal shards (one
per rank, no collective on the data path) and sum the shards' totals.

--impl reference times the reference's own CPU implementation of the path, the
naive nested-loop matcher (target/naive_pm.cu) built from its sources into
oracle/_ref/, on all host threads over a bounded sample of first vertices; if
that binary is absent, the oracle's restatement of the same matcher is timed.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import threading
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

WORKLOAD = dict(name="rmat20_k4_c4", scale=20, samples=1 << 24, a=0.57, b=0.19, c=0.19, seed=2)
PATTERNS = {"k4": "0111101111011110", "c4": "0101101001011010"}
L2_FLUSH_BYTES = 256 << 20


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


def graph_cache_path() -> Path:
    w = WORKLOAD
    d = Path(tempfile.gettempdir()) / "gat_bench"
    d.mkdir(exist_ok=True)
    return d / f"rmat{w['scale']}_{w['samples']}_{w['seed']}.bin"


def load_workload_graph(g):
    path = graph_cache_path()
    if path.exists():
        return g.Graph.load(str(path)), True
    w = WORKLOAD
    gr = g.Graph.rmat(w["scale"], w["samples"], w["a"], w["b"], w["c"], w["seed"])
    tmp = path.with_suffix(f".{os.getpid()}.tmp")
    gr.save(str(tmp))
    os.replace(tmp, path)
    return gr, False


class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines: list[str] = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for nm, val in zip(names, parts[5:9]):
                if val.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peaks() -> tuple[float, str]:
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profile_traffic(pattern: str) -> float | None:
    """DRAM bytes (read + write) of one full count of `pattern` on the
    workload graph, from the ncu capture summarised in profiles/."""
    p = ROOT / "profiles" / "traffic.json"
    if p.exists():
        try:
            d = json.loads(p.read_text()).get(WORKLOAD["name"], {})
            v = d.get(pattern) if isinstance(d, dict) else None
            return None if v is None else float(v["bytes_per_count"])
        except Exception:
            return None
    return None


# ----------------------------------------------------------------- reference

MAX_ROOT_SCANS = 200


class _Over(Exception):
    pass


def naive_scans(off, adj, pattern: str, v0: int, cap: int) -> int:
    """Full scans of V the naive matcher (target/naive_pm.cu:10-44) makes for
    root v0: one per partial embedding of 1 .. n-1 vertices.  Raises _Over
    past `cap`."""
    n = int(round(len(pattern) ** 0.5))
    nbr = [[j for j in range(n) if j != i and (pattern[i * n + j] == "1"
                                                or pattern[j * n + i] == "1")]
           for i in range(n)]
    import numpy as np

    count = 0
    emb = [v0]

    def rec():
        nonlocal count
        count += 1
        if count > cap:
            raise _Over
        k = len(emb)
        if k == n - 1:
            return
        prev = [j for j in nbr[k] if j < k]
        if not prev:
            raise _Over  # would scan every vertex: unbounded
        lists = sorted((adj[off[emb[j]]:off[emb[j] + 1]] for j in prev), key=len)
        cand = lists[0]
        for other in lists[1:]:
            if len(cand) == 0 or len(other) == 0:
                cand = cand[:0]
                break
            idx = np.minimum(np.searchsorted(other, cand), len(other) - 1)
            cand = cand[other[idx] == cand]
        cand = cand[~np.isin(cand, emb)]
        if count + len(cand) > cap:  # every candidate costs at least one scan
            raise _Over
        for u in cand.tolist():
            emb.append(u)
            rec()
            emb.pop()

    rec()
    return count


def sample_roots(gr, pattern: str, n_scans: int, seed: int = 12345):
    """Seeded uniform random first vertices whose naive-matcher cost is at
    most MAX_ROOT_SCANS scans of V (costlier roots are skipped); stops when
    the sum of scans reaches n_scans."""
    import numpy as np

    off, adj = gr.csr()
    V = len(off) - 1
    rng = np.random.default_rng(seed)
    roots, total, skipped = [], 0, 0
    for v in rng.permutation(V):
        if int(off[v + 1] - off[v]) + 1 > MAX_ROOT_SCANS:
            skipped += 1
            continue
        try:
            cost = naive_scans(off, adj, pattern, int(v), MAX_ROOT_SCANS)
        except _Over:
            skipped += 1
            continue
        roots.append(int(v))
        total += cost
        if total >= n_scans:
            break
    return roots, total, skipped


def cpu_naive_sample(gr, pattern: str, aut: int, budget_s: float = 15.0) -> dict:
    """Times the reference naive matcher on a bounded random sample of roots
    on all host threads, sized from a calibration run to take ~budget_s."""
    threads = os.cpu_count() or 1
    V = gr.v_cnt()
    binary = ROOT / "oracle/_ref/naive_sample"
    use_ref = binary.exists()
    if use_ref:
        gpath = graph_cache_path()
        if not gpath.exists():
            gr.save(str(gpath))
    else:
        sys.path.insert(0, str(ROOT / "oracle"))
        import pyoracle

        off, adj = gr.csr()

    def run(roots):
        t0 = time.perf_counter()
        if use_ref:
            out = subprocess.run([str(binary), str(graph_cache_path()), pattern, "-",
                                  str(threads)], input="\n".join(map(str, roots)) + "\n",
                                 capture_output=True, text=True, check=True).stdout.split()
            return int(out[1]), float(out[3])
        lab = pyoracle.naive_labelled_roots(off, adj, pattern, roots, threads)
        return lab, time.perf_counter() - t0

    scans = 4 * threads
    roots, total, skipped = sample_roots(gr, pattern, scans)
    labelled, secs = run(roots)
    per_scan = secs * threads / max(total, 1)
    scans = int(budget_s * threads / max(per_scan, 1e-6))
    roots, total, skipped = sample_roots(gr, pattern, scans)
    return {"run": run, "roots": roots, "total": total, "skipped": skipped, "aut": aut,
            "threads": threads, "V": V, "kind": "reference" if use_ref else "port",
            "pattern": pattern}


def cpu_baseline_step(plans: list[dict]) -> dict:
    """One timed pass of the naive matcher over every pattern's sample."""
    matches, secs, parts = 0.0, 0.0, []
    for p in plans:
        labelled, s = p["run"](p["roots"])
        matches += labelled / p["aut"]
        secs += s
        parts.append(f"pattern {p['pattern']}: {len(p['roots'])} seeded uniform random first "
                     f"vertices of {p['V']} costing <= {MAX_ROOT_SCANS} scans of V each "
                     f"({p['skipped']} costlier roots skipped), {p['total']} scans, "
                     f"{labelled} labelled embeddings ({labelled / p['aut']:.2f} matches) in "
                     f"{s:.2f} s")
    return {"value": matches / secs if secs > 0 else 0.0, "unit": "matches/s",
            "cores": plans[0]["threads"], "kind": plans[0]["kind"],
            "sample": "naive nested-loop matcher (target/naive_pm.cu) on all host threads; "
                      + "; ".join(parts), "seconds": secs}


def cpu_baseline_plans(gr, budget_s: float) -> list[dict]:
    import graphautotune_b200 as g

    return [cpu_naive_sample(gr, p, g.Pattern(p).automorphisms(), budget_s / len(PATTERNS))
            for p in PATTERNS.values()]


def run_reference(args):
    ws, rank, _ = dist_env()
    if rank != 0:
        return 0
    import graphautotune_b200 as g

    gr, _ = load_workload_graph(g)
    plans = cpu_baseline_plans(gr, 12.0)  # calibration = warm-up
    steps = [cpu_baseline_step(plans) for _ in range(args.steps)]
    value = statistics.median(s["value"] for s in steps)
    base = dict(steps[-1])
    secs = base.pop("seconds")
    line = {
        "impl": "reference", "metric": "matches/s (exact 4-clique + 4-cycle counts)",
        "value": value, "unit": "matches/s", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": secs * 1000,
        "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "int64",
        "data": "synthetic", "config": {"workload": WORKLOAD["name"], **WORKLOAD,
                                        "patterns": list(PATTERNS)},
        "cpu_baseline": {**base, "value": value},
        "e2e": {"value": value, "unit": "matches/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


# ----------------------------------------------------------------------- ours

def run_ours(args):
    import numpy as np
    import torch

    import graphautotune_b200 as g

    ws, rank, local = dist_env()
    torch.cuda.set_device(local)
    dist = None
    if ws > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                device_id=torch.device("cuda", local))

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()

    t0 = time.perf_counter()
    gr, cached = load_workload_graph(g)
    V, E, maxdeg = gr.info()
    t_gen = time.perf_counter() - t0
    t0 = time.perf_counter()
    gr.upload(degree_order=True)
    t_up = time.perf_counter() - t0
    cfg = g.Config.engine_default()
    ex = g.Executor(cfg)
    scheds = {k: g.Schedule(p, "exact", stats_graph=gr) for k, p in PATTERNS.items()}
    log(f"[rank {rank}] graph V={V} E={E} maxdeg={maxdeg} gen {t_gen:.2f}s "
        f"(cached={cached}) upload {t_up:.2f}s")

    flush = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device="cuda")

    def step():
        raws, ms, results = {}, 0.0, {}
        for k, s in scheds.items():
            raw, r = ex.count_shard(gr, s, rank, ws)
            raws[k] = (raw, r.divisor)
            ms += r.kernel_ms
            results[k] = r
        return raws, ms, results

    for _ in range(args.warmup):
        step()
        flush.zero_()
    barrier()
    sampler = ClockSampler(local)
    sampler.start()
    wall0 = time.perf_counter()
    dev_ms = 0.0
    per_pat_ms = {k: 0.0 for k in PATTERNS}
    launches = 0
    raws = None
    for _ in range(args.steps):
        raws, ms, results = step()
        dev_ms += ms
        for k, r in results.items():
            per_pat_ms[k] += r.kernel_ms
            launches += r.launches
        flush.zero_()
    barrier()
    wall = time.perf_counter() - wall0
    clocks = sampler.stop()

    # totals over ranks: sum of raw shard totals, max of device time
    from graphautotune_b200.dist import reduce_shards

    cnt_list, max_ms = reduce_shards([raws[k][0] for k in PATTERNS],
                                     [raws[k][1] for k in PATTERNS], dev_ms, device="cuda")
    counts = dict(zip(PATTERNS, cnt_list))
    ms_per_step = max_ms / args.steps
    matches = sum(counts.values())
    value = matches / (ms_per_step / 1000.0)

    line = None
    if rank == 0:
        # Roofline of the dominant launch, from an instrumented (untimed) run.
        dom = max(per_pat_ms, key=per_pat_ms.get)
        balg = ex.count(gr, scheds[dom], balg=True).balg_bytes if ws == 1 else \
            ex.count_shard(gr, scheds[dom], rank, ws)[1].balg_bytes
        dom_ms = per_pat_ms[dom] / args.steps
        peak, peak_kind = measured_peaks()
        achieved = balg / (dom_ms / 1000.0) / 1e9
        # End to end through the C ABI from pinned host buffers.
        off, adj = gr.csr()
        off_p = torch.from_numpy(off).pin_memory()
        adj_p = torch.from_numpy(adj).pin_memory()
        e2e_ms = []
        for i in range(max(1, min(3, args.steps))):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            g2 = g.Graph.from_csr(off_p.numpy(), adj_p.numpy(), check_symmetry=False)
            g2.upload(degree_order=True)
            tot = 0
            for k, s in scheds.items():
                tot += ex.count(g2, s).count
            torch.cuda.synchronize()
            e2e_ms.append((time.perf_counter() - t0) * 1000)
            assert tot == matches, (tot, matches)
            del g2
        e2e_value = matches / (statistics.median(e2e_ms) / 1000.0)
        cpu = cpu_baseline_step(cpu_baseline_plans(gr, 12.0))
        cpu.pop("seconds", None)
        line = {
            "metric": "matches/s (exact 4-clique + 4-cycle counts)",
            "value": value, "unit": "matches/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "int64",
            "data": "synthetic",
            "config": {"workload": WORKLOAD["name"], "graph": f"R-MAT scale 20, 2^24 samples "
                       f"(a,b,c)=(.57,.19,.19) seed 2 -> V={V}, E={E} directed, max degree "
                       f"{maxdeg}", "patterns": PATTERNS, "counts": counts,
                       "count_mode": "exact", "l2": "flushed between steps (256 MiB write)",
                       "engine": {"tile": cfg.threads_per_warp,
                                  "block": cfg.threads_per_block, "chunk": cfg.chunk},
                       "parallelism": f"work-queue shards x{ws}"},
            "per_pattern_ms": {k: v / args.steps for k, v in per_pat_ms.items()},
            "wall_ms_per_step": wall * 1000 / args.steps,
            "setup": {"graph_build_s": t_gen, "upload_s": t_up},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": profile_traffic(dom),
                         "kernel": ("4-cycle wedge kernels (one count)" if dom == "c4"
                                    else f"search_kernel ({dom})"),
                         "balg_bytes_per_launch": balg,
                         "peak_kind": peak_kind},
            "e2e": {"value": e2e_value, "unit": "matches/s",
                    "h2d_bytes_per_step": int(off.nbytes + adj.nbytes),
                    "d2h_bytes_per_step": 32 * len(PATTERNS), "ms_per_step":
                    statistics.median(e2e_ms)},
            "gpu_launches": launches,
            "clocks": clocks,
            "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def run_profile_case(args):
    """A bounded slice of one workload pattern's search, for profilers: the
    workload graph, `pattern` counted over one shard (default 0) of `parts`
    equal slices of the work queue (`--profile PATTERN:PARTS[:SHARD]`),
    warmup + steps launches (one search kernel each)."""
    import torch

    import graphautotune_b200 as g

    fields = args.profile.split(":")
    name, parts = fields[0], int(fields[1])
    shard = int(fields[2]) if len(fields) > 2 else 0
    torch.cuda.set_device(0)
    gr, _ = load_workload_graph(g)
    gr.upload(degree_order=True)
    ex = g.Executor(g.Config.engine_default())
    s = g.Schedule(PATTERNS[name], "exact", stats_graph=gr)
    for i in range(args.warmup + args.steps):
        raw, r = ex.count_shard(gr, s, shard, parts)
        log(f"{name} shard {shard}/{parts}: raw {raw} tasks {r.tasks} "
            f"kernel {r.kernel_ms:.2f} ms")
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--profile", default=None,
                    help="PATTERN:PARTS[:SHARD], e.g. c4:64:32 - one slice of the search, for ncu")
    args = ap.parse_args()
    if args.profile:
        sys.exit(run_profile_case(args))
    from graphautotune_b200 import _lib

    if not _lib.LIB_PATH.exists():
        from graphautotune_b200 import build

        build.build()
    if args.impl == "reference":
        sys.exit(run_reference(args))
    sys.exit(run_ours(args))


if __name__ == "__main__":
    main()
