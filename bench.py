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
oracle/_ref/, on all host threads over a degree-stratified sample of its
level-1 units (hub roots included), without loading libgat; the GPU line's
cpu_baseline holds the same estimate plus the oracle's OpenMP exact counters
on the pinned root ranges next to this engine's time on those ranges.
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


# ------------------------------------------------------------ CPU baselines
#
# Neither CPU leg loads libgat: the workload graph comes from the cached file
# or from oracle/synth.py (the same generator restated in numpy), |Aut| and
# the degree order from the oracle, the exact plans' order conditions from
# tests/golden/full_size_pins.json.

def host_workload_graph():
    """(offsets, neighbours) of the workload graph, without libgat."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import synth

    path = graph_cache_path()
    if path.exists():
        return synth.load_bin(path)
    w = WORKLOAD
    off, adj = synth.rmat(w["scale"], w["samples"], w["a"], w["b"], w["c"], w["seed"])
    tmp = path.with_suffix(f".{os.getpid()}.tmp")
    synth.save_bin(tmp, off, adj)
    os.replace(tmp, path)
    return off, adj


def workload_config(V: int, E: int, maxdeg: int) -> dict:
    """The `config` of both arms' JSON lines: the workload and nothing of
    either implementation."""
    return {"workload": WORKLOAD["name"],
            "graph": f"R-MAT scale {WORKLOAD['scale']}, 2^24 samples (a,b,c)=(.57,.19,.19) "
                     f"seed {WORKLOAD['seed']} -> V={V}, E={E} directed, max degree {maxdeg}",
            "patterns": PATTERNS, "count_mode": "exact",
            "l2": "flushed between steps (256 MiB write)"}


STRATA = 8          # level-1 units grouped by log4 of their root's degree
MAX_UNIT_SCANS = 64  # units whose naive search would scan V more often are skipped


class _Over(Exception):
    pass


def unit_scans(off, adj, nbr, v0: int, v1: int, cap: int) -> int:
    """Full scans of V the naive matcher (target/naive_pm.cu:10-44) makes
    below the level-1 unit (v0, v1): one per partial embedding of 2 .. n-1
    vertices.  Raises _Over past `cap`."""
    import numpy as np

    n = len(nbr)
    count = 0
    emb = [v0, v1]

    def rec():
        nonlocal count
        count += 1
        if count > cap:
            raise _Over
        k = len(emb)
        if k == n - 1:
            return
        prev = [j for j in nbr[k] if j < k]
        lists = sorted((adj[off[emb[j]]:off[emb[j] + 1]] for j in prev), key=len)
        cand = lists[0]
        for other in lists[1:]:
            if len(cand) == 0 or len(other) == 0:
                cand = cand[:0]
                break
            idx = np.minimum(np.searchsorted(other, cand), len(other) - 1)
            cand = cand[other[idx] == cand]
        cand = cand[~np.isin(cand, emb)]
        if count + len(cand) > cap:
            raise _Over
        for u in cand.tolist():
            emb.append(u)
            rec()
            emb.pop()

    rec()
    return count


def naive_plan(off, adj, pattern: str, scans_per_stratum: int, seed: int = 12345) -> dict:
    """A degree-stratified random sample of the naive matcher's level-1 units
    (v0, v1), v1 a neighbour of v0 (the pattern's vertices 0 and 1 are
    adjacent).  Stratum h holds the units whose root has degree in
    [4^h, 4^(h+1)) (the last one: every larger degree, the hubs); within a
    stratum units are drawn uniformly (roots by degree, then a neighbour)
    until their scans of V reach the stratum's share; units above
    MAX_UNIT_SCANS are skipped and counted."""
    import numpy as np

    n = int(round(len(pattern) ** 0.5))
    nbr = [[j for j in range(n) if j != i and (pattern[i * n + j] == "1"
                                                or pattern[j * n + i] == "1")]
           for i in range(n)]
    assert 1 in nbr[0], "units need pattern vertices 0 and 1 adjacent"
    deg = np.diff(off)
    h = np.minimum(np.floor(np.log(np.maximum(deg, 1)) / np.log(4)).astype(int), STRATA - 1)
    rng = np.random.default_rng(seed)
    units, strata = [], []
    for k in range(STRATA):
        vs = np.nonzero((h == k) & (deg > 0))[0]
        if len(vs) == 0:
            continue
        w = deg[vs].astype(np.float64)
        total_units = int(w.sum())
        got = scans = skipped = tries = 0
        while scans < scans_per_stratum and tries < 50 * scans_per_stratum:
            tries += 1
            v0 = int(vs[rng.choice(len(vs), p=w / w.sum())])
            v1 = int(adj[off[v0] + rng.integers(deg[v0])])
            try:
                c = unit_scans(off, adj, nbr, v0, v1, MAX_UNIT_SCANS)
            except _Over:
                skipped += 1
                continue
            units.append((v0, v1, k))
            got += 1
            scans += c
        strata.append({"stratum": k, "min_degree": 4 ** k, "units_total": total_units,
                       "units": got, "scans": scans, "skipped": skipped})
    return {"pattern": pattern, "units": units, "strata": strata}


def run_naive(plan: dict, threads: int) -> dict:
    """Times the reference's naive matcher (oracle/_ref/naive_sample, built
    from target/naive_pm.cu) on the plan's units on `threads` threads, and
    per stratum (labelled embeddings, thread-seconds)."""
    binary = ROOT / "oracle/_ref/naive_sample"
    lines = "\n".join(f"{a} {b} {c}" for a, b, c in plan["units"]) + "\n"
    out = subprocess.run([str(binary), str(graph_cache_path()), plan["pattern"], "-",
                          str(threads)], input=lines, capture_output=True, text=True,
                         check=True).stdout.splitlines()
    head = out[0].split()
    per = {}
    for ln in out[1:]:
        f = ln.split()
        per[int(f[1])] = (int(f[3]), float(f[5]))
    return {"labelled": int(head[1]), "seconds": float(head[3]), "per": per}


def naive_estimate(plans: list[dict], runs: list[dict], auts: list[int], threads: int) -> dict:
    """Whole-workload rate of the naive matcher from the stratified samples:
    every stratum's matches and thread-seconds scaled by its units over its
    sampled units; time on all threads = thread-seconds / threads."""
    matches = secs = 0.0
    found = {}
    for plan, run, aut in zip(plans, runs, auts):
        name = [k for k, v in PATTERNS.items() if v == plan["pattern"]][0]
        found[name] = 0.0
        for st in plan["strata"]:
            lab, tsec = run["per"].get(st["stratum"], (0, 0.0))
            if st["units"] == 0:
                continue
            scale = st["units_total"] / st["units"]
            matches += scale * lab / aut
            secs += scale * tsec / threads
            found[name] += lab / aut
    return {"value": matches / secs if secs > 0 else 0.0, "matches_on_sample": found,
            "estimated_workload_seconds": secs}


def naive_sample_text(plans: list[dict], runs: list[dict], threads: int) -> str:
    parts = []
    for plan, run in zip(plans, runs):
        name = [k for k, v in PATTERNS.items() if v == plan["pattern"]][0]
        st = "; ".join(f"deg>={s['min_degree']}: {s['units']} of {s['units_total']} units"
                       f"{', ' + str(s['skipped']) + ' skipped' if s['skipped'] else ''}"
                       for s in plan["strata"])
        parts.append(f"{name}: {len(plan['units'])} level-1 units (v0, v1) drawn per root-degree "
                     f"stratum [{st}], {run['labelled']} labelled embeddings in "
                     f"{run['seconds']:.2f} s")
    return ("reference naive nested-loop matcher (target/naive_pm.cu, oracle/_ref/naive_sample) "
            f"on {threads} host threads; strata weighted by their unit counts; units scanning V "
            f"more than {MAX_UNIT_SCANS} times skipped; " + " | ".join(parts))


def naive_plans(off, adj, budget_s: float, threads: int) -> list[dict]:
    """Stratified samples sized from a calibration run so one pass over both
    patterns takes about budget_s on `threads` threads."""
    probe = [naive_plan(off, adj, p, 4) for p in PATTERNS.values()]
    t = sum(run_naive(pl, threads)["seconds"] for pl in probe)
    sc = sum(s["scans"] for pl in probe for s in pl["strata"])
    per_scan = t / max(sc, 1)
    per_stratum = max(2, int(budget_s / max(per_scan, 1e-6) / (len(PATTERNS) * STRATA)))
    return [naive_plan(off, adj, p, per_stratum) for p in PATTERNS.values()]


def oracle_port(off, adj, threads: int) -> dict:
    """The oracle's OpenMP exact counters on the full-size pin ranges of the
    workload graph (hub roots included): plain backtracking under the exact
    plan's order conditions for the 4-clique, wedge aggregation at each
    cycle's smallest vertex for the 4-cycle, on the degree-ordered copy."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import pyoracle

    pins = json.loads((ROOT / "tests/golden/full_size_pins.json").read_text())["c2"]
    oo, oa = pyoracle.degree_order(off, adj)
    ranges, matches, secs, detail = {}, 0, 0.0, []
    for name, p in PATTERNS.items():
        pin = pins["patterns"][name]
        rs = pin.get("c4_ranges") or pin["plan_ranges"]
        ranges[name] = [(b, e) for b, e, _ in rs]
        t0 = time.perf_counter()
        if "c4_ranges" in pin:
            got = [pyoracle.c4_rooted(oo, oa, roots=(b, e), threads=threads) for b, e, _ in rs]
            div = 1
        else:
            q, less = pyoracle.plan_conditions(pin)
            got = [pyoracle.restricted_labelled(oo, oa, q, less, roots=(b, e), threads=threads)
                   for b, e, _ in rs]
            div = pin["divisor"]
        dt = time.perf_counter() - t0
        assert got == [x for _, _, x in rs], "oracle disagrees with its own pins"
        matches += sum(got) // div
        secs += dt
        detail.append(f"{name}: {len(rs)} root ranges, {sum(got) // div} matches in {dt:.2f} s")
    return {"value": matches / secs, "unit": "matches/s", "cores": threads, "kind": "port",
            "matches": matches, "seconds": secs, "ranges": ranges,
            "sample": "oracle exact counters (oracle/oracle.cpp, OpenMP) on the pinned root "
                      "ranges of the degree-ordered graph: " + "; ".join(detail)}


REF_CUDA_TIMEOUT_S = 75


def reference_cuda(patterns: dict, counts: dict | None = None) -> dict:
    """The reference's own CUDA engine on the same B200: target/pm.cu built
    for sm_100a from the reference sources (oracle/Makefile target ref_gpu,
    oracle/_ref/pm), run once per pattern on the workload graph file.  Its
    `Time:` line covers Executor::perform_search with the graph resident
    (target/pm.cu:56-64), the same region as this engine's device time; its
    `Answer:` is the reference engine's own number, not the exact count
    (restrictions outside the basic vertices are dropped, and per-level int
    counters overflow on large graphs).  Reported once, outside the steps."""
    import re

    binary = ROOT / "oracle/_ref/pm"
    if not binary.exists():
        return {"unavailable": "oracle/_ref/pm not built (make -C oracle ref_gpu)"}
    out = {"binary": "oracle/_ref/pm (target/pm.cu, sm_100a, default generated config)"}
    for name, p in patterns.items():
        try:
            r = subprocess.run([str(binary), str(graph_cache_path()), p], capture_output=True,
                               text=True, timeout=REF_CUDA_TIMEOUT_S)
        except subprocess.TimeoutExpired:
            out[name] = {"finished": False,
                         "note": f"no answer within {REF_CUDA_TIMEOUT_S} s (process stopped)"}
            continue
        ans = re.search(r"Answer: (-?\d+)", r.stdout)
        tm = re.search(r"Time: (\d+) us", r.stdout)
        rec = {"finished": r.returncode == 0 and tm is not None, "rc": r.returncode,
               "answer": int(ans.group(1)) if ans else None,
               "seconds": int(tm.group(1)) / 1e6 if tm else None}
        if rec["seconds"] and counts and name in counts:
            rec["exact_matches_per_s"] = counts[name] / rec["seconds"]
        if not rec["finished"]:
            rec["tail"] = (r.stdout + r.stderr)[-300:]
        out[name] = rec
    return out


def exact_counts() -> dict | None:
    """The workload's exact counts as pinned by the oracle
    (tests/golden/c2_oracle.json), for rates of engines that do not return
    them."""
    p = ROOT / "tests/golden/c2_oracle.json"
    try:
        d = json.loads(p.read_text())
        # the oracle's restatement of the reference engine counts each
        # 4-clique 4 times; the 4-cycle total is the whole-graph count
        return {"k4": int(d["k4"]["ref_engine_oracle"]) // 4,
                "c4": int(d["c4"]["exact_at_largest_vertex"])}
    except Exception:
        return None


def run_reference(args):
    ws, rank, _ = dist_env()
    if rank != 0:
        return 0
    sys.path.insert(0, str(ROOT / "oracle"))
    import pyoracle

    threads = os.cpu_count() or 1
    off, adj = host_workload_graph()
    V, E = len(off) - 1, len(adj)
    maxdeg = int((off[1:] - off[:-1]).max())
    auts = [pyoracle.automorphisms(p) for p in PATTERNS.values()]
    # each step about 150 / (steps + warmup) s, so the whole run takes minutes
    budget = max(1.0, min(12.0, 100.0 / max(1, args.steps + args.warmup)))
    plans = naive_plans(off, adj, budget, threads)
    for _ in range(args.warmup):
        [run_naive(pl, threads) for pl in plans]
    steps = []
    for _ in range(args.steps):
        runs = [run_naive(pl, threads) for pl in plans]
        steps.append((naive_estimate(plans, runs, auts, threads), runs))
    value = statistics.median(st["value"] for st, _ in steps)
    est, runs = steps[-1]
    line = {
        "impl": "reference", "metric": "matches/s (exact 4-clique + 4-cycle counts)",
        "value": value, "unit": "matches/s", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": sum(r["seconds"] for r in runs) * 1000,
        "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "int64",
        "data": "synthetic", "config": workload_config(V, E, maxdeg),
        "cpu_baseline": {"value": value, "unit": "matches/s", "cores": threads,
                         "kind": "reference", "sample": naive_sample_text(plans, runs, threads),
                         "matches_on_sample": est["matches_on_sample"],
                         "estimated_workload_seconds": est["estimated_workload_seconds"]},
        "e2e": {"value": value, "unit": "matches/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
        "reference_cuda": reference_cuda(PATTERNS, exact_counts()),
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
        e2e_ms, parts_ms = [], []
        for i in range(max(1, min(3, args.steps))):
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            g2 = g.Graph.from_csr(off_p.numpy(), adj_p.numpy(), check_symmetry=False,
                                  device=True)
            t1 = time.perf_counter()
            g2.upload(degree_order=True)
            t2 = time.perf_counter()
            tot = 0
            for k, s in scheds.items():
                tot += ex.count(g2, s).count
            torch.cuda.synchronize()
            t3 = time.perf_counter()
            e2e_ms.append((t3 - t0) * 1000)
            parts_ms.append({"graph_from_host_arrays": (t1 - t0) * 1000,
                             "upload": (t2 - t1) * 1000, "counts": (t3 - t2) * 1000})
            assert tot == matches, (tot, matches)
            del g2
        e2e_value = matches / (statistics.median(e2e_ms) / 1000.0)
        cpu = cpu_baselines(off, adj, ex, gr, scheds)
        line = {
            "metric": "matches/s (exact 4-clique + 4-cycle counts)",
            "value": value, "unit": "matches/s", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms_per_step, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "int64",
            "data": "synthetic",
            "config": workload_config(V, E, maxdeg),
            "counts": counts,
            "engine": {"tile": cfg.threads_per_warp, "block": cfg.threads_per_block,
                       "chunk": cfg.chunk, "parallelism": f"work-queue shards x{ws}"},
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
                    statistics.median(e2e_ms),
                    "breakdown_ms": parts_ms},
            "gpu_launches": launches,
            "clocks": clocks,
            "cpu_baseline": cpu,
        }
        print(json.dumps(line), flush=True)
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def cpu_baselines(off, adj, ex, gr, scheds) -> dict:
    """cpu_baseline of the GPU line: the reference's naive matcher on a
    stratified sample (about 10 s on all host threads; kind "reference"),
    with the oracle's OpenMP exact counters beside it on the pinned root
    ranges, and this engine's device time on the same ranges."""
    threads = os.cpu_count() or 1
    sys.path.insert(0, str(ROOT / "oracle"))
    import pyoracle

    auts = [pyoracle.automorphisms(p) for p in PATTERNS.values()]
    plans = naive_plans(off, adj, 10.0, threads)
    runs = [run_naive(pl, threads) for pl in plans]
    est = naive_estimate(plans, runs, auts, threads)
    port = oracle_port(off, adj, threads)
    gpu_ms, gpu_matches = 0.0, 0
    for name, rs in port.pop("ranges").items():
        for b, e in rs:
            raw, r = ex.count_range(gr, scheds[name], b, e)
            gpu_ms += r.kernel_ms
            gpu_matches += raw // r.divisor
    assert gpu_matches == port["matches"], (gpu_matches, port["matches"])
    port["engine_on_same_ranges"] = {"value": gpu_matches / (gpu_ms / 1000.0),
                                     "unit": "matches/s", "device_ms": gpu_ms}
    return {"value": est["value"], "unit": "matches/s", "cores": threads, "kind": "reference",
            "sample": naive_sample_text(plans, runs, threads),
            "matches_on_sample": est["matches_on_sample"],
            "estimated_workload_seconds": est["estimated_workload_seconds"],
            "oracle_port": port}


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
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--profile", default=None,
                    help="PATTERN:PARTS[:SHARD], e.g. c4:64:32 - one slice of the search, for ncu")
    args = ap.parse_args()
    if args.impl == "reference":
        # the reference arm never imports this package or loads libgat
        sys.exit(run_reference(args))
    from graphautotune_b200 import _lib

    if not _lib.LIB_PATH.exists():
        from graphautotune_b200 import build

        build.build()
    if args.profile:
        sys.exit(run_profile_case(args))
    sys.exit(run_ours(args))


if __name__ == "__main__":
    main()
