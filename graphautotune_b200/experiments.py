"""Drivers for the benchmark configurations other than bench.py's headline
(R-MAT 2^20, 4-clique + 4-cycle).  Each prints JSON lines.

    python -m graphautotune_b200.experiments c1      # ER 10^4 triangle: exact, ref, timing
    python -m graphautotune_b200.experiments c3      # R-MAT 2^22 house + 5-clique
    python -m graphautotune_b200.experiments c4 [--tune N]
                                                     # 21 patterns x 64 graphs: plain
                                                     # launches vs one batched launch
    python -m graphautotune_b200.experiments c5 [--model cm.npz]
                                                     # R-MAT 2^24: 6-clique in full, the
                                                     # other two patterns on slices with
                                                     # cost-model picks

Graphs are synthetic and seeded (splitmix64 streams in libgat), built on the
device.
"""
from __future__ import annotations

import argparse
import json
import math
import sys
import time

import numpy as np

import graphautotune_b200 as g

TRIANGLE = "011101110"
HOUSE_P2 = "0100110110010110110010100"
K5 = "0111110111110111110111110"


def emit(**kw):
    print(json.dumps(kw), flush=True)


def splitmix(x: int) -> int:
    x = (x + 0x9E3779B97F4A7C15) & (2**64 - 1)
    z = x
    z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & (2**64 - 1)
    z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & (2**64 - 1)
    return z ^ (z >> 31)


def c4_graph_spec(seed: int) -> dict:
    """Configuration 4's graph for `seed` (100..163): n log-uniform in
    [10^4, 10^6]; even seeds R-MAT with average degree 16 on 2^round(log2 n)
    vertices (R-MAT needs a power of two), odd seeds Barabasi-Albert with m
    drawn uniformly from 4..32."""
    u = (splitmix(seed) >> 11) / float(1 << 53)
    n = int(round(10 ** (4 + 2 * u)))
    if seed % 2 == 0:
        scale = max(1, int(round(math.log2(n))))
        return {"seed": seed, "kind": "rmat", "scale": scale, "samples": 8 << scale}
    m = 4 + (splitmix(seed ^ 0x5EED) % 29)
    return {"seed": seed, "kind": "ba", "n": n, "m": int(m)}


def make_graph(spec: dict, device: bool = True) -> "g.Graph":
    if spec["kind"] == "rmat":
        return g.Graph.rmat(spec["scale"], spec["samples"], 0.57, 0.19, 0.19, spec["seed"],
                            device=device)
    return g.Graph.barabasi_albert(spec["n"], spec["m"], spec["seed"], device=device)


def plain_config() -> "g.Config":
    """The engine's default configuration, as a user gets it without tuning
    (one launch per (pattern, graph) job is the 'plain' arm)."""
    return g.Config.engine_default()


def run_c1(args):
    gr = g.Graph.erdos_renyi(10000, 16.0, 1)
    V, E, md = gr.info()
    ex = g.Executor()
    for mode in ("exact", "ref"):
        s = g.Schedule(TRIANGLE, mode)
        r = ex.count(gr, s)
        times = [ex.count(gr, s).kernel_ms for _ in range(5)]
        emit(config="c1", mode=mode, V=V, E=E, count=r.count, kernel_ms=min(times),
             matches_per_s=(r.count if mode == "exact" else r.count / 3) / (min(times) / 1e3))


def run_c2(args):
    """R-MAT 2^20 (2^24 samples, seed 2): the 4-clique and the 4-cycle with
    the default configuration and with the configuration the in-process
    autotuner finds (tuner.tune_count: `--tune` measured points, proposals
    ranked by the cost model when --model is given); counts must agree."""
    from graphautotune_b200 import costmodel, tuner

    gr = g.Graph.rmat(20, 1 << 24, 0.57, 0.19, 0.19, 2, device=True)
    gr.upload(degree_order=True)
    V, E, md = gr.info()
    emit(config="c2", graph="R-MAT scale 20, 2^24 samples, seed 2", V=V, E=E, max_degree=md)
    for name, pat in (("k4", "0111101111011110"), ("c4", "0101101001011010")):
        s = g.Schedule(pat, "exact", stats_graph=gr)
        ex = g.Executor()
        ex.count(gr, s)
        rs = [ex.count(gr, s) for _ in range(3)]
        t_def = min(r.kernel_ms for r in rs)
        model = None
        if args.model:
            model = costmodel.TunerModel(costmodel.CostModel.load(args.model),
                                         costmodel.graph_features(gr),
                                         costmodel.plan_features(s))
        t0 = time.time()
        cfg, hist, counts = tuner.tune_count(gr, s, budget=max(args.tune, 4), model=model)
        ex_t = g.Executor(cfg)
        rt = [ex_t.count(gr, s) for _ in range(3)]
        t_tuned = min(r.kernel_ms for r in rt)
        assert rt[0].count == rs[0].count
        emit(config="c2", pattern=name, count=rs[0].count, default_ms=t_def, tuned_ms=t_tuned,
             tuned_vs_default=t_def / t_tuned, points=len(hist), tuning_s=time.time() - t0,
             kernel="dedicated" if s.dedicated_kernel else "schedule plan",
             tuned={k: getattr(cfg, k) for k in cfg._FIELDS})


def run_c3(args):
    """R-MAT 2^22 (2^26 samples, seed 3): house and 5-clique, exact and
    reference-compatible.  Every pattern is first timed on `--slices`
    work-queue slices spread over the whole queue (shards i*P/S of P), which
    gives the slices' throughput, their algorithmic GB/s and an estimate of
    the full count's time; the full count runs when the estimate is below
    `--max-seconds`."""
    t0 = time.time()
    gr = g.Graph.rmat(22, 1 << 26, 0.57, 0.19, 0.19, 3, device=True)
    V, E, md = gr.info()
    gr.upload(degree_order=True)
    emit(config="c3", graph="R-MAT scale 22, 2^26 samples, seed 3", V=V, E=E, max_degree=md,
         setup_s=time.time() - t0)
    ex = g.Executor()
    out = {}
    parts, nsl = args.parts, args.slices
    from graphautotune_b200 import tuner

    for name, pat in (("house", HOUSE_P2), ("k5", K5)):
        for mode in ("exact", "ref"):
            s = g.Schedule(pat, mode)
            if mode == "exact" and g.Schedule.variants(pat) > 1:
                s, tim = tuner.pick_schedule(ex, gr, pat, parts=parts, slices=2)
                emit(config="c3", pattern=name, schedule_variants=tim, picked=s.variant)
            raw = ms = gb = 0
            div = 1
            for i in range(nsl):
                sh = i * parts // nsl
                r0, rs = ex.count_shard(gr, s, sh, parts)
                raw += r0
                ms += rs.kernel_ms
                div = rs.divisor
                _, rbs = ex.count_shard(gr, s, sh, parts, balg=True)
                gb += rbs.balg_bytes
            est_s = ms * parts / nsl / 1e3
            emit(config="c3", pattern=name, mode=mode, slices=f"{nsl} of {parts}",
                 slice_kernel_ms=ms, slice_matches=raw / div,
                 slice_matches_per_s=raw / div / (ms / 1e3),
                 slice_alg_GBps=gb / (ms / 1e3) / 1e9, estimate_full_s=est_s)
            if est_s > args.max_seconds:
                continue
            r = ex.count(gr, s)
            out[(name, mode)] = r.count
            emit(config="c3", pattern=name, mode=mode, count=r.count, kernel_ms=r.kernel_ms,
                 matches_per_s=r.count / (r.kernel_ms / 1e3) if mode == "exact" else None)
    if ("house", "exact") in out and ("house", "ref") in out:
        emit(config="c3", check="ref house (P2 labelling) == exact house",
             ok=out[("house", "exact")] == out[("house", "ref")])
    if ("k5", "exact") in out and ("k5", "ref") in out:
        emit(config="c3", check="ref 5-clique == 5 x exact", ok=out[("k5", "ref")] ==
             5 * out[("k5", "exact")])


def c4_jobs(graphs, patterns):
    return [(gi, p) for gi in range(len(graphs)) for p in patterns]


def _spec_size(sp: dict) -> int:
    return 1 << sp["scale"] if sp["kind"] == "rmat" else sp["n"]


def run_c4(args):
    seeds = list(range(100, 100 + args.graphs))
    t0 = time.time()
    specs = [c4_graph_spec(s) for s in seeds]
    if args.smallest:
        # the K smallest graphs of the set (by vertex count), in seed order
        keep = sorted(sorted(specs, key=_spec_size)[:args.smallest], key=lambda sp: sp["seed"])
        specs = keep
    graphs = [make_graph(sp) for sp in specs]
    for gr in graphs:
        gr.upload(degree_order=True)
    pats = g.enumerate_patterns(5)
    scheds = {p: g.Schedule(p, "exact") for p in pats}
    tot_e = sum(gr.info()[1] for gr in graphs)
    emit(config="c4", graphs=len(graphs), patterns=len(pats), total_directed_edges=tot_e,
         setup_s=time.time() - t0, specs=specs)
    ex = g.Executor(plain_config())
    if args.estimate:
        # Per-job cost from `slices` spread-out slices of each job's work
        # queue, extrapolated (no full counts).
        P, nsl = args.estimate, 4
        total = 0.0
        for gi, gr in enumerate(graphs):
            per = []
            for p in pats:
                ms = sum(ex.count_shard(gr, scheds[p], i * P // nsl, P)[1].kernel_ms
                         for i in range(nsl))
                per.append(round(ms * P / nsl, 2))
            total += sum(per)
            emit(config="c4", estimate_graph=gi, spec=specs[gi], E=gr.info()[1],
                 est_ms_per_pattern=per, est_ms=sum(per))
        emit(config="c4", estimate_total_ms=total)
        return
    # plain: one default-config launch per job, each synchronised
    plain_counts, plain_ms, plain_wall = [], 0.0, 0.0
    t = time.perf_counter()
    for gi, gr in enumerate(graphs):
        gms = 0.0
        for p in pats:
            r = ex.count(gr, scheds[p])
            plain_counts.append(r.count)
            plain_ms += r.kernel_ms
            gms += r.kernel_ms
        emit(config="c4", arm="plain", graph=gi, kernel_ms=gms)
    plain_wall = (time.perf_counter() - t) * 1e3
    emit(config="c4", arm="plain", launches=len(plain_counts), kernel_ms=plain_ms,
         wall_ms=plain_wall)
    # batched: one persistent launch over all jobs, CUDA graph replay
    cfg = g.Config.engine_default()
    tscheds = dict(scheds)
    if args.tune:
        from graphautotune_b200 import tuner

        # data-aware schedules: each pattern's fastest exact plan variant on
        # slices of the set's largest graph
        big = max(graphs, key=lambda gr: gr.info()[1])
        t = time.perf_counter()
        chosen = {}
        for p in pats:
            tscheds[p], tim = tuner.pick_schedule(ex, big, p, parts=64, slices=4)
            chosen[p] = {"variant": tscheds[p].variant, "slice_ms": tim}
        emit(config="c4", arm="schedules", picked=chosen, seconds=time.perf_counter() - t)
    # Jobs whose pattern has a dedicated kernel (the 5-clique) keep it: they
    # are counted by the executor, the others in the one batched launch.
    dedicated = [p for p in pats if scheds[p].dedicated_kernel]
    bpats = [p for p in pats if p not in dedicated]
    b = g.Batch()
    for gr in graphs:
        for p in bpats:
            b.add(gr, tscheds[p])
    if args.tune:

        # Launch shapes are timed on a sample batch: one slice of 1/P of every
        # job's work queue, slices spread over the queues.
        P = args.tune_parts
        sample, screen = g.Batch(), g.Batch()
        for j, (gr, p) in enumerate((gr, p) for gr in graphs for p in bpats):
            sample.add_shard(gr, tscheds[p], (j * 7) % P, P)
            screen.add_shard(gr, tscheds[p], (j * 7) % (8 * P), 8 * P)
        model = None
        if args.model:
            # proposals ranked by the learned cost model (summed over the jobs)
            from graphautotune_b200 import costmodel

            gfs = [costmodel.graph_features(gr) for gr in graphs]
            pfs = {p: costmodel.plan_features(tscheds[p]) for p in pats}
            model = costmodel.BatchTunerModel(costmodel.CostModel.load(args.model),
                                              [(gf, pfs[p]) for gf in gfs for p in bpats])
        t = time.perf_counter()
        cfg, hist = tuner.tune_batch(sample, budget=args.tune, model=model, screen=screen)
        emit(config="c4", arm="tuner", sample=f"1/{P} of every job", history=hist,
             ranking="cost model" if model else "nearest measured point",
             tuning_s=time.perf_counter() - t)
    b.prepare(cfg, cuda_graph=True)

    def run_all():
        t = time.perf_counter()
        r = b.run()
        ms = r.kernel_ms
        dcounts = {}
        for gi, gr in enumerate(graphs):
            for p in dedicated:
                rd = ex.count(gr, scheds[p])
                dcounts[(gi, p)] = rd.count
                ms += rd.kernel_ms
        return (time.perf_counter() - t) * 1e3, ms, dcounts

    runs = [run_all()]
    while len(runs) < 3 and runs[-1][0] < 10000:  # long batches need no warm-up repeats
        runs.append(run_all())
    bc = iter(b.counts())
    dcounts = runs[-1][2]
    counts = [dcounts[(gi, p)] if p in dedicated else next(bc)
              for gi in range(len(graphs)) for p in pats]
    assert counts == plain_counts, "batched counts differ from the plain launches"
    best_wall = min(x[0] for x in runs)
    emit(config="c4", arm="batched", launches=1 + len(graphs) * len(dedicated),
         dedicated_kernel_jobs=len(graphs) * len(dedicated),
         kernel_ms=min(x[1] for x in runs),
         wall_ms=best_wall, config_used={k: getattr(cfg, k) for k in cfg._FIELDS},
         speedup_vs_plain_wall=plain_wall / best_wall, counts_equal=True,
         matches=sum(counts))


def _edges(n, pairs):
    s = ["0"] * (n * n)
    for u, v in pairs:
        s[u * n + v] = s[v * n + u] = "1"
    return "".join(s)


C5_PATTERNS = {
    "k6": _edges(6, [(i, j) for i in range(6) for j in range(i + 1, 6)]),
    "c6_chord": _edges(6, [(0, 1), (1, 2), (2, 3), (3, 4), (4, 5), (5, 0), (0, 3)]),
    "tri_path_7v": _edges(7, [(0, 1), (1, 2), (0, 2), (2, 3), (3, 4), (4, 5), (5, 6)]),
}


def c5_candidates() -> list[dict]:
    """The launch-shape sub-space measured exhaustively: tile x block x
    chunk x hub bitmaps, binary search, persistent grid."""
    from graphautotune_b200 import tuner

    base = tuner.default_point()
    out = []
    for tile in (4, 8, 16, 32):
        for block in (128, 256):
            for chunk in (1, 4, 16, 64):
                for hub in (0, 1):
                    d = dict(base)
                    d["engine_config.launch_config.threads_per_warp"] = tile
                    d["engine_config.launch_config.threads_per_block"] = block
                    d["engine_config.chunk"] = chunk
                    d["engine_config.hub_bitmaps"] = hub
                    out.append(d)
    return out


def eval_c5(model, parts: int = 256, n_candidates: int = 64, graph=None, names=None):
    """Configuration 5: the cost model picks a launch configuration for 6- and
    7-vertex patterns on R-MAT 2^24 (average degree 24, seed 4); compared with
    the default configuration and the best of the exhaustively measured
    candidates.  Every measurement counts the same slice of the work queue
    (shard 0 of `parts`) so that all configurations do identical work; counts
    must agree across configurations."""
    from graphautotune_b200 import costmodel, tuner

    t0 = time.time()
    gr = graph
    if gr is None:
        gr = g.Graph.rmat(24, 12 << 24, 0.57, 0.19, 0.19, 4, device=True)
        gr.upload(degree_order=True)
    V, E, md = gr.info()
    gf = costmodel.graph_features(gr)
    emit(config="c5", graph="R-MAT scale 24, 12*2^24 samples (avg degree 24), seed 4", V=V,
         E=E, max_degree=md, setup_s=time.time() - t0)
    default = tuner.default_point()
    allc = c5_candidates()
    # an evenly spread subset of the launch-shape space, with the default in it
    step = max(1, len(allc) // max(1, n_candidates))
    cands = allc[::step][:n_candidates]
    if all(tuner.fingerprint(c) != tuner.fingerprint(default) for c in cands):
        cands = [default] + cands[:-1]
    for name, pat in C5_PATTERNS.items():
        if names is not None and name not in names:
            continue
        s = g.Schedule(pat, "exact", stats_graph=gr)
        pf = costmodel.plan_features(s)
        # The slice: the middle shard of P, P grown from `parts` until the
        # default configuration counts it in under 3 s.
        P = parts
        while True:
            sh = P // 2
            t0 = time.time()
            _, r = g.Executor(tuner.to_config(default)).count_shard(gr, s, sh, P)
            emit(config="c5", pattern=name, sizing=f"shard {sh} of {P}", default_ms=r.kernel_ms)
            if r.kernel_ms < 100 or P >= parts << 8:
                break
            P <<= 2

        def measure(d):
            ex = g.Executor(tuner.to_config(d))
            raw, r = ex.count_shard(gr, s, sh, P)
            raw2, r2 = ex.count_shard(gr, s, sh, P)
            assert raw == raw2
            return raw, min(r.kernel_ms, r2.kernel_ms)

        # Every configuration is first timed on a slice 8x smaller; one more
        # than 4x slower there than the default is not measured on the full
        # slice (a bad launch shape can be 100x slower than a good one).
        def screen(d):
            return g.Executor(tuner.to_config(d)).count_shard(gr, s, 4 * P, 8 * P)[1].kernel_ms

        ts0 = screen(default)
        raw0, t_default = measure(default)
        emit(config="c5", pattern=name, slice=f"shard {sh} of {P}", default_ms=t_default)
        t_budget = time.time() + 60.0  # per pattern: candidates measured until then
        if t_default > 20000:
            emit(config="c5", pattern=name, skipped="slice too slow")
            continue
        picked, kept_default = costmodel.choose(model, gf, pf, cands, default)
        tsp = screen(picked)
        raw_p, t_pick = measure(picked) if tsp <= 4 * ts0 else (raw0, math.inf)
        emit(config="c5", pattern=name, model_pick_ms=t_pick, kept_default=kept_default)
        times, screened, cands_m = [], 0, []
        for d in cands:
            if times and time.time() > t_budget:
                break
            if screen(d) > 4 * ts0:
                screened += 1
                continue
            raw_c, t_c = measure(d)
            assert raw_c == raw0, "counts differ across configurations"
            times.append(t_c)
            cands_m.append(d)
        best = int(np.argmin(times))
        pred = model.predict(np.stack([costmodel.features(gf, pf, d) for d in cands_m]))
        rank_corr = float(np.corrcoef(np.argsort(np.argsort(pred)),
                                      np.argsort(np.argsort(times)))[0, 1]) \
            if len(times) > 2 else None
        best_ms = min(times[best], t_pick, t_default)
        emit(config="c5", pattern=name, slice_raw_count=raw0, default_ms=t_default,
             model_pick_ms=t_pick, best_measured_ms=best_ms,
             median_candidate_ms=float(np.median(times)),
             pick_vs_default=t_default / t_pick, pick_vs_best=best_ms / t_pick,
             kept_default=kept_default, screened_out=screened,
             spearman_pred_vs_measured=rank_corr, candidates=len(cands_m),
             picked={k.split(".")[-1]: v for k, v in picked.items()},
             best={k.split(".")[-1]: v for k, v in cands_m[best].items()})


def run_c5(args):
    """R-MAT 2^24 (12 * 2^24 samples, average degree 24, seed 4): the
    6-clique counted over the whole graph by the clique kernels (the launch
    configuration does not enter them), then, with --model, the 6-cycle with
    chord and the 7-vertex triangle + path on work-queue slices, where the
    cost model picks the launch configuration and is compared with the
    default and the best measured candidate (eval_c5)."""
    t0 = time.time()
    gr = g.Graph.rmat(24, 12 << 24, 0.57, 0.19, 0.19, 4, device=True)
    t_gen = time.time() - t0
    t0 = time.time()
    gr.upload(degree_order=True)
    V, E, md = gr.info()
    emit(config="c5", graph="R-MAT scale 24, 12*2^24 samples (avg degree 24), seed 4", V=V,
         E=E, max_degree=md, generate_on_device_s=t_gen, upload_s=time.time() - t0)
    # The 6-clique: the clique kernels on spread slices of the level-1 units
    # (the full count is out of reach of one call's time), and the schedule
    # plan path on the middle slice for comparison; counts must agree.
    ex = g.Executor()
    plan_cfg = g.Config.engine_default()
    plan_cfg.special_kernels = 0
    ex_plan = g.Executor(plan_cfg)
    s = g.Schedule(C5_PATTERNS["k6"], "exact", stats_graph=gr)
    P, nsl = args.parts, 8
    raw = ms = 0
    done = 0
    for i in range(nsl):
        sh = i * P // nsl
        r0, rs = ex.count_shard(gr, s, sh, P)
        raw += r0
        ms += rs.kernel_ms
        done += 1
        emit(config="c5", pattern="k6", slice=f"shard {sh} of {P}", count=r0,
             clique_kernels_ms=rs.kernel_ms)
        if ms > args.max_seconds * 1e3:
            break
    nsl = done
    emit(config="c5", pattern="k6", slices=f"{nsl} of {P}", slice_count=raw,
         slice_ms=ms, matches_per_s=raw / (ms / 1e3), estimate_full_s=ms * P / nsl / 1e3)
    sh = P // 2
    rc, rcs = ex.count_shard(gr, s, sh, P)
    rp, rps = ex_plan.count_shard(gr, s, sh, P)
    assert rc == rp, "clique kernels and schedule plan disagree"
    emit(config="c5", pattern="k6", slice=f"shard {sh} of {P}", count=rc,
         clique_kernels_ms=rcs.kernel_ms, schedule_plan_ms=rps.kernel_ms,
         speedup=rps.kernel_ms / rcs.kernel_ms)
    if args.model:
        from graphautotune_b200.costmodel import CostModel

        eval_c5(CostModel.load(args.model), parts=args.parts, graph=gr,
                names=["c6_chord", "tri_path_7v"], n_candidates=args.candidates)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("config", choices=["c1", "c2", "c3", "c4", "c5"])
    ap.add_argument("--graphs", type=int, default=64)
    ap.add_argument("--tune", type=int, default=0)
    ap.add_argument("--max-seconds", type=float, default=120.0)
    ap.add_argument("--parts", type=int, default=1024)
    ap.add_argument("--tune-parts", type=int, default=32)
    ap.add_argument("--model", default=None, help="c4: cost model file for the tuner")
    ap.add_argument("--smallest", type=int, default=0,
                    help="c4: only the K smallest of the graphs")
    ap.add_argument("--estimate", type=int, default=0,
                    help="c4: estimate every job from 4 slices of 1/N of its queue")
    ap.add_argument("--slices", type=int, default=8)
    ap.add_argument("--candidates", type=int, default=16,
                    help="c5: launch configurations measured per pattern")
    args = ap.parse_args()
    import torch

    torch.cuda.set_device(0)
    {"c1": run_c1, "c2": run_c2, "c3": run_c3, "c4": run_c4, "c5": run_c5}[args.config](args)


if __name__ == "__main__":
    sys.exit(main())
