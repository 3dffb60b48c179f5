"""In-process autotuner for launch shapes.

Mirrors the reference tuner (tuning/tuning/): a discrete config space over
flat dotted keys (tuning/tuning/config/base.py:170-222), the same md5
fingerprint of the sorted-key index list (base.py:259-262), random warm-up
configurations, simulated-annealing proposals ranked by a cost model
(role/manipulator.py:63-131: temperature 0.1, x0.9 per step), and a
record.json history of [value dict, seconds] pairs that is reloaded on start
(role/modeling.py:48-79).  The differences: a configuration is applied at
run time (no header export, no CMake rebuild per configuration), it is
measured in process with CUDA events, and the cost model is pluggable
(`model=`): by default the measured history itself (nearest measured point),
or the learned MLP of graphautotune_b200.costmodel.

PmDriver keeps the reference's process protocol instead: it runs the
pm-compatible CLI with the configuration file and a hash, and reads
<results>/<hash>/time.txt and count.txt (role/driver.py:88-132).
"""
from __future__ import annotations

import hashlib
import json
import math
import os
import random
import subprocess
from pathlib import Path

import graphautotune_b200 as g

INT_MAX = 2**31 - 1

# Flat key -> allowed values.  The first eight keys are the reference's
# (tuning/tuning/config/details.py:11-85, with this engine's value sets);
# the last two are this engine's own knobs.
SPACE: dict[str, list] = {
    "vertex_set_config.set_search_type": [0, 4, 16, 64, INT_MAX],
    "vertex_set_config.set_intersection_type": ["Parallel"],
    "vertex_set_config.vertex_store_type": ["Array"],
    "infra_config.graph_backend_type": ["InMemory"],
    "engine_config.launch_config.num_blocks": [0, 256, 512, 1024],
    "engine_config.launch_config.threads_per_block": [64, 128, 256],
    "engine_config.launch_config.threads_per_warp": [1, 4, 8, 16, 32],
    "engine_config.launch_config.max_regs": [32, 64, 96],
    "engine_config.chunk": [1, 4, 8, 16, 64],
    "engine_config.hub_bitmaps": [0, 1],
}
KEYS = sorted(SPACE)
TUNABLE = [k for k in KEYS if len(SPACE[k]) > 1]


def default_point() -> dict:
    c = g.Config.engine_default()
    return from_config(c)


def from_config(c: "g.Config") -> dict:
    d = {
        "vertex_set_config.set_search_type": c.set_search_type,
        "vertex_set_config.set_intersection_type": "Parallel",
        "vertex_set_config.vertex_store_type": "Array",
        "infra_config.graph_backend_type": "InMemory",
        "engine_config.launch_config.num_blocks": c.num_blocks,
        "engine_config.launch_config.threads_per_block": c.threads_per_block,
        "engine_config.launch_config.threads_per_warp": c.threads_per_warp,
        "engine_config.launch_config.max_regs": c.max_regs,
        "engine_config.chunk": c.chunk,
        "engine_config.hub_bitmaps": c.hub_bitmaps,
    }
    for k in KEYS:  # snap to the space
        if d[k] not in SPACE[k]:
            d[k] = min(SPACE[k], key=lambda v: abs(v - d[k]) if isinstance(v, int) else 0)
    return d


def to_config(d: dict) -> "g.Config":
    c = g.Config.engine_default()
    return c.parse(json.dumps(d))


def index_list(d: dict) -> list[int]:
    return [SPACE[k].index(d[k]) for k in KEYS]


def fingerprint(d: dict) -> str:
    return hashlib.md5(",".join(str(x) for x in index_list(d)).encode()).hexdigest()


def valid(d: dict) -> bool:
    return d["engine_config.launch_config.threads_per_block"] % \
        d["engine_config.launch_config.threads_per_warp"] == 0


def random_point(rng: random.Random) -> dict:
    while True:
        d = {k: rng.choice(SPACE[k]) for k in KEYS}
        if valid(d):
            return d


def random_walk(d: dict, rng: random.Random) -> dict:
    while True:
        k = rng.choice(TUNABLE)
        e = dict(d)
        e[k] = rng.choice([v for v in SPACE[k] if v != d[k]])
        if valid(e):
            return e


class History:
    """Measured (config, seconds) pairs, persisted as record.json; the best
    pair so far goes to best_config.json beside it (the file the reference's
    tuner names as CONF_PATH, tuning/tuning/common/const.py:27-30), as
    [value dict, seconds] like one record entry."""

    def __init__(self, path: str | None = None):
        self.path = Path(path) if path else None
        self.xs: list[dict] = []
        self.ys: list[float] = []
        if self.path and self.path.exists() and self.path.stat().st_size > 0:
            for x, y in json.loads(self.path.read_text()):
                self.xs.append(x)
                self.ys.append(float(y))

    def add(self, x: dict, y: float) -> None:
        self.xs.append(x)
        self.ys.append(y)
        if self.path:
            self.path.parent.mkdir(parents=True, exist_ok=True)
            self.path.write_text(json.dumps([[a, b] for a, b in zip(self.xs, self.ys)]))
            bx, by = self.best()
            (self.path.parent / "best_config.json").write_text(json.dumps([bx, by]))

    def seen(self, x: dict) -> bool:
        f = fingerprint(x)
        return any(fingerprint(a) == f for a in self.xs)

    def best(self) -> tuple[dict, float]:
        i = min(range(len(self.ys)), key=self.ys.__getitem__)
        return self.xs[i], self.ys[i]


class NearestModel:
    """Predicts the time of the closest measured point (index-space L1)."""

    def __init__(self, hist: History):
        self.h = hist

    def predict(self, xs: list[dict]) -> list[float]:
        out = []
        for x in xs:
            ix = index_list(x)
            best = min(range(len(self.h.xs)),
                       key=lambda i: sum(abs(a - b) for a, b in zip(ix, index_list(self.h.xs[i]))))
            out.append(self.h.ys[best])
        return out


def propose(model, hist: History, batch: int, rng: random.Random, n_iter: int = 40
            ) -> list[dict]:
    """Simulated annealing over the model's predictions (temperature 0.1,
    x0.9 per step), keeping the best `batch` unseen points."""
    pts = [random_point(rng) for _ in range(batch)]
    scores = model.predict(pts)
    pool: dict[str, tuple[float, dict]] = {}
    temp = 0.1
    for _ in range(n_iter):
        new = [random_walk(p, rng) for p in pts]
        ns = model.predict(new)
        for i in range(len(pts)):
            if ns[i] <= scores[i] or rng.random() < math.exp((scores[i] - ns[i]) / temp):
                pts[i], scores[i] = new[i], ns[i]
        for p, s in zip(new, ns):
            if not hist.seen(p):
                pool[fingerprint(p)] = (s, p)
        temp *= 0.9
    return [p for _, p in sorted(pool.values(), key=lambda t: t[0])[:batch]]


def pick_schedule(ex: "g.Executor", graph: "g.Graph", pattern: str, parts: int = 256,
                  slices: int = 4, stats_graph=None):
    """Data-aware schedule choice: times every distinct exact plan of the
    best-ranked vertex orders on `slices` spread slices (shards i*P/S of P)
    of its work queue and returns (fastest schedule, [(variant, ms)])."""
    n = g.Schedule.variants(pattern, "exact", stats_graph)
    timings, best = [], None
    for v in range(n):
        s = g.Schedule(pattern, "exact", stats_graph, variant=v)
        ms = sum(ex.count_shard(graph, s, i * parts // slices, parts)[1].kernel_ms
                 for i in range(slices))
        timings.append((v, ms))
        if best is None or ms < best[1]:
            best = (s, ms)
    return best[0], timings


def measure_batch(b: "g.Batch", d: dict, reps: int = 2) -> float:
    b.prepare(to_config(d), cuda_graph=True)
    b.run()
    return min(b.run().kernel_ms for _ in range(reps)) / 1e3


def tune_batch(b: "g.Batch", budget: int = 12, seed: int = 0, record: str | None = None,
               model=None, screen: "g.Batch | None" = None, screen_factor: float = 3.0
               ) -> tuple["g.Config", list]:
    """Measures the default point, a few random warm-up points, then model-ranked
    proposals, `budget` points in all; returns the best config.

    With a `screen` batch (a much smaller sample of the same jobs), every
    point is first timed there; a point more than `screen_factor` times
    slower than the best screened point so far is not measured on `b` and
    is recorded at its screened time scaled by the last measured
    full-to-screen ratio (a bad launch shape can be 1000x slower than a good
    one, and would otherwise dominate the tuning time)."""
    rng = random.Random(seed)
    hist = History(record)
    todo = [default_point()] + [random_point(rng) for _ in range(max(1, budget // 3))]
    best_screen, ratio = math.inf, None
    while len(hist.xs) < budget:
        if not todo:
            m = model or NearestModel(hist)
            todo = propose(m, hist, 3, rng)
            if not todo:
                todo = [random_point(rng)]
        d = todo.pop(0)
        if hist.seen(d) or not valid(d):
            continue
        ts = None
        if screen is not None:
            ts = measure_batch(screen, d, reps=1)
            if ratio is not None and ts > screen_factor * best_screen:
                hist.add(d, ts * ratio)
                continue
            best_screen = min(best_screen, ts)
        y = measure_batch(b, d)
        if ts:
            ratio = y / ts
        hist.add(d, y)
    best, _ = hist.best()
    return to_config(best), [[fingerprint(x), y] for x, y in zip(hist.xs, hist.ys)]


def tune_count(graph: "g.Graph", schedule: "g.Schedule", budget: int = 16, seed: int = 0,
               record: str | None = None, model=None, reps: int = 2
               ) -> tuple["g.Config", list, dict]:
    """In-process tuning of one (graph, pattern) count: the default point,
    a few random warm-up points, then proposals ranked by `model` (the
    learned cost model's TunerModel, or the nearest measured point), `budget`
    points measured in all by the count's device time (best of `reps`).
    Returns (best config, history, {fingerprint: count}); every point must
    give the same count."""
    rng = random.Random(seed)
    hist = History(record)
    todo = [default_point()] + [random_point(rng) for _ in range(max(1, budget // 3))]
    counts: dict[str, int] = {}
    while len(hist.xs) < budget:
        if not todo:
            todo = propose(model or NearestModel(hist), hist, 3, rng) or [random_point(rng)]
        d = todo.pop(0)
        if hist.seen(d) or not valid(d):
            continue
        ex = g.Executor(to_config(d))
        rs = [ex.count(graph, schedule) for _ in range(reps)]
        counts[fingerprint(d)] = rs[0].count
        hist.add(d, min(r.kernel_ms for r in rs) / 1e3)
    assert len(set(counts.values())) == 1, "configurations disagree on the count"
    best, _ = hist.best()
    return to_config(best), [[fingerprint(x), y] for x, y in zip(hist.xs, hist.ys)], counts


class PmDriver:
    """The reference driver's protocol (role/driver.py:88-132) over the
    pm-compatible CLI: runs `pm <graph> <pattern> <hash> --config <file>` and
    reads <results>/<hash>/time.txt; a non-zero exit maps to FLOAT_INF."""

    FLOAT_INF = 1e38

    def __init__(self, graph: str, pattern: str, workdir: str, mode: str = "exact"):
        self.graph, self.pattern, self.mode = graph, pattern, mode
        self.workdir = Path(workdir)
        self.pm = Path(__file__).resolve().parent / "bin" / "pm"

    def run(self, d: dict) -> float:
        h = fingerprint(d)
        cdir = self.workdir / "build_tuning" / h
        cdir.mkdir(parents=True, exist_ok=True)
        (cdir / "config.json").write_text(json.dumps(d))
        res = self.workdir / "tuning_results"
        r = subprocess.run([str(self.pm), self.graph, self.pattern, h, "--mode", self.mode,
                            "--config", str(cdir / "config.json"), "--results-dir", str(res)],
                           capture_output=True, text=True, env=dict(os.environ))
        if r.returncode != 0:
            return self.FLOAT_INF
        return float((res / h / "time.txt").read_text().strip())

    def count(self, d: dict) -> int:
        return int((self.workdir / "tuning_results" / fingerprint(d) / "count.txt").read_text())
