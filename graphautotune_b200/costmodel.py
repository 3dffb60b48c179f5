"""Learned cost model for schedule/configuration choice.

A 3-layer FP32 perceptron (libgat's gat_mlp_*: hand-written forward,
backward and Adam kernels) maps features of (plan, launch configuration,
data graph) to log run time.  It is trained on timings the engine itself
records (`collect`), and used to rank candidate configurations (`pick`),
replacing the reference tuner's XGBoost model over configuration indices
(tuning/tuning/role/modeling.py:81-102); the measured-search tuner
(graphautotune_b200.tuner) is its fallback, and measured times are what its
ranking is checked against.

    python -m graphautotune_b200.costmodel collect --runs 20000 --out data.npz
    python -m graphautotune_b200.costmodel train data.npz --out model.npz
    python -m graphautotune_b200.costmodel eval5 --model model.npz
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import math
import random
import sys
import time

import numpy as np

import graphautotune_b200 as g
from graphautotune_b200 import tuner
from graphautotune_b200._lib import check, lib

HIST_BUCKETS = 15
N_FEATURES = 7 + 11 + 5 + HIST_BUCKETS


def _bind():
    l = lib()
    P = C.c_void_p
    fp = C.POINTER(C.c_float)
    sigs = {
        "gat_mlp_create": (C.c_int, [C.c_int, C.c_uint64, C.POINTER(P)]),
        "gat_mlp_free": (None, [P]),
        "gat_mlp_num_params": (C.c_int, [P]),
        "gat_mlp_get_params": (C.c_int, [P, fp, C.c_int]),
        "gat_mlp_set_params": (C.c_int, [P, fp, C.c_int]),
        "gat_mlp_predict": (C.c_int, [P, fp, C.c_int, fp]),
        "gat_mlp_gradient": (C.c_int, [P, fp, fp, C.c_int, fp, fp]),
        "gat_mlp_train": (C.c_int, [P, fp, fp, C.c_int, C.c_int, C.c_int, C.c_float,
                                    C.c_uint64, fp]),
        "gat_mlp_last_error": (C.c_char_p, []),
    }
    for name, (res, args) in sigs.items():
        f = getattr(l, name)
        f.restype, f.argtypes = res, args
    return l


def _fp(a: np.ndarray):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def _check_mlp(rc: int) -> None:
    if rc != 0:
        raise g.GatError(rc, lib().gat_mlp_last_error().decode())


class MLP:
    """gat_mlp handle: in -> 64 -> 64 -> 1."""

    def __init__(self, in_features: int = N_FEATURES, seed: int = 0):
        self.l = _bind()
        self.h = C.c_void_p()
        self.in_features = in_features
        _check_mlp(self.l.gat_mlp_create(in_features, seed, C.byref(self.h)))

    def __del__(self):
        if getattr(self, "h", None) and self.h.value:
            self.l.gat_mlp_free(self.h)

    @property
    def num_params(self) -> int:
        return self.l.gat_mlp_num_params(self.h)

    def params(self) -> np.ndarray:
        out = np.zeros(self.num_params, np.float32)
        _check_mlp(self.l.gat_mlp_get_params(self.h, _fp(out), len(out)))
        return out

    def set_params(self, p: np.ndarray) -> None:
        p = np.ascontiguousarray(p, np.float32)
        _check_mlp(self.l.gat_mlp_set_params(self.h, _fp(p), len(p)))

    def predict(self, X: np.ndarray) -> np.ndarray:
        X = np.ascontiguousarray(X, np.float32)
        y = np.zeros(len(X), np.float32)
        _check_mlp(self.l.gat_mlp_predict(self.h, _fp(X), len(X), _fp(y)))
        return y

    def gradient(self, X: np.ndarray, T: np.ndarray) -> tuple[np.ndarray, float]:
        X = np.ascontiguousarray(X, np.float32)
        T = np.ascontiguousarray(T, np.float32)
        grad = np.zeros(self.num_params, np.float32)
        loss = C.c_float()
        _check_mlp(self.l.gat_mlp_gradient(self.h, _fp(X), _fp(T), len(X), _fp(grad),
                                           C.byref(loss)))
        return grad, loss.value

    def train(self, X: np.ndarray, T: np.ndarray, epochs: int = 200, batch: int = 256,
              lr: float = 1e-3, seed: int = 0) -> float:
        X = np.ascontiguousarray(X, np.float32)
        T = np.ascontiguousarray(T, np.float32)
        loss = C.c_float()
        _check_mlp(self.l.gat_mlp_train(self.h, _fp(X), _fp(T), len(X), epochs, batch, lr,
                                        seed, C.byref(loss)))
        return loss.value


# ------------------------------------------------------------------ features

def graph_features(graph: "g.Graph") -> np.ndarray:
    off, _ = graph.csr()
    deg = np.diff(off)
    V = max(len(deg), 1)
    E = int(off[-1])
    md = int(deg.max()) if len(deg) else 0
    hist = np.zeros(HIST_BUCKETS, np.float32)
    nz = deg[deg > 0]
    if len(nz):
        b = np.minimum(np.floor(np.log2(nz)).astype(int), HIST_BUCKETS - 1)
        hist += np.bincount(b, minlength=HIST_BUCKETS)[:HIST_BUCKETS] / V
    hub = float(deg[deg >= 512].sum()) / max(E, 1)
    return np.concatenate([[math.log10(V) / 7, math.log10(max(E, 1)) / 9,
                            math.log10(max(md, 1)) / 6, (E / V) / 64, hub], hist]).astype(
        np.float32)


def plan_features(sched: "g.Schedule") -> np.ndarray:
    raw = sched.plan_bytes()
    i32 = np.frombuffer(raw[:40], np.int32)
    n, basic, num_prefix, mode, collide, l1b, num_store, iep_num, num_terms, special = i32[:10]
    divisor = np.frombuffer(raw[40:48], np.int64)[0]
    kinds = np.frombuffer(raw[48 + 64:48 + 96], np.int8)[:num_prefix]
    edges = sched.pattern.adjacency().count("1") // 2
    return np.array([n / 10, basic / 10, num_prefix / 16, num_store / 8, iep_num / 8,
                     num_terms / 16, math.log2(max(int(divisor), 1)) / 10, float(l1b),
                     float((kinds == 2).sum()) / 8, edges / 45,
                     float(special != 0)], np.float32)


def config_features(d: dict) -> np.ndarray:
    s = d["vertex_set_config.set_search_type"]
    nb = d["engine_config.launch_config.num_blocks"]
    return np.array([math.log2(s + 1) / 31, float(nb == 0), math.log2(nb + 1) / 11,
                     math.log2(d["engine_config.launch_config.threads_per_block"]) / 8,
                     math.log2(d["engine_config.launch_config.threads_per_warp"]) / 5,
                     math.log2(d["engine_config.chunk"]) / 6,
                     float(d["engine_config.hub_bitmaps"])], np.float32)


def features(gf: np.ndarray, pf: np.ndarray, d: dict) -> np.ndarray:
    return np.concatenate([config_features(d), pf, gf]).astype(np.float32)


# ---------------------------------------------------------------- data

EXEC_BUDGET = 256 << 20  # scratch budget of the executors that gather timings


def training_graphs(count: int, seed0: int = 1000, max_log2: int = 16) -> list[dict]:
    """Graphs like configuration 4's, smaller: n log-uniform in
    [2^10, 2^max_log2], half R-MAT (average degree 16), half
    Barabasi-Albert (m in 4..32)."""
    from graphautotune_b200.experiments import splitmix

    specs = []
    for i in range(count):
        s = seed0 + i
        u = (splitmix(s) >> 11) / float(1 << 53)
        n = int(2 ** (10 + (max_log2 - 10) * u))
        if i % 2 == 0:
            scale = max(1, int(round(math.log2(n))))
            specs.append({"seed": s, "kind": "rmat", "scale": scale, "samples": 8 << scale})
        else:
            specs.append({"seed": s, "kind": "ba", "n": n, "m": 4 + splitmix(s ^ 7) % 29})
    return specs


def collect(runs: int, seed: int = 0, graphs: int = 24, max_ms: float = 200.0,
            log=None, max_seconds: float = 0.0, max_log2: int = 16,
            checkpoint: str | None = None, every: int = 500
            ) -> tuple[np.ndarray, np.ndarray]:
    """Times `runs` random (graph, pattern, configuration) counts (fewer if
    `max_seconds` > 0 runs out first).  With `checkpoint`, the rows gathered
    so far are saved there every `every` runs, and a run that finds the file
    keeps its rows and adds new ones (drawn from a stream seeded by the
    seed and the number of rows already there)."""
    from graphautotune_b200.experiments import make_graph

    rng = random.Random(seed)
    pats = g.enumerate_patterns(4) + g.enumerate_patterns(5)
    glist = []
    for sp in training_graphs(graphs, max_log2=max_log2):
        gr = make_graph(sp)
        gr.upload(degree_order=True)
        glist.append((gr, graph_features(gr)))
    # every pattern's first two exact plan variants, so that the model also
    # sees how plans of one pattern differ (later variants are often far
    # slower and would dominate the collection time)
    scheds = [g.Schedule(p, "exact", variant=v) for p in pats
              for v in range(min(2, g.Schedule.variants(p)))]
    pfs = [plan_features(s) for s in scheds]
    X, T = [], []
    if checkpoint:
        import os

        if os.path.exists(checkpoint):
            z = np.load(checkpoint)
            X, T = list(z["X"]), list(z["T"])
            rng = random.Random(seed * 1000003 + len(X))
            if log:
                log(f"resumed {len(X)} runs from {checkpoint}")
    # a few executors at a time (each keeps its scratch), with a modest
    # memory budget: thousands of random configurations are visited
    from collections import OrderedDict

    execs: "OrderedDict[str, g.Executor]" = OrderedDict()
    slow: set = set()
    t0 = time.time()
    while len(X) < runs and not (max_seconds > 0 and time.time() - t0 > max_seconds):
        gi, si = rng.randrange(len(glist)), rng.randrange(len(scheds))
        if (gi, si) in slow:
            continue
        d = tuner.random_point(rng)
        key = tuner.fingerprint(d)
        if key not in execs:
            cfg = tuner.to_config(d)
            cfg.memory_budget = EXEC_BUDGET
            execs[key] = g.Executor(cfg)
            if len(execs) > 8:
                execs.popitem(last=False)
        execs.move_to_end(key)
        gr, gf = glist[gi]
        r = execs[key].count(gr, scheds[si])
        if r.kernel_ms > max_ms:
            slow.add((gi, si))  # keep the data set cheap to gather
        X.append(features(gf, pfs[si], d))
        T.append(math.log(max(r.kernel_ms, 1e-3)))
        if checkpoint and len(X) % every == 0:
            np.savez(checkpoint, X=np.stack(X), T=np.array(T, np.float32))
        if log and len(X) % 1000 == 0:
            log(f"collected {len(X)} runs in {time.time() - t0:.1f}s")
    if checkpoint and X:
        np.savez(checkpoint, X=np.stack(X), T=np.array(T, np.float32))
    return np.stack(X), np.array(T, np.float32)


class CostModel:
    def __init__(self, mlp: MLP, mean: np.ndarray, std: np.ndarray):
        self.mlp, self.mean, self.std = mlp, mean, std

    def predict(self, X: np.ndarray) -> np.ndarray:
        return self.mlp.predict((X - self.mean) / self.std)

    def save(self, path: str) -> None:
        np.savez(path, params=self.mlp.params(), mean=self.mean, std=self.std)

    @classmethod
    def load(cls, path: str) -> "CostModel":
        z = np.load(path)
        m = MLP(len(z["mean"]))
        m.set_params(z["params"])
        return cls(m, z["mean"], z["std"])

    @classmethod
    def fit(cls, X: np.ndarray, T: np.ndarray, epochs: int = 200, seed: int = 0,
            lr: float = 1e-3) -> tuple["CostModel", float]:
        mean = X.mean(0)
        std = X.std(0) + 1e-6
        m = MLP(X.shape[1], seed)
        loss = m.train((X - mean) / std, T, epochs=epochs, lr=lr, seed=seed)
        return cls(m, mean, std), loss


class TunerModel:
    """Adapter so the tuner's simulated annealing ranks points with the MLP."""

    def __init__(self, model: CostModel, gf: np.ndarray, pf: np.ndarray):
        self.model, self.gf, self.pf = model, gf, pf

    def predict(self, xs: list[dict]) -> list[float]:
        X = np.stack([features(self.gf, self.pf, d) for d in xs])
        return self.model.predict(X).tolist()


class BatchTunerModel:
    """Ranks launch shapes for a whole batch: the log of the summed predicted
    times of its jobs, each job given by (graph features, plan features)."""

    def __init__(self, model: CostModel, jobs: list[tuple[np.ndarray, np.ndarray]]):
        self.model, self.jobs = model, jobs

    def predict(self, xs: list[dict]) -> list[float]:
        X = np.stack([features(gf, pf, d) for d in xs for gf, pf in self.jobs])
        p = self.model.predict(X).reshape(len(xs), len(self.jobs)).astype(np.float64)
        m = p.max(axis=1, keepdims=True)
        return (m[:, 0] + np.log(np.exp(p - m).sum(axis=1))).tolist()


def all_points() -> list[dict]:
    import itertools

    keys = tuner.KEYS
    out = []
    for vals in itertools.product(*(tuner.SPACE[k] for k in keys)):
        d = dict(zip(keys, vals))
        if tuner.valid(d):
            out.append(d)
    return out


def pick(model: CostModel, gf: np.ndarray, pf: np.ndarray, points: list[dict]) -> dict:
    X = np.stack([features(gf, pf, d) for d in points])
    return points[int(np.argmin(model.predict(X)))]


# The model leaves the default configuration only for a predicted gain of at
# least this factor: its ranking error on held-out graphs is of that order.
MIN_PREDICTED_GAIN = 1.15
# Plan variants need a larger predicted gain: the training runs hold only
# each pattern's first two variants, so predictions for the others are
# extrapolations.
MIN_PREDICTED_PLAN_GAIN = 1.5


def choose_schedule(model: CostModel, graph: "g.Graph", pattern: str,
                    point: dict | None = None, max_variants: int = 8,
                    min_gain: float = MIN_PREDICTED_PLAN_GAIN) -> tuple["g.Schedule", bool]:
    """The model's choice among the pattern's exact plan variants (vertex
    orders and their symmetry-breaking conditions, all counting the same
    subgraphs) under launch configuration `point` (default: the engine's),
    falling back to variant 0 - the reference cost formula's first choice,
    with the graph's sizes - unless the best prediction beats it by
    min_gain.  Returns (schedule, whether variant 0 was kept)."""
    point = point or tuner.default_point()
    n = min(max_variants, g.Schedule.variants(pattern, stats_graph=graph))
    scheds = [g.Schedule(pattern, "exact", stats_graph=graph, variant=v) for v in range(n)]
    gf = graph_features(graph)
    X = np.stack([features(gf, plan_features(s), point) for s in scheds])
    pred = model.predict(X)
    bi = int(np.argmin(pred))
    if pred[bi] + math.log(min_gain) <= pred[0]:
        return scheds[bi], False
    return scheds[0], True


def choose(model: CostModel, gf: np.ndarray, pf: np.ndarray, points: list[dict],
           default: dict, min_gain: float = MIN_PREDICTED_GAIN) -> tuple[dict, bool]:
    """The model's choice among `points`, falling back to `default` unless
    the best prediction beats the default's by min_gain.  Returns (point,
    whether the default was kept)."""
    cand = list(points)
    if all(tuner.fingerprint(d) != tuner.fingerprint(default) for d in cand):
        cand.append(default)
    X = np.stack([features(gf, pf, d) for d in cand])
    pred = model.predict(X)
    di = [tuner.fingerprint(d) for d in cand].index(tuner.fingerprint(default))
    bi = int(np.argmin(pred))
    if pred[bi] + math.log(min_gain) <= pred[di]:
        return cand[bi], False
    return default, True


# ---------------------------------------------------------------- CLI

def main():
    ap = argparse.ArgumentParser()
    sub = ap.add_subparsers(dest="cmd", required=True)
    c = sub.add_parser("collect")
    c.add_argument("--runs", type=int, default=20000)
    c.add_argument("--out", default="costmodel_data.npz")
    c.add_argument("--seed", type=int, default=0)
    c.add_argument("--max-seconds", type=float, default=0.0)
    c.add_argument("--max-log2", type=int, default=16)
    c.add_argument("--max-ms", type=float, default=200.0)
    t = sub.add_parser("train")
    t.add_argument("data")
    t.add_argument("--out", default="costmodel.npz")
    t.add_argument("--epochs", type=int, default=200)
    e = sub.add_parser("eval5")
    e.add_argument("--model", required=True)
    e.add_argument("--parts", type=int, default=256)
    e.add_argument("--candidates", type=int, default=48)
    a = ap.parse_args()
    import torch

    torch.cuda.set_device(0)
    if a.cmd == "collect":
        X, T = collect(a.runs, a.seed, log=lambda s: print(s, file=sys.stderr, flush=True),
                       max_seconds=a.max_seconds, max_log2=a.max_log2, max_ms=a.max_ms,
                       checkpoint=a.out)
        np.savez(a.out, X=X, T=T)
        print(json.dumps({"runs": len(X), "features": X.shape[1], "out": a.out}))
    elif a.cmd == "train":
        z = np.load(a.data)
        X, T = z["X"], z["T"]
        idx = np.random.default_rng(0).permutation(len(X))
        cut = int(0.9 * len(X))
        tr, te = idx[:cut], idx[cut:]
        t0 = time.time()
        model, loss = CostModel.fit(X[tr], T[tr], epochs=a.epochs)
        pred = model.predict(X[te])
        test_mse = float(np.mean((pred - T[te]) ** 2))
        base_mse = float(np.mean((T[tr].mean() - T[te]) ** 2))
        model.save(a.out)
        print(json.dumps({"train_mse": loss, "test_mse": test_mse,
                          "test_mse_predicting_mean": base_mse, "seconds": time.time() - t0,
                          "out": a.out}))
    elif a.cmd == "eval5":
        from graphautotune_b200.experiments import eval_c5

        eval_c5(CostModel.load(a.model), parts=a.parts, n_candidates=a.candidates)


if __name__ == "__main__":
    main()
