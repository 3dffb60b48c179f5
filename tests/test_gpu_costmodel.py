"""The learned cost model's CUDA kernels and what the trained network gains.

  * gradients of gat_mlp_gradient equal the float64 numpy restatement
    (oracle/mlp_ref.py) for random parameters and data
  * Adam training on the GPU fits a known smooth function
  * trained on engine timings from some graphs, the network's choice of a
    launch configuration on held-out graphs (with the default configuration
    as its fallback) is judged against the default configuration and against
    the best measured candidate; its predicted order correlates with the
    measured one
"""
import math
import random

import numpy as np
import pytest

import mlp_ref

pytestmark = pytest.mark.gpu


def test_mlp_gradients_match_cpu_reference(gat):
    from graphautotune_b200 import costmodel

    rng = np.random.default_rng(3)
    for n_in, n in ((37, 200), (5, 33), (64, 1000)):
        m = costmodel.MLP(n_in, seed=n)
        X = rng.normal(size=(n, n_in)).astype(np.float32)
        T = rng.normal(size=n).astype(np.float32)
        g_gpu, loss_gpu = m.gradient(X, T)
        loss_ref, g_ref = mlp_ref.loss_and_grad(m.params(), X, T, n_in)
        assert abs(loss_gpu - loss_ref) <= 1e-4 * max(1.0, abs(loss_ref))
        scale = np.abs(g_ref).max()
        assert np.allclose(g_gpu, g_ref, rtol=1e-3, atol=1e-5 * scale), \
            float(np.abs(g_gpu - g_ref).max())
        y = m.predict(X)
        assert np.allclose(y, mlp_ref.forward(m.params(), X, n_in)[0], rtol=1e-4, atol=1e-4)


def test_mlp_training_fits_a_smooth_function(gat):
    from graphautotune_b200 import costmodel

    rng = np.random.default_rng(0)
    X = rng.uniform(-1, 1, size=(4000, 8)).astype(np.float32)
    T = (np.sin(2 * X[:, 0]) + X[:, 1] * X[:, 2] + 0.5 * np.abs(X[:, 3])).astype(np.float32)
    m = costmodel.MLP(8, seed=1)
    before = float(np.mean((m.predict(X) - T) ** 2))
    after = m.train(X, T, epochs=150, batch=128, lr=3e-3, seed=2)
    assert after < 0.1 * before and after < 0.02, (before, after)


def test_trained_model_beats_choosing_without_it(gat):
    from graphautotune_b200 import costmodel, tuner
    from graphautotune_b200.experiments import make_graph

    specs = costmodel.training_graphs(10, seed0=5000, max_log2=13)
    graphs = []
    for sp in specs:
        gr = make_graph(sp)
        gr.upload(degree_order=True)
        graphs.append((gr, costmodel.graph_features(gr)))
    # patterns counted by the schedule-plan interpreter, whose launch shape
    # matters (the 4-cycle and cliques have dedicated kernels): the house,
    # the diamond and the tailed triangle
    pats = ["0100110110010110110010100", "0111101111001100", "0111101011001000"]
    scheds = [gat.Schedule(p, "exact") for p in pats]
    pfs = [costmodel.plan_features(s) for s in scheds]
    rng = random.Random(0)
    cands = [tuner.default_point()]
    while len(cands) < 16:
        d = tuner.random_point(rng)
        if all(tuner.fingerprint(d) != tuner.fingerprint(c) for c in cands):
            cands.append(d)
    cfgs = [tuner.to_config(d) for d in cands]
    for c in cfgs:
        c.memory_budget = costmodel.EXEC_BUDGET
    execs = [gat.Executor(c) for c in cfgs]
    groups = []  # (graph index, pattern index, X rows, measured ms)
    for gi, (gr, gf) in enumerate(graphs):
        for si, s in enumerate(scheds):
            times = []
            for ex in execs:
                ex.count(gr, s)
                times.append(min(ex.count(gr, s).kernel_ms for _ in range(2)))
            X = np.stack([costmodel.features(gf, pfs[si], d) for d in cands])
            groups.append((gi, si, X, np.array(times)))
    train = [x for x in groups if x[0] < 7]
    test = [x for x in groups if x[0] >= 7]
    Xtr = np.concatenate([x[2] for x in train])
    Ttr = np.log(np.concatenate([x[3] for x in train])).astype(np.float32)
    model, _ = costmodel.CostModel.fit(Xtr, Ttr, epochs=300, seed=0, lr=2e-3)
    vs_default, vs_best, corrs, kept = [], [], [], 0
    fps = [tuner.fingerprint(d) for d in cands]
    for gi, si, X, times in test:
        choice, k = costmodel.choose(model, graphs[gi][1], pfs[si], cands, cands[0])
        kept += k
        t = times[fps.index(tuner.fingerprint(choice))]
        vs_default.append(times[0] / t)
        vs_best.append(float(times.min()) / t)
        pred = model.predict(X)
        corrs.append(float(np.corrcoef(np.argsort(np.argsort(pred)),
                                       np.argsort(np.argsort(times)))[0, 1]))

    def gm(xs):
        return math.exp(sum(math.log(x) for x in xs) / len(xs))

    info = dict(vs_default=gm(vs_default), vs_best=gm(vs_best), kept_default=kept,
                groups=len(test), corr=float(np.mean(corrs)))
    print(info)
    # the choice is not slower than the default (geometric mean over the
    # held-out graph x pattern groups; measured 2.25x faster), it keeps at
    # least half the best measured candidate's speed (measured 0.66), and the
    # predicted order follows the measured one (measured 0.93)
    assert info["vs_default"] >= 1.0, info
    assert info["vs_best"] >= 0.5, info
    assert info["corr"] > 0.5, info


def test_model_ranks_schedule_variants(gat):
    """The model, trained on engine timings that include every pattern's
    first exact plan variants, chooses among the plan variants of patterns
    on held-out graphs (costmodel.choose_schedule, with variant 0 - the
    reference cost formula's first choice - as the fallback; a switch needs a
    1.5x predicted gain).  Judged by measured times against variant 0 and
    against the best variant: the choice must not lose more than 15 % to
    variant 0 (geometric mean over 8 held-out groups; measured 0.89, variant
    0 kept in 7 groups and one switch that ran slower) and must keep at least
    half the best variant's speed (measured 0.88)."""
    from graphautotune_b200 import costmodel
    from graphautotune_b200.experiments import make_graph

    X, T = costmodel.collect(1500, seed=7, graphs=12, max_ms=50.0, max_seconds=90.0,
                             max_log2=12)
    model, _ = costmodel.CostModel.fit(X, T, epochs=200, seed=0, lr=2e-3)
    ex = gat.Executor()
    vs_v0, vs_best, kept = [], [], 0
    for sp in costmodel.training_graphs(4, seed0=9100, max_log2=12):
        gr = make_graph(sp)
        gr.upload(degree_order=True)
        for p in ("0100110110010110110010100", "0000100110010110110110110"):
            n = min(8, gat.Schedule.variants(p, stats_graph=gr))
            times = []
            for v in range(n):
                s = gat.Schedule(p, "exact", stats_graph=gr, variant=v)
                ex.count(gr, s)
                times.append(min(ex.count(gr, s).kernel_ms for _ in range(2)))
            choice, k = costmodel.choose_schedule(model, gr, p)
            kept += k
            t = times[choice.variant]
            vs_v0.append(times[0] / t)
            vs_best.append(min(times) / t)

    def gm(xs):
        return math.exp(sum(math.log(x) for x in xs) / len(xs))

    info = dict(vs_variant0=gm(vs_v0), vs_best=gm(vs_best), kept_variant0=kept,
                groups=len(vs_v0))
    print(info)
    assert info["vs_variant0"] >= 0.85, info
    assert info["vs_best"] >= 0.5, info
