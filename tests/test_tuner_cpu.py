"""Host logic of the autotuner and the cost model, without a GPU: the config
space and its md5 fingerprints, the record.json history, simulated-annealing
proposals over a synthetic cost surface, the batch tuning loop with a fake
measurement, feature vectors, and the batch model's aggregation."""
import json
import math
import random

import numpy as np
import pytest


@pytest.fixture(scope="module")
def tuner(gat):
    from graphautotune_b200 import tuner
    return tuner


def test_points_round_trip_through_config(tuner):
    rng = random.Random(1)
    assert tuner.valid(tuner.default_point())
    for _ in range(200):
        d = tuner.random_point(rng)
        assert tuner.valid(d)
        assert tuner.from_config(tuner.to_config(d)) == d
        e = tuner.random_walk(d, rng)
        assert tuner.valid(e)
        assert sum(d[k] != e[k] for k in tuner.KEYS) == 1


def test_fingerprint_is_md5_of_sorted_key_indices(tuner):
    import hashlib

    d = tuner.default_point()
    idx = [tuner.SPACE[k].index(d[k]) for k in sorted(tuner.SPACE)]
    want = hashlib.md5(",".join(map(str, idx)).encode()).hexdigest()
    assert tuner.fingerprint(d) == want
    rng = random.Random(2)
    pts = {tuner.fingerprint(tuner.random_point(rng)) for _ in range(300)}
    assert len(pts) > 100  # distinct points, distinct fingerprints


def test_history_persists_as_record_json(tuner, tmp_path):
    path = tmp_path / "run" / "record.json"
    h = tuner.History(str(path))
    rng = random.Random(3)
    pts = [tuner.random_point(rng) for _ in range(5)]
    for i, p in enumerate(pts):
        h.add(p, 1.0 + i)
    rec = json.loads(path.read_text())
    assert [r[1] for r in rec] == [1.0, 2.0, 3.0, 4.0, 5.0]
    h2 = tuner.History(str(path))
    assert h2.best() == (pts[0], 1.0)
    assert all(h2.seen(p) for p in pts)
    # best_config.json (the reference tuner's CONF_PATH) holds the best pair
    assert json.loads((path.parent / "best_config.json").read_text()) == [pts[0], 1.0]
    h2.add(pts[1], 0.5)
    assert json.loads((path.parent / "best_config.json").read_text()) == [pts[1], 0.5]


def _bowl(tuner):
    """Synthetic cost: squared index distance to a fixed optimum."""
    opt = {k: tuner.SPACE[k][len(tuner.SPACE[k]) // 2] for k in tuner.KEYS}
    oi = tuner.index_list(opt)

    def cost(d):
        return float(sum((a - b) ** 2 for a, b in zip(tuner.index_list(d), oi)))
    return opt, cost


def test_annealing_proposals_descend_a_cost_surface(tuner):
    opt, cost = _bowl(tuner)

    class Model:
        def predict(self, xs):
            return [cost(x) for x in xs]

    rng = random.Random(4)
    h = tuner.History()
    props = tuner.propose(Model(), h, 3, rng, n_iter=60)
    assert len(props) == 3 and all(tuner.valid(p) for p in props)
    base = np.mean([cost(tuner.random_point(random.Random(i))) for i in range(50)])
    assert max(cost(p) for p in props) < base
    # proposals are never points already measured
    for p in props:
        h.add(p, cost(p))
    again = tuner.propose(Model(), h, 3, rng, n_iter=60)
    assert not any(h.seen(p) for p in again)


def test_tune_batch_loop_with_a_fake_measurement(tuner, monkeypatch):
    opt, cost = _bowl(tuner)
    calls = []

    def fake_measure(b, d, reps=2):
        calls.append(d)
        return 1.0 + cost(d)

    monkeypatch.setattr(tuner, "measure_batch", fake_measure)
    cfg, hist = tuner.tune_batch(object(), budget=10, seed=5)
    assert len(calls) == 10 and len(hist) == 10
    assert tuner.fingerprint(calls[0]) == tuner.fingerprint(tuner.default_point())
    best = min(calls, key=cost)
    assert tuner.from_config(cfg) == best
    assert len({tuner.fingerprint(c) for c in calls}) == 10  # no repeats


def test_feature_vectors(gat):
    from graphautotune_b200 import costmodel, tuner

    g = gat.Graph.barabasi_albert(500, 4, 6)
    gf = costmodel.graph_features(g)
    assert gf.shape == (20,) and np.all(np.isfinite(gf))
    for p in ("0111101111011110", "0100110110010110110010100"):
        pf = costmodel.plan_features(gat.Schedule(p, "exact"))
        assert pf.shape == (11,) and np.all(np.isfinite(pf))
        # the last plan feature flags a dedicated kernel (the 4-clique's)
        assert pf[-1] == (1.0 if p == "0111101111011110" else 0.0)
        x = costmodel.features(gf, pf, tuner.default_point())
        assert x.shape == (costmodel.N_FEATURES,) and np.all(np.isfinite(x))
    pts = costmodel.all_points()
    assert len(pts) > 100 and all(tuner.valid(p) for p in pts)


def test_batch_model_sums_predicted_job_times(gat):
    from graphautotune_b200 import costmodel, tuner

    class Fixed:
        """Predicts log-time = first configuration feature + job offset."""

        def predict(self, X):
            return X[:, 0] + X[:, -1]

    g1 = gat.Graph.barabasi_albert(300, 3, 7)
    g2 = gat.Graph.rmat(9, 2048, 0.57, 0.19, 0.19, 8)
    pf = costmodel.plan_features(gat.Schedule("0111101111011110", "exact"))
    jobs = [(costmodel.graph_features(g1), pf), (costmodel.graph_features(g2), pf)]
    bm = costmodel.BatchTunerModel(Fixed(), jobs)
    rng = random.Random(9)
    xs = [tuner.random_point(rng) for _ in range(4)]
    got = bm.predict(xs)
    for d, v in zip(xs, got):
        per = [float(Fixed().predict(costmodel.features(gf, p, d)[None, :])[0])
               for gf, p in jobs]
        assert math.isclose(v, math.log(sum(math.exp(t) for t in per)), rel_tol=1e-9)


def test_tune_batch_screens_out_slow_points(tuner, monkeypatch):
    """With a screen batch, points far slower than the best screened one are
    never measured on the full sample."""
    opt, cost = _bowl(tuner)
    full, screen = object(), object()
    full_calls = []

    def fake_measure(b, d, reps=2):
        t = 2.0 ** cost(d)  # steep: most random points are >3x the best
        if b is full:
            full_calls.append(d)
            return 8.0 * t
        return t

    monkeypatch.setattr(tuner, "measure_batch", fake_measure)
    cfg, hist = tuner.tune_batch(full, budget=12, seed=6, screen=screen)
    assert len(hist) == 12
    assert len(full_calls) < 12  # some points were screened out
    best_full = min(full_calls, key=cost)
    assert tuner.from_config(cfg) == best_full
    # screened points carry an estimate on the full-sample scale
    ys = dict(hist)
    for d in full_calls:
        assert math.isclose(ys[tuner.fingerprint(d)], 8.0 * 2.0 ** cost(d))


class _StubModel:
    """Stands in for a trained CostModel: predicted log-times chosen by a
    function of the feature rows."""

    def __init__(self, fn):
        self.fn = fn

    def predict(self, X):
        return np.array([self.fn(x) for x in X], np.float32)


def test_choose_keeps_the_default_unless_the_gain_is_large(gat, tuner):
    """costmodel.choose leaves the default configuration only when the best
    prediction is at least MIN_PREDICTED_GAIN times faster; the default is
    added to the candidates when missing."""
    from graphautotune_b200 import costmodel

    g = gat.Graph.barabasi_albert(600, 4, 3)
    gf = costmodel.graph_features(g)
    pf = costmodel.plan_features(gat.Schedule("0100110110010110110010100", "exact"))
    rng = random.Random(2)
    default = tuner.default_point()
    others = []
    while len(others) < 6:
        d = tuner.random_point(rng)
        if tuner.fingerprint(d) != tuner.fingerprint(default):
            others.append(d)
    target = tuner.fingerprint(others[3])
    rows = {tuner.fingerprint(d): costmodel.features(gf, pf, d).tobytes()
            for d in [default] + others}
    by_row = {v: k for k, v in rows.items()}

    def model_with(gain):
        # every point predicts 1.0 (log-time 0) except others[3], predicted
        # `gain` times faster than the default
        return _StubModel(lambda x: -math.log(gain) if by_row[x.tobytes()] == target else 0.0)

    pick, kept = costmodel.choose(model_with(1.05), gf, pf, others, default)
    assert kept and tuner.fingerprint(pick) == tuner.fingerprint(default)
    pick, kept = costmodel.choose(model_with(2.0), gf, pf, others, default)
    assert not kept and tuner.fingerprint(pick) == target


def test_choose_schedule_keeps_variant_zero_unless_the_gain_is_large(gat):
    """costmodel.choose_schedule ranks a pattern's exact plan variants and
    keeps variant 0 (the reference cost formula's choice) unless another is
    predicted MIN_PREDICTED_PLAN_GAIN times faster."""
    from graphautotune_b200 import costmodel

    g = gat.Graph.rmat(10, 1 << 13, 0.57, 0.19, 0.19, 3)
    pat = "0000100110010110110110110"
    n = gat.Schedule.variants(pat, stats_graph=g)
    assert n > 2
    pfs = [costmodel.plan_features(gat.Schedule(pat, "exact", stats_graph=g, variant=v))
           for v in range(min(8, n))]
    # the first variant whose plan features differ from variant 0's (the
    # features summarise a plan's shape, so many vertex orders look alike;
    # equal rows get equal predictions and the lowest index among them wins)
    keys = [pf.tobytes() for pf in pfs]
    t = next(v for v in range(1, len(pfs)) if keys[v] != keys[0])
    # a model that sees only the plan part of the row: variant t is
    # predicted faster by `gain`
    off = 7  # configuration features come first

    def model_with(gain):
        return _StubModel(lambda x: -math.log(gain)
                          if x[off:off + len(pfs[t])].tobytes() == keys[t] else 0.0)

    s, kept = costmodel.choose_schedule(model_with(1.2), g, pat)
    assert kept and s.variant == 0
    s, kept = costmodel.choose_schedule(model_with(3.0), g, pat)
    assert not kept and s.variant == t
