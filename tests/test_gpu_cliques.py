"""GPU parity of the bit-matrix k-clique kernels (cliques.cu).

Exact k-clique counts (4 <= k <= 7) through the dedicated kernels must equal
the oracle and the schedule-plan path (`special_kernels = 0`, itself pinned to
the reference's naive matcher) on whole graphs, on root ranges and on shards,
with and without hub bitmaps (which switches row building between bitmap
probes and list scans/searches).  One graph has a root whose lower list is
too long for the matrix to sit in shared memory, so its rows go through the
global scratch slice.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

CLIQUES = {k: "".join("0" if i == j else "1" for i in range(k) for j in range(k))
           for k in range(4, 8)}


def _executor(gat, **kw):
    c = gat.Config.engine_default()
    for k, v in kw.items():
        setattr(c, k, v)
    return gat.Executor(c)


@pytest.fixture(scope="module")
def executors(gat):
    return {"special": _executor(gat), "plain": _executor(gat, special_kernels=0),
            "nobitmap": _executor(gat, hub_bitmaps=0)}


def _dense_core_graph(gat, core=3300, p=0.3, attach=900, seed=11):
    """A random core of `core` vertices (edge probability p, degree about
    p * core) plus one vertex joined to `attach` core vertices: its degree is
    below every core degree, so on the degree-ordered copy all of its
    neighbours are lower ids and its lower list has `attach` entries."""
    rng = np.random.default_rng(seed)
    iu, ju = np.triu_indices(core, 1)
    keep = rng.random(len(iu)) < p
    src = [iu[keep], ju[keep]]
    star = rng.choice(core, attach, replace=False)
    src_s = np.concatenate([src[0], np.full(attach, core)])
    dst_s = np.concatenate([src[1], star])
    V = core + 1
    a = np.concatenate([src_s, dst_s]).astype(np.int64)
    b = np.concatenate([dst_s, src_s]).astype(np.int64)
    order = np.lexsort((b, a))
    a, b = a[order], b[order]
    off = np.zeros(V + 1, np.int64)
    np.add.at(off, a + 1, 1)
    off = np.cumsum(off)
    return gat.Graph.from_csr(off, b.astype(np.int32))


def _graphs(gat):
    from pathlib import Path

    golden = Path(__file__).resolve().parent / "golden" / "graphs"
    return {
        "er200": gat.Graph.load(str(golden / "er200.bin")),
        "ba3000": gat.Graph.barabasi_albert(3000, 8, 5),
        "rmat12": gat.Graph.rmat(12, 1 << 16, 0.57, 0.19, 0.19, 7),
    }


def test_cliques_match_oracle_and_plan(gat, oracle, executors):
    for name, g in _graphs(gat).items():
        off, adj = g.csr()
        for k, pat in CLIQUES.items():
            s = gat.Schedule(pat, "exact")
            r = executors["special"].count(g, s)
            assert r.launches == 2, (name, k, "clique kernels not used")
            plain = executors["plain"].count(g, s)
            assert plain.launches == 1
            assert r.count == plain.count, (name, k, r.count, plain.count)
            assert executors["nobitmap"].count(g, s).count == r.count, (name, k)
            if k == 4 or name == "er200":
                assert r.count == oracle.exact_count(off, adj, pat), (name, k)
            # the instrumented launch counts the same
            rb = executors["special"].count(g, s, balg=True)
            assert rb.count == r.count and rb.balg_bytes > 0


def test_cliques_on_a_larger_power_law_graph(gat, executors):
    g = gat.Graph.rmat(15, 1 << 19, 0.57, 0.19, 0.19, 3)
    for k in (4, 5, 6):
        s = gat.Schedule(CLIQUES[k], "exact")
        r = executors["special"].count(g, s)
        assert r.launches == 2
        assert r.count == executors["plain"].count(g, s).count, k
        assert r.count == executors["nobitmap"].count(g, s).count, k


def test_clique_ranges_and_shards_sum_to_the_whole(gat, executors):
    g = gat.Graph.rmat(13, 1 << 17, 0.57, 0.19, 0.19, 5)
    g.upload(degree_order=True)
    V, _, _ = g.info()
    ex, plain = executors["special"], executors["plain"]
    for k in (4, 5):
        s = gat.Schedule(CLIQUES[k], "exact")
        whole = ex.count(g, s).count
        cuts = [0, 1, 7, 300, V // 3, V // 2, V]
        total = 0
        for b, e in zip(cuts, cuts[1:]):
            got, _ = ex.count_range(g, s, b, e)
            want, _ = plain.count_range(g, s, b, e)
            assert got == want, (k, b, e)
            total += got
        assert total == whole
        # shards split the level-1 units (v0, v1) exactly as the plan path
        # does, rows of one root included
        shards = [ex.count_shard(g, s, i, 7)[0] for i in range(7)]
        assert shards == [plain.count_shard(g, s, i, 7)[0] for i in range(7)], k
        assert sum(shards) == whole


def test_clique_rows_in_global_scratch(gat, oracle, executors):
    g = _dense_core_graph(gat)
    g.upload(degree_order=True)
    oo, oa = g.ordered_csr()
    deg = np.diff(oo)
    V = len(deg)
    lower = np.array([np.searchsorted(oa[oo[v]:oo[v + 1]], v) for v in range(V)])
    star = int(np.argmax(lower))
    # rows of ceil(d / 32) | 1 words: about 900 x 29 words, more than the
    # 22 Ki words of matrix rows a CTA keeps in shared memory
    d = int(lower[star])
    assert d * (((d + 31) // 32) | 1) > 22 * 1024
    for k in (4, 5):
        s = gat.Schedule(CLIQUES[k], "exact")
        q, less = oracle.plan_conditions(s.dump())
        for b, e in ((star, star + 1), (0, 64), (1000, 1010)):
            got, _ = executors["special"].count_range(g, s, b, e)
            assert got == executors["plain"].count_range(g, s, b, e)[0], (k, b, e)
            assert got == executors["nobitmap"].count_range(g, s, b, e)[0], (k, b, e)
            assert got == oracle.restricted_labelled(oo, oa, q, less, roots=(b, e)), (k, b, e)
    s = gat.Schedule(CLIQUES[4], "exact")
    assert executors["special"].count(g, s).count == executors["plain"].count(g, s).count
