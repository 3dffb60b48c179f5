"""GPU: the degree-ordered copy is derived on the device from the uploaded
CSR (radix sort by degree, row scatter, segmented sort, lower-offset scan).
It must equal the host restatement below id for id, including graphs with
isolated vertices, no edges, and hubs."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def host_relabel(off, adj):
    """Vertex r of the result is the r-th vertex by decreasing degree, ties
    by id; every row sorted."""
    off = np.asarray(off, np.int64)
    adj = np.asarray(adj, np.int64)
    V = len(off) - 1
    deg = np.diff(off)
    order = np.argsort(-deg, kind="stable")
    nid = np.empty(V, np.int64)
    nid[order] = np.arange(V)
    noff = np.zeros(V + 1, np.int64)
    noff[1:] = np.cumsum(deg[order])
    nsrc = nid[np.repeat(np.arange(V), deg)]
    ndst = nid[adj]
    idx = np.lexsort((ndst, nsrc))
    return noff, ndst[idx].astype(np.int32)


def _graphs(gat, golden_graphs):
    out = list(golden_graphs.items())
    out.append(("rmat12", gat.Graph.rmat(12, 1 << 15, 0.57, 0.19, 0.19, 9)))
    out.append(("ba3000", gat.Graph.barabasi_albert(3000, 7, 4)))
    out.append(("er_sparse", gat.Graph.erdos_renyi(5000, 0.7, 3)))  # isolated vertices
    out.append(("no_edges", gat.Graph.from_csr(np.zeros(6, np.int64), np.zeros(0, np.int32))))
    return out


def test_device_relabel_equals_host(gat, golden_graphs):
    for name, g in _graphs(gat, golden_graphs):
        g.upload(degree_order=True)
        off, adj = g.csr()
        want_off, want_adj = host_relabel(off, adj)
        got_off, got_adj = g.ordered_csr()
        assert np.array_equal(got_off, want_off), name
        assert np.array_equal(got_adj, want_adj), name


def test_counts_on_device_relabelled_copy(gat, oracle):
    """Exact counts on the device-derived copy equal the oracle's, and a
    second upload (copies rebuilt) gives the same counts."""
    g = gat.Graph.rmat(11, 1 << 14, 0.57, 0.19, 0.19, 13)
    off, adj = g.csr()
    ex = gat.Executor(gat.Config.engine_default())
    pats = ["011101110", "0111101111011110", "0100110110010110110010100"]
    want = [oracle.exact_count(off, adj, p) for p in pats]
    for _ in range(2):
        g.upload(degree_order=True)
        assert [ex.count(g, gat.Schedule(p, "exact")).count for p in pats] == want


def test_device_generated_graphs_equal_host_generated(gat):
    """gat_graph_generate_device: R-MAT drawn on the GPU, and Erdos-Renyi /
    Barabasi-Albert edge lists deduplicated into CSR on the GPU, give the
    host generators' graphs entry for entry (self loops and duplicate samples
    included in the R-MAT draws), and the resident copy counts like an
    uploaded one."""
    cases = [
        ("rmat", (12, 1 << 15, 0.57, 0.19, 0.19, 9)),
        ("rmat", (16, 1 << 20, 0.57, 0.19, 0.19, 2)),
        ("rmat", (3, 100, 0.45, 0.15, 0.15, 1)),   # dense: many duplicates and loops
        ("ba", (3000, 7, 4)),
        ("er", (5000, 0.7, 3)),
    ]
    for kind, p in cases:
        if kind == "rmat":
            h, d = gat.Graph.rmat(*p), gat.Graph.rmat(*p, device=True)
        elif kind == "ba":
            h, d = gat.Graph.barabasi_albert(*p), gat.Graph.barabasi_albert(*p, device=True)
        else:
            h = gat.Graph.erdos_renyi(*p)
            d = gat.Graph._generate(0, (p[0], p[1], 0, 0, 0), p[2], True)
        assert h.info() == d.info(), (kind, p)
        ho, ha = h.csr()
        do, da = d.csr()
        assert np.array_equal(ho, do) and np.array_equal(ha, da), (kind, p)
        d.upload(degree_order=True)
        go, ga = d.ordered_csr()
        want_off, want_adj = host_relabel(ho, ha)
        assert np.array_equal(go, want_off) and np.array_equal(ga, want_adj), (kind, p)
    g = gat.Graph.rmat(13, 1 << 17, 0.57, 0.19, 0.19, 5, device=True)
    ex = gat.Executor()
    for pat in ("011101110", "0111101111011110", "0101101001011010"):
        s = gat.Schedule(pat, "exact")
        assert ex.count(g, s).count == ex.count(gat.Graph.rmat(13, 1 << 17, 0.57, 0.19, 0.19, 5),
                                                s).count


def test_from_csr_device_checks_rows_and_reads_back_lazily(gat, oracle):
    """gat_graph_from_csr_device: the caller's host CSR goes straight to the
    GPU and is checked there by the host validator's rules (first failing
    row reported); the host view reads the neighbours back on first use;
    counts equal those of the host-built graph."""
    import torch

    from graphautotune_b200._lib import GatError

    src = gat.Graph.rmat(12, 1 << 15, 0.57, 0.19, 0.19, 9)
    off, adj = src.csr()
    off_p = torch.from_numpy(off).pin_memory()
    adj_p = torch.from_numpy(adj).pin_memory()
    d = gat.Graph.from_csr(off_p.numpy(), adj_p.numpy(), check_symmetry=False, device=True)
    assert d.info() == src.info()
    d.upload(degree_order=True)
    ex = gat.Executor()
    for p in ("011101110", "0111101111011110", "0101101001011010",
              "0100110110010110110010100"):
        s = gat.Schedule(p, "exact")
        assert ex.count(d, s).count == ex.count(src, s).count == oracle.exact_count(off, adj, p)
        sr = gat.Schedule(p, "ref")
        assert ex.count(d, sr).count == ex.count(src, sr).count
    do, da = d.csr()
    assert np.array_equal(do, off) and np.array_equal(da, adj)
    # invalid inputs: the lowest failing row and its reason
    V = len(off) - 1
    row = int(np.argmax(np.diff(off) >= 3))
    cases = []
    a2 = adj.copy()
    a2[off[row]] = row
    cases.append((off, a2, "self loop"))
    a3 = adj.copy()
    a3[off[row]], a3[off[row] + 1] = a3[off[row] + 1], a3[off[row]]
    cases.append((off, a3, "row not strictly increasing"))
    a4 = adj.copy()
    a4[off[row]] = V + 7
    cases.append((off, a4, "neighbour id out of range"))
    o5 = off.copy()
    o5[row + 1] = o5[row] - 1
    cases.append((o5, adj, "offsets not monotone"))
    for o, a, why in cases:
        with pytest.raises(GatError) as err:
            gat.Graph.from_csr(o, a, check_symmetry=False, device=True)
        assert why in str(err.value), (why, str(err.value))
    empty = gat.Graph.from_csr(np.zeros(4, np.int64), np.zeros(0, np.int32), device=True)
    assert empty.info()[:2] == (3, 0)
