"""gat_count_noalloc: the counting entry point for callers that cannot
allocate device memory when they count (a framework allocator that already
owns the device, a stream that must not pick up cudaMalloc's implicit device
synchronisation, a fixed memory plan).  It must give the same count as the
ordinary executor entry point, call after call, while keeping all its scratch
in the library's static device array.

This file is named so pytest collects it last; it passes on its own in a
fresh process as well as after the rest of the suite.
"""
import ctypes as C
from pathlib import Path

import pytest

import plan_model

pytestmark = pytest.mark.gpu

GOLDEN = Path(__file__).resolve().parent / "golden" / "graphs"
PATTERNS = [
    ("011101110", "exact"), ("0111101111011110", "exact"), ("0101101001011010", "exact"),
    ("0100110110010110110010100", "exact"), ("0111110111110111110111110", "exact"),
    ("0111101111011110", "ref"), ("0100110110010110110010100", "ref"),
]


def _noalloc(lib):
    fn = lib.gat_count_noalloc
    fn.restype = C.c_int
    fn.argtypes = [C.c_void_p, C.c_void_p, C.c_int32, C.c_int64, C.c_int32, C.c_void_p,
                   C.c_void_p, C.c_void_p, C.c_void_p]
    return fn


def test_noalloc_matches_executor_on_repeated_calls(gat):
    import torch

    from graphautotune_b200 import _lib

    fn = _noalloc(_lib.lib())
    ex = gat.Executor()
    graphs = [gat.Graph.load(str(GOLDEN / "er200.bin")),
              gat.Graph.rmat(12, 1 << 15, 0.57, 0.19, 0.19, 9),
              gat.Graph.barabasi_albert(3000, 4, 7)]
    checked = 0
    for g in graphs:
        off, adj = g.csr()
        V, E, md = g.info()
        d_off = torch.from_numpy(off).cuda()
        d_adj = torch.from_numpy(adj).cuda()
        out = torch.empty(1, dtype=torch.int64, device="cuda")
        for p, mode in PATTERNS:
            s = gat.Schedule(p, mode)
            want = ex.count(g, s).count
            for _ in range(2):  # the static scratch keeps the previous call's data
                out.fill_(-12345)
                torch.cuda.synchronize()
                rc = fn(d_off.data_ptr(), d_adj.data_ptr(), V, E, md, s._h, None,
                        out.data_ptr(), None)
                assert rc == 0, _lib.lib().gat_last_error()
                torch.cuda.synchronize()
                assert int(out.item()) == want, (p, mode)
                checked += 1
    assert checked == 2 * len(graphs) * len(PATTERNS)


def test_noalloc_rejects_scratch_beyond_the_static_array(gat):
    import torch

    from graphautotune_b200 import _lib

    fn = _noalloc(_lib.lib())
    g = gat.Graph.load(str(GOLDEN / "er60.bin"))
    off, adj = g.csr()
    V, E, _ = g.info()
    d_off = torch.from_numpy(off).cuda()
    d_adj = torch.from_numpy(adj).cuda()
    out = torch.zeros(1, dtype=torch.int64, device="cuda")
    s = gat.Schedule("0111101111011110", "exact")  # one stored set per tile
    huge_degree = 1 << 26  # one CTA's stored sets would exceed the array
    rc = fn(d_off.data_ptr(), d_adj.data_ptr(), V, E, huge_degree, s._h, None,
            out.data_ptr(), None)
    assert rc == 5  # GAT_ERR_MEMORY
    assert b"static scratch" in _lib.lib().gat_last_error()


def test_noalloc_shrunk_grid_matches_executor_and_oracle(gat, oracle):
    """A stated maximum degree far above the graph's (still a valid upper
    bound) makes one CTA's slots so large that only a few CTAs fit in the
    static array: the grid is shrunk below one wave of the device.  The count
    must not change."""
    import torch

    from graphautotune_b200 import _lib

    fn = _noalloc(_lib.lib())
    ex = gat.Executor()
    g = gat.Graph.load(str(GOLDEN / "er200.bin"))
    off, adj = g.csr()
    V, E, md = g.info()
    d_off = torch.from_numpy(off).cuda()
    d_adj = torch.from_numpy(adj).cuda()
    out = torch.empty(1, dtype=torch.int64, device="cuda")
    cfg = gat.Config.engine_default()
    tiles = cfg.threads_per_block // cfg.threads_per_warp
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    big = 200_000
    for p in ("0111101111011110", "0111110111110111110111110"):
        s = gat.Schedule(p, "exact")
        stored = plan_model.parse(s.plan_bytes()).num_store
        assert stored >= 1
        per_cta = tiles * stored * big * 4
        assert ((64 << 20) - 2048) // per_cta < sms  # fewer CTAs than SMs
        want = ex.count(g, s).count
        assert want == oracle.exact_count(off, adj, p)
        for _ in range(2):
            out.fill_(-12345)
            torch.cuda.synchronize()
            rc = fn(d_off.data_ptr(), d_adj.data_ptr(), V, E, big, s._h, None,
                    out.data_ptr(), None)
            assert rc == 0, _lib.lib().gat_last_error()
            torch.cuda.synchronize()
            assert int(out.item()) == want, p


def test_noalloc_understated_degree_reports_an_error(gat):
    """max_degree below the true maximum: every stored set is cut to its
    slot and the call yields INT64_MIN instead of a count."""
    import torch

    from graphautotune_b200 import _lib

    fn = _noalloc(_lib.lib())
    g = gat.Graph.barabasi_albert(3000, 8, 5)
    off, adj = g.csr()
    V, E, md = g.info()
    assert md > 64
    d_off = torch.from_numpy(off).cuda()
    d_adj = torch.from_numpy(adj).cuda()
    out = torch.empty(1, dtype=torch.int64, device="cuda")
    s = gat.Schedule("0111101111011110", "exact")
    out.fill_(0)
    torch.cuda.synchronize()
    rc = fn(d_off.data_ptr(), d_adj.data_ptr(), V, E, 4, s._h, None, out.data_ptr(), None)
    assert rc == 0, _lib.lib().gat_last_error()
    torch.cuda.synchronize()
    assert int(out.item()) == -(1 << 63)
    # the next call with the right bound is unaffected
    rc = fn(d_off.data_ptr(), d_adj.data_ptr(), V, E, md, s._h, None, out.data_ptr(), None)
    assert rc == 0
    torch.cuda.synchronize()
    assert int(out.item()) == gat.Executor().count(g, s).count
