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
