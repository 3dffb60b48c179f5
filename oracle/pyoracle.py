"""Test infrastructure only: ctypes wrapper of the CPU oracle (liboracle.so).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may
import this module, and only as the checker.  The product never does.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "liboracle.so"
_lib = None


def build() -> None:
    subprocess.run(["make", "-C", str(HERE), "liboracle.so"], check=True,
                   capture_output=True)


def lib():
    global _lib
    if _lib is None:
        if not LIB.exists():
            build()
        l = C.CDLL(str(LIB))
        i64p, i32p = C.POINTER(C.c_int64), C.POINTER(C.c_int32)
        l.oracle_naive_labelled.restype = C.c_uint64
        l.oracle_naive_labelled.argtypes = [C.c_int32, i64p, i32p, C.c_char_p, C.c_int32,
                                            C.c_int32, C.c_int]
        l.oracle_naive_labelled_roots.restype = C.c_uint64
        l.oracle_naive_labelled_roots.argtypes = [C.c_int32, i64p, i32p, C.c_char_p, i32p,
                                                  C.c_int64, C.c_int]
        l.oracle_backtrack_labelled.restype = C.c_uint64
        l.oracle_backtrack_labelled.argtypes = l.oracle_naive_labelled.argtypes
        l.oracle_automorphisms.restype = C.c_int64
        l.oracle_automorphisms.argtypes = [C.c_char_p]
        l.oracle_ref_engine.restype = C.c_int
        l.oracle_ref_engine.argtypes = [C.c_int32, i64p, i32p, i32p, C.c_int32, C.c_int32,
                                        C.c_int32, C.c_int, i64p, C.POINTER(C.c_uint64)]
        l.oracle_restricted_labelled.restype = C.c_uint64
        l.oracle_restricted_labelled.argtypes = [C.c_int32, i64p, i32p, C.c_char_p, i32p,
                                                 C.c_int32, C.c_int32, C.c_int32, C.c_int]
        l.oracle_restricted_labelled_capped.restype = C.c_uint64
        l.oracle_restricted_labelled_capped.argtypes = [
            C.c_int32, i64p, i32p, C.c_char_p, i32p, C.c_int32, C.c_int32, C.c_int32, C.c_int,
            C.c_int64, C.POINTER(C.c_int)]
        l.oracle_c4_rooted.restype = C.c_uint64
        l.oracle_c4_rooted.argtypes = [C.c_int32, i64p, i32p, C.c_int32, C.c_int32, C.c_int,
                                       C.c_int]
        l.oracle_degree_order.restype = C.c_int
        l.oracle_degree_order.argtypes = [C.c_int32, i64p, i32p, i64p, i32p]
        l.oracle_intersect_size.restype = C.c_int32
        l.oracle_intersect_size.argtypes = [i32p, C.c_int32, i32p, C.c_int32]
        _lib = l
    return _lib


def _csr(off: np.ndarray, adj: np.ndarray):
    off = np.ascontiguousarray(off, np.int64)
    adj = np.ascontiguousarray(adj if len(adj) else np.zeros(1, np.int32), np.int32)
    return (len(off) - 1, off, adj,
            off.ctypes.data_as(C.POINTER(C.c_int64)),
            adj.ctypes.data_as(C.POINTER(C.c_int32)))


def naive_labelled(off, adj, pattern: str, roots=None, threads: int = 0) -> int:
    V, o, a, po, pa = _csr(off, adj)
    b, e = roots if roots else (0, V)
    return lib().oracle_naive_labelled(V, po, pa, pattern.encode(), b, e, threads)


def naive_labelled_roots(off, adj, pattern: str, roots, threads: int = 0) -> int:
    V, o, a, po, pa = _csr(off, adj)
    r = np.ascontiguousarray(roots, np.int32)
    return lib().oracle_naive_labelled_roots(V, po, pa, pattern.encode(),
                                             r.ctypes.data_as(C.POINTER(C.c_int32)), len(r),
                                             threads)


def backtrack_labelled(off, adj, pattern: str, roots=None, threads: int = 0) -> int:
    V, o, a, po, pa = _csr(off, adj)
    b, e = roots if roots else (0, V)
    return lib().oracle_backtrack_labelled(V, po, pa, pattern.encode(), b, e, threads)


def automorphisms(pattern: str) -> int:
    return lib().oracle_automorphisms(pattern.encode())


def exact_count(off, adj, pattern: str, threads: int = 0) -> int:
    lab = backtrack_labelled(off, adj, pattern, threads=threads)
    aut = automorphisms(pattern)
    assert lab % aut == 0
    return lab // aut


def encode_schedule(sd: dict) -> np.ndarray:
    """Flat ScheduleData encoding (see oracle.h) from a schedule dump."""
    basic = sd["basic_vertexes"]
    pre = sd["prefixs"]
    rest = [r[0] for r in sd["restrictions"]]
    out = [basic, len(pre), len(rest), len(sd["iep_vertex_id"]), len(sd["iep_ans_pos"])]
    for p in pre:
        out += [len(p), *p]
    out += sd["prefixs_father"] + sd["prefixs_size_only"]
    out += sd["sd_vertex_prefix_start"] + sd["loop_set_prefix_id"]
    out += sd["sd_restrictions_start"] + rest
    out += sd["iep_vertex_id"] + sd["iep_ans_pos"] + sd["iep_coef"]
    out += [int(x) for x in sd["iep_flag"]]
    return np.array(out, np.int32)


REF_UNDEFINED = (-2, -3)


def ref_engine(off, adj, sd: dict, roots=None, threads: int = 0):
    """(status, total, balg) of the reference engine semantics."""
    V, o, a, po, pa = _csr(off, adj)
    flat = encode_schedule(sd)
    b, e = roots if roots else (0, V)
    out = C.c_int64()
    balg = C.c_uint64()
    st = lib().oracle_ref_engine(V, po, pa, flat.ctypes.data_as(C.POINTER(C.c_int32)),
                                 len(flat), b, e, threads, C.byref(out), C.byref(balg))
    return st, out.value, balg.value


def intersect_size(a, b) -> int:
    a = np.ascontiguousarray(a, np.int32)
    b = np.ascontiguousarray(b, np.int32)
    return lib().oracle_intersect_size(a.ctypes.data_as(C.POINTER(C.c_int32)), len(a),
                                       b.ctypes.data_as(C.POINTER(C.c_int32)), len(b))


def restricted_labelled(off, adj, pattern: str, less, roots=None, threads: int = 0) -> int:
    """Labelled embeddings f of `pattern` with f(0) in roots=(begin, end) and
    f(a) < f(b) for every (a, b) in `less` (see oracle.h)."""
    V, o, a, po, pa = _csr(off, adj)
    b, e = roots if roots else (0, V)
    flat = np.ascontiguousarray(np.array(less, np.int32).reshape(-1) if len(less)
                                else np.zeros(2, np.int32))
    return lib().oracle_restricted_labelled(V, po, pa, pattern.encode(),
                                            flat.ctypes.data_as(C.POINTER(C.c_int32)),
                                            len(less), b, e, threads)


def restricted_labelled_capped(off, adj, pattern: str, less, roots, max_work: int,
                               threads: int = 0):
    """restricted_labelled, or None once about max_work candidates were
    examined without finishing."""
    V, o, a, po, pa = _csr(off, adj)
    b, e = roots
    flat = np.ascontiguousarray(np.array(less, np.int32).reshape(-1) if len(less)
                                else np.zeros(2, np.int32))
    over = C.c_int(0)
    r = lib().oracle_restricted_labelled_capped(V, po, pa, pattern.encode(),
                                                flat.ctypes.data_as(C.POINTER(C.c_int32)),
                                                len(less), b, e, threads, max_work,
                                                C.byref(over))
    return None if over.value else r


def c4_rooted(off, adj, roots=None, at_largest: bool = False, threads: int = 0) -> int:
    """4-cycles whose smallest (at_largest: largest) vertex lies in roots."""
    V, o, a, po, pa = _csr(off, adj)
    b, e = roots if roots else (0, V)
    return lib().oracle_c4_rooted(V, po, pa, b, e, 1 if at_largest else 0, threads)


def degree_order(off, adj):
    """(offsets, neighbours) relabelled by decreasing degree, ties by id."""
    V, o, a, po, pa = _csr(off, adj)
    no = np.empty(V + 1, np.int64)
    na = np.empty(max(int(o[-1]), 1), np.int32)
    rc = lib().oracle_degree_order(V, po, pa, no.ctypes.data_as(C.POINTER(C.c_int64)),
                                   na.ctypes.data_as(C.POINTER(C.c_int32)))
    assert rc == 0
    return no, na[:int(o[-1])]


def plan_conditions(dump: dict) -> tuple[str, list[tuple[int, int]]]:
    """For an exact schedule dump (or a pin record with the same "adj",
    "perm" and "restrictions" fields): the pattern in the plan's vertex order
    (vertex i of the input becomes perm[i]) and its order conditions as
    pairs (a, b) meaning f(a) < f(b).  The dump's restriction (i, u) means
    the vertex at level u takes a smaller id than the one at level i."""
    pat, perm = dump.get("pattern", dump.get("adj")), dump["perm"]
    n = len(perm)
    q = ["0"] * (n * n)
    for i in range(n):
        for j in range(n):
            if pat[i * n + j] == "1" or pat[j * n + i] == "1":
                q[perm[i] * n + perm[j]] = "1"
    return "".join(q), [(u, i) for i, u in dump["restrictions"]]
