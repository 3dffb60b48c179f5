"""Test / baseline infrastructure: numpy restatement of libgat's seeded R-MAT
generator (graphautotune_b200/csrc/graph.cpp gen_rmat + build_csr), so the
CPU legs of bench.py can build the workload graph without loading libgat.

Edge sample i draws from its own splitmix64 stream (state = splitmix64(seed)
+ i * 0xD1B54A32D192ED03); each 64-bit draw gives two 32-bit uniforms, one
per recursion level, low half first.  Level l picks the quadrant by
comparing the uniform against a, a+b, a+b+c scaled to 2^32.  The edge list is
symmetrised, self loops and duplicates are dropped and rows are sorted; the
result is written in the reference's binary layout
(infra/graph_backend.cuh:91-99,163-169: int32 V, int64 E, int64 offsets[V+1],
int32 neighbours[E]).

Only tests/ and bench.py's CPU legs use this module.
"""
from __future__ import annotations

from pathlib import Path

import numpy as np

M64 = np.uint64(0xFFFFFFFFFFFFFFFF)
GOLDEN = np.uint64(0x9E3779B97F4A7C15)
STREAM = np.uint64(0xD1B54A32D192ED03)


def _mix(z: np.ndarray) -> np.ndarray:
    z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
    z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
    return z ^ (z >> np.uint64(31))


def _first_draw(seed: int) -> np.uint64:
    with np.errstate(over="ignore"):
        return _mix(np.array([np.uint64(seed) + GOLDEN], np.uint64))[0]


def rmat_edges(scale: int, samples: int, a: float, b: float, c: float, seed: int,
               batch: int = 1 << 22):
    ta = np.uint64(int(a * 4294967296.0))
    tb = np.uint64(int((a + b) * 4294967296.0))
    tc = np.uint64(int((a + b + c) * 4294967296.0))
    base = _first_draw(seed)
    us, vs = [], []
    with np.errstate(over="ignore"):
        for s0 in range(0, samples, batch):
            i = np.arange(s0, min(samples, s0 + batch), dtype=np.uint64)
            state = base + i * STREAM
            u = np.zeros(len(i), np.uint32)
            v = np.zeros(len(i), np.uint32)
            bits = None
            for lvl in range(scale):
                if lvl % 2 == 0:
                    state = state + GOLDEN
                    bits = _mix(state)
                    r = bits & np.uint64(0xFFFFFFFF)
                else:
                    r = bits >> np.uint64(32)
                bu = (r >= tb).astype(np.uint32)
                bv = (((r >= ta) & (r < tb)) | (r >= tc)).astype(np.uint32)
                u = (u << np.uint32(1)) | bu
                v = (v << np.uint32(1)) | bv
            us.append(u)
            vs.append(v)
    return np.concatenate(us).astype(np.int64), np.concatenate(vs).astype(np.int64)


def csr_from_edges(V: int, u: np.ndarray, v: np.ndarray):
    keep = u != v
    u, v = u[keep], v[keep]
    key = np.unique(np.concatenate([u * V + v, v * V + u]))
    rows = key // V
    adj = (key % V).astype(np.int32)
    off = np.zeros(V + 1, np.int64)
    np.cumsum(np.bincount(rows, minlength=V), out=off[1:])
    return off, adj


def rmat(scale: int, samples: int, a: float, b: float, c: float, seed: int):
    u, v = rmat_edges(scale, samples, a, b, c, seed)
    return csr_from_edges(1 << scale, u, v)


def save_bin(path: str | Path, off: np.ndarray, adj: np.ndarray) -> None:
    V = len(off) - 1
    with open(path, "wb") as f:
        f.write(np.int32(V).tobytes())
        f.write(np.int64(len(adj)).tobytes())
        f.write(np.ascontiguousarray(off, np.int64).tobytes())
        f.write(np.ascontiguousarray(adj, np.int32).tobytes())


def load_bin(path: str | Path):
    with open(path, "rb") as f:
        V = int(np.frombuffer(f.read(4), np.int32)[0])
        E = int(np.frombuffer(f.read(8), np.int64)[0])
        off = np.frombuffer(f.read(8 * (V + 1)), np.int64).copy()
        adj = np.frombuffer(f.read(4 * E), np.int32).copy()
    return off, adj
