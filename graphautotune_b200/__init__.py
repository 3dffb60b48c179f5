"""GraphAutoTune-B200: subgraph counting on B200 behind the reference's API.

Host mirror of the reference's pattern-matching interface
(core/pattern.hpp Pattern, core/schedule.hpp Schedule,
infra/graph_backend.cuh GlobalMemoryGraph, engine/engine.cuh
Executor::perform_search, configs/*.hpp Config) over the C ABI in
include/gat.h.  Every computation runs in libgat (C++ host code and sm_100a
CUDA kernels); a missing library raises GatLibraryMissing.
"""
from __future__ import annotations

import ctypes as C
import json
from dataclasses import dataclass

import numpy as np

from ._lib import (
    MODE_EXACT,
    MODE_REF_COMPAT,
    UPLOAD_DEGREE_ORDER,
    GatError,
    GatLibraryMissing,
    check,
    gat_config,
    gat_stats,
    lib,
    read_string,
)

__all__ = [
    "Pattern", "Schedule", "Graph", "Config", "Executor", "CountResult",
    "GatError", "GatLibraryMissing", "enumerate_patterns", "MODE_EXACT",
    "MODE_REF_COMPAT",
]

_MODES = {"exact": MODE_EXACT, "ref": MODE_REF_COMPAT, "ref_compat": MODE_REF_COMPAT,
          MODE_EXACT: MODE_EXACT, MODE_REF_COMPAT: MODE_REF_COMPAT}


class _Handle:
    _free = None

    def __init__(self):
        self._h = C.c_void_p()

    def __del__(self):
        h = getattr(self, "_h", None)
        if h and h.value and self._free:
            try:
                getattr(lib(), self._free)(h)
            except Exception:
                pass
            h.value = None


class Pattern(_Handle):
    """Core::Pattern(adj_string) (core/pattern.hpp:22-39)."""

    _free = "gat_pattern_free"

    def __init__(self, adj: str):
        super().__init__()
        check(lib().gat_pattern_from_adj(adj.encode(), C.byref(self._h)))
        self.adj_input = adj

    def v_cnt(self) -> int:
        return lib().gat_pattern_vertices(self._h)

    def automorphisms(self) -> int:
        out = C.c_int64()
        check(lib().gat_pattern_automorphisms(self._h, C.byref(out)))
        return out.value

    def adjacency(self) -> str:
        n = self.v_cnt()
        buf = C.create_string_buffer(n * n + 1)
        check(lib().gat_pattern_adjacency(self._h, buf, n * n + 1))
        return buf.value.decode()


def enumerate_patterns(n: int) -> list[str]:
    """Connected n-vertex patterns (n <= 6), one per isomorphism class."""
    s = read_string(lib().gat_enumerate_patterns, n)
    return [x for x in s.split("\n") if x]


class Schedule(_Handle):
    """Core::Schedule(pattern) (core/schedule.hpp:864-958).

    mode "ref": the reference's own schedule and counting rules;
    mode "exact": a schedule for the exact subgraph count.
    """

    _free = "gat_schedule_free"

    def __init__(self, pattern: Pattern | str, mode: str | int = "exact",
                 stats_graph: "Graph | None" = None, variant: int = 0):
        super().__init__()
        if isinstance(pattern, str):
            pattern = Pattern(pattern)
        self.pattern = pattern
        self.mode = _MODES[mode]
        self.variant = variant
        g = stats_graph._h if stats_graph is not None else None
        check(lib().gat_schedule_build_variant(pattern._h, self.mode, g, variant,
                                               C.byref(self._h)))

    @staticmethod
    def variants(pattern: Pattern | str, mode: str | int = "exact",
                 stats_graph: "Graph | None" = None) -> int:
        """How many distinct plans Schedule(..., variant=i) offers."""
        if isinstance(pattern, str):
            pattern = Pattern(pattern)
        n = C.c_int32()
        g = stats_graph._h if stats_graph is not None else None
        check(lib().gat_schedule_variants(pattern._h, _MODES[mode], g, C.byref(n)))
        return n.value

    def dump(self) -> dict:
        return json.loads(read_string(lib().gat_schedule_dump, self._h))

    def plan_bytes(self) -> bytes:
        need = C.c_size_t(0)
        check(lib().gat_schedule_plan(self._h, None, 0, C.byref(need)))
        buf = C.create_string_buffer(need.value)
        check(lib().gat_schedule_plan(self._h, buf, need.value, C.byref(need)))
        return buf.raw

    @property
    def dedicated_kernel(self) -> int:
        """The device plan's `special` field: 0 when the plan interpreter
        counts it, 1 for the 4-cycle's wedge kernels, 2 for the clique
        kernels (exact mode; Executor counts use them unless
        Config.special_kernels says otherwise; batched launches interpret
        the plan)."""
        import struct

        return struct.unpack_from("<i", self.plan_bytes(), 36)[0]


@dataclass
class Config:
    """Runtime Config mirroring configs/config.hpp (+ engine knobs)."""

    set_search_type: int = 64
    set_intersection_type: int = 0
    vertex_store_type: int = 0
    graph_backend_type: int = 0
    num_blocks: int = 256
    threads_per_block: int = 128
    threads_per_warp: int = 1
    max_regs: int = 32
    chunk: int = 16
    hub_bitmaps: int = 1
    memory_budget: int = 0
    special_kernels: int = 1

    _FIELDS = ("set_search_type", "set_intersection_type", "vertex_store_type",
               "graph_backend_type", "num_blocks", "threads_per_block",
               "threads_per_warp", "max_regs", "chunk", "hub_bitmaps", "memory_budget",
               "special_kernels")

    @classmethod
    def _from_c(cls, c: gat_config) -> "Config":
        return cls(**{f: getattr(c, f) for f in cls._FIELDS})

    def to_c(self) -> gat_config:
        c = gat_config()
        for f in self._FIELDS:
            setattr(c, f, int(getattr(self, f)))
        return c

    @classmethod
    def reference_default(cls) -> "Config":
        """include/generated/default_config.hpp:5 values."""
        c = gat_config()
        lib().gat_config_default(C.byref(c))
        return cls._from_c(c)

    @classmethod
    def engine_default(cls) -> "Config":
        c = gat_config()
        lib().gat_config_engine_default(C.byref(c))
        return cls._from_c(c)

    def parse(self, text: str) -> "Config":
        """Applies a designated-initializer or config.json text."""
        c = self.to_c()
        check(lib().gat_config_parse(text.encode(), C.byref(c)))
        return Config._from_c(c)

    def format(self) -> str:
        buf = C.create_string_buffer(1024)
        c = self.to_c()
        check(lib().gat_config_format(C.byref(c), buf, 1024))
        return buf.value.decode()


class Graph(_Handle):
    """Infra::GlobalMemoryGraph (infra/graph_backend.cuh:15-170)."""

    _free = "gat_graph_free"

    def __init__(self):
        super().__init__()

    @classmethod
    def load(cls, path: str, binary: bool = True) -> "Graph":
        g = cls()
        check(lib().gat_graph_load(str(path).encode(), 1 if binary else 0, C.byref(g._h)))
        return g

    @classmethod
    def from_csr(cls, offsets: np.ndarray, adj: np.ndarray, check_symmetry: bool = True,
                 device: bool = False, stream: int | None = None) -> "Graph":
        """A graph from host CSR arrays; device=True copies them straight to
        the current GPU (gat_graph_from_csr_device) and checks them there."""
        off = np.ascontiguousarray(offsets, dtype=np.int64)
        a = np.ascontiguousarray(adj, dtype=np.int32)
        g = cls()
        if device:
            check(lib().gat_graph_from_csr_device(len(off) - 1, len(a), off.ctypes.data,
                                                  a.ctypes.data,
                                                  C.c_void_p(stream) if stream else None,
                                                  C.byref(g._h)))
        else:
            check(lib().gat_graph_from_csr(len(off) - 1, len(a), off.ctypes.data, a.ctypes.data,
                                           C.byref(g._h)))
        if check_symmetry:
            check(lib().gat_graph_validate(g._h, 1))
        return g

    @classmethod
    def erdos_renyi(cls, n: int, avg_degree: float, seed: int) -> "Graph":
        g = cls()
        check(lib().gat_graph_generate(0, n, avg_degree, 0, 0, 0, seed, C.byref(g._h)))
        return g

    @classmethod
    def rmat(cls, scale: int, samples: int, a: float = 0.57, b: float = 0.19,
             c: float = 0.19, seed: int = 0, device: bool = False) -> "Graph":
        """Seeded R-MAT graph; device=True draws and builds it on the current
        GPU (identical result, resident there afterwards)."""
        return cls._generate(1, (scale, samples, a, b, c), seed, device)

    @classmethod
    def barabasi_albert(cls, n: int, m: int, seed: int, device: bool = False) -> "Graph":
        return cls._generate(2, (n, m, 0, 0, 0), seed, device)

    @classmethod
    def _generate(cls, kind: int, p: tuple, seed: int, device: bool) -> "Graph":
        g = cls()
        if device:
            check(lib().gat_graph_generate_device(kind, *p, seed, None, C.byref(g._h)))
        else:
            check(lib().gat_graph_generate(kind, *p, seed, C.byref(g._h)))
        return g

    def save(self, path: str) -> None:
        check(lib().gat_graph_save(self._h, str(path).encode()))

    def info(self) -> tuple[int, int, int]:
        v, e, m = C.c_int32(), C.c_int64(), C.c_int32()
        check(lib().gat_graph_info(self._h, C.byref(v), C.byref(e), C.byref(m)))
        return v.value, e.value, m.value

    def v_cnt(self) -> int:
        return self.info()[0]

    def e_cnt(self) -> int:
        return self.info()[1]

    def max_degree(self) -> int:
        return self.info()[2]

    def csr(self) -> tuple[np.ndarray, np.ndarray]:
        """Copies of the host CSR arrays (int64 offsets, int32 neighbours)."""
        v, e, _ = self.info()
        po, pa = C.c_void_p(), C.c_void_p()
        check(lib().gat_graph_csr(self._h, C.byref(po), C.byref(pa)))
        off = np.ctypeslib.as_array(C.cast(po, C.POINTER(C.c_int64)), shape=(v + 1,)).copy()
        adj = (np.ctypeslib.as_array(C.cast(pa, C.POINTER(C.c_int32)), shape=(e,)).copy()
               if e > 0 else np.zeros(0, np.int32))
        return off, adj

    def upload(self, degree_order: bool = True, stream: int | None = None,
               hub_min_degree: int | None = None, hub_max_bytes: int | None = None) -> None:
        """GlobalMemoryGraph::to_device (graph_backend.cuh:102-118), plus the
        degree-ordered copy and hub bitmaps."""
        flags = UPLOAD_DEGREE_ORDER if degree_order else 0
        s = C.c_void_p(stream) if stream else None
        if hub_min_degree is None and hub_max_bytes is None:
            check(lib().gat_graph_upload(self._h, flags, s))
        else:
            check(lib().gat_graph_upload_ex(self._h, flags,
                                            512 if hub_min_degree is None else hub_min_degree,
                                            (1 << 30) if hub_max_bytes is None else hub_max_bytes,
                                            s))

    def hubs(self, ordered: bool = True) -> int:
        n = C.c_int32()
        check(lib().gat_graph_hubs(self._h, 1 if ordered else 0, C.byref(n)))
        return n.value

    def ordered_csr(self) -> tuple[np.ndarray, np.ndarray]:
        """The degree-ordered device copy (vertex r = r-th by decreasing
        degree, ties by id), read back from the GPU."""
        V, E, _ = self.info()
        off = np.empty(V + 1, np.int64)
        adj = np.empty(max(E, 1), np.int32)
        check(lib().gat_graph_ordered_csr(self._h, off.ctypes.data, adj.ctypes.data))
        return off, adj[:E]


@dataclass
class CountResult:
    count: int
    kernel_ms: float
    total_ms: float
    raw_sum: int
    divisor: int
    tasks: int
    balg_bytes: int
    grid: int
    block: int
    tile: int
    scratch_bytes: int
    launches: int = 1


class Executor(_Handle):
    """Engine::Executor (engine/engine.cuh:157-265)."""

    _free = "gat_executor_free"

    def __init__(self, config: Config | None = None):
        super().__init__()
        cfg = (config or Config.engine_default()).to_c()
        check(lib().gat_executor_create(C.byref(cfg), C.byref(self._h)))

    def count(self, graph: Graph, schedule: Schedule, stream: int | None = None,
              balg: bool = False) -> CountResult:
        out = C.c_uint64()
        st = gat_stats()
        fn = lib().gat_executor_count_balg if balg else lib().gat_executor_count
        check(fn(self._h, graph._h, schedule._h, C.c_void_p(stream) if stream else None,
                 C.byref(out), C.byref(st)))
        cnt = out.value
        if schedule.mode == MODE_REF_COMPAT and cnt >= 1 << 63:
            cnt -= 1 << 64
        return CountResult(cnt, st.kernel_ms, st.total_ms, st.raw_sum, st.divisor, st.tasks,
                           st.balg_bytes, st.grid, st.block, st.tile, st.scratch_bytes, st.launches)

    def count_range(self, graph: Graph, schedule: Schedule, root_begin: int, root_end: int,
                    stream: int | None = None) -> tuple[int, CountResult]:
        """Undivided signed total over first vertices in [root_begin, root_end)."""
        raw = C.c_int64()
        st = gat_stats()
        check(lib().gat_executor_count_range(self._h, graph._h, schedule._h,
                                             C.c_void_p(stream) if stream else None,
                                             root_begin, root_end, C.byref(raw), C.byref(st)))
        return raw.value, CountResult(raw.value, st.kernel_ms, st.total_ms, st.raw_sum,
                                      st.divisor, st.tasks, st.balg_bytes, st.grid, st.block,
                                      st.tile, st.scratch_bytes, st.launches)

    def count_shard(self, graph: Graph, schedule: Schedule, shard: int, num_shards: int,
                    stream: int | None = None, balg: bool = False) -> tuple[int, CountResult]:
        """Undivided signed total of one equal slice of the work queue."""
        raw = C.c_int64()
        st = gat_stats()
        fn = lib().gat_executor_count_shard_balg if balg else lib().gat_executor_count_shard
        check(fn(self._h, graph._h, schedule._h, C.c_void_p(stream) if stream else None,
                 shard, num_shards, C.byref(raw), C.byref(st)))
        return raw.value, CountResult(raw.value, st.kernel_ms, st.total_ms, st.raw_sum,
                                      st.divisor, st.tasks, st.balg_bytes, st.grid, st.block,
                                      st.tile, st.scratch_bytes, st.launches)

    def perform_search(self, graph: Graph, schedule: Schedule) -> int:
        """long long Executor::perform_search(DeviceContext&)."""
        return self.count(graph, schedule).count


class Batch(_Handle):
    """Many (schedule, graph) counts in one persistent launch (gat_batch_*)."""

    _free = "gat_batch_free"

    def __init__(self):
        super().__init__()
        check(lib().gat_batch_create(C.byref(self._h)))
        self._keep: list = []  # graphs and schedules must outlive the batch

    def add(self, graph: Graph, schedule: Schedule) -> int:
        j = C.c_int32()
        check(lib().gat_batch_add(self._h, graph._h, schedule._h, C.byref(j)))
        self._keep.append((graph, schedule, False))
        return j.value

    def add_shard(self, graph: Graph, schedule: Schedule, shard: int, num_shards: int) -> int:
        """One equal slice of the job's work queue; counts() reports the
        slice's undivided raw total for it."""
        j = C.c_int32()
        check(lib().gat_batch_add_shard(self._h, graph._h, schedule._h, shard, num_shards,
                                        C.byref(j)))
        self._keep.append((graph, schedule, True))
        return j.value

    def prepare(self, config: Config | None = None, cuda_graph: bool = True) -> None:
        cfg = (config or Config.engine_default()).to_c()
        check(lib().gat_batch_prepare(self._h, C.byref(cfg), 1 if cuda_graph else 0))

    def run(self) -> CountResult:
        st = gat_stats()
        check(lib().gat_batch_run(self._h, C.byref(st)))
        return CountResult(0, st.kernel_ms, st.total_ms, 0, 1, st.tasks, 0, st.grid, st.block,
                           st.tile, st.scratch_bytes, st.launches)

    def counts(self) -> list[int]:
        n = lib().gat_batch_size(self._h)
        arr = (C.c_uint64 * max(n, 1))()
        check(lib().gat_batch_counts(self._h, arr, n))
        out = []
        for (g, s, sliced), v in zip(self._keep, arr[:n]):
            signed = sliced or s.mode == MODE_REF_COMPAT  # raw slice totals can be < 0
            out.append(v - (1 << 64) if signed and v >= 1 << 63 else v)
        return out

    def __len__(self) -> int:
        return lib().gat_batch_size(self._h)
