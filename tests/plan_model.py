"""Test helper: a slow Python model of how the CUDA engine interprets a
device plan (struct GatPlan, graphautotune_b200/csrc/gat_plan.h).

It lets the planners be checked against the oracle on the CPU: if the model
of a plan gives the oracle's count, the plan is right, and the GPU tests then
check that the kernel implements the same semantics.
"""
from __future__ import annotations

import ctypes as C
from bisect import bisect_left

MAXV, MAXP, MAXT = 10, 32, 64
ALIAS, STORE, COUNT = 0, 1, 2
INF = 2**31 - 1


class GatPlan(C.Structure):
    _fields_ = [
        ("n", C.c_int32), ("basic", C.c_int32), ("num_prefix", C.c_int32),
        ("mode", C.c_int32), ("collide_clear", C.c_int32), ("level1_bounded", C.c_int32),
        ("num_store", C.c_int32), ("iep_num", C.c_int32), ("num_terms", C.c_int32),
        ("special", C.c_int32), ("divisor", C.c_int64),
        ("lane_last", C.c_int32), ("pad1", C.c_int32),
        ("p_level", C.c_int8 * MAXP), ("p_father", C.c_int8 * MAXP),
        ("p_kind", C.c_int8 * MAXP), ("p_slot", C.c_int8 * MAXP),
        ("p_trunc", C.c_uint16 * MAXP), ("p_excl", C.c_uint16 * MAXP),
        ("l_loop", C.c_int8 * MAXV), ("l_pbegin", C.c_int8 * (MAXV + 1)),
        ("l_bound", C.c_uint16 * MAXV), ("l_distinct", C.c_uint16 * MAXV),
        ("iep_prefix", C.c_int8 * MAXP), ("iep_sub", C.c_uint16 * MAXP),
        ("iep_bound", C.c_uint16 * MAXP),
        ("t_slot", C.c_int8 * MAXT), ("t_close", C.c_int8 * MAXT),
        ("t_coef", C.c_int32 * MAXT),
    ]


def parse(raw: bytes) -> GatPlan:
    assert len(raw) == C.sizeof(GatPlan), (len(raw), C.sizeof(GatPlan))
    return GatPlan.from_buffer_copy(raw)


def run(P: GatPlan, off, adj) -> tuple[int, int]:
    """Returns (raw signed total, divisor)."""
    V = len(off) - 1
    rows = [list(adj[off[v]:off[v + 1]]) for v in range(V)]
    basic = P.basic
    emb = [0] * MAXV
    sets: list = [None] * P.num_prefix

    def minmask(m):
        r = INF
        for j in range(MAXV):
            if m >> j & 1:
                r = min(r, emb[j])
        return r

    def level_sets(k, v, collided):
        nb = rows[v]
        for p in range(P.l_pbegin[k], P.l_pbegin[k + 1]):
            kind = P.p_kind[p]
            if collided:
                sets[p] = 0 if kind == COUNT else []
                continue
            T = minmask(P.p_trunc[p])
            nbt = nb[:bisect_left(nb, T)]
            if kind == ALIAS:
                sets[p] = nbt
                continue
            F = sets[P.p_father[p]]
            Ft = F[:bisect_left(F, T)]
            inter = sorted(set(Ft) & set(nbt))
            if kind == STORE:
                sets[p] = inter
            else:
                ex = {emb[j] for j in range(MAXV) if P.p_excl[p] >> j & 1}
                sets[p] = sum(1 for x in inter if x not in ex)

    def iep():
        vals = []
        for x in range(P.iep_num):
            p = P.iep_prefix[x]
            if P.p_kind[p] == COUNT:
                vals.append(sets[p])
                continue
            S = sets[p]
            S = S[:bisect_left(S, minmask(P.iep_bound[x]))]
            ss = set(S)
            sub = sum(1 for j in range(basic) if P.iep_sub[x] >> j & 1 and emb[j] in ss)
            vals.append(len(S) - sub)
        local, cur, last = 0, 1, -1
        for g in range(P.num_terms):
            a = vals[P.t_slot[g]]
            cur = a if g == last + 1 else cur * a
            if P.t_close[g]:
                last = g
                local += cur * P.t_coef[g]
        return local

    total = 0

    def search(k):
        nonlocal total
        lp = P.l_loop[k]
        L = sets[lp]
        cnt = bisect_left(L, minmask(P.l_bound[k]))
        for i in range(cnt):
            cand = L[i]
            hit = any(emb[j] == cand for j in range(MAXV) if P.l_distinct[k] >> j & 1)
            if hit and not P.collide_clear:
                continue
            emb[k] = cand
            level_sets(k, cand, hit)
            if k == basic - 1:
                total += iep()
            else:
                search(k + 1)

    for v0 in range(V):
        emb[0] = v0
        level_sets(0, v0, False)
        for v1 in rows[v0]:
            if P.level1_bounded and v1 >= v0:
                break
            emb[1] = v1
            level_sets(1, v1, False)
            if basic == 2:
                total += iep()
            else:
                search(2)
    return total, P.divisor
