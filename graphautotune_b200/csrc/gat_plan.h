/* The device plan: a flat, pointer-free description of one pattern's search
 * that the CUDA engine interprets.  It plays the role of the reference's
 * Core::ScheduleData (core/schedule.hpp:984-1022), which is passed by value
 * to every kernel there, but it is a different encoding: one record per
 * prefix set and per enumeration level, bit masks over embedded levels for
 * bounds and exclusions, and the inclusion-exclusion terms flattened.
 *
 * Levels 0 .. basic-1 are enumerated vertex by vertex.  A prefix set belongs
 * to the level of its last vertex: it is either N(v_level) itself (alias),
 * N(v_level) intersected with its father set (materialised in scratch), or a
 * count of that intersection (count only).  After level basic-1 the
 * remaining independent suffix vertices are counted by inclusion-exclusion
 * over the IEP sets.
 *
 * "min mask" fields encode min{ v_j : bit j set } (no bits = +infinity).
 */
#ifndef GAT_PLAN_H
#define GAT_PLAN_H
#include <stdint.h>

#define GAT_MAX_VERTICES 10
#define GAT_MAX_PREFIX 32
#define GAT_MAX_TERMS 64

#define GAT_SPECIAL_C4 1
#define GAT_SPECIAL_CLIQUE 2

enum {
    GAT_SET_ALIAS = 0,  /* N(v_level), truncated by p_trunc */
    GAT_SET_STORE = 1,  /* N(v_level) n father, materialised */
    GAT_SET_COUNT = 2   /* |N(v_level) n father|, minus p_excl, below p_trunc */
};

typedef struct GatPlan {
    int32_t n;             /* pattern vertices */
    int32_t basic;         /* enumerated levels, 2 <= basic <= n */
    int32_t num_prefix;
    int32_t mode;          /* 0 exact, 1 reference-compatible */
    int32_t collide_clear; /* 1: a candidate equal to an embedded vertex
                              empties that level's sets and the unit goes on
                              (reference); 0: the candidate is skipped */
    int32_t level1_bounded;/* 1: level-1 candidates are v1 < v0 */
    int32_t num_store;     /* materialised prefixes = scratch slots per tile */
    int32_t iep_num;       /* IEP value slots */
    int32_t num_terms;     /* IEP subgroups */
    int32_t special;       /* 0: interpret this plan; GAT_SPECIAL_C4 /
                              GAT_SPECIAL_CLIQUE: the exact 4-cycle or
                              k-clique count has a dedicated kernel (the
                              plan stays valid as its fallback) */
    int64_t divisor;       /* final count = sum / divisor */
    int32_t lane_last;     /* 1: every prefix of level basic-1 is COUNT and
                              every IEP slot is one of them (<= 8 slots), so
                              lanes may take last-level candidates one each */
    int32_t pad1;

    int8_t p_level[GAT_MAX_PREFIX];
    int8_t p_father[GAT_MAX_PREFIX];
    int8_t p_kind[GAT_MAX_PREFIX];
    int8_t p_slot[GAT_MAX_PREFIX];     /* scratch slot (STORE) or -1 */
    uint16_t p_trunc[GAT_MAX_PREFIX];  /* min mask: drop elements >= it */
    uint16_t p_excl[GAT_MAX_PREFIX];   /* COUNT: levels whose vertex is not
                                          counted */

    int8_t l_loop[GAT_MAX_VERTICES];        /* loop-set prefix of level k */
    int8_t l_pbegin[GAT_MAX_VERTICES + 1];  /* prefixes of level k:
                                               [l_pbegin[k], l_pbegin[k+1]) */
    uint16_t l_bound[GAT_MAX_VERTICES];     /* min mask: candidate < it */
    uint16_t l_distinct[GAT_MAX_VERTICES];  /* levels the candidate is
                                               compared against */

    int8_t iep_prefix[GAT_MAX_PREFIX];
    uint16_t iep_sub[GAT_MAX_PREFIX];   /* ALIAS/STORE: subtract each v_j
                                           (bit j) found in the set */
    uint16_t iep_bound[GAT_MAX_PREFIX]; /* ALIAS/STORE: count only elements
                                           below this min mask */
    int8_t t_slot[GAT_MAX_TERMS];
    int8_t t_close[GAT_MAX_TERMS];
    int32_t t_coef[GAT_MAX_TERMS];
} GatPlan;

#endif
