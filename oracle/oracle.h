/* Test infrastructure only: the CPU oracle for the pattern-counting path.
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may
 * load this library, and only as the checker.  The product (libgat) never
 * links or calls it.
 *
 * Every function restates reference behaviour on plain CSR arrays:
 *   int64 offs[V+1], int32 adj[E]  (sorted, deduplicated, symmetric lists;
 *   infra/graph_backend.cuh:91-99 is the reference layout).
 *
 * Parity pins: oracle_naive_labelled is checked against the reference's own
 * naive_pm binary (oracle/_ref) on seeded graphs, oracle_ref_engine against
 * the reference engine (pm) counts, and the reference's single numeric test
 * (tests/test_vertex_set.cu:76, |{1..30} n {2,4..60}| = 15) through
 * oracle_intersect_size.  See tests/golden/.
 */
#ifndef GAT_ORACLE_H
#define GAT_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Labelled, non-induced, injective embeddings of the pattern (n x n '0'/'1'
 * row-major adjacency, symmetrised from the lower triangle exactly like
 * core/pattern.hpp:22-39), restating target/naive_pm.cu:10-44: at depth d
 * every vertex i of the graph is tried; i is rejected if already chosen or if
 * a pattern edge (j, d) has no graph edge (choose[j], i).  Only first-level
 * vertices in [root_begin, root_end) are tried (the full count uses [0, V)).
 * Returns the 64-bit count (the reference keeps an int). */
uint64_t oracle_naive_labelled(int32_t V, const int64_t *offs,
                               const int32_t *adj, const char *pattern,
                               int32_t root_begin, int32_t root_end,
                               int threads);

/* oracle_naive_labelled over an explicit list of first-level vertices (a
 * bounded sample of roots). */
uint64_t oracle_naive_labelled_roots(int32_t V, const int64_t *offs,
                                     const int32_t *adj, const char *pattern,
                                     const int32_t *roots, int64_t num,
                                     int threads);

/* Same count as oracle_naive_labelled, with candidates drawn from the
 * neighbour list of one earlier adjacent pattern vertex instead of all V
 * (the result is identical; only untouched candidates are skipped). */
uint64_t oracle_backtrack_labelled(int32_t V, const int64_t *offs,
                                   const int32_t *adj, const char *pattern,
                                   int32_t root_begin, int32_t root_end,
                                   int threads);

/* |Aut(pattern)|: permutations that map the pattern onto itself
 * (core/schedule.hpp:173-191). */
int64_t oracle_automorphisms(const char *pattern);

/* The reference engine's per-unit semantics (engine/engine.cuh:232-428,
 * engine/engine_kernel.cuh:40-432, implementations/array_vertex_set.cuh),
 * evaluated depth-first on the CPU.  `sd` is a flat encoding of
 * Core::ScheduleData (core/schedule.hpp:984-1022):
 *   [0] basic_vertexes  [1] total_prefix_num  [2] restrictions count R
 *   [3] iep_prefix_num  [4] subgroups_num
 *   then, in order:
 *   prefixs:  for each prefix: depth, data[depth]
 *   prefixs_father[P], prefixs_size_only[P],
 *   vertex_prefix_start[basic+1], loop_set_prefix_id[basic],
 *   restrictions_start[basic+1], restrictions[R] (the .first of each pair),
 *   iep_vertex_id[iep_prefix_num], iep_ans_pos[S], iep_coef[S], iep_flag[S]
 * Returns 0 and writes the signed 64-bit total to *out, or a negative code:
 *   -1 malformed encoding, -2 the reference would read an uninitialised
 *   restriction slot (undefined result), -3 a loop set is a size-only prefix
 *   created after level 0 (the reference reads an unmaterialised set).
 * `balg` (may be NULL) receives the algorithmic bytes of the set operations:
 * 4*(|A|+|B|) per intersection plus 4*|C| per materialised output. */
int oracle_ref_engine(int32_t V, const int64_t *offs, const int32_t *adj,
                      const int32_t *sd, int32_t sd_len, int32_t root_begin,
                      int32_t root_end, int threads, int64_t *out,
                      uint64_t *balg);

/* Labelled embeddings f of the pattern with f(0) in [root_begin, root_end)
 * and f(less[2i]) < f(less[2i+1]) for every i < nless (pattern vertex
 * indices).  With an exact plan's vertex order and symmetry-breaking
 * conditions, this is the plan's undivided total over those roots; it is
 * found by plain backtracking (candidates from neighbour lists, the last
 * vertex counted), sharing nothing with the engine's prefix sets or
 * inclusion-exclusion.  Summed over all roots and divided by the plan's
 * divisor it is naive_pm's Answer / |Aut|. */
uint64_t oracle_restricted_labelled(int32_t V, const int64_t *offs, const int32_t *adj,
                                    const char *pattern, const int32_t *less,
                                    int32_t nless, int32_t root_begin, int32_t root_end,
                                    int threads);

/* As oracle_restricted_labelled, giving up (returning 0 with *over = 1)
 * once about max_work candidates have been examined (max_work < 0: no cap). */
uint64_t oracle_restricted_labelled_capped(int32_t V, const int64_t *offs,
                                           const int32_t *adj, const char *pattern,
                                           const int32_t *less, int32_t nless,
                                           int32_t root_begin, int32_t root_end, int threads,
                                           int64_t max_work, int *over);

/* 4-cycles counted at a corner: for each v0 in [root_begin, root_end),
 * sum over x of C(c, 2), c = common neighbours v1 of v0 and x with v1 and x
 * above v0 (at_largest = 0: cycles whose smallest vertex is v0) or below it
 * (at_largest = 1: cycles whose largest vertex is v0).  Over all roots both
 * give the 4-cycle count (naive_pm's Answer / 8). */
uint64_t oracle_c4_rooted(int32_t V, const int64_t *offs, const int32_t *adj,
                          int32_t root_begin, int32_t root_end, int at_largest,
                          int threads);

/* The graph relabelled by decreasing degree, ties by smaller id first
 * (vertex r of the result is the r-th in that order), rows sorted.  Writes
 * V+1 offsets and E neighbours. */
int oracle_degree_order(int32_t V, const int64_t *offs, const int32_t *adj,
                        int64_t *new_offs, int32_t *new_adj);

/* |a n b| for two sorted int32 lists (array_vertex_set.cuh:160-200). */
int32_t oracle_intersect_size(const int32_t *a, int32_t na, const int32_t *b,
                              int32_t nb);

#ifdef __cplusplus
}
#endif
#endif
