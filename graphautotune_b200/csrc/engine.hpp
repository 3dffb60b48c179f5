// Host-side interface of the CUDA search engine.
#pragma once
#include <cuda_runtime.h>

#include <cstdint>
#include <string>

#include "gat_plan.h"

namespace gat {

// A graph resident on the device.  `task_off` arrays index the level-1
// units: lo_off[v] = number of entries u < v in rows before v (rows are
// sorted, so a row's entries u < v are its prefix).
struct DevGraphView {
    int32_t V = 0;
    int64_t E = 0;
    const int64_t *off = nullptr;
    const int32_t *adj = nullptr;
    const int64_t *lo_off = nullptr;
    int64_t lo_total = 0;  // lo_off[V]
    int32_t max_degree = 0;
    int32_t max_lower = 0;  // max over v of lo_off[v + 1] - lo_off[v]
    // Hub bitmaps: bit x of row hub_slot[v] is set iff x is in N(v), for
    // the vertices with hub_slot[v] >= 0 (null when none were built).
    const int32_t *hub_slot = nullptr;
    const uint32_t *bitmaps = nullptr;
    int64_t bitmap_words = 0;  // words per row = ceil(V / 32)
};

// Fills one V-bit row per hub (rows must be zeroed first).
cudaError_t build_hub_bitmaps(const int64_t *off, const int32_t *adj,
                              const int32_t *hubs, int32_t nhubs, int64_t words,
                              uint32_t *bitmaps, cudaStream_t stream);

// lo_off[v] = sum over u < v of |{w in N(u) : w < u}| (V+1 entries), from a
// device CSR with sorted rows (relabel.cu).
cudaError_t lower_offsets_device(const int64_t *off, const int32_t *adj, int32_t V,
                                 int64_t *lo_off, cudaStream_t stream);
// Whether relabel_by_degree_device takes a graph of this size.
bool relabel_fits_device(int32_t V, int64_t E);
// The copy relabelled by decreasing degree (ties by id), rows sorted, built
// from a device CSR into caller-allocated new_off (V+1) and new_adj (E).
cudaError_t relabel_by_degree_device(const int64_t *off, const int32_t *adj, int32_t V,
                                     int64_t E, int32_t max_degree, int64_t *new_off,
                                     int32_t *new_adj, cudaStream_t stream);

struct LaunchShape {
    int grid = 0;         // CTAs
    int block = 128;      // threads per CTA
    int tile = 32;        // lanes cooperating on one unit
    int chunk = 16;       // level-1 units taken per queue grab
    int linear_below = 0; // lists shorter than this are scanned linearly
    int64_t task_begin = 0;  // level-1 unit range [task_begin, task_end);
    int64_t task_end = -1;   // -1: all units
    bool use_bitmaps = true; // use the graph's hub bitmaps when present
};

// Device counters used by one search: work-queue cursor, signed 64-bit
// total (two's complement in an unsigned word), algorithmic bytes, error
// flags.
struct DevCounters {
    unsigned long long cursor;
    unsigned long long result;
    unsigned long long bytes;
    unsigned long long error;
};

// Exact 4-cycle count by wedge aggregation over smallest vertices
// [v_begin, v_end) (plans with special == GAT_SPECIAL_C4), tallied in shared
// memory (cycles.cu).  Roots below heavy_end take a CTA each; the others a
// warp each, which defers roots with many wedges to the CTA kernel.
struct C4Aux {
    unsigned long long light_cursor;
    unsigned long long deferred_count;
    unsigned long long root_cursor;
    unsigned long long pad;
};
struct C4Launch {
    DevGraphView g;
    int64_t v_begin = 0, v_end = 0, heavy_end = 0;
    int light_grid = 0, root_grid = 0;
    DevCounters *ctr = nullptr;
    C4Aux *aux = nullptr;
    int32_t *deferred = nullptr;   // room for every light root
    int32_t *cursors = nullptr;    // root_grid x cursor_stride list positions
    int64_t cursor_stride = 0;     // >= the largest degree
    bool stats = false;
};
int c4_light_blocks_per_sm(bool stats);
int c4_root_blocks_per_sm(bool wide, bool stats);
cudaError_t launch_c4(const C4Launch &launch, cudaStream_t st);

// Exact k-clique count (4 <= k <= 7) over the level-1 units [u_begin, u_end)
// of the K_k exact plan: unit lo_off[v0] + i is (v0, i-th lower neighbour),
// whose cliques have v0 as largest and that neighbour as second largest
// vertex (plans with special == GAT_SPECIAL_CLIQUE), by bit-matrix induced subgraphs
// of each root's lower list (cliques.cu).  Needs lo_off, every lower list of
// at most kCliqueMaxLower entries, and adj readable 4 ints past its end.
// `rows` holds cta_grid slices of rows_stride words when
// clique_rows_words(max lower degree) > 0, else it may be null.
constexpr int kCliqueMaxLower = 2048;
constexpr int kCliqueCtaThreads = 512;  // threads of the CTA-per-root kernel
struct CliqueAux {
    unsigned long long warp_cursor;
    unsigned long long cta_cursor;
    unsigned long long pad[2];
};
struct CliqueLaunch {
    DevGraphView g;
    int k = 4;
    int64_t v_begin = 0, v_end = 0;  // roots holding the units [u_begin, u_end)
    int64_t u_begin = 0, u_end = 0;  // level-1 units (v0, v1 < v0) numbered by lo_off
    int warp_grid = 0, cta_grid = 0;
    DevCounters *ctr = nullptr;
    CliqueAux *aux = nullptr;
    uint32_t *rows = nullptr;
    int64_t rows_stride = 0;
    bool stats = false;
};
int64_t clique_rows_words(int32_t max_lower);
void clique_blocks_per_sm(int k, bool stats, int *warp_occ, int *cta_occ);
cudaError_t launch_clique(const CliqueLaunch &launch, cudaStream_t st);

// Graph construction on the device (gen.cu).  Both write off[V + 1] (caller
// allocated) and allocate *adj with pad_ints ints past the E entries; E is
// the number of directed entries of the symmetric, loop-free, deduplicated
// CSR with sorted rows.
// R-MAT exactly as graph.cpp gen_rmat + build_csr compute it.
cudaError_t rmat_csr_device(int scale, int64_t samples, double a, double b, double c,
                            uint64_t seed, int64_t *off, int32_t **adj, int64_t pad_ints,
                            int64_t *E, cudaStream_t st);
// Checks a device CSR by the host validate() rules without symmetry; *flag
// ends as ~0 when every row passes, else (first failing row << 3) | reason.
enum : unsigned { kCsrOffsets = 1, kCsrRange = 2, kCsrLoop = 3, kCsrOrder = 4 };
cudaError_t csr_check_device(const int64_t *off, const int32_t *adj, int32_t V, int64_t E,
                             unsigned long long *flag, cudaStream_t st);
// An undirected edge list of n (u, v) pairs (device memory) on V vertices.
cudaError_t pairs_csr_device(const int32_t *pairs, int64_t n, int32_t V, int64_t *off,
                             int32_t **adj, int64_t pad_ints, int64_t *E, cudaStream_t st);

// Batched launches: host code fills an array of batch_job_bytes()-sized job
// records (one per (plan, graph) pair), copies it and the chunk-aligned
// virtual start of every job to the device, and launches one persistent
// kernel over all of them.  `results` receives one signed 64-bit raw total
// per job; cursor and results must be zero before the launch.
size_t batch_job_bytes();
void batch_fill_job(void *dst, const GatPlan *d_plan, const GatPlan &h_plan,
                    const DevGraphView &g, int linear_below, bool use_bitmaps, int shard = 0,
                    int num_shards = 0);
int64_t batch_job_tasks(const void *job);
int batch_blocks_per_sm(int tile, int block);
cudaError_t launch_batch(const void *d_jobs, const int64_t *d_vstart, int32_t num_jobs,
                         int64_t vtotal, int tile, int grid, int block, int chunk,
                         unsigned long long *d_cursor, unsigned long long *d_results,
                         int32_t *scratch, int64_t stride, cudaStream_t st);

// Counts `plan` on a caller-owned device CSR without allocating: counters,
// plan and per-tile set scratch live in the library's static device array
// (GAT_NOALLOC_SCRATCH_BYTES, include/gat.h).  Writes the count (raw sum /
// divisor, or LLONG_MIN on a device-side error) to d_count on `stream`.
// Returns a gat_status.
int count_noalloc(const GatPlan &plan, const int64_t *d_off, const int32_t *d_adj,
                  int32_t V, int64_t E, int32_t max_degree, const LaunchShape &shape,
                  long long *d_count, cudaStream_t stream, std::string *err);

enum : unsigned long long {
    GAT_DEVERR_SCRATCH = 1ull,  // a stored set would overflow its slot
    GAT_DEVERR_TABLE = 2ull,    // a shared-memory count table ran out of slots
    GAT_DEVERR_WAIT = 4ull,     // a bulk copy did not complete within the wait bound
};

// Shared memory one tile needs.
size_t tile_smem_bytes();
// Largest CTA count per SM for this tile/block/stats combination.
int blocks_per_sm(int tile, int block, bool stats);
// Scratch ints one tile needs for `plan` on a graph with this max degree.
int64_t tile_scratch_ints(const GatPlan &plan, int32_t max_degree);

// Launches the search kernel.  `counters` must be zeroed before the launch
// (done here with cudaMemsetAsync on `stream`).  Returns a cudaError_t.
cudaError_t launch_search(const GatPlan *d_plan, const GatPlan &h_plan,
                          const DevGraphView &g, const LaunchShape &shape,
                          int32_t *scratch, int64_t scratch_stride,
                          DevCounters *counters, bool stats,
                          cudaStream_t stream);

}  // namespace gat
