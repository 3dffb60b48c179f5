/* libgat: B200 subgraph-counting engine, C ABI.
 *
 * Drop-in boundary for GraphAutoTune's pattern-matching path.  Each entry
 * point names the reference interface it replaces (paths inside the
 * reference project).  Plain pointers, sizes and status codes only; no C++
 * or CUDA types cross this boundary (CUDA streams are passed as void*).
 *
 * Error behaviour: the reference exits the process on CUDA errors
 * (utils/cuda_utils.cuh:7-16 gpuErrchk) and throws on I/O errors
 * (target/pm.cu:16,24).  Here every call returns a gat_status; the message
 * of the last failure on the calling thread is available from
 * gat_last_error().  No call exits the process.
 *
 * Threading: handles are not internally locked; use one host thread per
 * executor.  Graph and schedule handles may be shared read-only.
 */
#ifndef GAT_H
#define GAT_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum gat_status {
    GAT_OK = 0,
    GAT_ERR_ARGUMENT = 1,    /* null pointer, size out of range */
    GAT_ERR_PATTERN = 2,     /* malformed, disconnected or too large pattern */
    GAT_ERR_IO = 3,          /* file missing, truncated or malformed */
    GAT_ERR_CUDA = 4,        /* a CUDA runtime call failed */
    GAT_ERR_MEMORY = 5,      /* allocation failed or memory budget too small */
    GAT_ERR_UNDEFINED = 6,   /* the reference engine's result is undefined for
                                this schedule (reads uninitialised state) */
    GAT_ERR_DEVICE = 7,      /* the kernel reported an internal error */
    GAT_ERR_STATE = 8,       /* handle in the wrong state (e.g. not uploaded) */
    GAT_ERR_CONFIG = 9       /* unparsable or out-of-range configuration */
} gat_status;

/* Count semantics. */
typedef enum gat_mode {
    GAT_MODE_EXACT = 0,      /* number of (non-induced) subgraphs isomorphic to
                                the pattern = labelled embeddings / |Aut| */
    GAT_MODE_REF_COMPAT = 1  /* the value Executor::perform_search returns for
                                the reference's own schedule
                                (engine/engine.cuh:232-265) */
} gat_mode;

typedef struct gat_pattern gat_pattern;
typedef struct gat_schedule gat_schedule;
typedef struct gat_graph gat_graph;
typedef struct gat_executor gat_executor;

const char *gat_last_error(void);
const char *gat_version(void);

/* ------------------------------------------------------------- pattern --
 * Replaces Core::Pattern(const std::string&) (core/pattern.hpp:22-39):
 * n*n characters '0'/'1', row-major, symmetrised from either triangle,
 * 1 <= n <= 10 (MAX_VERTEXES, consts/general_consts.hpp:3). */
int gat_pattern_from_adj(const char *adj, gat_pattern **out);
int gat_pattern_vertices(const gat_pattern *p);
/* |Aut(p)| (core/schedule.hpp:189-191). */
int gat_pattern_automorphisms(const gat_pattern *p, int64_t *out);
/* Writes the symmetrised n*n adjacency string (+ NUL) into buf. */
int gat_pattern_adjacency(const gat_pattern *p, char *buf, size_t cap);
void gat_pattern_free(gat_pattern *p);
/* All connected n-vertex patterns (n <= 6) up to isomorphism, each as its
 * lexicographically smallest adjacency string, sorted, concatenated with
 * '\n'.  *needed receives the byte count including the final NUL. */
int gat_enumerate_patterns(int n, char *buf, size_t cap, size_t *needed);

/* ------------------------------------------------------------ schedule --
 * Replaces Core::Schedule(const Pattern&) (core/schedule.hpp:864-958) and
 * Core::ScheduleData (core/schedule.hpp:984-1022).
 *   GAT_MODE_REF_COMPAT: the reference's own schedule (same vertex order,
 *     restrictions, prefixes and IEP groups), executed with the reference
 *     engine's counting rules.
 *   GAT_MODE_EXACT: a schedule for the exact count; `stats_graph` (nullable)
 *     supplies data-graph statistics for ranking candidate vertex orders in
 *     place of the reference's fixed v=5000, e=1e6, tri=1e4
 *     (core/schedule.hpp:909-910). */
int gat_schedule_build(const gat_pattern *p, int mode,
                       const gat_graph *stats_graph, gat_schedule **out);
/* Data-aware schedule choice (no reference counterpart: the reference keeps
 * the first schedule its cost formula ranks best, core/schedule.hpp:878-926).
 * For GAT_MODE_EXACT, *count receives the number of distinct exact plans
 * among the best-ranked vertex orders (at most 16; 1 for other modes), and
 * gat_schedule_build_variant builds plan `variant` of them (0 = the one
 * gat_schedule_build returns).  Every variant counts the same subgraphs; a
 * caller times them on a slice of the work queue and keeps the fastest. */
int gat_schedule_variants(const gat_pattern *p, int mode,
                          const gat_graph *stats_graph, int32_t *count);
int gat_schedule_build_variant(const gat_pattern *p, int mode,
                               const gat_graph *stats_graph, int32_t variant,
                               gat_schedule **out);
int gat_schedule_mode(const gat_schedule *s);
/* JSON with the fields of Schedule::output() (core/schedule.hpp:752-784)
 * plus the chosen permutation and restrictions.  *needed = bytes incl NUL. */
int gat_schedule_dump(const gat_schedule *s, char *buf, size_t cap,
                      size_t *needed);
/* Copies the device plan (struct GatPlan, graphautotune_b200/csrc/gat_plan.h)
 * into buf; *needed = sizeof(GatPlan). */
int gat_schedule_plan(const gat_schedule *s, void *buf, size_t cap,
                      size_t *needed);
void gat_schedule_free(gat_schedule *s);

/* -------------------------------------------------------------- config --
 * Runtime form of the compile-time Config (configs/config.hpp:10-14,
 * vertex_set_config.hpp:3-17, infra_config.hpp:3-5, engine_config.hpp:3-11).
 * The first eight fields keep the reference's names and meaning; the rest
 * are this engine's own knobs. */
typedef struct gat_config {
    int32_t set_search_type;       /* lists shorter than this are scanned
                                      linearly; 0 = always binary,
                                      INT32_MAX = always linear */
    int32_t set_intersection_type; /* 0 Parallel (tile-cooperative),
                                      1 Serial (one lane per unit) */
    int32_t vertex_store_type;     /* 0 Array (1 Bitmap is not implemented
                                      in the reference either) */
    int32_t graph_backend_type;    /* 0 InMemory */
    int32_t num_blocks;            /* CTAs; 0 = persistent grid sized from
                                      occupancy (SMs x resident CTAs) */
    int32_t threads_per_block;     /* 32..256 */
    int32_t threads_per_warp;      /* lanes per unit: 1,2,4,8,16,32 */
    int32_t max_regs;              /* accepted for compatibility; register
                                      use is fixed when the library is built */
    int32_t chunk;                 /* level-1 units per work-queue grab (per
                                      lane for two-level plans, whose lanes
                                      take units one each) */
    int32_t hub_bitmaps;           /* 1: intersect against the graph's hub
                                      bitmaps where cheaper; 0: never */
    int64_t memory_budget;         /* bytes of set scratch the executor may
                                      hold for the schedule-plan search;
                                      0 = 4 GiB */
    int32_t special_kernels;       /* 1: patterns with a dedicated kernel use
                                      it (exact 4-cycle, exact 4- to
                                      7-cliques) and plans use the
                                      lane-per-candidate last level; 2: the
                                      lane path but no dedicated kernel;
                                      0: the plan interpreter alone */
    int32_t reserved1;
    int64_t reserved[3];
} gat_config;

/* Defaults: the reference's generated default_config.hpp
 * (include/generated/default_config.hpp:5): set_search_type 64, Parallel,
 * Array, InMemory, 256 blocks, 128 threads, 1 thread per warp, 32 regs. */
void gat_config_default(gat_config *c);
/* This engine's tuned starting point (persistent grid, 32-lane tiles). */
void gat_config_engine_default(gat_config *c);
/* Parses either the designated-initializer text the tuner writes into
 * default_config.hpp (tuning/tuning/config/base.py:224-242, e.g.
 * "{.vertex_set_config = {.set_search_type = 64, ...}, ...}") or the flat
 * JSON value dict of config.json (tuning/tuning/role/driver.py:50-51, keys
 * like "engine_config.launch_config.num_blocks").  Unmentioned fields keep
 * their current values. */
int gat_config_parse(const char *text, gat_config *c);
/* Writes the designated-initializer form (the text the tuner would emit). */
int gat_config_format(const gat_config *c, char *buf, size_t cap);

/* --------------------------------------------------------------- graph --
 * Replaces Infra::GlobalMemoryGraph (infra/graph_backend.cuh:15-170).
 * Binary layout: int32 V, int64 E (directed entries), int64 offsets[V+1],
 * int32 neighbours[E]; text layout: "V E" then E lines "u v". */
int gat_graph_load(const char *path, int binary, gat_graph **out);
/* Copies caller CSR arrays.  Rows must be strictly increasing, ids in
 * [0, V), no self loops (checked, O(E)); the lists must also be symmetric,
 * which gat_graph_validate(g, 1) checks in O(E log d). */
int gat_graph_from_csr(int32_t V, int64_t E, const int64_t *offsets,
                       const int32_t *adj, gat_graph **out);
/* As gat_graph_from_csr, but the arrays go straight to the current device
 * (one host-to-device copy each on `stream`; from pinned host memory the
 * copy runs at full PCIe speed) and the row rules are checked there by a
 * kernel; the host view reads the neighbours back only when asked for
 * (gat_graph_csr, gat_graph_save, gat_graph_validate).  The caller's arrays
 * may be freed when the call returns.  Replaces GlobalMemoryGraph's load +
 * to_device (infra/graph_backend.cuh:102-118) for callers that hold the CSR
 * in host memory already. */
int gat_graph_from_csr_device(int32_t V, int64_t E, const int64_t *offsets,
                              const int32_t *adj, void *stream, gat_graph **out);
int gat_graph_validate(const gat_graph *g, int check_symmetry);
/* Seeded synthetic graphs (splitmix64 streams).  kind: 0 Erdos-Renyi
 * (p0 = n, p1 = avg degree), 1 R-MAT (p0 = scale, p1 = edge samples,
 * p2..p4 = a, b, c), 2 Barabasi-Albert (p0 = n, p1 = m). */
int gat_graph_generate(int kind, double p0, double p1, double p2, double p3,
                       double p4, uint64_t seed, gat_graph **out);
/* The same seeded graphs built on the current device: R-MAT edges are drawn
 * there (the same splitmix64 streams, so the graph is identical to
 * gat_graph_generate's), Erdos-Renyi and Barabasi-Albert edge lists are drawn
 * on the host; symmetrising, dropping self loops and duplicates and sorting
 * the rows run on the device, and the CSR is copied back for the host view.
 * The device copy stays resident (gat_graph_upload then only adds the
 * degree-ordered copy and hub bitmaps).  Replaces the reference's host-side
 * graph construction (infra/graph_backend.cuh:23-89) and
 * utils/graph_transform.cu:6-28 for synthetic inputs. */
int gat_graph_generate_device(int kind, double p0, double p1, double p2, double p3,
                              double p4, uint64_t seed, void *stream, gat_graph **out);
int gat_graph_save(const gat_graph *g, const char *path);
int gat_graph_info(const gat_graph *g, int32_t *V, int64_t *E,
                   int32_t *max_degree);
/* Host CSR view (valid until gat_graph_free). */
int gat_graph_csr(const gat_graph *g, const int64_t **offsets,
                  const int32_t **adj);
/* Copies the graph to the current device (GlobalMemoryGraph::to_device,
 * graph_backend.cuh:102-118; the device copy is owned and freed by the
 * handle).  flags: GAT_UPLOAD_DEGREE_ORDER also builds a copy relabelled by
 * decreasing degree, which exact-mode counts use (exact counts do not depend
 * on vertex ids; reference-compatible counts always use the ids as given). */
#define GAT_UPLOAD_DEGREE_ORDER 1
int gat_graph_upload(gat_graph *g, int flags, void *stream);
/* As gat_graph_upload, also building hub bitmaps: one V-bit row (bit x set
 * iff x is a neighbour) for every vertex of degree >= hub_min_degree, largest
 * degree first, as many as fit in hub_max_bytes (0 disables).
 * gat_graph_upload uses the defaults below.  With GAT_UPLOAD_DEGREE_ORDER,
 * the given-id copy's bitmaps (used only by reference-compatible counts) are
 * built on first use, with these parameters. */
#define GAT_HUB_MIN_DEGREE_DEFAULT 512
#define GAT_HUB_MAX_BYTES_DEFAULT (1LL << 30)
int gat_graph_upload_ex(gat_graph *g, int flags, int64_t hub_min_degree,
                        int64_t hub_max_bytes, void *stream);
/* Number of hub bitmaps on the given device copy (0: ids as given, whose
 * bitmaps this call builds if they are still pending; 1: degree-ordered). */
int gat_graph_hubs(const gat_graph *g, int ordered_copy, int32_t *nhubs);
/* Copies the degree-ordered device copy (uploaded with
 * GAT_UPLOAD_DEGREE_ORDER) into host buffers of V+1 offsets and E
 * neighbours.  Vertex r of that copy is the r-th vertex by decreasing degree,
 * ties by id; exact counts by root range (gat_executor_count_range) name
 * roots by these ids.  No reference counterpart: the reference counts on the
 * ids as loaded. */
int gat_graph_ordered_csr(const gat_graph *g, int64_t *offsets, int32_t *adj);
void gat_graph_free(gat_graph *g);

/* -------------------------------------------------------------- engine --
 * Replaces Engine::Executor<config>(set_size, device) and
 * long long Executor::perform_search(DeviceContext&)
 * (engine/engine.cuh:157-265). */
typedef struct gat_stats {
    double kernel_ms;        /* device time of the search launch(es) */
    double total_ms;         /* host wall time of the call */
    int64_t raw_sum;         /* signed engine total before the divisor */
    int64_t divisor;         /* embeddings per subgraph left by the plan */
    uint64_t tasks;          /* level-1 units in the work queue */
    uint64_t balg_bytes;     /* algorithmic bytes (when collected) */
    int32_t grid, block, tile, launches;
    int64_t scratch_bytes;
} gat_stats;

int gat_executor_create(const gat_config *c, gat_executor **out);
void gat_executor_free(gat_executor *e);
/* Counts `s` in `g` (uploaded, or uploaded on demand).  For GAT_MODE_EXACT
 * *count is the subgraph count; for GAT_MODE_REF_COMPAT it holds the
 * reference's signed long long result (two's complement).  stream may be
 * NULL (default stream).  The call returns after the count is on the host.
 * stats may be NULL. */
int gat_executor_count(gat_executor *e, gat_graph *g, const gat_schedule *s,
                       void *stream, uint64_t *count, gat_stats *stats);
/* As gat_executor_count, and also measures the algorithmic bytes of every
 * set operation (4(|A|+|B|) per intersection + 4|C| per stored output) with
 * an instrumented launch. */
int gat_executor_count_balg(gat_executor *e, gat_graph *g,
                            const gat_schedule *s, void *stream,
                            uint64_t *count, gat_stats *stats);
/* Counts only the units whose first vertex v0 lies in [root_begin,
 * root_end) (the reference's first-level chunking, engine.cuh:246-261, made
 * an API: the unit of sampling and of sharding across GPUs).  For exact
 * schedules on a degree-ordered upload the roots are relabelled ids.
 * *raw_sum receives the undivided signed total; the caller sums the shards
 * and divides by stats->divisor. */
int gat_executor_count_range(gat_executor *e, gat_graph *g,
                             const gat_schedule *s, void *stream,
                             int32_t root_begin, int32_t root_end,
                             int64_t *raw_sum, gat_stats *stats);
/* Counts shard `shard` of `num_shards` equal slices of the level-1 work
 * queue (balanced by units, not by vertices, so power-law rows spread
 * evenly).  One process per GPU calls it with its rank; the shards' raw sums
 * add up to the whole-graph raw sum (divide by stats->divisor). */
int gat_executor_count_shard(gat_executor *e, gat_graph *g,
                             const gat_schedule *s, void *stream,
                             int32_t shard, int32_t num_shards,
                             int64_t *raw_sum, gat_stats *stats);
/* As gat_executor_count_shard, with the algorithmic bytes of the slice's
 * set operations measured as in gat_executor_count_balg. */
int gat_executor_count_shard_balg(gat_executor *e, gat_graph *g,
                                  const gat_schedule *s, void *stream,
                                  int32_t shard, int32_t num_shards,
                                  int64_t *raw_sum, gat_stats *stats);
/* ---------------------------------------------------------------- batch --
 * No single reference counterpart: the reference runs one pm process per
 * (pattern, graph, config) (tuning/tuning/role/driver.py:88-132).  A batch
 * counts many (schedule, graph) jobs of uneven size in ONE persistent launch:
 * the jobs' level-1 work queues are concatenated (each rounded up to a whole
 * chunk) and drained by one atomic cursor, so small jobs do not leave the GPU
 * idle.  gat_batch_prepare fixes the launch shape from `c`, uploads graphs
 * that are not resident yet, builds the job table and, with use_cuda_graph,
 * captures memset + launch + result copy into a CUDA graph that
 * gat_batch_run replays.  Counts follow each schedule's mode. */
typedef struct gat_batch gat_batch;
int gat_batch_create(gat_batch **out);
int gat_batch_add(gat_batch *b, gat_graph *g, const gat_schedule *s,
                  int32_t *job_index);
/* As gat_batch_add, for one equal slice of the job's level-1 work queue
 * (the slicing of gat_executor_count_shard).  Its entry in gat_batch_counts
 * is the slice's undivided signed total.  Used to time launch shapes on a
 * sample of every job. */
int gat_batch_add_shard(gat_batch *b, gat_graph *g, const gat_schedule *s,
                        int32_t shard, int32_t num_shards, int32_t *job_index);
int gat_batch_prepare(gat_batch *b, const gat_config *c, int use_cuda_graph);
int gat_batch_run(gat_batch *b, gat_stats *stats);
int gat_batch_counts(const gat_batch *b, uint64_t *counts, size_t n);
int gat_batch_size(const gat_batch *b);
void gat_batch_free(gat_batch *b);

/* ------------------------------------------------------- cost model --
 * Replaces the tuner's XGBoost regressor (tuning/tuning/role/modeling.py:
 * 16-162) with a 3-layer FP32 perceptron (in -> 64 -> 64 -> 1, ReLU) whose
 * forward, backward and Adam kernels are this library's own.  Features and
 * targets are row-major float arrays on the host (n rows x in_features);
 * the model predicts whatever target it was trained on (log seconds in
 * graphautotune_b200.costmodel).  Parameters are one flat vector:
 * W1[in][64], b1[64], W2[64][64], b2[64], w3[64], b3. */
typedef struct gat_mlp gat_mlp;
int gat_mlp_create(int in_features, uint64_t seed, gat_mlp **out);
void gat_mlp_free(gat_mlp *net);
int gat_mlp_num_params(const gat_mlp *net);
int gat_mlp_get_params(const gat_mlp *net, float *out, int n);
int gat_mlp_set_params(gat_mlp *net, const float *in, int n);
int gat_mlp_predict(const gat_mlp *net, const float *X, int n, float *y);
/* Full-batch mean squared error and its gradient (no update). */
int gat_mlp_gradient(const gat_mlp *net, const float *X, const float *T, int n,
                     float *grad_out, float *loss);
/* Mini-batch Adam (beta1 0.9, beta2 0.999) over seeded shuffles. */
int gat_mlp_train(gat_mlp *net, const float *X, const float *T, int n, int epochs,
                  int batch, float lr, uint64_t seed, float *final_loss);
const char *gat_mlp_last_error(void);

/* ------------------------------------------------------ allocation-free --
 * No counterpart in the reference.  For callers that cannot allocate device
 * memory when they count: a host framework whose caching allocator already
 * owns the device's memory (a cudaMalloc next to it fails or fragments the
 * pool), a latency-critical stream that must not pick up the implicit device
 * synchronisation cudaMalloc/cudaFree bring, or a deployment whose device
 * memory is fixed before the first request.  The graph stays in the caller's
 * device memory (int64 offsets[V+1], int32 neighbours[E], sorted
 * deduplicated rows, ids as given); set scratch, counters and the plan live
 * in one static device array of GAT_NOALLOC_SCRATCH_BYTES that every device
 * loading this library holds until the process exits.  The grid is shrunk
 * until every resident tile's stored sets (stored prefixes x max_degree
 * ints) fit in the array; a schedule whose single CTA would not fit is
 * rejected with GAT_ERR_MEMORY.  Hub bitmaps are not used.
 * max_degree must be at least the graph's largest row length: it sizes each
 * tile's slots.  The kernel never writes past a slot; when a set would
 * exceed one (max_degree stated too small) it reports an internal error and
 * *d_count receives INT64_MIN.
 * The first call on each device looks up the array's device address
 * (cudaGetSymbolAddress), so make that first call before any stream capture
 * on the device.  Every call reuses the same array, so calls whose work
 * overlaps on the GPU (other streams, other host threads) race and return
 * wrong counts: serialise them.  *d_count (device memory, written in order on
 * `stream`) receives the count gat_executor_count would return, or
 * INT64_MIN if the kernel reported an internal error.  The plan travels in
 * a kernel's parameter block, so the schedule may be freed once the call
 * returns.  Nothing in this call
 * allocates (no cudaMalloc/cudaFree, no allocating library routine). */
#define GAT_NOALLOC_SCRATCH_BYTES (64u << 20)
int gat_count_noalloc(const int64_t *d_offsets, const int32_t *d_adj, int32_t V,
                      int64_t E, int32_t max_degree, const gat_schedule *s,
                      const gat_config *c, int64_t *d_count, void *stream);
/* One-shot convenience: executor from config (NULL = engine default). */
int gat_count(gat_graph *g, const gat_schedule *s, const gat_config *c,
              uint64_t *count, gat_stats *stats);

#ifdef __cplusplus
}
#endif
#endif
