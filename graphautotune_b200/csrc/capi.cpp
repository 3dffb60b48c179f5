// C ABI of libgat (include/gat.h).
#include <cuda_runtime.h>

#include <algorithm>
#include <cctype>
#include <chrono>
#include <climits>
#include <cstring>
#include <memory>
#include <string>

#include "../../include/gat.h"
#include "engine.hpp"
#include "gat_internal.hpp"
#include "graph.hpp"

using namespace gat;

namespace {

thread_local std::string g_last_error;

int fail(int code, const std::string &msg) {
    g_last_error = msg;
    return code;
}

int cuda_fail(cudaError_t e, const char *what) {
    return fail(GAT_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

int copy_out(const std::string &s, char *buf, size_t cap, size_t *needed) {
    if (needed) *needed = s.size() + 1;
    if (!buf) return GAT_OK;
    if (cap < s.size() + 1) return fail(GAT_ERR_ARGUMENT, "buffer too small");
    std::memcpy(buf, s.c_str(), s.size() + 1);
    return GAT_OK;
}

}  // namespace

struct gat_pattern {
    Pattern p;
};

struct gat_schedule {
    int mode = 0;
    bool trivial = false;  // n <= 2: counted on the host
    Pattern pattern;
    RefSchedule ref;
    PlanInfo plan;
    std::string json;
};

struct DevCopy {
    int64_t *off = nullptr;
    int32_t *adj = nullptr;
    int64_t *lo_off = nullptr;
    int64_t lo_total = 0;
    int32_t max_degree = 0;
    int32_t max_lower = 0;  // longest lower list (entries below the row's vertex)
    bool ready = false;
    std::vector<int64_t> lo_host;   // host copy of lo_off
    std::vector<int64_t> off_host;  // host copy of off
    int32_t *hub_slot = nullptr;    // per vertex: bitmap row or -1
    int32_t *hubs = nullptr;        // row -> vertex
    uint32_t *bitmaps = nullptr;
    int32_t nhubs = 0;
    int64_t bitmap_words = 0;
    void release() {
        cudaFree(off);
        cudaFree(adj);
        cudaFree(lo_off);
        cudaFree(hub_slot);
        cudaFree(hubs);
        cudaFree(bitmaps);
        hub_slot = nullptr;
        hubs = nullptr;
        bitmaps = nullptr;
        nhubs = 0;
        bitmap_words = 0;
        off = nullptr;
        adj = nullptr;
        lo_off = nullptr;
        lo_total = 0;
        max_degree = 0;
        max_lower = 0;
        ready = false;
        lo_host.clear();
        off_host.clear();
    }
};

struct gat_graph {
    HostGraph host;
    DevCopy dev;          // ids as given
    DevCopy dev_ordered;  // relabelled by decreasing degree
    int device = -1;
    // Hub bitmap parameters of the last upload.  With the degree-ordered
    // copy present, the given-id copy's bitmaps (used only by
    // reference-compatible counts) are built on first use.
    int64_t hub_min_degree = GAT_HUB_MIN_DEGREE_DEFAULT;
    int64_t hub_max_bytes = GAT_HUB_MAX_BYTES_DEFAULT;
    bool dev_hubs_pending = false;
    // Built on the device (gat_graph_generate_device,
    // gat_graph_from_csr_device): host.off is filled, host.adj is read back
    // from the resident copy on first use.
    bool host_adj_pending = false;
    ~gat_graph() {
        dev.release();
        dev_ordered.release();
    }
};

struct gat_executor {
    gat_config cfg{};
    int device = 0;
    int sms = 0;
    int32_t *scratch = nullptr;
    size_t scratch_bytes = 0;
    bool scratch_clean = false;  // all-zero (the 4-cycle kernel's invariant)
    DevCounters *ctr = nullptr;
    DevCounters *host_ctr = nullptr;  // pinned
    GatPlan *d_plan = nullptr;
    GatPlan *h_plan = nullptr;  // pinned
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    ~gat_executor() {
        cudaFree(scratch);
        cudaFree(ctr);
        cudaFree(d_plan);
        cudaFreeHost(host_ctr);
        cudaFreeHost(h_plan);
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
    }
};

namespace {
// Reads host.adj back from the resident device copy when the graph was built
// on the device and the host neighbours were not needed until now.
int ensure_host_adj(gat_graph *g) {
    if (!g->host_adj_pending) return GAT_OK;
    int cur = -1;
    cudaError_t e = cudaGetDevice(&cur);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
    if (cur != g->device || !g->dev.ready)
        return fail(GAT_ERR_STATE, "graph built on another device: make it current to read it");
    std::vector<int32_t> adj(size_t(g->host.E));
    if (g->host.E > 0 &&
        (e = cudaMemcpy(adj.data(), g->dev.adj, sizeof(int32_t) * size_t(g->host.E),
                        cudaMemcpyDeviceToHost)) != cudaSuccess)
        return cuda_fail(e, "graph read-back");
    g->host.adj.swap(adj);
    g->host_adj_pending = false;
    return GAT_OK;
}
}  // namespace

extern "C" {

const char *gat_last_error(void) { return g_last_error.c_str(); }
const char *gat_version(void) { return "libgat 0.1 (sm_100a)"; }

// ------------------------------------------------------------ pattern

int gat_pattern_from_adj(const char *adj, gat_pattern **out) {
    if (!adj || !out) return fail(GAT_ERR_ARGUMENT, "null argument");
    *out = nullptr;
    Pattern p;
    if (!Pattern::parse(adj, p))
        return fail(GAT_ERR_PATTERN,
                    "pattern must be n*n characters '0'/'1' with 1 <= n <= 10");
    *out = new gat_pattern{p};
    return GAT_OK;
}

int gat_pattern_vertices(const gat_pattern *p) { return p ? p->p.n : 0; }

int gat_pattern_automorphisms(const gat_pattern *p, int64_t *out) {
    if (!p || !out) return fail(GAT_ERR_ARGUMENT, "null argument");
    *out = (int64_t)automorphisms(p->p).size();
    return GAT_OK;
}

int gat_pattern_adjacency(const gat_pattern *p, char *buf, size_t cap) {
    if (!p) return fail(GAT_ERR_ARGUMENT, "null argument");
    return copy_out(p->p.adjacency(), buf, cap, nullptr);
}

void gat_pattern_free(gat_pattern *p) { delete p; }

int gat_enumerate_patterns(int n, char *buf, size_t cap, size_t *needed) {
    if (n < 1 || n > 6) return fail(GAT_ERR_ARGUMENT, "n must be in [1, 6]");
    std::string s;
    for (auto &x : enumerate_connected_patterns(n)) {
        if (!s.empty()) s += '\n';
        s += x;
    }
    return copy_out(s, buf, cap, needed);
}

// ----------------------------------------------------------- schedule

namespace {
GraphStats stats_of(const gat_graph *g) {
    GraphStats gs;
    if (g && g->host.V > 0) {
        gs.v = g->host.V;
        gs.e = g->host.E / 2;
        gs.tri = std::max<int64_t>(1, gs.e / 10);
    }
    return gs;
}
}  // namespace

int gat_schedule_variants(const gat_pattern *p, int mode, const gat_graph *stats_graph,
                          int32_t *count) {
    if (!p || !count) return fail(GAT_ERR_ARGUMENT, "null argument");
    if (mode != GAT_MODE_EXACT || p->p.n <= 2) {
        *count = 1;
        return GAT_OK;
    }
    PlanInfo pi;
    std::string err;
    int n = 0;
    if (!plan_exact(p->p, stats_of(stats_graph), pi, &err, 0, &n))
        return fail(GAT_ERR_PATTERN, err);
    *count = n;
    return GAT_OK;
}

int gat_schedule_build(const gat_pattern *p, int mode,
                       const gat_graph *stats_graph, gat_schedule **out) {
    return gat_schedule_build_variant(p, mode, stats_graph, 0, out);
}

int gat_schedule_build_variant(const gat_pattern *p, int mode, const gat_graph *stats_graph,
                               int32_t variant, gat_schedule **out) {
    if (!p || !out) return fail(GAT_ERR_ARGUMENT, "null argument");
    *out = nullptr;
    if (variant < 0 || (variant > 0 && (mode != GAT_MODE_EXACT || p->p.n <= 2)))
        return fail(GAT_ERR_ARGUMENT, "schedule variant out of range");
    if (mode != GAT_MODE_EXACT && mode != GAT_MODE_REF_COMPAT)
        return fail(GAT_ERR_ARGUMENT, "unknown mode");
    auto s = std::make_unique<gat_schedule>();
    s->mode = mode;
    s->pattern = p->p;
    std::string err;
    if (mode == GAT_MODE_REF_COMPAT) {
        if (!build_ref_schedule(p->p, s->ref, &err)) return fail(GAT_ERR_PATTERN, err);
        s->json = ref_schedule_json(s->ref);
        if (p->p.n <= 2) {
            s->trivial = true;
        } else if (!plan_from_ref(s->ref, s->plan, &err)) {
            // Keep the schedule (it can be dumped) but mark it uncountable.
            s->plan = PlanInfo{};
            s->plan.summary = err;
        }
    } else {
        if (p->p.n <= 2) {
            if (!pattern_connected(p->p)) return fail(GAT_ERR_PATTERN, "pattern is not connected");
            s->trivial = true;
            s->json = "{\"mode\":\"exact\",\"trivial\":true}";
        } else {
            if (!plan_exact(p->p, stats_of(stats_graph), s->plan, &err, variant)) {
                if (variant > 0 && err == "no such schedule variant")
                    return fail(GAT_ERR_ARGUMENT, "schedule variant out of range");
                return fail(GAT_ERR_PATTERN, err);
            }
            std::string perm, r;
            for (size_t i = 0; i < s->plan.perm.size(); i++)
                perm += (i ? "," : "") + std::to_string(s->plan.perm[i]);
            for (size_t i = 0; i < s->plan.restrictions.size(); i++)
                r += std::string(i ? "," : "") + "[" +
                     std::to_string(s->plan.restrictions[i].first) + "," +
                     std::to_string(s->plan.restrictions[i].second) + "]";
            s->json = "{\"mode\":\"exact\",\"pattern\":\"" + p->p.adjacency() +
                      "\",\"perm\":[" + perm + "],\"restrictions\":[" + r +
                      "],\"basic_vertexes\":" + std::to_string(s->plan.plan.basic) +
                      ",\"divisor\":" + std::to_string(s->plan.plan.divisor) +
                      ",\"aut\":" + std::to_string(s->plan.aut) + "}";
        }
    }
    *out = s.release();
    return GAT_OK;
}

int gat_schedule_mode(const gat_schedule *s) { return s ? s->mode : -1; }

int gat_schedule_dump(const gat_schedule *s, char *buf, size_t cap,
                      size_t *needed) {
    if (!s) return fail(GAT_ERR_ARGUMENT, "null argument");
    return copy_out(s->json, buf, cap, needed);
}

int gat_schedule_plan(const gat_schedule *s, void *buf, size_t cap,
                      size_t *needed) {
    if (!s) return fail(GAT_ERR_ARGUMENT, "null argument");
    if (needed) *needed = sizeof(GatPlan);
    if (s->trivial || s->plan.plan.n == 0)
        return fail(GAT_ERR_UNDEFINED, s->trivial ? "trivial schedule has no plan"
                                                  : s->plan.summary);
    if (!buf) return GAT_OK;
    if (cap < sizeof(GatPlan)) return fail(GAT_ERR_ARGUMENT, "buffer too small");
    std::memcpy(buf, &s->plan.plan, sizeof(GatPlan));
    return GAT_OK;
}

void gat_schedule_free(gat_schedule *s) { delete s; }

// ------------------------------------------------------------- config

void gat_config_default(gat_config *c) {
    if (!c) return;
    std::memset(c, 0, sizeof(*c));
    c->set_search_type = 64;
    c->set_intersection_type = 0;
    c->vertex_store_type = 0;
    c->graph_backend_type = 0;
    c->num_blocks = 256;
    c->threads_per_block = 128;
    c->threads_per_warp = 1;
    c->max_regs = 32;
    c->chunk = 16;
    c->hub_bitmaps = 1;
    c->special_kernels = 1;
    c->memory_budget = 0;
}

void gat_config_engine_default(gat_config *c) {
    if (!c) return;
    gat_config_default(c);
    c->set_search_type = 0;
    c->num_blocks = 0;
    c->threads_per_block = 256;
    c->threads_per_warp = 32;
    c->max_regs = 64;
    c->chunk = 8;
}

namespace {
bool set_field(gat_config *c, const std::string &key, const std::string &val) {
    auto ident = [&](int64_t &out) {
        if (val == "Parallel" || val == "Array" || val == "InMemory") {
            out = 0;
            return true;
        }
        if (val == "Serial" || val == "Bitmap") {
            out = 1;
            return true;
        }
        if (val == "INT_MAX") {
            out = INT32_MAX;
            return true;
        }
        if (val.empty()) return false;
        char *end = nullptr;
        long long x = std::strtoll(val.c_str(), &end, 10);
        if (*end != '\0') return false;
        out = x;
        return true;
    };
    std::string k = key.substr(key.rfind('.') + 1);
    int64_t x = 0;
    if (!ident(x)) return false;
    auto i32 = [&](int32_t &f) {
        if (x < INT32_MIN || x > INT32_MAX) return false;
        f = (int32_t)x;
        return true;
    };
    if (k == "set_search_type") return i32(c->set_search_type);
    if (k == "set_intersection_type") return i32(c->set_intersection_type);
    if (k == "vertex_store_type") return i32(c->vertex_store_type);
    if (k == "graph_backend_type") return i32(c->graph_backend_type);
    if (k == "num_blocks") return i32(c->num_blocks);
    if (k == "threads_per_block") return i32(c->threads_per_block);
    if (k == "threads_per_warp") return i32(c->threads_per_warp);
    if (k == "max_regs") return i32(c->max_regs);
    if (k == "chunk") return i32(c->chunk);
    if (k == "hub_bitmaps") return i32(c->hub_bitmaps);
    if (k == "special_kernels") return i32(c->special_kernels);
    if (k == "memory_budget") {
        c->memory_budget = x;
        return true;
    }
    return true;  // unknown keys are ignored, like the C++ designated
                  // initializer ignores nothing but the tuner may add fields
}
}  // namespace

int gat_config_parse(const char *text, gat_config *c) {
    if (!text || !c) return fail(GAT_ERR_ARGUMENT, "null argument");
    std::string s(text);
    size_t i = 0;
    auto is_id = [](char ch) {
        return std::isalnum((unsigned char)ch) || ch == '_' || ch == '.';
    };
    int found = 0;
    while (i < s.size()) {
        std::string key;
        if (s[i] == '.' && i + 1 < s.size() &&
            (std::isalpha((unsigned char)s[i + 1]) || s[i + 1] == '_')) {
            size_t j = i + 1;
            while (j < s.size() && (std::isalnum((unsigned char)s[j]) || s[j] == '_')) j++;
            key = s.substr(i + 1, j - i - 1);
            i = j;
            while (i < s.size() && std::isspace((unsigned char)s[i])) i++;
            if (i >= s.size() || s[i] != '=') continue;
            i++;
        } else if (s[i] == '"') {
            size_t j = s.find('"', i + 1);
            if (j == std::string::npos) break;
            key = s.substr(i + 1, j - i - 1);
            i = j + 1;
            while (i < s.size() && std::isspace((unsigned char)s[i])) i++;
            if (i >= s.size() || s[i] != ':') continue;
            i++;
        } else {
            i++;
            continue;
        }
        while (i < s.size() && std::isspace((unsigned char)s[i])) i++;
        if (i < s.size() && s[i] == '{') continue;  // nested struct
        std::string val;
        if (i < s.size() && s[i] == '"') {
            size_t j = s.find('"', i + 1);
            if (j == std::string::npos) break;
            val = s.substr(i + 1, j - i - 1);
            i = j + 1;
        } else {
            size_t j = i;
            while (j < s.size() && (is_id(s[j]) || s[j] == '-')) j++;
            val = s.substr(i, j - i);
            i = j;
        }
        if (!set_field(c, key, val))
            return fail(GAT_ERR_CONFIG, "bad value '" + val + "' for " + key);
        found++;
    }
    if (found == 0) return fail(GAT_ERR_CONFIG, "no configuration fields found");
    return GAT_OK;
}

int gat_config_format(const gat_config *c, char *buf, size_t cap) {
    if (!c) return fail(GAT_ERR_ARGUMENT, "null argument");
    auto st = [](int v) {
        return v == INT32_MAX ? std::string("2147483647") : std::to_string(v);
    };
    std::string s = "{.vertex_set_config = {.set_search_type = " +
                     st(c->set_search_type) + ", .set_intersection_type = " +
                     (c->set_intersection_type ? "Serial" : "Parallel") +
                     ", .vertex_store_type = " +
                     (c->vertex_store_type ? "Bitmap" : "Array") +
                     "}, .infra_config = {.graph_backend_type = InMemory}, "
                     ".engine_config = {.launch_config = {.num_blocks = " +
                     std::to_string(c->num_blocks) + ", .threads_per_block = " +
                     std::to_string(c->threads_per_block) +
                     ", .threads_per_warp = " + std::to_string(c->threads_per_warp) +
                     ", .max_regs = " + std::to_string(c->max_regs) + "}}}";
    return copy_out(s, buf, cap, nullptr);
}

// -------------------------------------------------------------- graph

int gat_graph_load(const char *path, int binary, gat_graph **out) {
    if (!path || !out) return fail(GAT_ERR_ARGUMENT, "null argument");
    *out = nullptr;
    auto g = std::make_unique<gat_graph>();
    std::string err;
    bool ok = binary ? load_binary(path, g->host, &err) : load_text(path, g->host, &err);
    if (!ok) return fail(GAT_ERR_IO, err);
    if (!validate(g->host, false, &err)) return fail(GAT_ERR_IO, "invalid CSR: " + err);
    *out = g.release();
    return GAT_OK;
}

int gat_graph_from_csr(int32_t V, int64_t E, const int64_t *offsets,
                       const int32_t *adj, gat_graph **out) {
    if (!out || V < 0 || E < 0 || !offsets || (E > 0 && !adj))
        return fail(GAT_ERR_ARGUMENT, "bad CSR arguments");
    *out = nullptr;
    auto g = std::make_unique<gat_graph>();
    g->host.V = V;
    g->host.E = E;
    g->host.off.assign(offsets, offsets + V + 1);
    g->host.adj.assign(adj, adj + E);
    std::string err;
    if (!validate(g->host, false, &err)) return fail(GAT_ERR_ARGUMENT, "invalid CSR: " + err);
    *out = g.release();
    return GAT_OK;
}

int gat_graph_validate(const gat_graph *g, int check_symmetry) {
    if (!g) return fail(GAT_ERR_ARGUMENT, "null argument");
    int rc = ensure_host_adj(const_cast<gat_graph *>(g));
    if (rc != GAT_OK) return rc;
    std::string err;
    if (!validate(g->host, check_symmetry != 0, &err))
        return fail(GAT_ERR_ARGUMENT, "invalid CSR: " + err);
    return GAT_OK;
}

int gat_graph_generate(int kind, double p0, double p1, double p2, double p3,
                       double p4, uint64_t seed, gat_graph **out) {
    if (!out) return fail(GAT_ERR_ARGUMENT, "null argument");
    *out = nullptr;
    auto g = std::make_unique<gat_graph>();
    if (kind == 0) {
        if (p0 < 0 || p0 > INT32_MAX || p1 < 0) return fail(GAT_ERR_ARGUMENT, "bad ER parameters");
        gen_erdos_renyi((int32_t)p0, p1, seed, g->host);
    } else if (kind == 1) {
        if (p0 < 1 || p0 > 30 || p1 < 0 || p2 < 0 || p3 < 0 || p4 < 0 || p2 + p3 + p4 > 1)
            return fail(GAT_ERR_ARGUMENT, "bad R-MAT parameters");
        gen_rmat((int)p0, (int64_t)p1, p2, p3, p4, seed, g->host);
    } else if (kind == 2) {
        if (p0 < 0 || p0 > INT32_MAX || p1 < 1) return fail(GAT_ERR_ARGUMENT, "bad BA parameters");
        gen_barabasi_albert((int32_t)p0, (int32_t)p1, seed, g->host);
    } else {
        return fail(GAT_ERR_ARGUMENT, "unknown generator");
    }
    *out = g.release();
    return GAT_OK;
}

int gat_graph_save(const gat_graph *g, const char *path) {
    if (!g || !path) return fail(GAT_ERR_ARGUMENT, "null argument");
    int rc = ensure_host_adj(const_cast<gat_graph *>(g));
    if (rc != GAT_OK) return rc;
    std::string err;
    if (!save_binary(path, g->host, &err)) return fail(GAT_ERR_IO, err);
    return GAT_OK;
}

int gat_graph_info(const gat_graph *g, int32_t *V, int64_t *E, int32_t *max_degree) {
    if (!g) return fail(GAT_ERR_ARGUMENT, "null argument");
    if (V) *V = g->host.V;
    if (E) *E = g->host.E;
    if (max_degree) *max_degree = g->host.max_degree();
    return GAT_OK;
}

int gat_graph_csr(const gat_graph *g, const int64_t **offsets, const int32_t **adj) {
    if (!g || !offsets || !adj) return fail(GAT_ERR_ARGUMENT, "null argument");
    int rc = ensure_host_adj(const_cast<gat_graph *>(g));
    if (rc != GAT_OK) return rc;
    *offsets = g->host.off.data();
    *adj = g->host.adj.data();
    return GAT_OK;
}

namespace {
// Device rows are allocated 4 ints longer than the edge list: kernels that
// read aligned 16-byte groups (cliques.cu) may touch up to 3 entries past
// the last row.
constexpr int64_t kAdjPadInts = 4;
int64_t adj_alloc_ints(int64_t E) { return E + kAdjPadInts; }

// Completes a device copy whose off and adj are in place: lo_off is derived
// on the device, and both offset arrays are kept on the host too (range and
// shard arithmetic reads them).  `off_known` is the host's copy of off when
// there is one; otherwise off is read back.
int finish_copy(DevCopy &d, int32_t V, int32_t max_degree, const std::vector<int64_t> *off_known,
                cudaStream_t st) {
    cudaError_t e;
    if ((e = cudaMalloc(&d.lo_off, sizeof(int64_t) * (size_t(V) + 1))) != cudaSuccess) {
        d.release();
        return fail(GAT_ERR_MEMORY, std::string("device graph allocation: ") + cudaGetErrorString(e));
    }
    d.lo_host.resize(size_t(V) + 1);
    if (off_known)
        d.off_host = *off_known;
    else
        d.off_host.resize(size_t(V) + 1);
    if ((e = lower_offsets_device(d.off, d.adj, V, d.lo_off, st)) != cudaSuccess ||
        (e = cudaMemcpyAsync(d.lo_host.data(), d.lo_off, sizeof(int64_t) * (size_t(V) + 1),
                             cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
        (!off_known &&
         (e = cudaMemcpyAsync(d.off_host.data(), d.off, sizeof(int64_t) * (size_t(V) + 1),
                              cudaMemcpyDeviceToHost, st)) != cudaSuccess) ||
        (e = cudaStreamSynchronize(st)) != cudaSuccess) {
        d.release();
        return cuda_fail(e, "graph upload");
    }
    d.lo_total = d.lo_host[size_t(V)];
    d.max_degree = max_degree;
    int64_t ml = 0;
    for (size_t v = 0; v < size_t(V); v++) ml = std::max(ml, d.lo_host[v + 1] - d.lo_host[v]);
    d.max_lower = (int32_t)ml;
    d.ready = true;
    return GAT_OK;
}

int upload_copy(const HostGraph &h, DevCopy &d, cudaStream_t st) {
    d.release();
    cudaError_t e;
    if ((e = cudaMalloc(&d.off, sizeof(int64_t) * (h.V + 1))) != cudaSuccess ||
        (e = cudaMalloc(&d.adj, sizeof(int32_t) * adj_alloc_ints(h.E))) != cudaSuccess) {
        d.release();
        return fail(GAT_ERR_MEMORY, std::string("device graph allocation: ") + cudaGetErrorString(e));
    }
    if ((e = cudaMemcpyAsync(d.off, h.off.data(), sizeof(int64_t) * (h.V + 1),
                             cudaMemcpyHostToDevice, st)) != cudaSuccess ||
        (h.E > 0 && (e = cudaMemcpyAsync(d.adj, h.adj.data(), sizeof(int32_t) * h.E,
                                         cudaMemcpyHostToDevice, st)) != cudaSuccess)) {
        d.release();
        return cuda_fail(e, "graph upload");
    }
    return finish_copy(d, h.V, h.max_degree(), &h.off, st);
}

// The degree-ordered copy, derived on the device from the resident copy
// `src` of h (graphs whose edge count CUB's segmented sort cannot index are
// relabelled on the host and uploaded instead).
int derive_ordered_copy(const HostGraph &h, const DevCopy &src, DevCopy &d, cudaStream_t st) {
    if (!relabel_fits_device(h.V, h.E)) {
        HostGraph r;
        relabel_by_degree(h, r, nullptr);
        return upload_copy(r, d, st);
    }
    d.release();
    cudaError_t e;
    if ((e = cudaMalloc(&d.off, sizeof(int64_t) * (h.V + 1))) != cudaSuccess ||
        (e = cudaMalloc(&d.adj, sizeof(int32_t) * adj_alloc_ints(h.E))) != cudaSuccess) {
        d.release();
        return fail(GAT_ERR_MEMORY, std::string("device graph allocation: ") + cudaGetErrorString(e));
    }
    const int32_t md = h.max_degree();
    if ((e = relabel_by_degree_device(src.off, src.adj, h.V, h.E, md, d.off, d.adj, st)) !=
        cudaSuccess) {
        d.release();
        return cuda_fail(e, "degree relabel");
    }
    return finish_copy(d, h.V, md, nullptr, st);
}

// Hub bitmaps for the vertices of degree >= min_degree, largest degree first,
// as many as fit in max_bytes.
void release_hubs(DevCopy &d) {
    cudaFree(d.hub_slot);
    cudaFree(d.hubs);
    cudaFree(d.bitmaps);
    d.hub_slot = nullptr;
    d.hubs = nullptr;
    d.bitmaps = nullptr;
    d.nhubs = 0;
    d.bitmap_words = 0;
}

int upload_hubs(DevCopy &d, int32_t V, int64_t min_degree, int64_t max_bytes,
                cudaStream_t st) {
    if (min_degree <= 0 || max_bytes <= 0 || V == 0) return GAT_OK;
    const std::vector<int64_t> &off = d.off_host;
    auto degree = [&](int32_t v) { return off[size_t(v) + 1] - off[size_t(v)]; };
    const int64_t words = (int64_t(V) + 31) / 32;
    std::vector<int32_t> cand;
    for (int32_t v = 0; v < V; v++)
        if (degree(v) >= min_degree) cand.push_back(v);
    std::stable_sort(cand.begin(), cand.end(),
                     [&](int32_t x, int32_t y) { return degree(x) > degree(y); });
    const int64_t fit = max_bytes / (words * 4);
    if ((int64_t)cand.size() > fit) cand.resize(size_t(fit));
    if (cand.empty()) return GAT_OK;
    std::vector<int32_t> slot(size_t(V), -1);
    for (size_t i = 0; i < cand.size(); i++) slot[cand[i]] = (int32_t)i;
    cudaError_t e;
    const size_t bm_bytes = size_t(cand.size()) * size_t(words) * 4;
    if ((e = cudaMalloc(&d.hub_slot, sizeof(int32_t) * V)) != cudaSuccess ||
        (e = cudaMalloc(&d.hubs, sizeof(int32_t) * cand.size())) != cudaSuccess ||
        (e = cudaMalloc(&d.bitmaps, bm_bytes)) != cudaSuccess)
        return fail(GAT_ERR_MEMORY, std::string("hub bitmap allocation: ") + cudaGetErrorString(e));
    if ((e = cudaMemcpyAsync(d.hub_slot, slot.data(), sizeof(int32_t) * V,
                             cudaMemcpyHostToDevice, st)) != cudaSuccess ||
        (e = cudaMemcpyAsync(d.hubs, cand.data(), sizeof(int32_t) * cand.size(),
                             cudaMemcpyHostToDevice, st)) != cudaSuccess ||
        (e = cudaMemsetAsync(d.bitmaps, 0, bm_bytes, st)) != cudaSuccess ||
        (e = build_hub_bitmaps(d.off, d.adj, d.hubs, (int32_t)cand.size(), words, d.bitmaps,
                               st)) != cudaSuccess ||
        (e = cudaStreamSynchronize(st)) != cudaSuccess)
        return cuda_fail(e, "hub bitmaps");
    d.nhubs = (int32_t)cand.size();
    d.bitmap_words = words;
    return GAT_OK;
}

// Builds the given-id copy's hub bitmaps if the last upload deferred them.
int ensure_dev_hubs(gat_graph *g, cudaStream_t st) {
    if (!g->dev_hubs_pending || !g->dev.ready) return GAT_OK;
    g->dev_hubs_pending = false;
    return upload_hubs(g->dev, g->host.V, g->hub_min_degree, g->hub_max_bytes, st);
}
}  // namespace

int gat_graph_generate_device(int kind, double p0, double p1, double p2, double p3, double p4,
                              uint64_t seed, void *stream, gat_graph **out) {
    if (!out) return fail(GAT_ERR_ARGUMENT, "null argument");
    *out = nullptr;
    cudaStream_t st = (cudaStream_t)stream;
    auto g = std::make_unique<gat_graph>();
    DevCopy &d = g->dev;
    int32_t V = 0;
    int64_t E = 0;
    cudaError_t e = cudaSuccess;
    std::vector<std::pair<int32_t, int32_t>> edges;
    if (kind == 1) {
        if (p0 < 1 || p0 > 30 || p1 < 0 || p2 < 0 || p3 < 0 || p4 < 0 || p2 + p3 + p4 > 1)
            return fail(GAT_ERR_ARGUMENT, "bad R-MAT parameters");
        V = int32_t(1) << (int)p0;
    } else if (kind == 0) {
        if (p0 < 0 || p0 > INT32_MAX || p1 < 0) return fail(GAT_ERR_ARGUMENT, "bad ER parameters");
        V = (int32_t)p0;
        gen_erdos_renyi_edges(V, p1, seed, edges);
    } else if (kind == 2) {
        if (p0 < 0 || p0 > INT32_MAX || p1 < 1) return fail(GAT_ERR_ARGUMENT, "bad BA parameters");
        V = (int32_t)p0;
        gen_barabasi_albert_edges(V, (int32_t)p1, seed, edges);
    } else {
        return fail(GAT_ERR_ARGUMENT, "unknown generator");
    }
    if ((e = cudaMalloc(&d.off, sizeof(int64_t) * (size_t(V) + 1))) != cudaSuccess) {
        d.release();
        return fail(GAT_ERR_MEMORY, std::string("device graph allocation: ") + cudaGetErrorString(e));
    }
    if (kind == 1) {
        e = rmat_csr_device((int)p0, (int64_t)p1, p2, p3, p4, seed, d.off, &d.adj,
                            kAdjPadInts, &E, st);
    } else {
        int32_t *pairs = nullptr;
        const size_t bytes = sizeof(int32_t) * 2 * std::max<size_t>(edges.size(), 1);
        if ((e = cudaMalloc(&pairs, bytes)) == cudaSuccess &&
            (edges.empty() ||
             (e = cudaMemcpyAsync(pairs, edges.data(), sizeof(int32_t) * 2 * edges.size(),
                                  cudaMemcpyHostToDevice, st)) == cudaSuccess))
            e = pairs_csr_device(pairs, (int64_t)edges.size(), V, d.off, &d.adj,
                                 kAdjPadInts, &E, st);
        const cudaError_t f = cudaStreamSynchronize(st);
        if (e == cudaSuccess) e = f;
        cudaFree(pairs);
    }
    if (e != cudaSuccess) {
        d.release();
        return cuda_fail(e, "device graph build");
    }
    HostGraph &h = g->host;
    h.V = V;
    h.E = E;
    h.off.resize(size_t(V) + 1);
    if ((e = cudaMemcpyAsync(h.off.data(), d.off, sizeof(int64_t) * (size_t(V) + 1),
                             cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
        (e = cudaStreamSynchronize(st)) != cudaSuccess) {
        d.release();
        return cuda_fail(e, "device graph read-back");
    }
    int rc = finish_copy(d, V, h.max_degree(), &h.off, st);
    if (rc != GAT_OK) return rc;
    int dev = 0;
    if ((e = cudaGetDevice(&dev)) != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
    g->device = dev;
    g->host_adj_pending = true;
    *out = g.release();
    return GAT_OK;
}

int gat_graph_from_csr_device(int32_t V, int64_t E, const int64_t *offsets,
                              const int32_t *adj, void *stream, gat_graph **out) {
    if (!out || V < 0 || E < 0 || !offsets || (E > 0 && !adj))
        return fail(GAT_ERR_ARGUMENT, "bad CSR arguments");
    *out = nullptr;
    cudaStream_t st = (cudaStream_t)stream;
    auto g = std::make_unique<gat_graph>();
    DevCopy &d = g->dev;
    unsigned long long *flag = nullptr;
    cudaError_t e;
    if ((e = cudaMalloc(&d.off, sizeof(int64_t) * (size_t(V) + 1))) != cudaSuccess ||
        (e = cudaMalloc(&d.adj, sizeof(int32_t) * adj_alloc_ints(E))) != cudaSuccess ||
        (e = cudaMalloc(&flag, sizeof(unsigned long long))) != cudaSuccess) {
        d.release();
        cudaFree(flag);
        return fail(GAT_ERR_MEMORY, std::string("device graph allocation: ") + cudaGetErrorString(e));
    }
    HostGraph &h = g->host;
    h.V = V;
    h.E = E;
    h.off.assign(offsets, offsets + size_t(V) + 1);
    unsigned long long bad = ~0ull;
    if ((e = cudaMemcpyAsync(d.off, offsets, sizeof(int64_t) * (size_t(V) + 1),
                             cudaMemcpyHostToDevice, st)) != cudaSuccess ||
        (E > 0 && (e = cudaMemcpyAsync(d.adj, adj, sizeof(int32_t) * size_t(E),
                                       cudaMemcpyHostToDevice, st)) != cudaSuccess) ||
        (e = csr_check_device(d.off, d.adj, V, E, flag, st)) != cudaSuccess ||
        (e = cudaMemcpyAsync(&bad, flag, sizeof(bad), cudaMemcpyDeviceToHost, st)) !=
            cudaSuccess ||
        (e = cudaStreamSynchronize(st)) != cudaSuccess) {
        d.release();
        cudaFree(flag);
        return cuda_fail(e, "graph upload");
    }
    cudaFree(flag);
    if (V > 0 && (h.off[0] != 0 || h.off[size_t(V)] != E))
        bad = std::min<unsigned long long>(bad, kCsrOffsets);
    if (bad != ~0ull) {
        static const char *why[] = {"", "offsets not monotone or outside [0, E]",
                                    "neighbour id out of range", "self loop",
                                    "row not strictly increasing"};
        d.release();
        return fail(GAT_ERR_ARGUMENT, "invalid CSR: row " + std::to_string(bad >> 3) + ": " +
                                          why[bad & 7u]);
    }
    int rc = finish_copy(d, V, h.max_degree(), &h.off, st);
    if (rc != GAT_OK) return rc;
    int dev = 0;
    if ((e = cudaGetDevice(&dev)) != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
    g->device = dev;
    g->host_adj_pending = true;
    *out = g.release();
    return GAT_OK;
}

int gat_graph_upload_ex(gat_graph *g, int flags, int64_t hub_min_degree,
                        int64_t hub_max_bytes, void *stream) {
    if (!g) return fail(GAT_ERR_ARGUMENT, "null argument");
    cudaStream_t st = (cudaStream_t)stream;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
    const int32_t V = g->host.V;
    // A graph's host CSR never changes, so a copy already resident on this
    // device (built there by gat_graph_generate_device, or uploaded before)
    // is kept; its hub bitmaps are rebuilt for the requested parameters.
    int rc = GAT_OK;
    if (g->dev.ready && g->device == dev)
        release_hubs(g->dev);
    else if ((rc = ensure_host_adj(g)) == GAT_OK)
        rc = upload_copy(g->host, g->dev, st);
    g->hub_min_degree = hub_min_degree;
    g->hub_max_bytes = hub_max_bytes;
    g->dev_hubs_pending = (flags & GAT_UPLOAD_DEGREE_ORDER) != 0;
    if (rc == GAT_OK && !g->dev_hubs_pending)
        rc = upload_hubs(g->dev, V, hub_min_degree, hub_max_bytes, st);
    if (rc != GAT_OK) return rc;
    if (flags & GAT_UPLOAD_DEGREE_ORDER) {
        if (g->dev_ordered.ready && g->device == dev) {
            release_hubs(g->dev_ordered);
            rc = GAT_OK;
        } else {
            // graphs too large for the device relabel are relabelled on the host
            if (!relabel_fits_device(V, g->host.E)) rc = ensure_host_adj(g);
            if (rc == GAT_OK) rc = derive_ordered_copy(g->host, g->dev, g->dev_ordered, st);
        }
        if (rc == GAT_OK)
            rc = upload_hubs(g->dev_ordered, V, hub_min_degree, hub_max_bytes, st);
        if (rc != GAT_OK) return rc;
    } else {
        g->dev_ordered.release();
    }
    g->device = dev;
    return GAT_OK;
}

int gat_graph_upload(gat_graph *g, int flags, void *stream) {
    return gat_graph_upload_ex(g, flags, GAT_HUB_MIN_DEGREE_DEFAULT, GAT_HUB_MAX_BYTES_DEFAULT,
                               stream);
}

int gat_graph_hubs(const gat_graph *g, int ordered_copy, int32_t *nhubs) {
    if (!g || !nhubs) return fail(GAT_ERR_ARGUMENT, "null argument");
    if (!ordered_copy) {
        // the given-id copy's bitmaps may still be pending: build them now
        int rc = ensure_dev_hubs(const_cast<gat_graph *>(g), nullptr);
        if (rc != GAT_OK) return rc;
    }
    *nhubs = ordered_copy ? g->dev_ordered.nhubs : g->dev.nhubs;
    return GAT_OK;
}

int gat_graph_ordered_csr(const gat_graph *g, int64_t *offsets, int32_t *adj) {
    if (!g || !offsets || !adj) return fail(GAT_ERR_ARGUMENT, "null argument");
    const DevCopy &d = g->dev_ordered;
    if (!d.ready) return fail(GAT_ERR_STATE, "no degree-ordered copy uploaded");
    cudaError_t e;
    if ((e = cudaMemcpy(offsets, d.off, sizeof(int64_t) * (size_t(g->host.V) + 1),
                        cudaMemcpyDeviceToHost)) != cudaSuccess ||
        (g->host.E > 0 && (e = cudaMemcpy(adj, d.adj, sizeof(int32_t) * size_t(g->host.E),
                                          cudaMemcpyDeviceToHost)) != cudaSuccess))
        return cuda_fail(e, "ordered copy read-back");
    return GAT_OK;
}

void gat_graph_free(gat_graph *g) { delete g; }

// ------------------------------------------------------------- engine

int gat_executor_create(const gat_config *c, gat_executor **out) {
    if (!out) return fail(GAT_ERR_ARGUMENT, "null argument");
    *out = nullptr;
    auto e = std::make_unique<gat_executor>();
    if (c)
        e->cfg = *c;
    else
        gat_config_engine_default(&e->cfg);
    const gat_config &k = e->cfg;
    int t = k.set_intersection_type == 1 ? 1 : k.threads_per_warp;
    if (t != 1 && t != 2 && t != 4 && t != 8 && t != 16 && t != 32)
        return fail(GAT_ERR_CONFIG, "threads_per_warp must be 1, 2, 4, 8, 16 or 32");
    if (k.threads_per_block < 32 || k.threads_per_block > 256 ||
        k.threads_per_block % 32 != 0)
        return fail(GAT_ERR_CONFIG, "threads_per_block must be a multiple of 32 in [32, 256]");
    if (k.num_blocks < 0) return fail(GAT_ERR_CONFIG, "num_blocks must be >= 0");
    if (k.vertex_store_type != 0 || k.graph_backend_type != 0)
        return fail(GAT_ERR_CONFIG, "only Array vertex sets and the InMemory backend exist");
    cudaError_t ce;
    if ((ce = cudaGetDevice(&e->device)) != cudaSuccess) return cuda_fail(ce, "cudaGetDevice");
    if ((ce = cudaDeviceGetAttribute(&e->sms, cudaDevAttrMultiProcessorCount, e->device)) !=
        cudaSuccess)
        return cuda_fail(ce, "device attributes");
    if ((ce = cudaMalloc(&e->ctr, sizeof(DevCounters))) != cudaSuccess ||
        (ce = cudaMalloc(&e->d_plan, sizeof(GatPlan))) != cudaSuccess ||
        (ce = cudaMallocHost(&e->host_ctr, sizeof(DevCounters))) != cudaSuccess ||
        (ce = cudaMallocHost(&e->h_plan, sizeof(GatPlan))) != cudaSuccess ||
        (ce = cudaEventCreate(&e->ev0)) != cudaSuccess ||
        (ce = cudaEventCreate(&e->ev1)) != cudaSuccess)
        return cuda_fail(ce, "executor allocation");
    *out = e.release();
    return GAT_OK;
}

void gat_executor_free(gat_executor *e) { delete e; }

namespace {

// The exact 4-cycle count through the wedge-aggregation kernels (cycles.cu):
// per-root counts are tallied in shared memory, so the scratch is only the
// deferred-root list and the root kernel's list cursors.
int run_c4(gat_executor *e, const DevGraphView &view, const DevCopy &dc, int64_t vb,
           int64_t ve, LaunchShape shape, cudaStream_t strm, bool balg, uint64_t *count,
           gat_stats *stats, std::chrono::steady_clock::time_point t0) {
    const bool wide = view.max_degree >= 65536;
    const int locc = c4_light_blocks_per_sm(balg);
    const int rocc = c4_root_blocks_per_sm(wide, balg);
    if (locc <= 0 || rocc <= 0) return fail(GAT_ERR_CUDA, "4-cycle kernels do not fit on the device");
    // Heavy roots: the leading run of ids with degree >= kC4HeavyDegree (on a
    // degree-ordered copy, exactly the vertices of that degree) take a CTA
    // each from the start.
    constexpr int64_t kC4HeavyDegree = 256;
    int64_t H = 0;
    while (H < view.V && dc.off_host[H + 1] - dc.off_host[H] >= kC4HeavyDegree) H++;
    const int light_grid = e->sms * locc;
    const int root_grid = e->cfg.num_blocks > 0 ? std::min(e->cfg.num_blocks, e->sms * rocc)
                                                : e->sms * rocc;
    const int64_t stride = std::max<int64_t>(view.max_degree, 1);
    auto al = [](int64_t b) { return (b + 255) / 256 * 256; };
    const int64_t aux_bytes = al(sizeof(C4Aux));
    const int64_t def_bytes = al(std::max<int64_t>(view.V, 1) * 4);
    const int64_t cur_bytes = al(int64_t(root_grid) * stride * 4);
    const size_t need = size_t(aux_bytes + def_bytes + cur_bytes);
    cudaError_t ce;
    if (need > e->scratch_bytes) {
        cudaFree(e->scratch);
        e->scratch = nullptr;
        e->scratch_bytes = 0;
        if ((ce = cudaMalloc(&e->scratch, need)) != cudaSuccess)
            return fail(GAT_ERR_MEMORY, std::string("4-cycle scratch: ") + cudaGetErrorString(ce));
        e->scratch_bytes = need;
    }
    e->scratch_clean = false;
    unsigned char *base = reinterpret_cast<unsigned char *>(e->scratch);
    C4Launch L;
    L.g = view;
    L.v_begin = vb;
    L.v_end = ve;
    L.heavy_end = H;
    L.light_grid = light_grid;
    L.root_grid = root_grid;
    L.ctr = e->ctr;
    L.aux = reinterpret_cast<C4Aux *>(base);
    L.deferred = reinterpret_cast<int32_t *>(base + aux_bytes);
    L.cursors = reinterpret_cast<int32_t *>(base + aux_bytes + def_bytes);
    L.cursor_stride = stride;
    L.stats = balg;
    cudaEventRecord(e->ev0, strm);
    ce = launch_c4(L, strm);
    if (ce != cudaSuccess) return cuda_fail(ce, "4-cycle launch");
    cudaEventRecord(e->ev1, strm);
    if ((ce = cudaMemcpyAsync(e->host_ctr, e->ctr, sizeof(DevCounters), cudaMemcpyDeviceToHost,
                              strm)) != cudaSuccess ||
        (ce = cudaStreamSynchronize(strm)) != cudaSuccess)
        return cuda_fail(ce, "4-cycle count");
    if (e->host_ctr->error) return fail(GAT_ERR_DEVICE, "4-cycle kernel reported an internal error");
    float ms = 0;
    cudaEventElapsedTime(&ms, e->ev0, e->ev1);
    const int64_t raw = (int64_t)e->host_ctr->result;
    *count = (uint64_t)raw;
    gat_stats st{};
    st.kernel_ms = ms;
    st.raw_sum = raw;
    st.divisor = 1;
    st.tasks = (uint64_t)(ve - vb);
    st.balg_bytes = e->host_ctr->bytes;
    st.grid = root_grid;
    st.block = 1024;
    st.tile = shape.tile;
    st.launches = (std::max(vb, H) < ve ? 1 : 0) + 1;
    st.scratch_bytes = (int64_t)need;
    st.total_ms =
        std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    if (stats) *stats = st;
    return GAT_OK;
}

// The exact k-clique count through the bit-matrix kernels (cliques.cu) over
// roots [vb, ve).  Scratch: the root cursors, and per-CTA matrix rows only
// when the graph's longest lower list does not fit in shared memory.
int run_clique(gat_executor *e, const DevGraphView &view, const std::vector<int64_t> &lo_host,
               int k, int64_t ub, int64_t ue, cudaStream_t strm, bool balg, uint64_t *count,
               gat_stats *stats, std::chrono::steady_clock::time_point t0) {
    // roots whose units meet [ub, ue): from the one holding unit ub to the
    // last one starting before ue
    const int64_t vb = std::upper_bound(lo_host.begin(), lo_host.end(), ub) - lo_host.begin() - 1;
    const int64_t ve = std::lower_bound(lo_host.begin(), lo_host.end(), ue) - lo_host.begin();
    int wocc = 0, cocc = 0;
    clique_blocks_per_sm(k, balg, &wocc, &cocc);
    if (wocc <= 0 || cocc <= 0) return fail(GAT_ERR_CUDA, "clique kernels do not fit on the device");
    const int warp_grid = e->sms * wocc;
    const int cta_grid = e->cfg.num_blocks > 0 ? std::min(e->cfg.num_blocks, e->sms * cocc)
                                               : e->sms * cocc;
    auto al = [](int64_t b) { return (b + 255) / 256 * 256; };
    const int64_t aux_bytes = al(sizeof(CliqueAux));
    const int64_t stride = clique_rows_words(view.max_lower);
    const int64_t rows_bytes = al(int64_t(cta_grid) * stride * 4);
    const size_t need = size_t(aux_bytes + rows_bytes);
    cudaError_t ce;
    if (need > e->scratch_bytes) {
        cudaFree(e->scratch);
        e->scratch = nullptr;
        e->scratch_bytes = 0;
        if ((ce = cudaMalloc(&e->scratch, need)) != cudaSuccess)
            return fail(GAT_ERR_MEMORY, std::string("clique scratch: ") + cudaGetErrorString(ce));
        e->scratch_bytes = need;
    }
    e->scratch_clean = false;
    unsigned char *base = reinterpret_cast<unsigned char *>(e->scratch);
    CliqueLaunch L;
    L.g = view;
    L.k = k;
    L.v_begin = std::max<int64_t>(vb, 0);
    L.v_end = std::min<int64_t>(ve, view.V);
    L.u_begin = ub;
    L.u_end = ue;
    L.warp_grid = warp_grid;
    L.cta_grid = cta_grid;
    L.ctr = e->ctr;
    L.aux = reinterpret_cast<CliqueAux *>(base);
    L.rows = stride > 0 ? reinterpret_cast<uint32_t *>(base + aux_bytes) : nullptr;
    L.rows_stride = stride;
    L.stats = balg;
    cudaEventRecord(e->ev0, strm);
    ce = launch_clique(L, strm);
    if (ce != cudaSuccess) return cuda_fail(ce, "clique launch");
    cudaEventRecord(e->ev1, strm);
    if ((ce = cudaMemcpyAsync(e->host_ctr, e->ctr, sizeof(DevCounters), cudaMemcpyDeviceToHost,
                              strm)) != cudaSuccess ||
        (ce = cudaStreamSynchronize(strm)) != cudaSuccess)
        return cuda_fail(ce, "clique count");
    if (e->host_ctr->error) return fail(GAT_ERR_DEVICE, "clique kernel reported an internal error");
    float ms = 0;
    cudaEventElapsedTime(&ms, e->ev0, e->ev1);
    const int64_t raw = (int64_t)e->host_ctr->result;
    *count = (uint64_t)raw;
    gat_stats st{};
    st.kernel_ms = ms;
    st.raw_sum = raw;
    st.divisor = 1;
    st.tasks = (uint64_t)(ue - ub);
    st.balg_bytes = e->host_ctr->bytes;
    st.grid = cta_grid;
    st.block = kCliqueCtaThreads;
    st.tile = 32;
    st.launches = ue > ub ? 2 : 0;
    st.scratch_bytes = (int64_t)need;
    st.total_ms =
        std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    if (stats) *stats = st;
    return GAT_OK;
}

int count_impl(gat_executor *e, gat_graph *g, const gat_schedule *s, void *stream,
               uint64_t *count, gat_stats *stats, bool balg, int64_t root_begin = -1,
               int64_t root_end = -1, int shard = 0, int num_shards = 0) {
    auto t0 = std::chrono::steady_clock::now();
    if (!e || !g || !s || !count) return fail(GAT_ERR_ARGUMENT, "null argument");
    gat_stats st{};
    cudaStream_t strm = (cudaStream_t)stream;
    if (s->trivial) {
        int64_t c = 0;
        if (s->mode == GAT_MODE_EXACT)
            c = s->pattern.n == 1 ? g->host.V : g->host.E / 2;
        *count = (uint64_t)c;
        st.raw_sum = c;
        st.divisor = 1;
        if (stats) *stats = st;
        return GAT_OK;
    }
    const GatPlan &plan = s->plan.plan;
    if (plan.n == 0) return fail(GAT_ERR_UNDEFINED, s->plan.summary);
    DevCopy *dc = nullptr;
    if (s->mode == GAT_MODE_EXACT) {
        if (!g->dev.ready) {
            int rc = gat_graph_upload(g, GAT_UPLOAD_DEGREE_ORDER, stream);
            if (rc != GAT_OK) return rc;
        }
        dc = g->dev_ordered.ready ? &g->dev_ordered : &g->dev;
    } else {
        if (!g->dev.ready) {
            int rc = gat_graph_upload(g, 0, stream);
            if (rc != GAT_OK) return rc;
        }
        int rc = ensure_dev_hubs(g, strm);
        if (rc != GAT_OK) return rc;
        dc = &g->dev;
    }
    DevGraphView view;
    view.V = g->host.V;
    view.E = g->host.E;
    view.off = dc->off;
    view.adj = dc->adj;
    view.lo_off = dc->lo_off;
    view.lo_total = dc->lo_total;
    view.max_degree = dc->max_degree;
    view.max_lower = dc->max_lower;
    view.hub_slot = dc->hub_slot;
    view.bitmaps = dc->bitmaps;
    view.bitmap_words = dc->bitmap_words;

    LaunchShape shape;
    shape.tile = e->cfg.set_intersection_type == 1 ? 1 : e->cfg.threads_per_warp;
    shape.block = e->cfg.threads_per_block;
    shape.chunk = e->cfg.chunk > 0 ? e->cfg.chunk : 16;
    // Two-level plans on the lane path give every lane its own level-1
    // unit, so one grab holds `chunk` units per lane.
    if (plan.basic == 2 && plan.lane_last && e->cfg.special_kernels != 0)
        shape.chunk *= shape.tile;
    shape.linear_below = e->cfg.set_search_type;
    shape.use_bitmaps = e->cfg.hub_bitmaps != 0;
    const bool ranged = root_begin >= 0 || num_shards > 0;
    if (num_shards > 0) {
        if (shard < 0 || shard >= num_shards)
            return fail(GAT_ERR_ARGUMENT, "shard index out of range");
        const int64_t total = plan.level1_bounded ? view.lo_total : view.E;
        shape.task_begin = total * shard / num_shards;
        shape.task_end = total * (shard + 1) / num_shards;
    }
    if (root_begin >= 0) {
        if (root_end < root_begin || root_end > view.V)
            return fail(GAT_ERR_ARGUMENT, "root range outside [0, V]");
        const int64_t *toff = plan.level1_bounded ? dc->lo_host.data() : dc->off_host.data();
        shape.task_begin = toff[root_begin];
        shape.task_end = toff[root_end];
    }
    if (plan.special == GAT_SPECIAL_CLIQUE && s->mode == GAT_MODE_EXACT &&
        e->cfg.special_kernels == 1 && view.lo_off != nullptr &&
        view.max_lower <= kCliqueMaxLower) {
        // The level-1 units of this call (whole graph, root range or shard),
        // exactly as the plan path numbers them.
        const int64_t ub = ranged ? shape.task_begin : 0;
        const int64_t ue = ranged ? shape.task_end : view.lo_total;
        return run_clique(e, view, dc->lo_host, plan.n, ub, ue, strm, balg, count, stats, t0);
    }
    if (plan.special == GAT_SPECIAL_C4 && s->mode == GAT_MODE_EXACT &&
        e->cfg.special_kernels == 1) {
        // First-vertex range of this call: whole graph, a root range, or the
        // vertices whose level-1 units start inside the shard's unit range.
        int64_t vb = 0, ve = view.V;
        if (root_begin >= 0) {
            vb = root_begin;
            ve = root_end;
        } else if (num_shards > 0) {
            // Roots are split by their upper neighbours (the 4-cycle kernels'
            // units): shard k takes the roots whose units start in its slice.
            const auto &of = dc->off_host;
            const auto &lo = dc->lo_host;
            auto first_root = [&](int64_t u) {
                int64_t a = 0, n = view.V;
                while (n > 0) {
                    const int64_t h = n >> 1;
                    if (of[a + h] - lo[a + h] < u) {
                        a += h + 1;
                        n -= h + 1;
                    } else {
                        n = h;
                    }
                }
                return a;
            };
            const int64_t total = view.E - view.lo_total;
            vb = first_root(total * shard / num_shards);
            ve = shard + 1 == num_shards ? view.V : first_root(total * (shard + 1) / num_shards);
        }
        return run_c4(e, view, *dc, vb, ve, shape, strm, balg, count, stats, t0);
    }
    int occ = blocks_per_sm(shape.tile, shape.block, balg);
    if (occ <= 0) return fail(GAT_ERR_CUDA, "kernel does not fit on the device");
    shape.grid = e->cfg.num_blocks > 0 ? e->cfg.num_blocks : e->sms * occ;
    e->scratch_clean = false;
    const int64_t stride = tile_scratch_ints(plan, view.max_degree);
    const int64_t tiles_per_block = shape.block / shape.tile;
    const int64_t budget = e->cfg.memory_budget > 0 ? e->cfg.memory_budget : (int64_t(4) << 30);
    int64_t per_block = tiles_per_block * stride * (int64_t)sizeof(int32_t);
    if (plan.num_store > 0) {
        int64_t max_grid = budget / per_block;
        if (max_grid < 1)
            return fail(GAT_ERR_MEMORY, "memory budget below one CTA's scratch");
        if (shape.grid > max_grid) shape.grid = (int)max_grid;
    }
    size_t need = (size_t)(plan.num_store > 0 ? per_block * shape.grid : 4);
    cudaError_t ce;
    if (need > e->scratch_bytes) {
        cudaFree(e->scratch);
        e->scratch = nullptr;
        e->scratch_bytes = 0;
        if ((ce = cudaMalloc(&e->scratch, need)) != cudaSuccess)
            return fail(GAT_ERR_MEMORY, std::string("scratch allocation: ") + cudaGetErrorString(ce));
        e->scratch_bytes = need;
    }
    *e->h_plan = plan;
    if (e->cfg.special_kernels == 0) e->h_plan->lane_last = 0;
    if ((ce = cudaMemcpyAsync(e->d_plan, e->h_plan, sizeof(GatPlan), cudaMemcpyHostToDevice,
                              strm)) != cudaSuccess)
        return cuda_fail(ce, "plan upload");
    cudaEventRecord(e->ev0, strm);
    ce = launch_search(e->d_plan, plan, view, shape, e->scratch, stride, e->ctr, balg, strm);
    if (ce != cudaSuccess) return cuda_fail(ce, "search launch");
    cudaEventRecord(e->ev1, strm);
    if ((ce = cudaMemcpyAsync(e->host_ctr, e->ctr, sizeof(DevCounters), cudaMemcpyDeviceToHost,
                              strm)) != cudaSuccess ||
        (ce = cudaStreamSynchronize(strm)) != cudaSuccess)
        return cuda_fail(ce, "search");
    float ms = 0;
    cudaEventElapsedTime(&ms, e->ev0, e->ev1);
    if (e->host_ctr->error) return fail(GAT_ERR_DEVICE, "kernel reported an internal error");
    int64_t raw = (int64_t)e->host_ctr->result;
    if (ranged) {
        *count = (uint64_t)raw;  // partial sums are divided by the caller
    } else {
        if (plan.divisor <= 0 || raw % plan.divisor != 0)
            return fail(GAT_ERR_DEVICE, "engine total is not a multiple of the plan divisor");
        *count = (uint64_t)(raw / plan.divisor);
    }
    st.kernel_ms = ms;
    st.raw_sum = raw;
    st.divisor = plan.divisor;
    st.tasks = ranged ? (uint64_t)(shape.task_end - shape.task_begin)
                      : (plan.level1_bounded ? (uint64_t)view.lo_total : (uint64_t)view.E);
    st.balg_bytes = e->host_ctr->bytes;
    st.grid = shape.grid;
    st.block = shape.block;
    st.tile = shape.tile;
    st.launches = 1;
    st.scratch_bytes = plan.num_store > 0 ? per_block * shape.grid : 0;
    st.total_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0)
                      .count();
    if (stats) *stats = st;
    return GAT_OK;
}

}  // namespace

int gat_executor_count(gat_executor *e, gat_graph *g, const gat_schedule *s, void *stream,
                       uint64_t *count, gat_stats *stats) {
    return count_impl(e, g, s, stream, count, stats, false);
}

int gat_executor_count_balg(gat_executor *e, gat_graph *g, const gat_schedule *s,
                            void *stream, uint64_t *count, gat_stats *stats) {
    return count_impl(e, g, s, stream, count, stats, true);
}

int gat_executor_count_range(gat_executor *e, gat_graph *g, const gat_schedule *s,
                             void *stream, int32_t root_begin, int32_t root_end,
                             int64_t *raw_sum, gat_stats *stats) {
    if (root_begin < 0) return fail(GAT_ERR_ARGUMENT, "negative root");
    uint64_t c = 0;
    int rc = count_impl(e, g, s, stream, &c, stats, false, root_begin, root_end);
    if (rc == GAT_OK && raw_sum) *raw_sum = (int64_t)c;
    return rc;
}

int gat_executor_count_shard(gat_executor *e, gat_graph *g, const gat_schedule *s,
                             void *stream, int32_t shard, int32_t num_shards,
                             int64_t *raw_sum, gat_stats *stats) {
    if (num_shards < 1) return fail(GAT_ERR_ARGUMENT, "num_shards must be >= 1");
    uint64_t c = 0;
    int rc = count_impl(e, g, s, stream, &c, stats, false, -1, -1, shard, num_shards);
    if (rc == GAT_OK && raw_sum) *raw_sum = (int64_t)c;
    return rc;
}

int gat_executor_count_shard_balg(gat_executor *e, gat_graph *g, const gat_schedule *s,
                                  void *stream, int32_t shard, int32_t num_shards,
                                  int64_t *raw_sum, gat_stats *stats) {
    if (num_shards < 1) return fail(GAT_ERR_ARGUMENT, "num_shards must be >= 1");
    uint64_t c = 0;
    int rc = count_impl(e, g, s, stream, &c, stats, true, -1, -1, shard, num_shards);
    if (rc == GAT_OK && raw_sum) *raw_sum = (int64_t)c;
    return rc;
}

}  // extern "C"

// ------------------------------------------------------------------ batch

struct gat_batch {
    struct Job {
        gat_graph *g;
        const gat_schedule *s;
        int shard = 0, num_shards = 0;  // num_shards > 0: one slice of the work queue
    };
    std::vector<Job> jobs;
    gat_config cfg{};
    bool prepared = false, use_graph = false;
    int tile = 32, block = 256, grid = 0, chunk = 8;
    int64_t vtotal = 0, stride = 0;
    GatPlan *d_plans = nullptr;
    void *d_jobs = nullptr;
    int64_t *d_vstart = nullptr;
    unsigned long long *d_cursor = nullptr, *d_results = nullptr, *h_results = nullptr;
    int32_t *d_scratch = nullptr;
    size_t scratch_bytes = 0;
    cudaStream_t stream = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    std::vector<int64_t> divisors;
    std::vector<int> modes;
    std::vector<int64_t> raw;
    void release_device() {
        if (exec) cudaGraphExecDestroy(exec);
        if (graph) cudaGraphDestroy(graph);
        exec = nullptr;
        graph = nullptr;
        cudaFree(d_plans);
        cudaFree(d_jobs);
        cudaFree(d_vstart);
        cudaFree(d_cursor);
        cudaFree(d_results);
        cudaFree(d_scratch);
        cudaFreeHost(h_results);
        d_plans = nullptr;
        d_jobs = nullptr;
        d_vstart = nullptr;
        d_cursor = nullptr;
        d_results = nullptr;
        d_scratch = nullptr;
        h_results = nullptr;
        scratch_bytes = 0;
        prepared = false;
    }
    ~gat_batch() {
        release_device();
        if (ev0) cudaEventDestroy(ev0);
        if (ev1) cudaEventDestroy(ev1);
        if (stream) cudaStreamDestroy(stream);
    }
};

extern "C" {

int gat_batch_create(gat_batch **out) {
    if (!out) return fail(GAT_ERR_ARGUMENT, "null argument");
    auto b = std::make_unique<gat_batch>();
    cudaError_t e;
    if ((e = cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking)) != cudaSuccess ||
        (e = cudaEventCreate(&b->ev0)) != cudaSuccess ||
        (e = cudaEventCreate(&b->ev1)) != cudaSuccess)
        return cuda_fail(e, "batch stream");
    *out = b.release();
    return GAT_OK;
}

void gat_batch_free(gat_batch *b) { delete b; }

int gat_batch_add(gat_batch *b, gat_graph *g, const gat_schedule *s, int32_t *job_index) {
    if (!b || !g || !s) return fail(GAT_ERR_ARGUMENT, "null argument");
    if (s->trivial) return fail(GAT_ERR_ARGUMENT, "patterns of at most two vertices have no plan");
    if (s->plan.plan.n == 0) return fail(GAT_ERR_UNDEFINED, s->plan.summary);
    b->jobs.push_back({g, s});
    b->prepared = false;
    if (job_index) *job_index = (int32_t)b->jobs.size() - 1;
    return GAT_OK;
}

int gat_batch_add_shard(gat_batch *b, gat_graph *g, const gat_schedule *s, int32_t shard,
                        int32_t num_shards, int32_t *job_index) {
    if (num_shards < 1 || shard < 0 || shard >= num_shards)
        return fail(GAT_ERR_ARGUMENT, "shard index out of range");
    int32_t idx = -1;
    const int rc = gat_batch_add(b, g, s, &idx);
    if (rc != GAT_OK) return rc;
    b->jobs[size_t(idx)].shard = shard;
    b->jobs[size_t(idx)].num_shards = num_shards;
    if (job_index) *job_index = idx;
    return GAT_OK;
}

int gat_batch_prepare(gat_batch *b, const gat_config *c, int use_cuda_graph) {
    if (!b) return fail(GAT_ERR_ARGUMENT, "null argument");
    if (b->jobs.empty()) return fail(GAT_ERR_STATE, "empty batch");
    b->release_device();
    if (c)
        b->cfg = *c;
    else
        gat_config_engine_default(&b->cfg);
    b->tile = b->cfg.set_intersection_type == 1 ? 1 : b->cfg.threads_per_warp;
    b->block = b->cfg.threads_per_block;
    b->chunk = b->cfg.chunk > 0 ? b->cfg.chunk : 8;
    if (b->block < 32 || b->block > 256 || b->block % 32 || b->block % b->tile)
        return fail(GAT_ERR_CONFIG, "bad threads_per_block / threads_per_warp");
    const size_t J = b->jobs.size();
    const size_t jb = batch_job_bytes();
    std::vector<unsigned char> host_jobs(J * jb);
    std::vector<GatPlan> plans(J);
    std::vector<int64_t> vstart(J);
    b->divisors.assign(J, 1);
    b->modes.assign(J, 0);
    cudaError_t e;
    if ((e = cudaMalloc(&b->d_plans, sizeof(GatPlan) * J)) != cudaSuccess)
        return fail(GAT_ERR_MEMORY, "batch plans");
    int64_t stride = 0, vt = 0;
    for (size_t j = 0; j < J; j++) {
        gat_graph *g = b->jobs[j].g;
        const gat_schedule *s = b->jobs[j].s;
        const bool exact = s->mode == GAT_MODE_EXACT;
        if (!g->dev.ready || (exact && !g->dev_ordered.ready)) {
            int rc = gat_graph_upload(g, exact ? GAT_UPLOAD_DEGREE_ORDER : 0, b->stream);
            if (rc != GAT_OK) return rc;
        }
        if (!(exact && g->dev_ordered.ready)) {
            int rc = ensure_dev_hubs(g, b->stream);
            if (rc != GAT_OK) return rc;
        }
        const DevCopy &dc = (exact && g->dev_ordered.ready) ? g->dev_ordered : g->dev;
        DevGraphView v;
        v.V = g->host.V;
        v.E = g->host.E;
        v.off = dc.off;
        v.adj = dc.adj;
        v.lo_off = dc.lo_off;
        v.lo_total = dc.lo_total;
        v.max_degree = dc.max_degree;
        v.hub_slot = dc.hub_slot;
        v.bitmaps = dc.bitmaps;
        v.bitmap_words = dc.bitmap_words;
        plans[j] = s->plan.plan;
        if (b->cfg.special_kernels == 0) plans[j].lane_last = 0;
        batch_fill_job(host_jobs.data() + j * jb, b->d_plans + j, plans[j], v,
                       b->cfg.set_search_type, b->cfg.hub_bitmaps != 0, b->jobs[j].shard,
                       b->jobs[j].num_shards);
        stride = std::max<int64_t>(stride, tile_scratch_ints(plans[j], v.max_degree));
        vstart[j] = vt;
        const int64_t n = batch_job_tasks(host_jobs.data() + j * jb);
        vt += (n + b->chunk - 1) / b->chunk * b->chunk;
        b->divisors[j] = plans[j].divisor;
        b->modes[j] = s->mode;
    }
    b->vtotal = vt;
    b->stride = stride;
    int occ = batch_blocks_per_sm(b->tile, b->block);
    if (occ <= 0) return fail(GAT_ERR_CUDA, "batch kernel does not fit on the device");
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    b->grid = b->cfg.num_blocks > 0 ? b->cfg.num_blocks : sms * occ;
    const int64_t per_block = int64_t(b->block / b->tile) * stride * 4;
    const int64_t budget = b->cfg.memory_budget > 0 ? b->cfg.memory_budget : (int64_t(4) << 30);
    if (per_block > 0) {
        if (per_block > budget) return fail(GAT_ERR_MEMORY, "memory budget below one CTA's scratch");
        b->grid = (int)std::min<int64_t>(b->grid, budget / per_block);
    }
    b->scratch_bytes = size_t(std::max<int64_t>(per_block * b->grid, 4));
    if ((e = cudaMalloc(&b->d_jobs, J * jb)) != cudaSuccess ||
        (e = cudaMalloc(&b->d_vstart, sizeof(int64_t) * J)) != cudaSuccess ||
        (e = cudaMalloc(&b->d_cursor, sizeof(unsigned long long))) != cudaSuccess ||
        (e = cudaMalloc(&b->d_results, sizeof(unsigned long long) * J)) != cudaSuccess ||
        (e = cudaMalloc(&b->d_scratch, b->scratch_bytes)) != cudaSuccess ||
        (e = cudaMallocHost(&b->h_results, sizeof(unsigned long long) * J)) != cudaSuccess)
        return fail(GAT_ERR_MEMORY, std::string("batch tables: ") + cudaGetErrorString(e));
    if ((e = cudaMemcpyAsync(b->d_plans, plans.data(), sizeof(GatPlan) * J,
                             cudaMemcpyHostToDevice, b->stream)) != cudaSuccess ||
        (e = cudaMemcpyAsync(b->d_jobs, host_jobs.data(), J * jb, cudaMemcpyHostToDevice,
                             b->stream)) != cudaSuccess ||
        (e = cudaMemcpyAsync(b->d_vstart, vstart.data(), sizeof(int64_t) * J,
                             cudaMemcpyHostToDevice, b->stream)) != cudaSuccess ||
        (e = cudaStreamSynchronize(b->stream)) != cudaSuccess)
        return cuda_fail(e, "batch upload");
    b->use_graph = use_cuda_graph != 0;
    if (b->use_graph) {
        if ((e = cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal)) !=
            cudaSuccess)
            return cuda_fail(e, "begin capture");
        cudaMemsetAsync(b->d_cursor, 0, sizeof(unsigned long long), b->stream);
        cudaMemsetAsync(b->d_results, 0, sizeof(unsigned long long) * J, b->stream);
        cudaError_t le = launch_batch(b->d_jobs, b->d_vstart, (int32_t)J, b->vtotal, b->tile,
                                      b->grid, b->block, b->chunk, b->d_cursor, b->d_results,
                                      b->d_scratch, b->stride, b->stream);
        cudaMemcpyAsync(b->h_results, b->d_results, sizeof(unsigned long long) * J,
                        cudaMemcpyDeviceToHost, b->stream);
        e = cudaStreamEndCapture(b->stream, &b->graph);
        if (le != cudaSuccess) return cuda_fail(le, "batch launch (capture)");
        if (e != cudaSuccess) return cuda_fail(e, "end capture");
        if ((e = cudaGraphInstantiate(&b->exec, b->graph, 0)) != cudaSuccess)
            return cuda_fail(e, "graph instantiate");
    }
    b->prepared = true;
    return GAT_OK;
}

int gat_batch_run(gat_batch *b, gat_stats *stats) {
    if (!b) return fail(GAT_ERR_ARGUMENT, "null argument");
    if (!b->prepared) return fail(GAT_ERR_STATE, "batch not prepared");
    auto t0 = std::chrono::steady_clock::now();
    const size_t J = b->jobs.size();
    cudaError_t e;
    cudaEventRecord(b->ev0, b->stream);
    if (b->use_graph) {
        e = cudaGraphLaunch(b->exec, b->stream);
    } else {
        cudaMemsetAsync(b->d_cursor, 0, sizeof(unsigned long long), b->stream);
        cudaMemsetAsync(b->d_results, 0, sizeof(unsigned long long) * J, b->stream);
        e = launch_batch(b->d_jobs, b->d_vstart, (int32_t)J, b->vtotal, b->tile, b->grid,
                         b->block, b->chunk, b->d_cursor, b->d_results, b->d_scratch, b->stride,
                         b->stream);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(b->h_results, b->d_results, sizeof(unsigned long long) * J,
                                cudaMemcpyDeviceToHost, b->stream);
    }
    if (e != cudaSuccess) return cuda_fail(e, "batch launch");
    cudaEventRecord(b->ev1, b->stream);
    if ((e = cudaStreamSynchronize(b->stream)) != cudaSuccess) return cuda_fail(e, "batch run");
    b->raw.assign(J, 0);
    for (size_t j = 0; j < J; j++) {
        b->raw[j] = (int64_t)b->h_results[j];
        // a whole job's total is a multiple of its divisor; a slice's need not be
        if (b->jobs[j].num_shards == 0 &&
            (b->divisors[j] <= 0 || b->raw[j] % b->divisors[j] != 0))
            return fail(GAT_ERR_DEVICE, "job total is not a multiple of its plan divisor");
    }
    if (stats) {
        gat_stats st{};
        float ms = 0;
        cudaEventElapsedTime(&ms, b->ev0, b->ev1);
        st.kernel_ms = ms;
        st.total_ms = std::chrono::duration<double, std::milli>(
                          std::chrono::steady_clock::now() - t0)
                          .count();
        st.grid = b->grid;
        st.block = b->block;
        st.tile = b->tile;
        st.launches = 1;
        st.tasks = (uint64_t)b->vtotal;
        st.scratch_bytes = (int64_t)b->scratch_bytes;
        *stats = st;
    }
    return GAT_OK;
}

int gat_batch_counts(const gat_batch *b, uint64_t *counts, size_t n) {
    if (!b || !counts) return fail(GAT_ERR_ARGUMENT, "null argument");
    if (b->raw.size() != b->jobs.size()) return fail(GAT_ERR_STATE, "batch has not run");
    if (n < b->jobs.size()) return fail(GAT_ERR_ARGUMENT, "output too small");
    for (size_t j = 0; j < b->jobs.size(); j++)
        counts[j] = b->jobs[j].num_shards > 0 ? (uint64_t)b->raw[j]
                                              : (uint64_t)(b->raw[j] / b->divisors[j]);
    return GAT_OK;
}

int gat_batch_size(const gat_batch *b) { return b ? (int)b->jobs.size() : 0; }

int gat_count_noalloc(const int64_t *d_offsets, const int32_t *d_adj, int32_t V, int64_t E,
                      int32_t max_degree, const gat_schedule *s, const gat_config *c,
                      int64_t *d_count, void *stream) {
    if (!d_offsets || (E > 0 && !d_adj) || !s || !d_count || V < 0 || E < 0 ||
        max_degree < 0)
        return fail(GAT_ERR_ARGUMENT, "bad arguments");
    if (s->trivial)
        return fail(GAT_ERR_ARGUMENT, "patterns of at most two vertices have no device plan");
    if (s->plan.plan.n == 0) return fail(GAT_ERR_UNDEFINED, s->plan.summary);
    gat_config cfg;
    if (c)
        cfg = *c;
    else
        gat_config_engine_default(&cfg);
    LaunchShape shape;
    shape.tile = cfg.set_intersection_type == 1 ? 1 : cfg.threads_per_warp;
    shape.block = cfg.threads_per_block;
    shape.chunk = cfg.chunk > 0 ? cfg.chunk : 16;
    shape.linear_below = cfg.set_search_type;
    if (shape.block < 32 || shape.block > 256 || shape.block % 32 != 0)
        return fail(GAT_ERR_CONFIG, "threads_per_block must be a multiple of 32 in [32, 256]");
    std::string err;
    int rc = count_noalloc(s->plan.plan, d_offsets, d_adj, V, E, max_degree, shape,
                           reinterpret_cast<long long *>(d_count), (cudaStream_t)stream, &err);
    if (rc != GAT_OK) return fail(rc, err);
    return GAT_OK;
}

int gat_count(gat_graph *g, const gat_schedule *s, const gat_config *c, uint64_t *count,
              gat_stats *stats) {
    gat_executor *e = nullptr;
    int rc = gat_executor_create(c, &e);
    if (rc != GAT_OK) return rc;
    rc = gat_executor_count(e, g, s, nullptr, count, stats);
    gat_executor_free(e);
    return rc;
}

}  // extern "C"
