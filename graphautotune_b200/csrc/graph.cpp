#include "graph.hpp"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <fstream>
#include <map>
#include <numeric>

namespace gat {

int32_t HostGraph::max_degree() const {
    int64_t m = 0;
    for (int32_t v = 0; v < V; v++) m = std::max(m, degree(v));
    return (int32_t)m;
}

bool load_binary(const std::string &path, HostGraph &g, std::string *err) {
    g = HostGraph{};
    std::FILE *f = std::fopen(path.c_str(), "rb");
    if (!f) {
        if (err) *err = "cannot open " + path;
        return false;
    }
    bool ok = std::fread(&g.V, sizeof(int32_t), 1, f) == 1 &&
              std::fread(&g.E, sizeof(int64_t), 1, f) == 1 && g.V >= 0 &&
              g.E >= 0;
    if (ok) {
        g.off.resize(size_t(g.V) + 1);
        g.adj.resize(size_t(g.E));
        ok = std::fread(g.off.data(), sizeof(int64_t), g.off.size(), f) ==
                 g.off.size() &&
             std::fread(g.adj.data(), sizeof(int32_t), g.adj.size(), f) ==
                 g.adj.size();
    }
    std::fclose(f);
    if (!ok) {
        if (err) *err = "truncated or malformed binary graph " + path;
        g = HostGraph{};
        return false;
    }
    return true;
}

bool save_binary(const std::string &path, const HostGraph &g, std::string *err) {
    std::FILE *f = std::fopen(path.c_str(), "wb");
    if (!f) {
        if (err) *err = "cannot write " + path;
        return false;
    }
    bool ok = std::fwrite(&g.V, sizeof(int32_t), 1, f) == 1 &&
              std::fwrite(&g.E, sizeof(int64_t), 1, f) == 1 &&
              std::fwrite(g.off.data(), sizeof(int64_t), g.off.size(), f) ==
                  g.off.size() &&
              std::fwrite(g.adj.data(), sizeof(int32_t), g.adj.size(), f) ==
                  g.adj.size();
    ok = (std::fclose(f) == 0) && ok;
    if (!ok && err) *err = "short write to " + path;
    return ok;
}

bool load_text(const std::string &path, HostGraph &g, std::string *err) {
    g = HostGraph{};
    std::ifstream in(path);
    if (!in.is_open()) {
        if (err) *err = "cannot open " + path;
        return false;
    }
    long long v_cnt = 0, e_cnt = 0;
    if (!(in >> v_cnt >> e_cnt) || v_cnt < 0 || e_cnt < 0 ||
        v_cnt > INT32_MAX) {
        if (err) *err = "bad header in " + path;
        return false;
    }
    std::vector<std::pair<int64_t, int64_t>> raw;
    raw.reserve(size_t(e_cnt));
    std::map<int64_t, int32_t> ids;
    for (long long i = 0; i < e_cnt; i++) {
        long long u, v;
        if (!(in >> u >> v)) {
            if (err) *err = "truncated edge list in " + path;
            return false;
        }
        raw.emplace_back(u, v);
        ids[u] = 0;
        ids[v] = 0;
    }
    if ((long long)ids.size() > v_cnt) {
        if (err) *err = "more distinct vertices than declared in " + path;
        return false;
    }
    int32_t next = 0;
    for (auto &kv : ids) kv.second = next++;
    std::vector<std::pair<int32_t, int32_t>> edges;
    edges.reserve(raw.size());
    for (auto &e : raw) edges.emplace_back(ids[e.first], ids[e.second]);
    build_csr((int32_t)v_cnt, edges, g);
    return true;
}

void build_csr(int32_t V, const std::vector<std::pair<int32_t, int32_t>> &edges,
               HostGraph &g) {
    g = HostGraph{};
    g.V = V;
    std::vector<int64_t> deg(size_t(V) + 1, 0);
    for (auto &e : edges)
        if (e.first != e.second) {
            deg[e.first]++;
            deg[e.second]++;
        }
    std::vector<int64_t> pos(size_t(V) + 1, 0);
    for (int32_t v = 0; v < V; v++) pos[v + 1] = pos[v] + deg[v];
    std::vector<int32_t> tmp(size_t(pos[V]));
    std::vector<int64_t> fill(pos.begin(), pos.end() - 1);
    for (auto &e : edges)
        if (e.first != e.second) {
            tmp[fill[e.first]++] = e.second;
            tmp[fill[e.second]++] = e.first;
        }
    std::vector<int64_t> kept(size_t(V), 0);
#pragma omp parallel for schedule(dynamic, 1024)
    for (int32_t v = 0; v < V; v++) {
        auto b = tmp.begin() + pos[v], e = tmp.begin() + pos[v + 1];
        std::sort(b, e);
        kept[v] = std::unique(b, e) - b;
    }
    g.off.assign(size_t(V) + 1, 0);
    for (int32_t v = 0; v < V; v++) g.off[v + 1] = g.off[v] + kept[v];
    g.E = g.off[V];
    g.adj.resize(size_t(g.E));
#pragma omp parallel for schedule(dynamic, 1024)
    for (int32_t v = 0; v < V; v++)
        std::copy(tmp.begin() + pos[v], tmp.begin() + pos[v] + kept[v],
                  g.adj.begin() + g.off[v]);
}

namespace {
// First problem of row v (nullptr if none); offsets are known to be sane.
const char *row_problem(const HostGraph &g, int32_t v, bool check_symmetry) {
    for (int64_t i = g.off[v]; i < g.off[v + 1]; i++) {
        const int32_t u = g.adj[i];
        if (u < 0 || u >= g.V) return "neighbour id out of range";
        if (u == v) return "self loop";
        if (i > g.off[v] && g.adj[i - 1] >= u) return "row not strictly increasing";
    }
    if (check_symmetry)
        for (int64_t i = g.off[v]; i < g.off[v + 1]; i++) {
            const int32_t u = g.adj[i];
            auto b = g.adj.begin() + g.off[u], e = g.adj.begin() + g.off[u + 1];
            if (!std::binary_search(b, e, v)) return "not symmetric";
        }
    return nullptr;
}
}  // namespace

bool validate(const HostGraph &g, bool check_symmetry, std::string *err) {
    auto fail = [&](const char *m) {
        if (err) *err = m;
        return false;
    };
    if (g.V < 0 || (int64_t)g.off.size() != int64_t(g.V) + 1)
        return fail("offset array size mismatch");
    if (g.off[0] != 0 || g.off[g.V] != g.E || (int64_t)g.adj.size() != g.E)
        return fail("edge count mismatch");
    for (int32_t v = 0; v < g.V; v++)
        if (g.off[v + 1] < g.off[v]) return fail("offsets not monotone");
    // Rows in parallel; the row checks of the symmetry pass read other rows,
    // so the structural checks of every row come first.  The message is
    // that of the lowest failing row, as a serial scan would report it.
    for (int pass = 0; pass < (check_symmetry ? 2 : 1); pass++) {
        int32_t bad = g.V;
#pragma omp parallel for schedule(dynamic, 4096) reduction(min : bad)
        for (int32_t v = 0; v < g.V; v++)
            if (v < bad && row_problem(g, v, pass == 1)) bad = v;
        if (bad < g.V) return fail(row_problem(g, bad, pass == 1));
    }
    return true;
}

uint64_t splitmix64_next(uint64_t &state) {
    uint64_t z = (state += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

namespace {
double uniform01(uint64_t &s) {
    return double(splitmix64_next(s) >> 11) * (1.0 / 9007199254740992.0);
}
uint64_t stream_state(uint64_t seed, uint64_t i) {
    uint64_t s = seed;
    uint64_t base = splitmix64_next(s);
    return base + i * 0xD1B54A32D192ED03ull;
}
}  // namespace

void gen_erdos_renyi(int32_t n, double avg_degree, uint64_t seed, HostGraph &g) {
    std::vector<std::pair<int32_t, int32_t>> edges;
    gen_erdos_renyi_edges(n, avg_degree, seed, edges);
    build_csr(n, edges, g);
}

void gen_erdos_renyi_edges(int32_t n, double avg_degree, uint64_t seed,
                           std::vector<std::pair<int32_t, int32_t>> &edges) {
    edges.clear();
    double p = n > 1 ? avg_degree / double(n - 1) : 0.0;
    if (p > 0 && p < 1) {
        uint64_t s = stream_state(seed, 0);
        double lq = std::log(1.0 - p);
        int64_t v = 1, w = -1;
        while (v < n) {
            double r = uniform01(s);
            w += 1 + (int64_t)std::floor(std::log(1.0 - r) / lq);
            while (w >= v && v < n) {
                w -= v;
                v++;
            }
            if (v < n) edges.emplace_back((int32_t)v, (int32_t)w);
        }
    } else if (p >= 1) {
        for (int32_t v = 1; v < n; v++)
            for (int32_t w = 0; w < v; w++) edges.emplace_back(v, w);
    }
}

void gen_rmat(int scale, int64_t samples, double a, double b, double c,
              uint64_t seed, HostGraph &g) {
    const uint64_t ta = uint64_t(a * 4294967296.0);
    const uint64_t tb = uint64_t((a + b) * 4294967296.0);
    const uint64_t tc = uint64_t((a + b + c) * 4294967296.0);
    std::vector<std::pair<int32_t, int32_t>> edges(static_cast<size_t>(samples));
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < samples; i++) {
        uint64_t s = stream_state(seed, uint64_t(i));
        uint32_t u = 0, v = 0;
        uint64_t bits = 0;
        for (int l = 0; l < scale; l++) {
            if ((l & 1) == 0) bits = splitmix64_next(s);
            uint64_t r = (l & 1) ? (bits >> 32) : (bits & 0xFFFFFFFFull);
            uint32_t bu = r >= tb, bv = (r >= ta && r < tb) || r >= tc;
            u = (u << 1) | bu;
            v = (v << 1) | bv;
        }
        edges[size_t(i)] = {(int32_t)u, (int32_t)v};
    }
    build_csr(int32_t(1) << scale, edges, g);
}

void gen_barabasi_albert(int32_t n, int32_t m, uint64_t seed, HostGraph &g) {
    std::vector<std::pair<int32_t, int32_t>> edges;
    gen_barabasi_albert_edges(n, m, seed, edges);
    build_csr(std::max(n, 0), edges, g);
}

void gen_barabasi_albert_edges(int32_t n, int32_t m, uint64_t seed,
                               std::vector<std::pair<int32_t, int32_t>> &edges) {
    edges.clear();
    if (m < 1 || n <= m) return;
    uint64_t s = stream_state(seed, 0);
    // `ends` holds every edge endpoint, so a uniform pick from it is a pick
    // proportional to degree.
    std::vector<int32_t> ends;
    ends.reserve(size_t(n) * m * 2);
    for (int32_t i = 0; i <= m; i++)
        for (int32_t j = 0; j < i; j++) {
            edges.emplace_back(i, j);
            ends.push_back(i);
            ends.push_back(j);
        }
    std::vector<int32_t> pick;
    for (int32_t v = m + 1; v < n; v++) {
        pick.clear();
        while ((int32_t)pick.size() < m) {
            int32_t t = ends[splitmix64_next(s) % ends.size()];
            if (std::find(pick.begin(), pick.end(), t) == pick.end())
                pick.push_back(t);
        }
        for (int32_t t : pick) {
            edges.emplace_back(v, t);
            ends.push_back(v);
            ends.push_back(t);
        }
    }
}

void relabel_by_degree(const HostGraph &in, HostGraph &out,
                       std::vector<int32_t> *new_of_old) {
    const int32_t V = in.V;
    std::vector<int32_t> order(static_cast<size_t>(V));
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int32_t x, int32_t y) {
        return in.degree(x) > in.degree(y);
    });
    std::vector<int32_t> nid(static_cast<size_t>(V));
    for (int32_t r = 0; r < V; r++) nid[order[r]] = r;
    out = HostGraph{};
    out.V = V;
    out.E = in.E;
    out.off.assign(size_t(V) + 1, 0);
    for (int32_t r = 0; r < V; r++) out.off[r + 1] = out.off[r] + in.degree(order[r]);
    out.adj.resize(size_t(in.E));
#pragma omp parallel for schedule(dynamic, 1024)
    for (int32_t r = 0; r < V; r++) {
        int32_t o = order[r];
        int64_t w = out.off[r];
        for (int64_t i = in.off[o]; i < in.off[o + 1]; i++)
            out.adj[w++] = nid[in.adj[i]];
        std::sort(out.adj.begin() + out.off[r], out.adj.begin() + out.off[r + 1]);
    }
    if (new_of_old) *new_of_old = nid;
}

}  // namespace gat
