// Test infrastructure only: CPU oracle for the pattern-counting path.
// See oracle.h for the contract.  Only tests/, __graft_entry__.smoke() and
// bench.py's CPU-baseline leg load this library, as the checker; the product
// never links it.  Parity of this restatement is pinned against the
// reference's own binaries (oracle/_ref) through tests/golden/.
#include "oracle.h"

#include <omp.h>

#include <algorithm>
#include <atomic>
#include <cstring>
#include <numeric>
#include <string>
#include <vector>

namespace {

// Pattern adjacency, restating core/pattern.hpp:22-49: n is the first n with
// n*n == len; edge (i, j) exists if either triangle of the string says '1'.
struct Pat {
    int n = 0;
    unsigned char e[10][10] = {};
    explicit Pat(const char *s) {
        int len = (int)std::strlen(s);
        for (int k = 1; k < len; k++) {
            if (k * k == len) {
                n = k;
                break;
            }
        }
        if (n > 10) n = 0;
        for (int i = 0; i < n; i++)
            for (int j = 0; j < i; j++)
                if (s[i * n + j] == '1' || s[j * n + i] == '1')
                    e[i][j] = e[j][i] = 1;
    }
};

struct CSR {
    int32_t V;
    const int64_t *offs;
    const int32_t *adj;
    int64_t deg(int32_t v) const { return offs[v + 1] - offs[v]; }
    const int32_t *nb(int32_t v) const { return adj + offs[v]; }
    // graph_backend.cuh:140-147: search the shorter list.
    bool has_edge(int32_t u, int32_t v) const {
        if (deg(u) > deg(v)) std::swap(u, v);
        const int32_t *b = nb(u), *e = b + deg(u);
        const int32_t *t = std::lower_bound(b, e, v);
        return t != e && *t == v;
    }
};

// target/naive_pm.cu:10-44, with a 64-bit accumulator.
uint64_t naive_rec(const CSR &g, const Pat &p, int depth, int32_t *choose) {
    if (depth == p.n) return 1;
    uint64_t ans = 0;
    for (int32_t i = 0; i < g.V; i++) {
        bool ok = true;
        for (int j = 0; j < depth; j++) {
            bool in_pattern = p.e[j][depth];
            bool already = choose[j] == i;
            if (already || (in_pattern && !g.has_edge(choose[j], i))) {
                ok = false;
                break;
            }
        }
        if (ok) {
            choose[depth] = i;
            ans += naive_rec(g, p, depth + 1, choose);
        }
    }
    return ans;
}

uint64_t backtrack_rec(const CSR &g, const Pat &p, int depth,
                       int32_t *choose) {
    if (depth == p.n) return 1;
    // Candidate source: the smallest neighbour list among earlier pattern
    // neighbours; all vertices if there is none.
    int src = -1;
    for (int j = 0; j < depth; j++)
        if (p.e[j][depth] && (src < 0 || g.deg(choose[j]) < g.deg(choose[src])))
            src = j;
    uint64_t ans = 0;
    int64_t cnt = src < 0 ? g.V : g.deg(choose[src]);
    const int32_t *list = src < 0 ? nullptr : g.nb(choose[src]);
    for (int64_t t = 0; t < cnt; t++) {
        int32_t i = list ? list[t] : (int32_t)t;
        bool ok = true;
        for (int j = 0; j < depth && ok; j++) {
            if (choose[j] == i) ok = false;
            else if (p.e[j][depth] && j != src && !g.has_edge(choose[j], i))
                ok = false;
        }
        if (ok) {
            choose[depth] = i;
            ans += backtrack_rec(g, p, depth + 1, choose);
        }
    }
    return ans;
}

// ---------------------------------------------------------------- reference
// engine semantics

struct SD {
    int basic = 0, P = 0, R = 0, I = 0, S = 0;
    std::vector<std::vector<int>> pre;
    std::vector<int> father, size_only, vps, loop, rs, rest, vid, pos, coef,
        flag, level;
};

bool parse_sd(const int32_t *a, int32_t len, SD &sd) {
    int k = 0;
    auto take = [&](int &dst) {
        if (k >= len) return false;
        dst = a[k++];
        return true;
    };
    auto take_vec = [&](std::vector<int> &v, int cnt) {
        if (cnt < 0 || k + cnt > len) return false;
        v.assign(a + k, a + k + cnt);
        k += cnt;
        return true;
    };
    if (!take(sd.basic) || !take(sd.P) || !take(sd.R) || !take(sd.I) ||
        !take(sd.S))
        return false;
    if (sd.basic < 1 || sd.basic > 10 || sd.P < 1 || sd.P > 64) return false;
    sd.pre.resize(sd.P);
    sd.level.resize(sd.P);
    for (int i = 0; i < sd.P; i++) {
        int d;
        if (!take(d) || d < 1 || d > 10 || !take_vec(sd.pre[i], d))
            return false;
        sd.level[i] = sd.pre[i].back();
        if (sd.level[i] < 0 || sd.level[i] >= sd.basic) return false;
    }
    if (!take_vec(sd.father, sd.P) || !take_vec(sd.size_only, sd.P) ||
        !take_vec(sd.vps, sd.basic + 1) || !take_vec(sd.loop, sd.basic) ||
        !take_vec(sd.rs, sd.basic + 1) || !take_vec(sd.rest, sd.R) ||
        !take_vec(sd.vid, sd.I) || !take_vec(sd.pos, sd.S) ||
        !take_vec(sd.coef, sd.S) || !take_vec(sd.flag, sd.S))
        return false;
    for (int f : sd.father)
        if (f < -1 || f >= sd.P) return false;
    for (int v : sd.vps)
        if (v < 0 || v > sd.P) return false;
    for (int i = 1; i < sd.basic; i++)
        if (sd.loop[i] < 0 || sd.loop[i] >= sd.P) return false;
    for (int v : sd.vid)
        if (v < 0 || v >= sd.P) return false;
    for (int v : sd.pos)
        if (v < 0 || v >= sd.I) return false;
    for (int v : sd.rest)
        if (v < 0 || v >= sd.basic) return false;
    return true;
}

struct RefSet {
    const int32_t *data = nullptr;
    int64_t size = 0;
};

struct RefUnit {
    const CSR &g;
    const SD &sd;
    std::vector<std::vector<int32_t>> buf;
    std::vector<RefSet> set;
    int32_t emb[10];
    int64_t total = 0;
    uint64_t balg = 0;

    RefUnit(const CSR &g_, const SD &sd_)
        : g(g_), sd(sd_), buf(sd_.P), set(sd_.P) {}

    static bool contains(const RefSet &s, int32_t x) {
        const int32_t *e = s.data + s.size;
        const int32_t *t = std::lower_bound(s.data, e, x);
        return t != e && *t == x;
    }

    // engine_kernel.cuh:343-432 (get_iep_answer_kernel).
    void final_step() {
        int64_t ans[64];
        for (int x = 0; x < sd.I; x++) {
            int p = sd.vid[x];
            const RefSet &s = set[p];
            if (sd.size_only[p]) {
                ans[x] = s.size;
            } else {
                int64_t hit = 0;
                for (int j = 0; j < sd.basic; j++)
                    if (s.size > 0 && contains(s, emb[j])) hit++;
                ans[x] = s.size - hit;
            }
        }
        int64_t local = 0, val = 1;
        int last = -1;
        for (int gid = 0; gid < sd.S; gid++) {
            if (gid == last + 1)
                val = ans[sd.pos[gid]];
            else
                val *= ans[sd.pos[gid]];
            if (sd.flag[gid]) {
                last = gid;
                local += val * sd.coef[gid];
            }
        }
        total += local;
    }

    // engine.cuh:267-398 + engine_kernel.cuh:109-338: extend the unit at
    // level k to level k+1.
    void search(int k) {
        if (k == sd.basic - 1) {
            final_step();
            return;
        }
        const RefSet L = set[sd.loop[k + 1]];
        int32_t minv = g.V;
        for (int i = sd.rs[k + 1]; i < sd.rs[k + 2]; i++)
            minv = std::min(minv, emb[sd.rest[i]]);
        // utils/cuda_utils.cuh:59-73 lower_bound.
        int64_t cnt = std::lower_bound(L.data, L.data + L.size, minv) - L.data;
        for (int64_t idx = 0; idx < cnt; idx++) {
            int32_t v = L.data[idx];
            emb[k + 1] = v;
            bool ap = false;
            for (int j = 0; j <= k; j++) ap |= emb[j] == v;
            const int32_t *nv = g.nb(v);
            int64_t dv = g.deg(v);
            for (int p = sd.vps[k + 1]; p < sd.vps[k + 2]; p++) {
                if (ap) {
                    set[p] = RefSet{set[p].data, 0};
                    continue;
                }
                int f = sd.father[p];
                if (f == -1) {
                    set[p] = RefSet{nv, dv};
                    continue;
                }
                const RefSet &F = set[f];
                balg += 4ull * (uint64_t)(dv + F.size);
                const RefSet &a = dv <= F.size ? RefSet{nv, dv} : F;
                const RefSet &b = dv <= F.size ? F : RefSet{nv, dv};
                if (!sd.size_only[p]) {
                    std::vector<int32_t> &o = buf[p];
                    o.clear();
                    for (int64_t t = 0; t < a.size; t++)
                        if (contains(b, a.data[t])) o.push_back(a.data[t]);
                    set[p] = RefSet{o.data(), (int64_t)o.size()};
                    balg += 4ull * o.size();
                } else {
                    int64_t c = 0;
                    for (int64_t t = 0; t < a.size; t++) {
                        int32_t u = a.data[t];
                        bool emb_hit = false;
                        for (int j = 0; j <= k; j++) emb_hit |= emb[j] == u;
                        if (!emb_hit && contains(b, u)) c++;
                    }
                    set[p] = RefSet{nullptr, c};
                }
            }
            search(k + 1);
        }
    }
};

// -------------------------------------------------------- order-restricted
// labelled counting (full-size pins of the exact plans)
//
// Labelled embeddings f of the pattern, vertex by vertex in pattern order,
// with f(a) < f(b) for every listed pair.  Candidates for vertex k come from
// the shortest neighbour list among its earlier pattern neighbours, cut to
// the open interval the pairs already allow; the others are checked with
// has_edge.  The last vertex is counted, not recursed into.  None of this
// shares code or structure with the engine's prefix sets or its
// inclusion-exclusion.
struct Restricted {
    const CSR &g;
    const Pat &p;
    int lower[10][10];  // lower[k] = earlier a with f(a) < f(k)
    int nlower[10] = {};
    int upper[10][10];  // upper[k] = earlier b with f(k) < f(b)
    int nupper[10] = {};
    int32_t f[10];
    // Work cap: candidates examined, charged to a shared budget in blocks;
    // once it runs out every call returns at once and `over` is set.
    std::atomic<int64_t> *budget = nullptr;
    std::atomic<int> *over = nullptr;
    int64_t local = 0;
    bool charge(int64_t n) {
        if (!budget) return true;
        local += n;
        if (local >= 4096) {
            if (budget->fetch_sub(local) - local < 0) over->store(1);
            local = 0;
        }
        return over->load(std::memory_order_relaxed) == 0;
    }
    Restricted(const CSR &g_, const Pat &p_, const int32_t *less, int32_t nless)
        : g(g_), p(p_) {
        for (int i = 0; i < nless; i++) {
            const int a = less[2 * i], b = less[2 * i + 1];
            if (a < b)
                lower[b][nlower[b]++] = a;
            else
                upper[a][nupper[a]++] = b;
        }
    }
    uint64_t place(int k) {
        int src = -1;
        for (int j = 0; j < k; j++)
            if (p.e[j][k] && (src < 0 || g.deg(f[j]) < g.deg(f[src]))) src = j;
        int64_t lo = -1, hi = g.V;  // open interval (lo, hi)
        for (int i = 0; i < nlower[k]; i++) lo = std::max<int64_t>(lo, f[lower[k][i]]);
        for (int i = 0; i < nupper[k]; i++) hi = std::min<int64_t>(hi, f[upper[k][i]]);
        if (hi - lo < 2) return 0;
        const int32_t *b, *e;
        std::vector<int32_t> all;
        if (src >= 0) {
            const int32_t *nb = g.nb(f[src]);
            b = std::upper_bound(nb, nb + g.deg(f[src]), (int32_t)lo);
            e = std::lower_bound(b, nb + g.deg(f[src]), (int32_t)hi);
        } else {
            all.resize(size_t(hi - lo - 1));
            std::iota(all.begin(), all.end(), (int32_t)(lo + 1));
            b = all.data();
            e = b + all.size();
        }
        uint64_t n = 0;
        if (!charge(e - b)) return 0;
        for (const int32_t *it = b; it < e; ++it) {
            const int32_t x = *it;
            bool ok = true;
            for (int j = 0; j < k && ok; j++)
                ok = f[j] != x && (!p.e[j][k] || j == src || g.has_edge(f[j], x));
            if (!ok) continue;
            if (k + 1 == p.n) {
                n++;
            } else {
                f[k] = x;
                n += place(k + 1);
            }
        }
        return n;
    }
};

// Sum over roots v0 in [rb, re) of sum_x C(c(v0, x), 2), where c counts the
// common neighbours v1 of v0 and x with v1 and x both above v0 (at_largest
// = 0) or both below it (at_largest = 1): every 4-cycle once, at its
// smallest (largest) vertex and the vertex opposite it.
uint64_t c4_rooted(const CSR &g, int32_t rb, int32_t re, bool at_largest, int threads) {
    uint64_t total = 0;
#pragma omp parallel num_threads(threads) reduction(+ : total)
    {
        std::vector<uint32_t> c(size_t(g.V), 0);
        std::vector<int32_t> touched;
#pragma omp for schedule(dynamic, 1)
        for (int32_t v0 = rb; v0 < re; v0++) {
            touched.clear();
            const int32_t *n0 = g.nb(v0);
            const int64_t d0 = g.deg(v0);
            for (int64_t i = 0; i < d0; i++) {
                const int32_t v1 = n0[i];
                if (at_largest ? v1 >= v0 : v1 <= v0) continue;
                const int32_t *n1 = g.nb(v1);
                const int64_t d1 = g.deg(v1);
                for (int64_t j = 0; j < d1; j++) {
                    const int32_t x = n1[j];
                    if (at_largest ? x >= v0 : x <= v0) continue;
                    if (c[x]++ == 0) touched.push_back(x);
                }
            }
            for (int32_t x : touched) {
                total += uint64_t(c[x]) * (c[x] - 1) / 2;
                c[x] = 0;
            }
        }
    }
    return total;
}

}  // namespace

extern "C" {

uint64_t oracle_naive_labelled(int32_t V, const int64_t *offs,
                               const int32_t *adj, const char *pattern,
                               int32_t root_begin, int32_t root_end,
                               int threads) {
    CSR g{V, offs, adj};
    Pat p(pattern);
    if (p.n == 0) return 0;
    root_begin = std::max(root_begin, 0);
    root_end = std::min(root_end, V);
    uint64_t total = 0;
    if (threads <= 0) threads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 1) reduction(+ : total) \
    num_threads(threads)
    for (int32_t v0 = root_begin; v0 < root_end; v0++) {
        int32_t choose[10];
        choose[0] = v0;
        total += naive_rec(g, p, 1, choose);
    }
    return total;
}

uint64_t oracle_naive_labelled_roots(int32_t V, const int64_t *offs,
                                     const int32_t *adj, const char *pattern,
                                     const int32_t *roots, int64_t num,
                                     int threads) {
    CSR g{V, offs, adj};
    Pat p(pattern);
    if (p.n == 0) return 0;
    uint64_t total = 0;
    if (threads <= 0) threads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 1) reduction(+ : total) \
    num_threads(threads)
    for (int64_t i = 0; i < num; i++) {
        int64_t v0 = roots[i];
        if (v0 < 0 || v0 >= V) continue;
        int32_t choose[10];
        choose[0] = (int32_t)v0;
        total += naive_rec(g, p, 1, choose);
    }
    return total;
}

uint64_t oracle_backtrack_labelled(int32_t V, const int64_t *offs,
                                   const int32_t *adj, const char *pattern,
                                   int32_t root_begin, int32_t root_end,
                                   int threads) {
    CSR g{V, offs, adj};
    Pat p0(pattern);
    if (p0.n == 0) return 0;
    // Relabel the pattern into breadth-first order from vertex 0 so every
    // later vertex has an earlier neighbour (the labelled count does not
    // depend on the labelling; the search time does).
    int order[10], pos[10], cnt = 0;
    bool seen[10] = {};
    order[cnt++] = 0;
    seen[0] = true;
    while (cnt < p0.n) {
        int nxt = -1;
        for (int v = 0; v < p0.n && nxt < 0; v++)
            if (!seen[v])
                for (int i = 0; i < cnt; i++)
                    if (p0.e[v][order[i]]) {
                        nxt = v;
                        break;
                    }
        if (nxt < 0)
            for (int v = 0; v < p0.n; v++)
                if (!seen[v]) {
                    nxt = v;
                    break;
                }
        seen[nxt] = true;
        order[cnt++] = nxt;
    }
    for (int i = 0; i < p0.n; i++) pos[order[i]] = i;
    Pat p(pattern);
    for (int i = 0; i < p0.n; i++)
        for (int j = 0; j < p0.n; j++) p.e[pos[i]][pos[j]] = p0.e[i][j];
    root_begin = std::max(root_begin, 0);
    root_end = std::min(root_end, V);
    uint64_t total = 0;
    if (threads <= 0) threads = omp_get_max_threads();
#pragma omp parallel for schedule(dynamic, 1) reduction(+ : total) \
    num_threads(threads)
    for (int32_t v0 = root_begin; v0 < root_end; v0++) {
        int32_t choose[10];
        choose[0] = v0;
        total += backtrack_rec(g, p, 1, choose);
    }
    return total;
}

int64_t oracle_automorphisms(const char *pattern) {
    Pat p(pattern);
    if (p.n == 0) return 0;
    int perm[10];
    std::iota(perm, perm + p.n, 0);
    int64_t cnt = 0;
    do {
        bool same = true;
        for (int i = 0; i < p.n && same; i++)
            for (int j = 0; j < p.n; j++)
                if (p.e[i][j] != p.e[perm[i]][perm[j]]) {
                    same = false;
                    break;
                }
        cnt += same;
    } while (std::next_permutation(perm, perm + p.n));
    return cnt;
}

int oracle_ref_engine(int32_t V, const int64_t *offs, const int32_t *adj,
                      const int32_t *sd_flat, int32_t sd_len,
                      int32_t root_begin, int32_t root_end, int threads,
                      int64_t *out, uint64_t *balg) {
    SD sd;
    if (!parse_sd(sd_flat, sd_len, sd)) return -1;
    // Restriction ranges used by prepare_v_storage_kernel for vertices
    // 1..basic-1 must stay inside the initialised part of
    // ScheduleData::restrictions (core/schedule.hpp:1015-1021).
    // ... and name vertices already chosen (slot k and above is stale).
    for (int k = 1; k < sd.basic; k++)
        for (int i = sd.rs[k]; i < sd.rs[k + 1]; i++)
            if (i >= sd.R || sd.rest[i] >= k) return -2;
    for (int k = 2; k < sd.basic; k++) {
        int p = sd.loop[k];
        if (sd.size_only[p] && sd.father[p] != -1) return -3;
    }
    CSR g{V, offs, adj};
    root_begin = std::max(root_begin, 0);
    root_end = std::min(root_end, V);
    if (threads <= 0) threads = omp_get_max_threads();
    int64_t total = 0;
    uint64_t bytes = 0;
#pragma omp parallel num_threads(threads) reduction(+ : total, bytes)
    {
        RefUnit u(g, sd);
        // one root at a time: hub roots can hold most of the work
#pragma omp for schedule(dynamic, 1)
        for (int32_t v0 = root_begin; v0 < root_end; v0++) {
            // first_extend_kernel (engine_kernel.cuh:40-60): prefix 0 is
            // N(v0), the level-0 embedding is v0.
            u.emb[0] = v0;
            u.set[0] = RefSet{g.nb(v0), g.deg(v0)};
            u.search(0);
        }
        total += u.total;
        bytes += u.balg;
    }
    *out = total;
    if (balg) *balg = bytes;
    return 0;
}

int32_t oracle_intersect_size(const int32_t *a, int32_t na, const int32_t *b,
                              int32_t nb) {
    int32_t c = 0;
    for (int32_t i = 0; i < na; i++)
        if (std::binary_search(b, b + nb, a[i])) c++;
    return c;
}

uint64_t oracle_restricted_labelled(int32_t V, const int64_t *offs, const int32_t *adj,
                                    const char *pattern, const int32_t *less,
                                    int32_t nless, int32_t root_begin, int32_t root_end,
                                    int threads) {
    return oracle_restricted_labelled_capped(V, offs, adj, pattern, less, nless, root_begin,
                                             root_end, threads, -1, nullptr);
}

uint64_t oracle_restricted_labelled_capped(int32_t V, const int64_t *offs,
                                           const int32_t *adj, const char *pattern,
                                           const int32_t *less, int32_t nless,
                                           int32_t root_begin, int32_t root_end, int threads,
                                           int64_t max_work, int *over) {
    if (over) *over = 0;
    Pat p(pattern);
    if (p.n < 2 || nless < 0) return 0;
    for (int i = 0; i < 2 * nless; i++)
        if (less[i] < 0 || less[i] >= p.n) return 0;
    CSR g{V, offs, adj};
    root_begin = std::max(root_begin, 0);
    root_end = std::min(root_end, V);
    if (root_begin >= root_end) return 0;
    if (threads <= 0) threads = omp_get_max_threads();
    // Work units: (root, index of the level-1 candidate in N(root)) when
    // pattern vertex 1 is adjacent to vertex 0 (hub roots then spread over
    // the threads), else one unit per root.
    const bool by_edge = p.e[0][1];
    std::vector<int64_t> start(size_t(root_end - root_begin) + 1, 0);
    for (int32_t v = root_begin; v < root_end; v++)
        start[v - root_begin + 1] = start[v - root_begin] + (by_edge ? g.deg(v) : 1);
    const int64_t units = start.back();
    uint64_t total = 0;
    std::atomic<int64_t> budget{max_work};
    std::atomic<int> exceeded{0};
#pragma omp parallel num_threads(threads) reduction(+ : total)
    {
        Restricted r(g, p, less, nless);
        if (max_work >= 0) {
            r.budget = &budget;
            r.over = &exceeded;
        }
        int32_t row = root_begin;
#pragma omp for schedule(dynamic, 256)
        for (int64_t u = 0; u < units; u++) {
            if (start[row - root_begin] > u || start[row - root_begin + 1] <= u)
                row = root_begin + int32_t(std::upper_bound(start.begin(), start.end(), u) -
                                           start.begin() - 1);
            r.f[0] = row;
            if (!by_edge) {
                total += r.place(1);
                continue;
            }
            const int32_t x = g.nb(row)[u - start[row - root_begin]];
            bool ok = x != row;
            for (int i = 0; i < r.nlower[1] && ok; i++) ok = x > r.f[r.lower[1][i]];
            for (int i = 0; i < r.nupper[1] && ok; i++) ok = x < r.f[r.upper[1][i]];
            if (!ok) continue;
            if (p.n == 2) {
                total += 1;
                continue;
            }
            r.f[1] = x;
            total += r.place(2);
        }
    }
    if (over) *over = exceeded.load();
    return exceeded.load() ? 0 : total;
}

uint64_t oracle_c4_rooted(int32_t V, const int64_t *offs, const int32_t *adj,
                          int32_t root_begin, int32_t root_end, int at_largest,
                          int threads) {
    CSR g{V, offs, adj};
    root_begin = std::max(root_begin, 0);
    root_end = std::min(root_end, V);
    if (root_begin >= root_end) return 0;
    if (threads <= 0) threads = omp_get_max_threads();
    return c4_rooted(g, root_begin, root_end, at_largest != 0, threads);
}

int oracle_degree_order(int32_t V, const int64_t *offs, const int32_t *adj,
                        int64_t *new_offs, int32_t *new_adj) {
    if (V < 0) return -1;
    std::vector<int32_t> by_rank(static_cast<size_t>(V));
    std::iota(by_rank.begin(), by_rank.end(), 0);
    std::stable_sort(by_rank.begin(), by_rank.end(), [&](int32_t a, int32_t b) {
        return offs[a + 1] - offs[a] > offs[b + 1] - offs[b];
    });
    std::vector<int32_t> rank(static_cast<size_t>(V));
    for (int32_t r = 0; r < V; r++) rank[by_rank[r]] = r;
    new_offs[0] = 0;
    for (int32_t r = 0; r < V; r++)
        new_offs[r + 1] = new_offs[r] + (offs[by_rank[r] + 1] - offs[by_rank[r]]);
#pragma omp parallel for schedule(dynamic, 1024)
    for (int32_t r = 0; r < V; r++) {
        const int32_t v = by_rank[r];
        int32_t *out = new_adj + new_offs[r];
        for (int64_t i = offs[v]; i < offs[v + 1]; i++) *out++ = rank[adj[i]];
        std::sort(new_adj + new_offs[r], new_adj + new_offs[r + 1]);
    }
    return 0;
}

}  // extern "C"
