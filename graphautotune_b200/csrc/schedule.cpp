// Pattern handling, the reference-compatible schedule generator, and the two
// planners (reference-compatible and exact) that turn a schedule into the
// device plan interpreted by the CUDA engine.
//
// The reference-compatible generator must pick the same vertex order and the
// same restriction set as core/schedule.hpp:864-958, so the decision sequence
// (candidate order, tie breaking, the floating-point cost formula) is kept
// step for step; the data structures are this library's own.
#include <algorithm>
#include <cmath>
#include <map>
#include <numeric>
#include <queue>
#include <set>
#include <sstream>

#include "gat_internal.hpp"

namespace gat {

// ------------------------------------------------------------------ pattern

int Pattern::edges() const {
    int c = 0;
    for (int i = 0; i < n; i++) c += __builtin_popcount(row[i]);
    return c / 2;
}

bool Pattern::operator==(const Pattern &o) const {
    if (n != o.n) return false;
    for (int i = 0; i < n; i++)
        if (row[i] != o.row[i]) return false;
    return true;
}

Pattern Pattern::permuted(const std::vector<int> &perm) const {
    Pattern q;
    q.n = n;
    for (int i = 0; i < n; i++)
        for (int j = 0; j < n; j++)
            if (has(i, j)) q.add(perm[i], perm[j]);
    return q;
}

std::string Pattern::adjacency() const {
    std::string s(size_t(n) * n, '0');
    for (int i = 0; i < n; i++)
        for (int j = 0; j < n; j++)
            if (has(i, j)) s[size_t(i) * n + j] = '1';
    return s;
}

bool Pattern::parse(const std::string &s, Pattern &out) {
    out = Pattern{};
    int len = (int)s.size();
    int n = 0;
    for (int k = 1; k < len; k++)
        if (k * k == len) {
            n = k;
            break;
        }
    if (n < 1 || n > kMaxV) return false;
    for (char c : s)
        if (c != '0' && c != '1') return false;
    out.n = n;
    for (int i = 0; i < n; i++)
        for (int j = 0; j < i; j++)
            if (s[size_t(i) * n + j] == '1' || s[size_t(j) * n + i] == '1')
                out.add(i, j);
    return true;
}

bool pattern_valid(const Pattern &p) {
    for (int i = 1; i < p.n; i++)
        if ((p.row[i] & ((1u << i) - 1u)) == 0) return false;
    return true;
}

bool pattern_connected(const Pattern &p) {
    if (p.n == 0) return false;
    uint32_t seen = 1, frontier = 1;
    while (frontier) {
        uint32_t next = 0;
        for (int i = 0; i < p.n; i++)
            if (frontier >> i & 1) next |= p.row[i];
        next &= ~seen;
        seen |= next;
        frontier = next;
    }
    return seen == (1u << p.n) - 1u;
}

int iep_suffix_count(const Pattern &p) {
    for (int k = 2; k <= p.n - 2; k++) {
        int first = p.n - k;
        uint32_t later = ((1u << p.n) - 1u) & ~((1u << (first + 1)) - 1u);
        if (p.row[first] & later) return k - 1;
    }
    return p.n - 2;
}

std::vector<std::vector<int>> automorphisms(const Pattern &p) {
    std::vector<std::vector<int>> out;
    std::vector<int> perm(p.n);
    std::iota(perm.begin(), perm.end(), 0);
    do {
        if (p.permuted(perm) == p) out.push_back(perm);
    } while (std::next_permutation(perm.begin(), perm.end()));
    return out;
}

// ------------------------------------------------ restriction generation
// Symmetry-breaking candidates as the reference derives them
// (core/schedule.hpp:193-360).

namespace {

using Cycles = std::vector<std::vector<int>>;

// Cycle decomposition, each cycle started at its smallest unused vertex.
Cycles cycles_of(const std::vector<int> &perm) {
    int n = (int)perm.size();
    std::vector<char> used(n, 0);
    Cycles res;
    for (int i = 0; i < n; i++) {
        if (used[i]) continue;
        std::vector<int> c{i};
        used[i] = 1;
        for (int x = perm[i]; !used[x]; x = perm[x]) {
            used[x] = 1;
            c.push_back(x);
        }
        res.push_back(std::move(c));
    }
    return res;
}

// Kahn's algorithm over the pair list (duplicates counted per occurrence).
bool acyclic(const Pairs &pairs, int n) {
    std::vector<int> indeg(n, 0);
    for (auto &e : pairs) indeg[e.second]++;
    std::queue<int> q;
    for (int i = 0; i < n; i++)
        if (indeg[i] == 0) q.push(i);
    int seen = 0;
    while (!q.empty()) {
        int x = q.front();
        q.pop();
        seen++;
        for (auto &e : pairs)
            if (e.first == x && --indeg[e.second] == 0) q.push(e.second);
    }
    return seen == n;
}

void pair_search(const Pairs &dag, std::vector<std::vector<int>> autos,
                 std::vector<Cycles> cyc, std::vector<Pairs> &out, int n) {
    std::vector<std::vector<int>> keep_a;
    std::vector<Cycles> keep_c;
    for (size_t i = 0; i < autos.size(); i++) {
        Pairs test = dag;
        for (auto &e : dag)
            test.emplace_back(autos[i][e.first], autos[i][e.second]);
        if (acyclic(test, n)) {
            keep_a.push_back(autos[i]);
            keep_c.push_back(cyc[i]);
        }
    }
    if (keep_a.size() == 1) {
        out.push_back(dag);
        return;
    }
    for (size_t i = 0; i < keep_c.size(); i++) {
        for (const auto &c : keep_c[i]) {
            if (c.size() != 2) continue;
            auto next_a = keep_a;
            auto next_c = keep_c;
            next_a.erase(next_a.begin() + i);
            next_c.erase(next_c.begin() + i);
            Pairs next = dag;
            next.emplace_back(c[0], c[1]);
            pair_search(next, next_a, next_c, out, n);
        }
    }
}

// Permutations of 0..n-1 whose values satisfy value[first] < value[second]
// for every pair (core/schedule.hpp:126-146); -1 for n >= 10.
long long count_in_complete(int n, const Pairs &r) {
    if (n >= 10) return -1;
    std::vector<int> d(n);
    std::iota(d.begin(), d.end(), 0);
    long long c = 0;
    do {
        bool ok = true;
        for (auto &e : r)
            if (!(d[e.first] < d[e.second])) {
                ok = false;
                break;
            }
        c += ok;
    } while (std::next_permutation(d.begin(), d.end()));
    return c;
}

std::vector<Pairs> restriction_candidates(const Pattern &p) {
    auto autos = automorphisms(p);
    std::vector<Cycles> cyc;
    for (auto &a : autos) cyc.push_back(cycles_of(a));
    Pairs base;
    std::vector<std::vector<int>> rest_a;
    std::vector<Cycles> rest_c;
    for (size_t i = 0; i < autos.size(); i++) {
        int twos = 0;
        std::pair<int, int> found{0, 0};
        for (auto &c : cyc[i]) {
            if (c.size() == 2) {
                twos++;
                found = {c[0], c[1]};
            } else if (c.size() != 1) {
                twos = -1;
                break;
            }
        }
        if (twos == 1) {
            base.push_back(found);
        } else {
            rest_a.push_back(autos[i]);
            rest_c.push_back(cyc[i]);
        }
    }
    std::vector<Pairs> all;
    pair_search(base, rest_a, rest_c, all, p.n);
    long long want = count_in_complete(p.n, {}) / (long long)autos.size();
    std::vector<Pairs> ok;
    for (auto &r : all)
        if (count_in_complete(p.n, r) == want) ok.push_back(r);
    return ok;
}

}  // namespace

namespace {

// Survival fractions of a restriction list: f[i] = the share of the n!
// labellings of the pattern's vertices by 0..n-1 in which restrictions
// 0..i all hold (value of .first above value of .second), then made
// conditional: f[i] / f[i-1].  Counts are integers and n! is exact in a
// double, so the shares are computed as count / n! before the division.
std::vector<double> survival_fractions(int n, const Pairs &rs) {
    const int nr = (int)rs.size();
    std::vector<double> f(nr, 0.0);
    std::vector<int> lab(n);
    std::iota(lab.begin(), lab.end(), 0);
    do {
        int held = 0;
        while (held < nr && lab[rs[held].first] > lab[rs[held].second]) held++;
        for (int i = 0; i < held; i++) f[i] += 1;
    } while (std::next_permutation(lab.begin(), lab.end()));
    double orders = 1;
    for (int i = 2; i <= n; i++) orders *= i;
    for (double &x : f) x /= orders;
    for (int i = nr - 1; i > 0; --i) f[i] /= f[i - 1];
    return f;
}

// Position (1-based, counting upwards) of vertex j among the earlier
// neighbours of vertex u, or 0 when j is not one of them.
int backward_rank(const Pattern &p, int j, int u) {
    if (j >= u || !p.has(j, u)) return 0;
    int r = 0;
    for (int x = 0; x <= j; x++) r += p.has(x, u) ? 1 : 0;
    return r;
}

}  // namespace

// The reference's cost formula for a vertex order with restrictions
// (core/schedule.hpp:362-437), on a random graph with edge density
// p0 = E / V^2 and triangle closure p1 = tri * V / E^2.  Levels are visited
// from the last enumerated one down to level 0; each level adds the search
// cost of every later enumerated vertex that intersects with it (visited in
// decreasing order), is thinned by the survival fractions of the
// restrictions on it, and is multiplied by its expected candidate count.
// The operation order is the reference's: the ranking of candidate orders
// compares these doubles, so any reordering could pick another schedule.
double estimate_restrictions(const Pattern &p, const Pairs &restrictions,
                             int v_cnt, int64_t e_cnt, long long tri_cnt) {
    const int n = p.n;
    const int enumerated = n - iep_suffix_count(p);
    Pairs rs = restrictions;
    std::sort(rs.begin(), rs.end());
    const std::vector<double> keep = survival_fractions(n, rs);
    const double p0 = e_cnt * 1.0 / v_cnt / v_cnt;
    const double p1 = tri_cnt * 1.0 * v_cnt / e_cnt / e_cnt;
    double val = 1;
    for (int level = enumerated - 1; level >= 0; --level) {
        for (int later = enumerated - 1; later > level; --later) {
            const int r = backward_rank(p, level, later);
            if (r > 1)
                val += v_cnt * p0 * std::pow(p1, r - 2) * std::log2(p0 * v_cnt);
        }
        for (size_t j = 0; j < rs.size(); j++)
            if (rs[j].second == level) val *= keep[j];
        int fwd = 0;
        for (int j = 0; j < level; j++) fwd += p.has(j, level) ? 1 : 0;
        val *= level ? v_cnt * p0 * std::pow(p1, fwd - 1) : (double)v_cnt;
    }
    return val;
}

// --------------------------------------------------------------- structure

namespace {

int insert_prefix(Structure &st, const std::vector<int> &d) {
    if (d.empty()) return -1;
    for (size_t i = 0; i < st.prefix.size(); i++)
        if (st.prefix[i] == d) return (int)i;
    std::vector<int> parent(d.begin(), d.end() - 1);
    int f = insert_prefix(st, parent);
    st.prefix.push_back(d);
    st.father.push_back(f);
    return (int)st.prefix.size() - 1;
}

// (-1)^(s-1) (s-1)!: the signed number of connected graphs on s labelled
// vertices weighted by (-1)^edges, i.e. the Moebius value of a block of
// size s in the partition lattice.
long long block_moebius(int s) {
    long long f = 1;
    for (int i = 2; i < s; i++) f *= i;
    return (s % 2 == 1) ? f : -f;
}

struct IepGroup {
    std::vector<std::vector<int>> blocks;
    long long coef;
};

// Set partitions of the suffix in the reference's enumeration order
// (core/schedule.hpp:526-572): a new block first, then the existing blocks.
void set_partitions(int depth, std::vector<int> &id, int blocks, int k,
                    std::vector<IepGroup> &out) {
    if (depth == k) {
        IepGroup g;
        g.coef = 1;
        for (int b = 0; b < blocks; b++) {
            std::vector<int> cur;
            for (int v = 0; v < k; v++)
                if (id[v] == b) cur.push_back(v);
            g.coef *= block_moebius((int)cur.size());
            g.blocks.push_back(cur);
        }
        out.push_back(g);
        return;
    }
    id[depth] = blocks;
    set_partitions(depth + 1, id, blocks + 1, k, out);
    for (int b = 0; b < blocks; b++) {
        id[depth] = b;
        set_partitions(depth + 1, id, blocks, k, out);
    }
}

}  // namespace

bool build_structure(const Pattern &p, int suffix, Structure &st,
                     std::string *err) {
    st = Structure{};
    if (!pattern_valid(p)) {
        if (err) *err = "pattern order has a vertex with no earlier neighbour";
        return false;
    }
    st.n = p.n;
    st.suffix = suffix;
    st.basic = p.n - suffix;
    if (st.basic < 1) {
        if (err) *err = "no basic vertex";
        return false;
    }
    for (int i = 0; i < st.basic; i++) {
        std::vector<int> d;
        for (int j = 0; j < i; j++)
            if (p.has(i, j)) d.push_back(j);
        insert_prefix(st, d);
    }
    std::vector<IepGroup> groups;
    std::vector<int> id(suffix, 0);
    set_partitions(0, id, 0, suffix, groups);
    for (auto &g : groups) {
        for (size_t b = 0; b < g.blocks.size(); b++) {
            std::vector<int> d;
            for (int i = 0; i < st.basic; i++)
                for (int v : g.blocks[b])
                    if (p.has(i, st.basic + v)) {
                        d.push_back(i);
                        break;
                    }
            int pid = insert_prefix(st, d);
            if (pid < 0) {
                if (err) *err = "suffix vertex without basic neighbour";
                return false;
            }
            auto it = std::find(st.iep_vertex_id.begin(),
                                st.iep_vertex_id.end(), pid);
            int slot = (int)(it - st.iep_vertex_id.begin());
            if (it == st.iep_vertex_id.end()) st.iep_vertex_id.push_back(pid);
            st.iep_ans_pos.push_back(slot);
            bool last = b + 1 == g.blocks.size();
            st.iep_coef.push_back(last ? (int)g.coef : 0);
            st.iep_flag.push_back(last ? 1 : 0);
        }
    }
    // Order prefixes by (last vertex, insertion index) and remap fathers and
    // IEP slots (core/schedule.hpp:614-652).
    int P = (int)st.prefix.size();
    std::vector<int> order(P);
    std::iota(order.begin(), order.end(), 0);
    std::sort(order.begin(), order.end(), [&](int a, int b) {
        return std::make_pair(st.prefix[a].back(), a) <
               std::make_pair(st.prefix[b].back(), b);
    });
    std::vector<int> inv(P);
    for (int i = 0; i < P; i++) inv[order[i]] = i;
    std::vector<std::vector<int>> pre2(P);
    std::vector<int> fa2(P);
    for (int i = 0; i < P; i++) {
        pre2[i] = st.prefix[order[i]];
        int f = st.father[order[i]];
        fa2[i] = f < 0 ? -1 : inv[f];
    }
    st.prefix = pre2;
    st.father = fa2;
    for (auto &v : st.iep_vertex_id) v = inv[v];
    // Loop sets and per-vertex prefix ranges (core/schedule.hpp:786-818).
    st.loop_prefix.assign(1, -1);
    for (int i = 1; i < st.basic; i++) {
        std::vector<int> d;
        for (int j = 0; j < i; j++)
            if (p.has(j, i)) d.push_back(j);
        auto it = std::find(st.prefix.begin(), st.prefix.end(), d);
        if (it == st.prefix.end()) {
            if (err) *err = "loop-set prefix missing";
            return false;
        }
        st.loop_prefix.push_back((int)(it - st.prefix.begin()));
    }
    int cur = 0;
    for (int i = 0; i < st.basic; i++) {
        st.vertex_prefix_start.push_back(cur);
        while (cur < P && st.prefix[cur].back() == i) cur++;
    }
    st.vertex_prefix_start.push_back(P);
    // A prefix without children only ever needs its size
    // (core/schedule.hpp:847-862).
    std::vector<int> child(P, 0);
    for (int i = 0; i < P; i++)
        if (st.father[i] >= 0) child[st.father[i]] = 1;
    st.size_only.resize(P);
    for (int i = 0; i < P; i++) st.size_only[i] = child[i] ? 0 : 1;
    return true;
}

// -------------------------------------------------- reference schedule

bool build_ref_schedule(const Pattern &p, RefSchedule &s, std::string *err) {
    s = RefSchedule{};
    s.pattern = p;
    if (p.n < 2) {
        if (err) *err = "pattern needs at least 2 vertices";
        return false;
    }
    if (p.n >= 10) {
        if (err)
            *err = "the reference validates restrictions only below 10 "
                   "vertices";
        return false;
    }
    std::vector<int> perm(p.n), best_perm;
    std::iota(perm.begin(), perm.end(), 0);
    Pairs best_r;
    int best_k = -1;
    double best_cost = 1e18;
    bool have = false;
    do {
        Pattern q = p.permuted(perm);
        if (!pattern_valid(q)) continue;
        int k = iep_suffix_count(q);
        if (k < best_k) continue;
        if (k > best_k) {
            best_k = k;
            best_cost = 1e18;
            have = false;
        }
        for (const Pairs &r : restriction_candidates(q)) {
            double est = estimate_restrictions(q, r, 5000, 1000000, 10000);
            if (!have || est < best_cost) {
                have = true;
                best_cost = est;
                best_perm = perm;
                best_r = r;
            }
        }
    } while (std::next_permutation(perm.begin(), perm.end()));
    if (!have) {
        if (err) *err = "pattern is not connected";
        return false;
    }
    s.perm = best_perm;
    s.best_restrictions = best_r;
    s.permuted = p.permuted(best_perm);
    if (!build_structure(s.permuted, iep_suffix_count(s.permuted), s.st, err))
        return false;
    const int basic = s.st.basic;
    // Restrictions sorted by (second, first); those on IEP vertices dropped
    // (core/schedule.hpp:820-831).
    Pairs sorted = best_r;
    std::sort(sorted.begin(), sorted.end(), [](auto &a, auto &b) {
        if (a.second != b.second) return a.second < b.second;
        return a.first < b.first;
    });
    for (auto &e : sorted)
        if (e.second < basic) s.restrictions.push_back(e);
    // The start scan is bounded by basic_vertexes rather than the list
    // length (core/schedule.hpp:834-844).  After std::remove_if the slots
    // past the kept elements still hold the sorted list's values there, so
    // reads up to the original length are reproduced; a read beyond it is
    // undefined in the reference and flagged.
    auto slot = [&](int i, bool &defined) -> std::pair<int, int> {
        if (i < (int)s.restrictions.size()) return s.restrictions[i];
        if (i < (int)sorted.size()) {
            s.ub_read = true;
            return sorted[i];
        }
        s.ub_read = true;
        defined = false;
        return {0, 0};
    };
    bool defined = true;
    int cs = 0;
    for (int i = 0; i < basic; i++) {
        while (cs < basic && defined) {
            auto r = slot(cs, defined);
            if (!defined) break;
            if (r.second < i)
                cs++;
            else
                break;
        }
        s.restrictions_start.push_back(cs);
    }
    if (!defined) s.ub_uninit = true;
    s.sd_restrictions_start = s.restrictions_start;
    s.sd_restrictions_start.push_back((int)s.restrictions.size());
    // Ranges the engine reads for vertices 1..basic-1 must lie inside the
    // initialised restriction slots and name already-chosen vertices.
    for (int k = 1; k < basic; k++)
        for (int i = s.sd_restrictions_start[k];
             i < s.sd_restrictions_start[k + 1]; i++)
            if (i >= (int)s.restrictions.size() ||
                s.restrictions[i].first >= k)
                s.ub_uninit = true;
    for (int k = 2; k < basic; k++) {
        int lp = s.st.loop_prefix[k];
        if (s.st.size_only[lp] && s.st.father[lp] != -1) s.ub_loopset = true;
    }
    s.aut = (int64_t)automorphisms(p).size();
    return true;
}

namespace {
void json_vec(std::ostringstream &o, const std::vector<int> &v) {
    o << "[";
    for (size_t i = 0; i < v.size(); i++) o << (i ? "," : "") << v[i];
    o << "]";
}
void json_pairs(std::ostringstream &o, const Pairs &v) {
    o << "[";
    for (size_t i = 0; i < v.size(); i++)
        o << (i ? "," : "") << "[" << v[i].first << "," << v[i].second << "]";
    o << "]";
}
}  // namespace

std::string ref_schedule_json(const RefSchedule &s) {
    std::ostringstream o;
    o << "{\"pattern\":\"" << s.pattern.adjacency() << "\",\"n\":"
      << s.pattern.n << ",\"aut\":" << s.aut << ",\"perm\":";
    json_vec(o, s.perm);
    o << ",\"best_restrictions\":";
    json_pairs(o, s.best_restrictions);
    o << ",\"iep_suffix_vertexes\":" << s.st.suffix
      << ",\"basic_vertexes\":" << s.st.basic << ",\"prefixs\":[";
    for (size_t i = 0; i < s.st.prefix.size(); i++) {
        o << (i ? "," : "");
        json_vec(o, s.st.prefix[i]);
    }
    o << "],\"prefixs_father\":";
    json_vec(o, s.st.father);
    o << ",\"prefixs_size_only\":";
    json_vec(o, s.st.size_only);
    o << ",\"loop_set_prefix_id\":";
    json_vec(o, s.st.loop_prefix);
    std::vector<int> vps(s.st.vertex_prefix_start.begin(),
                         s.st.vertex_prefix_start.end() - 1);
    o << ",\"vertex_prefix_start\":";
    json_vec(o, vps);
    o << ",\"restrictions\":";
    json_pairs(o, s.restrictions);
    o << ",\"restrictions_start\":";
    json_vec(o, s.restrictions_start);
    o << ",\"sd_restrictions_start\":";
    json_vec(o, s.sd_restrictions_start);
    o << ",\"sd_vertex_prefix_start\":";
    json_vec(o, s.st.vertex_prefix_start);
    o << ",\"iep_vertex_id\":";
    json_vec(o, s.st.iep_vertex_id);
    o << ",\"iep_ans_pos\":";
    json_vec(o, s.st.iep_ans_pos);
    o << ",\"iep_coef\":";
    json_vec(o, s.st.iep_coef);
    o << ",\"iep_flag\":";
    json_vec(o, s.st.iep_flag);
    o << ",\"ub_read\":" << (s.ub_read ? "true" : "false") << "}";
    return o.str();
}

// ------------------------------------------------------ pattern catalogue

std::vector<std::string> enumerate_connected_patterns(int n) {
    std::vector<std::string> out;
    if (n < 1 || n > 7) return out;
    int m = n * (n - 1) / 2;
    std::vector<std::pair<int, int>> slots;
    for (int i = 0; i < n; i++)
        for (int j = i + 1; j < n; j++) slots.emplace_back(i, j);
    std::set<std::string> seen;
    std::vector<int> perm(n);
    for (uint32_t mask = 0; mask < (1u << m); mask++) {
        Pattern p;
        p.n = n;
        for (int b = 0; b < m; b++)
            if (mask >> b & 1) p.add(slots[b].first, slots[b].second);
        if (!pattern_connected(p)) continue;
        std::iota(perm.begin(), perm.end(), 0);
        std::string best;
        do {
            std::string s = p.permuted(perm).adjacency();
            if (best.empty() || s < best) best = s;
        } while (std::next_permutation(perm.begin(), perm.end()));
        if (seen.insert(best).second) out.push_back(best);
    }
    std::sort(out.begin(), out.end());
    return out;
}

}  // namespace gat
