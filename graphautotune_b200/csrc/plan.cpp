// Device plans.
//
// plan_from_ref: the reference engine's count for a reference schedule,
//   reproducing engine_kernel.cuh's per-unit rules (restriction ranges,
//   collision clearing, which embedded vertices each size-only set excludes,
//   and which IEP sets are subtracted).
//
// plan_exact: the true non-induced subgraph count.  Vertex order and IEP
//   structure come from the same structure builder; symmetry breaking uses
//   the Grochow-Kellis conditions ("each fixed vertex is the largest of its
//   orbit under the stabiliser of the earlier ones"), which select exactly
//   one embedding per subgraph.  Conditions on IEP suffix vertices cannot be
//   enforced inside inclusion-exclusion; they are dropped and the count is
//   divided by the (verified constant) number of surviving embeddings per
//   subgraph.
#include <algorithm>
#include <cstring>
#include <map>
#include <numeric>
#include <sstream>

#include "gat_internal.hpp"

namespace gat {

namespace {

uint16_t levels_below(int k) { return uint16_t((1u << k) - 1u); }

bool check_sizes(const Structure &st, std::string *err) {
    if ((int)st.prefix.size() > GAT_MAX_PREFIX ||
        (int)st.iep_vertex_id.size() > GAT_MAX_PREFIX ||
        (int)st.iep_ans_pos.size() > GAT_MAX_TERMS) {
        if (err) *err = "schedule exceeds plan capacity";
        return false;
    }
    return true;
}

void fill_common(const Structure &st, GatPlan &pl) {
    pl.n = st.n;
    pl.basic = st.basic;
    pl.num_prefix = (int)st.prefix.size();
    pl.iep_num = (int)st.iep_vertex_id.size();
    pl.num_terms = (int)st.iep_ans_pos.size();
    for (int p = 0; p < GAT_MAX_PREFIX; p++) pl.p_slot[p] = -1;
    for (int p = 0; p < pl.num_prefix; p++) {
        pl.p_level[p] = (int8_t)st.prefix[p].back();
        pl.p_father[p] = (int8_t)st.father[p];
    }
    const int basic = std::min(st.basic, GAT_MAX_VERTICES);
    for (int k = 0; k <= basic; k++)
        pl.l_pbegin[k] = (int8_t)st.vertex_prefix_start[k];
    for (int k = 1; k < basic; k++) pl.l_loop[k] = (int8_t)st.loop_prefix[k];
    pl.l_loop[0] = -1;
    for (int x = 0; x < pl.iep_num; x++)
        pl.iep_prefix[x] = (int8_t)st.iep_vertex_id[x];
    for (int t = 0; t < pl.num_terms; t++) {
        pl.t_slot[t] = (int8_t)st.iep_ans_pos[t];
        pl.t_close[t] = (int8_t)st.iep_flag[t];
        pl.t_coef[t] = st.iep_coef[t];
    }
}

void assign_slots(GatPlan &pl) {
    pl.num_store = 0;
    for (int p = 0; p < pl.num_prefix; p++)
        if (pl.p_kind[p] == GAT_SET_STORE) pl.p_slot[p] = (int8_t)pl.num_store++;
    // Lane-per-candidate last level: nothing at level basic-1 is stored
    // (each set is a count with a father, or the candidate's own list), and
    // at most 8 sets there and 8 IEP slots.
    const int k = pl.basic - 1;
    bool ok = pl.basic >= 2 && pl.iep_num >= 1 && pl.iep_num <= 8 &&
              pl.l_pbegin[k + 1] - pl.l_pbegin[k] <= 8;
    for (int p = pl.l_pbegin[k]; ok && p < pl.l_pbegin[k + 1]; p++)
        ok = (pl.p_kind[p] == GAT_SET_COUNT && pl.p_father[p] >= 0) ||
             pl.p_kind[p] == GAT_SET_ALIAS;
    pl.lane_last = ok ? 1 : 0;
}

uint16_t deps_mask(const std::vector<int> &d) {
    uint16_t m = 0;
    for (int v : d) m |= uint16_t(1u << v);
    return m;
}

// Grochow-Kellis symmetry-breaking conditions with the "largest of its
// orbit" convention, fixing vertices in index order.  Returns pairs (i, u)
// with i < u meaning v_u < v_i.
Pairs gk_conditions(const Pattern &q, std::vector<std::vector<int>> group) {
    Pairs r;
    for (int i = 0; i < q.n && group.size() > 1; i++) {
        std::vector<char> in(q.n, 0);
        for (auto &s : group) in[s[i]] = 1;
        for (int u = 0; u < q.n; u++)
            if (in[u] && u != i) r.emplace_back(i, u);
        std::vector<std::vector<int>> keep;
        for (auto &s : group)
            if (s[i] == i) keep.push_back(s);
        group.swap(keep);
    }
    return r;
}

// Aut(q) for q = p.permuted(pi), from Aut(p) by conjugation, in
// lexicographic order.
std::vector<std::vector<int>> conjugate_group(
    const std::vector<std::vector<int>> &autp, const std::vector<int> &pi) {
    int n = (int)pi.size();
    std::vector<std::vector<int>> out;
    for (auto &s : autp) {
        std::vector<int> t(n);
        for (int i = 0; i < n; i++) t[pi[i]] = pi[s[i]];
        out.push_back(t);
    }
    std::sort(out.begin(), out.end());
    return out;
}

// For every subgraph copy, the number of its embeddings whose values satisfy
// all conditions in r; returns that number if it is the same for all copies,
// else 0.  Copies are enumerated as the labellings of the pattern by values
// 0..n-1 (any copy in any data graph is order-isomorphic to one of these).
int64_t per_copy_multiplicity(const Pattern &q, const Pairs &r) {
    int n = q.n;
    std::vector<int> lab(n);
    std::iota(lab.begin(), lab.end(), 0);
    std::map<uint64_t, int64_t> per;
    do {
        uint64_t key = 0;
        for (int a = 0; a < n; a++)
            for (int b = a + 1; b < n; b++)
                if (q.has(a, b)) {
                    int x = std::min(lab[a], lab[b]), y = std::max(lab[a], lab[b]);
                    key |= 1ull << (x * n + y);
                }
        bool ok = true;
        for (auto &e : r)
            if (!(lab[e.second] < lab[e.first])) {
                ok = false;
                break;
            }
        per[key] += ok ? 1 : 0;
    } while (std::next_permutation(lab.begin(), lab.end()));
    int64_t c = -1;
    for (auto &kv : per) {
        if (c < 0) c = kv.second;
        if (kv.second != c) return 0;
    }
    return c < 0 ? 0 : c;
}

}  // namespace

bool plan_from_ref(const RefSchedule &s, PlanInfo &out, std::string *err) {
    out = PlanInfo{};
    if (s.ub_uninit) {
        if (err)
            *err = "reference result undefined: a restriction range reads an "
                   "uninitialised slot";
        return false;
    }
    if (s.ub_loopset) {
        if (err)
            *err = "reference result undefined: a loop set is an "
                   "unmaterialised size-only prefix";
        return false;
    }
    const Structure &st = s.st;
    if (!check_sizes(st, err)) return false;
    GatPlan &pl = out.plan;
    pl = GatPlan{};
    fill_common(st, pl);
    pl.mode = 1;
    pl.collide_clear = 1;
    pl.divisor = 1;
    for (int k = 1; k < st.basic; k++) {
        uint16_t b = 0;
        for (int i = s.sd_restrictions_start[k]; i < s.sd_restrictions_start[k + 1];
             i++)
            b |= uint16_t(1u << s.restrictions[i].first);
        pl.l_bound[k] = b;
        pl.l_distinct[k] = levels_below(k);
    }
    pl.level1_bounded = (pl.l_bound[1] & 1u) ? 1 : 0;
    for (int p = 0; p < pl.num_prefix; p++) {
        int lvl = pl.p_level[p];
        if (st.father[p] < 0) {
            pl.p_kind[p] = GAT_SET_ALIAS;
        } else if (st.size_only[p]) {
            pl.p_kind[p] = GAT_SET_COUNT;
            pl.p_excl[p] = levels_below(lvl);
        } else {
            pl.p_kind[p] = GAT_SET_STORE;
        }
        pl.p_trunc[p] = 0;
    }
    for (int x = 0; x < pl.iep_num; x++) {
        int p = pl.iep_prefix[x];
        pl.iep_sub[x] = st.size_only[p] ? 0 : levels_below(st.basic);
        pl.iep_bound[x] = 0;
    }
    assign_slots(pl);
    out.perm = s.perm;
    out.restrictions = s.restrictions;
    out.aut = s.aut;
    out.summary = "ref-compatible plan";
    return true;
}

namespace {
struct ExactCand {
    std::vector<int> perm;
    Pattern q;
    Pairs r;
    int k = 0;
    int64_t div = 1;
    double cost = 0;
};

// Device plan of one candidate vertex order (see plan_exact).
bool build_exact_plan(const Pattern &p, const ExactCand &best, int64_t aut, PlanInfo &out,
                      std::string *err);
}  // namespace

bool plan_exact(const Pattern &p, const GraphStats &gs, PlanInfo &out, std::string *err,
                int variant, int *num_variants) {
    out = PlanInfo{};
    if (p.n < 3) {
        if (err) *err = "exact plans need at least 3 vertices";
        return false;
    }
    if (!pattern_connected(p)) {
        if (err) *err = "pattern is not connected";
        return false;
    }
    auto autp = automorphisms(p);
    int kmax = 0;
    std::vector<int> perm(p.n);
    std::iota(perm.begin(), perm.end(), 0);
    do {
        Pattern q = p.permuted(perm);
        if (pattern_valid(q)) kmax = std::max(kmax, iep_suffix_count(q));
    } while (std::next_permutation(perm.begin(), perm.end()));

    // Every vertex order with the most IEP suffix vertices, cheapest first by
    // the reference's cost formula (ties in permutation order).
    std::vector<ExactCand> cands;
    for (int k = kmax; k >= 1 && cands.empty(); k--) {
        std::iota(perm.begin(), perm.end(), 0);
        do {
            Pattern q = p.permuted(perm);
            if (!pattern_valid(q) || iep_suffix_count(q) < k) continue;
            Pairs r = gk_conditions(q, conjugate_group(autp, perm));
            int basic = p.n - k;
            Pairs rb;
            for (auto &e : r)
                if (e.second < basic) rb.push_back(e);
            int64_t div = 1;
            Pairs used = r;
            if (k >= 2) {
                div = per_copy_multiplicity(q, rb);
                if (div <= 0) continue;
                used = rb;
            }
            double cost = estimate_restrictions(q, used, (int)gs.v, gs.e, gs.tri);
            cands.push_back(ExactCand{perm, q, used, k, div, cost});
        } while (std::next_permutation(perm.begin(), perm.end()));
    }
    if (cands.empty()) {
        if (err) *err = "no exact schedule found";
        return false;
    }
    std::stable_sort(cands.begin(), cands.end(),
                     [](const ExactCand &x, const ExactCand &y) { return x.cost < y.cost; });
    // Variant i = the i-th distinct device plan in that order (orders that
    // differ by an automorphism give the same plan).
    constexpr int kMaxVariants = 16;
    std::vector<GatPlan> seen;
    bool found = false;
    for (const ExactCand &c : cands) {
        PlanInfo pi;
        if (!build_exact_plan(p, c, (int64_t)autp.size(), pi, err)) continue;
        bool dup = false;
        for (const GatPlan &g : seen) dup |= std::memcmp(&g, &pi.plan, sizeof(GatPlan)) == 0;
        if (dup) continue;
        seen.push_back(pi.plan);
        if ((int)seen.size() - 1 == variant) {
            out = std::move(pi);
            found = true;
        }
        if ((found && !num_variants) || (int)seen.size() >= kMaxVariants) break;
    }
    if (num_variants) *num_variants = (int)seen.size();
    if (!found) {
        if (err && !seen.empty()) *err = "no such schedule variant";
        return false;
    }
    return true;
}

namespace {
bool build_exact_plan(const Pattern &p, const ExactCand &best, int64_t aut, PlanInfo &out,
                      std::string *err) {
    out = PlanInfo{};
    Structure st;
    if (!build_structure(best.q, best.k, st, err)) return false;
    if (!check_sizes(st, err)) return false;
    const int basic = st.basic, n = p.n;
    GatPlan &pl = out.plan;
    pl = GatPlan{};
    fill_common(st, pl);
    pl.mode = 0;
    pl.collide_clear = 0;
    pl.divisor = best.div;
    // Candidate bounds per level, and the bound on the single IEP vertex.
    uint16_t bound[kMaxV] = {};
    for (auto &e : best.r) bound[e.second] |= uint16_t(1u << e.first);
    for (int k = 1; k < basic; k++) {
        pl.l_bound[k] = bound[k];
        uint16_t deps = deps_mask(st.prefix[st.loop_prefix[k]]);
        pl.l_distinct[k] = uint16_t(levels_below(k) & ~deps & ~bound[k]);
    }
    pl.level1_bounded = (pl.l_bound[1] & 1u) ? 1 : 0;
    std::vector<uint16_t> iep_u(pl.iep_num, 0);
    for (int x = 0; x < pl.iep_num; x++) {
        int pid = st.iep_vertex_id[x];
        uint16_t u = best.k == 1 ? bound[n - 1] : 0;
        iep_u[x] = u;
        uint16_t d = deps_mask(st.prefix[pid]);
        pl.iep_bound[x] = u;
        pl.iep_sub[x] = uint16_t(levels_below(basic) & ~d & ~u);
    }
    // Truncation: a prefix set only needs elements below every consumer's
    // bound; the usable part of each bound is its vertices at or before the
    // set's own level.  Consumers are loop uses, IEP uses, and (through
    // them) the consumers of child sets.  Masks meet by intersection; the
    // empty mask means "keep everything".
    const int P = pl.num_prefix;
    std::vector<std::vector<uint16_t>> uses(P);
    for (int k = 1; k < basic; k++) uses[st.loop_prefix[k]].push_back(bound[k]);
    for (int x = 0; x < pl.iep_num; x++)
        uses[st.iep_vertex_id[x]].push_back(iep_u[x]);
    std::vector<uint16_t> trunc(P, 0);
    std::vector<char> has_trunc(P, 0);
    // Children have larger ids than fathers after sorting by level, so a
    // reverse sweep sees every child before its father.
    std::vector<std::vector<uint16_t>> all_uses = uses;
    for (int q = P - 1; q >= 0; q--) {
        int f = st.father[q];
        if (f >= 0)
            for (uint16_t m : all_uses[q]) all_uses[f].push_back(m);
    }
    for (int q = 0; q < P; q++) {
        uint16_t lvl_mask = levels_below(pl.p_level[q] + 1);
        uint16_t m = 0xFFFF;
        bool any = false;
        for (uint16_t u : all_uses[q]) {
            m &= uint16_t(u & lvl_mask);
            any = true;
        }
        trunc[q] = any ? m : 0;
    }
    for (int q = 0; q < P; q++) {
        int lvl = pl.p_level[q];
        pl.p_trunc[q] = trunc[q];
        if (st.father[q] < 0) {
            pl.p_kind[q] = GAT_SET_ALIAS;
            continue;
        }
        bool count_ok = false;
        if (st.size_only[q]) {
            // Only IEP uses remain for a childless set; it can be counted at
            // creation if every exclusion and bound is already known.
            count_ok = true;
            for (int x = 0; x < pl.iep_num; x++) {
                if (st.iep_vertex_id[x] != q) continue;
                uint16_t need = pl.iep_sub[x] | pl.iep_bound[x];
                if (need & ~levels_below(lvl + 1)) count_ok = false;
            }
            bool is_iep = false;
            for (int x = 0; x < pl.iep_num; x++)
                if (st.iep_vertex_id[x] == q) is_iep = true;
            if (!is_iep) count_ok = false;
        }
        if (count_ok) {
            pl.p_kind[q] = GAT_SET_COUNT;
            uint16_t ex = 0, bd = 0;
            for (int x = 0; x < pl.iep_num; x++)
                if (st.iep_vertex_id[x] == q) {
                    ex = pl.iep_sub[x];
                    bd = pl.iep_bound[x];
                }
            pl.p_excl[q] = ex;
            pl.p_trunc[q] = bd;  // a count set's bound is its own IEP bound
        } else {
            pl.p_kind[q] = GAT_SET_STORE;
        }
    }
    assign_slots(pl);
    out.perm = best.perm;
    out.restrictions = best.r;
    out.aut = aut;
    std::ostringstream o;
    o << "exact plan: suffix " << best.k << ", divisor " << best.div
      << ", cost " << best.cost;
    out.summary = o.str();
    // The 4-cycle (4 vertices, 4 edges, every degree 2) has a dedicated
    // wedge-aggregation kernel; this plan remains its fallback.
    if (p.n == 4 && p.edges() == 4) {
        bool cyc = true;
        for (int i = 0; i < 4; i++) cyc &= __builtin_popcount(p.row[i]) == 2;
        if (cyc) pl.special = GAT_SPECIAL_C4;
    }
    // Complete patterns on 4..7 vertices have the bit-matrix clique kernels
    // when the plan roots each clique at its largest vertex: every enumerated
    // level below all earlier ones and divisor 1 (so the counted vertex is
    // the smallest).
    if (p.n >= 4 && p.n <= 7 && p.edges() == p.n * (p.n - 1) / 2 && pl.divisor == 1 &&
        pl.level1_bounded) {
        bool chain = true;
        for (int k = 1; k < pl.basic; k++) chain &= pl.l_bound[k] == (1u << k) - 1u;
        if (chain) pl.special = GAT_SPECIAL_CLIQUE;
    }
    return true;
}
}  // namespace

}  // namespace gat
