// Internal host-side types of libgat: pattern, reference-compatible schedule,
// the exact planner and the device plan that the CUDA engine interprets.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

#include "gat_plan.h"

namespace gat {

constexpr int kMaxV = GAT_MAX_VERTICES;

// A pattern graph on n <= 10 vertices, adjacency as bit rows.
// Parsing follows core/pattern.hpp:22-39: n is the first n in [1, len) with
// n*n == len, and (i, j) is an edge if either triangle of the string holds '1'.
struct Pattern {
    int n = 0;
    uint16_t row[kMaxV] = {};
    bool has(int u, int v) const { return (row[u] >> v) & 1u; }
    void add(int u, int v) {
        row[u] |= uint16_t(1u << v);
        row[v] |= uint16_t(1u << u);
    }
    int edges() const;
    bool operator==(const Pattern &o) const;
    // New vertex perm[i] plays the role of old vertex i
    // (core/pattern.hpp:74-82).
    Pattern permuted(const std::vector<int> &perm) const;
    std::string adjacency() const;
    static bool parse(const std::string &s, Pattern &out);
};

// Every vertex after the first is adjacent to an earlier one
// (core/pattern.hpp:85-101).
bool pattern_valid(const Pattern &p);
bool pattern_connected(const Pattern &p);
// Number of trailing vertices that are pairwise independent, as
// core/schedule.hpp:66-83 computes it (never below 1 for n >= 3).
int iep_suffix_count(const Pattern &p);
// Automorphisms in lexicographic (std::next_permutation) order
// (core/schedule.hpp:173-187).
std::vector<std::vector<int>> automorphisms(const Pattern &p);

using Pairs = std::vector<std::pair<int, int>>;

// The data-graph independent part of a schedule: prefixes (dependency sets),
// fathers, loop sets and IEP bookkeeping, built from a permuted pattern and a
// suffix size the way core/schedule.hpp:575-862 does.
struct Structure {
    int n = 0, basic = 0, suffix = 0;
    std::vector<std::vector<int>> prefix;  // sorted ascending vertex ids
    std::vector<int> father;               // -1: none
    std::vector<int> size_only;            // 1: no child prefix
    std::vector<int> loop_prefix;          // per basic vertex, [0] = -1
    std::vector<int> vertex_prefix_start;  // per basic vertex, + total at end
    std::vector<int> iep_vertex_id;        // IEP slot -> prefix id
    std::vector<int> iep_ans_pos;          // subgroup -> IEP slot
    std::vector<int> iep_coef;             // subgroup -> coefficient
    std::vector<int> iep_flag;             // subgroup -> closes a group
};

bool build_structure(const Pattern &permuted, int suffix, Structure &out,
                     std::string *err);

// A schedule reproducing the reference's Core::Schedule for the same pattern
// string, field for field (core/schedule.hpp:864-958, 984-1022).
struct RefSchedule {
    Pattern pattern;           // as given
    Pattern permuted;          // pattern after best_perm
    std::vector<int> perm;
    Pairs best_restrictions;   // in generation order
    Structure st;
    Pairs restrictions;        // sorted by (second, first), second < basic
    std::vector<int> restrictions_start;     // basic entries
    std::vector<int> sd_restrictions_start;  // basic + 1 entries
    bool ub_read = false;      // the start scan evaluated an element past the
                               // end of the filtered list
    bool ub_uninit = false;    // a restriction range reaches a ScheduleData
                               // slot the reference never initialises, or an
                               // embedding slot not yet chosen
    bool ub_loopset = false;   // a loop set is an unmaterialised size-only
                               // prefix
    int64_t aut = 0;
};

bool build_ref_schedule(const Pattern &p, RefSchedule &out, std::string *err);
std::string ref_schedule_json(const RefSchedule &s);

// Estimated cost of a restriction set (core/schedule.hpp:362-437) with the
// given graph statistics.
double estimate_restrictions(const Pattern &p, const Pairs &restrictions,
                             int v_cnt, int64_t e_cnt, long long tri_cnt);

// Plans.
enum class Mode { Exact = 0, RefCompat = 1 };

struct PlanInfo {
    GatPlan plan{};
    std::vector<int> perm;         // pattern vertex order
    Pairs restrictions;            // (i, u): v_u < v_i
    int64_t aut = 0;
    std::string summary;
};

// Device plan reproducing the reference engine's count for this schedule.
bool plan_from_ref(const RefSchedule &s, PlanInfo &out, std::string *err);

struct GraphStats {
    int64_t v = 5000, e = 1000000, tri = 10000;  // reference defaults
};

// Device plan for the exact (non-induced subgraph) count.  Candidate vertex
// orders are ranked by the reference's cost formula; `variant` picks the
// variant-th distinct plan in that ranking (0 = the cheapest), and
// *num_variants (when given) receives how many distinct plans there are
// (at most 16).
bool plan_exact(const Pattern &p, const GraphStats &gs, PlanInfo &out, std::string *err,
                int variant = 0, int *num_variants = nullptr);

// All connected patterns on n vertices, one per isomorphism class, each in
// its lexicographically smallest adjacency string.
std::vector<std::string> enumerate_connected_patterns(int n);

}  // namespace gat
