// Test infrastructure (oracle side): dumps the reference's own Core::Schedule
// for a list of pattern adjacency strings, one JSON object per line.
//
// This driver is compiled against the reference headers where they lie
// (include/core/schedule.hpp) by oracle/Makefile into oracle/_ref/; it never
// ships with the product.  The JSON it prints is the golden schedule set that
// the product's schedule generator is checked against
// (tests/golden/ref_schedules.jsonl, made by tests/golden/make_golden.py).
//
// Reads patterns (one per line) from stdin.  For each it records:
//  * the best permutation and restriction list the reference picks
//    (schedule.hpp:864-958; printed on stdout by the constructor, captured
//    here by swapping std::cout's buffer),
//  * every public Schedule member (schedule.hpp:592-612),
//  * the ScheduleData view the kernels see (schedule.hpp:984-1022),
//  * whether build_restrictions (schedule.hpp:820-845) evaluated
//    restrictions[i] with i >= restrictions.size() in its while condition
//    (an out-of-bounds read whose result is undefined).
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#include "core/schedule.hpp"

static void print_vec(std::ostream &o, const std::vector<int> &v) {
    o << "[";
    for (size_t i = 0; i < v.size(); i++) o << (i ? "," : "") << v[i];
    o << "]";
}

static std::vector<int> parse_ints_after(const std::string &text,
                                         const std::string &tag) {
    std::vector<int> out;
    size_t p = text.find(tag);
    if (p == std::string::npos) return out;
    size_t e = text.find('\n', p);
    std::string line = text.substr(p + tag.size(), e - p - tag.size());
    std::string cur;
    for (char c : line) {
        if (c >= '0' && c <= '9') {
            cur.push_back(c);
        } else {
            if (!cur.empty()) out.push_back(std::stoi(cur));
            cur.clear();
        }
    }
    if (!cur.empty()) out.push_back(std::stoi(cur));
    return out;
}

int main() {
    std::string adj;
    while (std::cin >> adj) {
        Core::Pattern p{adj};
        std::stringstream captured;
        std::streambuf *old = std::cout.rdbuf(captured.rdbuf());
        Core::Schedule s{p};
        Core::ScheduleData sd{s};
        int aut = Core::get_isomorphism_multiplicity(p);
        std::cout.rdbuf(old);
        std::string text = captured.str();

        std::vector<int> perm = parse_ints_after(text, "Best Permutation:");
        std::vector<int> best_r = parse_ints_after(text, "Best Restrictions:");

        // Re-run the while-condition of build_restrictions with a bounds
        // check, to flag the out-of-bounds evaluation.
        bool ub_read = false;
        {
            int cs = 0;
            int sz = (int)s.restrictions.size();
            for (int i = 0; i < s.basic_vertexes && !ub_read; i++) {
                while (cs < s.basic_vertexes) {
                    if (cs >= sz) {
                        ub_read = true;
                        break;
                    }
                    if (s.restrictions[cs].second < i)
                        cs++;
                    else
                        break;
                }
            }
        }

        std::ostream &o = std::cout;
        o << "{\"pattern\":\"" << adj << "\",\"n\":" << p.v_cnt()
          << ",\"aut\":" << aut << ",\"perm\":";
        print_vec(o, perm);
        o << ",\"best_restrictions\":[";
        for (size_t i = 0; i + 1 < best_r.size(); i += 2)
            o << (i ? "," : "") << "[" << best_r[i] << "," << best_r[i + 1]
              << "]";
        o << "],\"iep_suffix_vertexes\":" << s.iep_suffix_vertexes
          << ",\"basic_vertexes\":" << s.basic_vertexes << ",\"prefixs\":[";
        for (size_t i = 0; i < s.prefixs.size(); i++) {
            std::vector<int> d(s.prefixs[i].data,
                               s.prefixs[i].data + s.prefixs[i].depth);
            o << (i ? "," : "");
            print_vec(o, d);
        }
        o << "],\"prefixs_father\":";
        print_vec(o, s.prefixs_father);
        o << ",\"prefixs_size_only\":";
        print_vec(o, s.prefixs_size_only);
        o << ",\"loop_set_prefix_id\":";
        print_vec(o, s.loop_set_prefix_id);
        o << ",\"vertex_prefix_start\":";
        print_vec(o, s.vertex_prefix_start);
        o << ",\"restrictions\":[";
        for (size_t i = 0; i < s.restrictions.size(); i++)
            o << (i ? "," : "") << "[" << s.restrictions[i].first << ","
              << s.restrictions[i].second << "]";
        o << "],\"restrictions_start\":";
        print_vec(o, s.restrictions_start);
        o << ",\"sd_restrictions_start\":[";
        for (int i = 0; i <= s.basic_vertexes; i++)
            o << (i ? "," : "") << sd.restrictions_start[i];
        o << "],\"sd_vertex_prefix_start\":[";
        for (int i = 0; i <= s.basic_vertexes; i++)
            o << (i ? "," : "") << sd.vertex_prefix_start[i];
        o << "],\"iep_vertex_id\":";
        print_vec(o, s.iep_info.iep_vertex_id);
        o << ",\"iep_ans_pos\":";
        print_vec(o, s.iep_info.iep_ans_pos);
        o << ",\"iep_coef\":";
        print_vec(o, s.iep_info.iep_coef);
        o << ",\"iep_flag\":[";
        for (size_t i = 0; i < s.iep_info.iep_flag.size(); i++)
            o << (i ? "," : "") << (s.iep_info.iep_flag[i] ? 1 : 0);
        o << "],\"ub_read\":" << (ub_read ? "true" : "false") << "}"
          << std::endl;
    }
    return 0;
}
