// Test / baseline infrastructure (oracle side): runs the reference's own naive
// nested-loop matcher (target/naive_pm.cu:10-44, pattern_matching_func) on a
// bounded sample of first-level vertices, on all host threads.
//
// The reference file is compiled where it lies (oracle/Makefile passes
// -I <reference root>); its main() is renamed so this driver can call the
// recursive matcher directly with the first pattern vertex pinned:
// pattern_matching_func(1, {v0}, graph, pattern) counts the labelled
// embeddings whose pattern vertex 0 maps to v0, so summing it over all v0
// equals naive_pm's Answer (target/naive_pm.cu:53-72).  The reference keeps
// the count in an int; per-v0 counts on the sampled roots stay far below
// 2^31, and the sum here is 64-bit.
//
// usage: naive_sample <graph.bin> <pattern_adj> <first_v0> <num_v0> <stride>
//                     [threads]
//   samples v0 = first_v0 + i*stride, i in [0, num_v0), v0 < V
//        naive_sample <graph.bin> <pattern_adj> - <threads>
//   reads work units from stdin, one per line: "v0" (a whole root) or
//   "v0 v1" (the embeddings whose pattern vertices 0 and 1 map to v0 and v1:
//   pattern_matching_func(2, {v0, v1}, ...), which is the part of root v0's
//   search below the level-1 candidate v1; the caller passes only v1 that
//   the matcher's level-1 checks accept), optionally followed by a group id
//   in [0, 64) (default 0)
// prints one line: "labelled <sum> seconds <t> roots <k> threads <T>", then
// one line per group that had units: "group <g> labelled <sum> thread_seconds
// <s> units <n>" (thread_seconds sums the per-unit wall times)
#include <omp.h>

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

#define main reference_naive_pm_main
#include "target/naive_pm.cu"
#undef main

int main(int argc, char **argv) {
    bool from_stdin = argc >= 4 && std::string(argv[3]) == "-";
    if (argc < 6 && !from_stdin) {
        std::fprintf(stderr,
                     "usage: %s graph.bin pattern first num stride [threads]\n"
                     "       %s graph.bin pattern - [threads] < roots\n",
                     argv[0], argv[0]);
        return 2;
    }
    std::ifstream f{argv[1], std::ios::binary};
    if (!f.is_open()) {
        std::fprintf(stderr, "cannot open %s\n", argv[1]);
        return 2;
    }
    Infra::GlobalMemoryGraph<default_config> g{f, true};
    Core::Pattern p{std::string(argv[2])};
    std::vector<long long> roots, second;  // second[i] < 0: whole root
    std::vector<int> group;
    int threads = omp_get_max_threads();
    if (from_stdin) {
        if (argc > 4) threads = std::atoi(argv[4]);
        std::string line;
        while (std::getline(std::cin, line)) {
            std::istringstream is(line);
            long long v, w;
            if (!(is >> v) || v < 0 || v >= g.v_cnt()) continue;
            int grp = 0;
            if (!(is >> w)) w = -1;
            else if (!(is >> grp) || grp < 0 || grp >= 64) grp = 0;
            if (w >= g.v_cnt()) continue;
            roots.push_back(v);
            second.push_back(w);
            group.push_back(grp);
        }
    } else {
        long long first = std::atoll(argv[3]);
        long long num = std::atoll(argv[4]);
        long long stride = std::atoll(argv[5]);
        if (argc > 6) threads = std::atoi(argv[6]);
        for (long long i = 0; i < num; i++) {
            long long v = first + i * stride;
            if (v >= g.v_cnt()) break;
            roots.push_back(v);
            second.push_back(-1);
            group.push_back(0);
        }
    }
    std::vector<long long> g_lab(64, 0), g_units(64, 0);
    std::vector<double> g_sec(64, 0.0);
    long long total = 0;
    auto t0 = std::chrono::steady_clock::now();
#pragma omp parallel for schedule(dynamic, 1) reduction(+ : total) \
    num_threads(threads)
    for (long long i = 0; i < (long long)roots.size(); i++) {
        auto u0 = std::chrono::steady_clock::now();
        std::vector<int> choose{(int)roots[i]};
        long long c;
        if (second[i] >= 0) {
            choose.push_back((int)second[i]);
            c = pattern_matching_func(2, choose, g, p);
        } else {
            c = pattern_matching_func(1, choose, g, p);
        }
        total += c;
        double us = std::chrono::duration<double>(std::chrono::steady_clock::now() - u0).count();
#pragma omp critical
        {
            g_lab[group[i]] += c;
            g_sec[group[i]] += us;
            g_units[group[i]]++;
        }
    }
    auto t1 = std::chrono::steady_clock::now();
    double sec = std::chrono::duration<double>(t1 - t0).count();
    std::printf("labelled %lld seconds %.6f roots %zu threads %d\n", total,
                sec, roots.size(), threads);
    for (int k = 0; k < 64; k++)
        if (g_units[k])
            std::printf("group %d labelled %lld thread_seconds %.6f units %lld\n", k,
                        g_lab[k], g_sec[k], g_units[k]);
    return 0;
}
