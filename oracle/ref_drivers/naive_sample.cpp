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
//   reads the roots (one per line) from stdin
// prints one line: "labelled <sum> seconds <t> roots <k> threads <T>"
#include <omp.h>

#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <iostream>
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
    std::vector<long long> roots;
    int threads = omp_get_max_threads();
    if (from_stdin) {
        if (argc > 4) threads = std::atoi(argv[4]);
        long long v;
        while (std::cin >> v)
            if (v >= 0 && v < g.v_cnt()) roots.push_back(v);
    } else {
        long long first = std::atoll(argv[3]);
        long long num = std::atoll(argv[4]);
        long long stride = std::atoll(argv[5]);
        if (argc > 6) threads = std::atoi(argv[6]);
        for (long long i = 0; i < num; i++) {
            long long v = first + i * stride;
            if (v >= g.v_cnt()) break;
            roots.push_back(v);
        }
    }
    long long total = 0;
    auto t0 = std::chrono::steady_clock::now();
#pragma omp parallel for schedule(dynamic, 1) reduction(+ : total) \
    num_threads(threads)
    for (long long i = 0; i < (long long)roots.size(); i++) {
        std::vector<int> choose{(int)roots[i]};
        total += pattern_matching_func(1, choose, g, p);
    }
    auto t1 = std::chrono::steady_clock::now();
    double sec = std::chrono::duration<double>(t1 - t0).count();
    std::printf("labelled %lld seconds %.6f roots %zu threads %d\n", total,
                sec, roots.size(), threads);
    return 0;
}
