// pm-compatible command line (target/pm.cu:14-90).
//
//   pm <graph.bin> <pattern_adj> [hash_code] [--mode exact|ref]
//      [--config <file with designated initializer or config.json>]
//      [--results-dir DIR] [--text] [--variant N]
//
// Prints "Answer: N" and "Time: X us (Y s)" like the reference (pm.cu:70-82);
// with a hash code it writes <results-dir>/<hash>/time.txt (seconds) and
// count.txt (utils/utils.hpp:12-52), the files the tuning driver reads
// (tuning/tuning/role/driver.py:124-128).  The timed region is the count
// call with the graph already resident, as in pm.cu:60-64.  The default mode
// is ref (the reference's semantics); --mode exact gives subgraph counts.
// Exit status is non-zero on any error, which the driver maps to an
// infinite time (driver.py:118-122).  --variant N (exact mode) counts with
// exact plan variant N (gat_schedule_build_variant), so a process-based
// tuner can time the variants too.
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <sstream>
#include <string>
#include <sys/stat.h>

#include "../../include/gat.h"

static int die(const char *what) {
    std::fprintf(stderr, "pm: %s: %s\n", what, gat_last_error());
    return 1;
}

static bool mkdir_p(const std::string &path) {
    std::string cur;
    std::stringstream ss(path);
    std::string part;
    if (!path.empty() && path[0] == '/') cur = "/";
    while (std::getline(ss, part, '/')) {
        if (part.empty()) continue;
        cur += part + "/";
        mkdir(cur.c_str(), 0755);
    }
    struct stat st;
    return stat(path.c_str(), &st) == 0 && S_ISDIR(st.st_mode);
}

int main(int argc, char **argv) {
    std::string graph, pattern, hash, results_dir = "tuning_results", config_file;
    int mode = GAT_MODE_REF_COMPAT;
    int variant = 0;
    bool binary = true;
    int pos = 0;
    for (int i = 1; i < argc; i++) {
        std::string a = argv[i];
        if (a == "--mode" && i + 1 < argc) {
            std::string m = argv[++i];
            mode = (m == "exact") ? GAT_MODE_EXACT : GAT_MODE_REF_COMPAT;
        } else if (a == "--config" && i + 1 < argc) {
            config_file = argv[++i];
        } else if (a == "--results-dir" && i + 1 < argc) {
            results_dir = argv[++i];
        } else if (a == "--text") {
            binary = false;
        } else if (a == "--variant" && i + 1 < argc) {
            variant = std::atoi(argv[++i]);
        } else if (pos == 0) {
            graph = a;
            pos++;
        } else if (pos == 1) {
            pattern = a;
            pos++;
        } else if (pos == 2) {
            hash = a;
            pos++;
        }
    }
    if (pos < 2) {
        std::fprintf(stderr, "Usage: pm <graph_name> <pattern_str> [hash_code] "
                             "[--mode exact|ref] [--config FILE] "
                             "[--results-dir DIR] [--text] [--variant N]\n");
        return 2;
    }
    std::printf("Graph Name: %s\n", graph.c_str());
    if (!hash.empty()) std::printf("Hash Code: %s\n", hash.c_str());

    gat_config cfg;
    gat_config_engine_default(&cfg);
    if (!config_file.empty()) {
        std::ifstream f(config_file);
        if (!f.is_open()) {
            std::fprintf(stderr, "pm: cannot open %s\n", config_file.c_str());
            return 1;
        }
        std::stringstream ss;
        ss << f.rdbuf();
        if (gat_config_parse(ss.str().c_str(), &cfg) != GAT_OK) return die("config");
    }
    gat_pattern *p = nullptr;
    gat_schedule *s = nullptr;
    gat_graph *g = nullptr;
    gat_executor *e = nullptr;
    if (gat_pattern_from_adj(pattern.c_str(), &p) != GAT_OK) return die("pattern");
    if (gat_graph_load(graph.c_str(), binary ? 1 : 0, &g) != GAT_OK) return die("graph");
    if (gat_schedule_build_variant(p, mode, g, variant, &s) != GAT_OK) return die("schedule");
    int32_t V = 0, md = 0;
    int64_t E = 0;
    gat_graph_info(g, &V, &E, &md);
    std::printf("Vertex Count: %d\nEdge Count: %lld\nMax Degree: %d\n", V, (long long)E, md);
    if (gat_graph_upload(g, mode == GAT_MODE_EXACT ? GAT_UPLOAD_DEGREE_ORDER : 0, nullptr) !=
        GAT_OK)
        return die("upload");
    if (gat_executor_create(&cfg, &e) != GAT_OK) return die("executor");
    std::printf("Enter the Search...\n");
    uint64_t count = 0;
    gat_stats st{};
    auto t0 = std::chrono::high_resolution_clock::now();
    if (gat_executor_count(e, g, s, nullptr, &count, &st) != GAT_OK) return die("search");
    auto t1 = std::chrono::high_resolution_clock::now();
    long long us = std::chrono::duration_cast<std::chrono::microseconds>(t1 - t0).count();
    std::printf("Time: %lld us (%g s)\n", us, double(us) / 1e6);
    if (mode == GAT_MODE_REF_COMPAT)
        std::printf("Answer: %lld\n", (long long)count);
    else
        std::printf("Answer: %llu\n", (unsigned long long)count);
    if (!hash.empty()) {
        std::string dir = results_dir + "/" + hash;
        if (!mkdir_p(dir)) {
            std::fprintf(stderr, "pm: cannot create %s\n", dir.c_str());
            return 1;
        }
        std::ofstream tf(dir + "/time.txt"), cf(dir + "/count.txt");
        if (!tf.is_open() || !cf.is_open()) {
            std::fprintf(stderr, "pm: cannot write result files\n");
            return 1;
        }
        tf << double(us) / 1e6 << std::endl;
        if (mode == GAT_MODE_REF_COMPAT)
            cf << (long long)count << std::endl;
        else
            cf << (unsigned long long)count << std::endl;
    }
    gat_executor_free(e);
    gat_schedule_free(s);
    gat_graph_free(g);
    gat_pattern_free(p);
    return 0;
}
