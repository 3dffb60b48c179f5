// Host CSR graphs: the reference's binary and text formats, seeded synthetic
// generators, and degree relabelling.
#pragma once
#include <cstdint>
#include <string>
#include <utility>
#include <vector>

namespace gat {

// Sorted, deduplicated, symmetric adjacency without self loops; offsets are
// int64 and neighbour ids int32 (infra/graph_backend.cuh:15-17,91-99).
struct HostGraph {
    int32_t V = 0;
    int64_t E = 0;  // directed entries = 2 x undirected edges
    std::vector<int64_t> off;
    std::vector<int32_t> adj;
    int64_t degree(int32_t v) const { return off[v + 1] - off[v]; }
    int32_t max_degree() const;
};

// Binary layout: int32 V, int64 E, int64 off[V+1], int32 adj[E]
// (graph_backend.cuh:91-99 reader, :163-169 writer).
bool load_binary(const std::string &path, HostGraph &g, std::string *err);
bool save_binary(const std::string &path, const HostGraph &g, std::string *err);
// Text layout: "V E" then E lines "u v"; ids are renumbered in increasing
// order of appearance value, self loops dropped, lists symmetrised, sorted
// and deduplicated (graph_backend.cuh:23-89).
bool load_text(const std::string &path, HostGraph &g, std::string *err);

// Undirected edge list -> CSR (drops self loops and duplicates).
void build_csr(int32_t V, const std::vector<std::pair<int32_t, int32_t>> &edges,
               HostGraph &g);
// Checks the CSR invariants (monotone offsets, ids in range, sorted unique
// rows, no self loops, symmetric).  `check_symmetry` is O(E log d).
bool validate(const HostGraph &g, bool check_symmetry, std::string *err);

// splitmix64 (Steele, Lea, Flood 2014): the one generator used for every
// synthetic graph; stream i of seed s starts at state mix(s) + i * gamma.
uint64_t splitmix64_next(uint64_t &state);

// Erdos-Renyi G(n, p) with p = avg_degree / (n - 1), by geometric skipping
// (Batagelj & Brandes 2005).
void gen_erdos_renyi(int32_t n, double avg_degree, uint64_t seed, HostGraph &g);
// R-MAT (Chakrabarti, Zhan, Faloutsos 2004): `samples` edge draws on 2^scale
// vertices with quadrant probabilities a, b, c (d = 1 - a - b - c); sample i
// uses its own splitmix64 stream, so the result does not depend on threads.
void gen_rmat(int scale, int64_t samples, double a, double b, double c,
              uint64_t seed, HostGraph &g);
// Barabasi-Albert preferential attachment: a clique on m + 1 vertices, then
// each new vertex joins m distinct existing vertices drawn in proportion to
// degree.
void gen_barabasi_albert(int32_t n, int32_t m, uint64_t seed, HostGraph &g);
// The undirected edge lists those two generators pass to build_csr.
void gen_erdos_renyi_edges(int32_t n, double avg_degree, uint64_t seed,
                           std::vector<std::pair<int32_t, int32_t>> &edges);
void gen_barabasi_albert_edges(int32_t n, int32_t m, uint64_t seed,
                               std::vector<std::pair<int32_t, int32_t>> &edges);

// Relabels vertices by decreasing degree (ties: increasing old id); new id 0
// is the largest hub.  `new_of_old` receives the map.
void relabel_by_degree(const HostGraph &in, HostGraph &out,
                       std::vector<int32_t> *new_of_old);

}  // namespace gat
