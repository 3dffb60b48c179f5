// Graph construction on the device: the seeded R-MAT generator and the
// edge-list -> CSR build (symmetrise, drop self loops and duplicates, sort
// rows) that the reference does on the host when it loads a text graph
// (infra/graph_backend.cuh:23-89) and that utils/graph_transform.cu:6-28
// does as a separate pass.  The result is bit-identical to the host build
// (graph.cpp gen_rmat + build_csr): the same per-sample splitmix64 streams,
// the same quadrant thresholds, and a CSR with the same sorted unique rows.
//
// One edge key per direction, (u << 32) | v, is radix-sorted by CUB (the
// toolkit's library sort), duplicates are removed by CUB's unique selection,
// and a kernel finds each row's start by binary search over the sorted keys.
#include <cub/cub.cuh>

#include "engine.hpp"

namespace gat {
namespace {

constexpr uint64_t kGolden = 0x9E3779B97F4A7C15ull;
constexpr uint64_t kStream = 0xD1B54A32D192ED03ull;
constexpr uint64_t kDropped = ~0ull;  // a self loop's key: sorts after every edge

__host__ __device__ __forceinline__ uint64_t mix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}

// Sample i: both directions of its edge, or two dropped keys for a loop.
__global__ void rmat_keys_kernel(int scale, int64_t samples, uint64_t base, uint64_t ta,
                                 uint64_t tb, uint64_t tc, uint64_t *__restrict__ keys) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= samples) return;
    uint64_t s = base + (uint64_t)i * kStream;
    uint32_t u = 0, v = 0;
    uint64_t bits = 0;
    for (int l = 0; l < scale; l++) {
        if ((l & 1) == 0) {
            s += kGolden;
            bits = mix64(s);
        }
        const uint64_t r = (l & 1) ? (bits >> 32) : (bits & 0xFFFFFFFFull);
        const uint32_t bu = r >= tb, bv = (r >= ta && r < tb) || r >= tc;
        u = (u << 1) | bu;
        v = (v << 1) | bv;
    }
    const bool loop = u == v;
    keys[2 * i] = loop ? kDropped : ((uint64_t)u << 32) | v;
    keys[2 * i + 1] = loop ? kDropped : ((uint64_t)v << 32) | u;
}

__global__ void pair_keys_kernel(const int32_t *__restrict__ pairs, int64_t n,
                                 uint64_t *__restrict__ keys) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint32_t u = (uint32_t)pairs[2 * i], v = (uint32_t)pairs[2 * i + 1];
    const bool loop = u == v;
    keys[2 * i] = loop ? kDropped : ((uint64_t)u << 32) | v;
    keys[2 * i + 1] = loop ? kDropped : ((uint64_t)v << 32) | u;
}

// off[v] = first key index with row >= v (keys sorted, unique, dropped keys
// past E); adj[i] = column of key i.
__global__ void row_starts_kernel(const uint64_t *__restrict__ keys, int64_t E, int32_t V,
                                  int64_t *__restrict__ off) {
    const int64_t v = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (v > V) return;
    const uint64_t x = (uint64_t)v << 32;
    int64_t lo = 0, n = E;
    while (n > 0) {
        const int64_t h = n >> 1;
        const bool right = keys[lo + h] < x;
        lo = right ? lo + h + 1 : lo;
        n = right ? n - h - 1 : h;
    }
    off[v] = lo;
}

__global__ void columns_kernel(const uint64_t *__restrict__ keys, int64_t E,
                               int32_t *__restrict__ adj) {
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < E) adj[i] = (int32_t)(keys[i] & 0xFFFFFFFFull);
}

unsigned blocks(int64_t n) { return (unsigned)((n + 255) / 256); }

template <class F>
cudaError_t with_temp(F &&call, cudaStream_t st) {
    size_t bytes = 0;
    cudaError_t e = call(nullptr, bytes);
    if (e != cudaSuccess) return e;
    void *tmp = nullptr;
    if ((e = cudaMallocAsync(&tmp, bytes ? bytes : 1, st)) != cudaSuccess) return e;
    e = call(tmp, bytes);
    const cudaError_t f = cudaFreeAsync(tmp, st);
    return e != cudaSuccess ? e : f;
}

// keys[0, nkeys) (both directions of every sample) -> CSR in off / *adj.
cudaError_t keys_to_csr(uint64_t *keys, int64_t nkeys, int32_t V, int64_t *off, int32_t **adj,
                        int64_t pad_ints, int64_t *E_out, cudaStream_t st) {
    uint64_t *sorted = nullptr;
    int64_t *nsel = nullptr;
    cudaError_t e;
    if ((e = cudaMallocAsync(&sorted, 8 * size_t(nkeys > 0 ? nkeys : 1), st)) != cudaSuccess ||
        (e = cudaMallocAsync(&nsel, sizeof(int64_t), st)) != cudaSuccess)
        return e;
    // rows need bits(V - 1) above the 32 column bits; the dropped key has
    // all of those bits set, so it still sorts last
    int vbits = 1;
    while (vbits < 31 && (int64_t(1) << vbits) < V) vbits++;
    const int end_bit = 32 + vbits;
    e = with_temp(
        [&](void *t, size_t &b) {
            return cub::DeviceRadixSort::SortKeys(t, b, keys, sorted, nkeys, 0, end_bit, st);
        },
        st);
    if (e == cudaSuccess)
        e = with_temp(
            [&](void *t, size_t &b) {
                return cub::DeviceSelect::Unique(t, b, sorted, keys, nsel, nkeys, st);
            },
            st);
    int64_t nu = 0, E = 0;
    if (e == cudaSuccess &&
        (e = cudaMemcpyAsync(&nu, nsel, sizeof(int64_t), cudaMemcpyDeviceToHost, st)) ==
            cudaSuccess &&
        (e = cudaStreamSynchronize(st)) == cudaSuccess) {
        uint64_t last = 0;
        if (nu > 0 &&
            (e = cudaMemcpy(&last, keys + nu - 1, 8, cudaMemcpyDeviceToHost)) != cudaSuccess)
            nu = 0;
        E = (nu > 0 && last == kDropped) ? nu - 1 : nu;
    }
    if (e == cudaSuccess) e = cudaMalloc(adj, sizeof(int32_t) * size_t(E + pad_ints));
    if (e == cudaSuccess) {
        row_starts_kernel<<<blocks(int64_t(V) + 1), 256, 0, st>>>(keys, E, V, off);
        if (E > 0) columns_kernel<<<blocks(E), 256, 0, st>>>(keys, E, *adj);
        e = cudaGetLastError();
    }
    const cudaError_t f1 = cudaFreeAsync(sorted, st), f2 = cudaFreeAsync(nsel, st);
    if (e == cudaSuccess) e = f1 != cudaSuccess ? f1 : f2;
    *E_out = E;
    return e;
}

// A warp per row: the CSR rules the host's validate() checks without
// symmetry (offsets monotone and inside [0, E], ids in [0, V), no self loop,
// rows strictly increasing).  The lowest failing row wins: *flag takes
// min(row << 3 | reason).
__global__ void csr_check_kernel(const int64_t *__restrict__ off,
                                 const int32_t *__restrict__ adj, int32_t V, int64_t E,
                                 unsigned long long *flag) {
    const int64_t v = ((int64_t)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (v >= V) return;
    const int64_t b = off[v], e = off[v + 1];
    unsigned reason = 0;
    if (b < 0 || e < b || e > E || (v == 0 && b != 0) || (v == V - 1 && e != E)) {
        reason = kCsrOffsets;
    } else {
        // rows are warp-uniform, so every lane runs every chunk
        for (int64_t base = b; base < e; base += 32) {
            const int64_t i = base + lane;
            unsigned r = 0;
            if (i < e) {
                const int32_t u = adj[i];
                if (u < 0 || u >= V) r = kCsrRange;
                else if (u == v) r = kCsrLoop;
                else if (i > b && adj[i - 1] >= u) r = kCsrOrder;
            }
            // the host check reports the first failing entry's reason
            const unsigned m = __ballot_sync(0xffffffffu, r != 0);
            if (m) {
                reason = __shfl_sync(0xffffffffu, r, __ffs(m) - 1);
                break;
            }
        }
    }
    if (lane == 0 && reason)
        atomicMin(flag, ((unsigned long long)v << 3) | reason);
}

}  // namespace

cudaError_t csr_check_device(const int64_t *off, const int32_t *adj, int32_t V, int64_t E,
                             unsigned long long *flag, cudaStream_t st) {
    cudaError_t e = cudaMemsetAsync(flag, 0xFF, sizeof(unsigned long long), st);
    if (e != cudaSuccess || V <= 0) return e;
    csr_check_kernel<<<blocks(int64_t(V) * 32), 256, 0, st>>>(off, adj, V, E, flag);
    return cudaGetLastError();
}

cudaError_t rmat_csr_device(int scale, int64_t samples, double a, double b, double c,
                            uint64_t seed, int64_t *off, int32_t **adj, int64_t pad_ints,
                            int64_t *E, cudaStream_t st) {
    const uint64_t ta = uint64_t(a * 4294967296.0);
    const uint64_t tb = uint64_t((a + b) * 4294967296.0);
    const uint64_t tc = uint64_t((a + b + c) * 4294967296.0);
    const uint64_t base = mix64(seed + kGolden);
    uint64_t *keys = nullptr;
    cudaError_t e = cudaMallocAsync(&keys, 16 * size_t(samples > 0 ? samples : 1), st);
    if (e != cudaSuccess) return e;
    if (samples > 0) {
        rmat_keys_kernel<<<blocks(samples), 256, 0, st>>>(scale, samples, base, ta, tb, tc,
                                                          keys);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess)
        e = keys_to_csr(keys, 2 * samples, int32_t(1) << scale, off, adj, pad_ints, E, st);
    const cudaError_t f = cudaFreeAsync(keys, st);
    return e != cudaSuccess ? e : f;
}

cudaError_t pairs_csr_device(const int32_t *pairs, int64_t n, int32_t V, int64_t *off,
                             int32_t **adj, int64_t pad_ints, int64_t *E, cudaStream_t st) {
    uint64_t *keys = nullptr;
    cudaError_t e = cudaMallocAsync(&keys, 16 * size_t(n > 0 ? n : 1), st);
    if (e != cudaSuccess) return e;
    if (n > 0) {
        pair_keys_kernel<<<blocks(n), 256, 0, st>>>(pairs, n, keys);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = keys_to_csr(keys, 2 * n, V, off, adj, pad_ints, E, st);
    const cudaError_t f = cudaFreeAsync(keys, st);
    return e != cudaSuccess ? e : f;
}

}  // namespace gat
