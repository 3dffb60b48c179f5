// Exact 4-cycle count by wedge aggregation in shared memory (sm_100a).
//
// Every 4-cycle is counted once, at its smallest vertex v0 together with the
// vertex x opposite v0: its other two vertices are common neighbours of v0
// and x above v0.  So
//   count = sum_{v0} sum_{x > v0} C(c(v0, x), 2),
//   c(v0, x) = |{ v1 in N(v0) : v1 > v0, x in N(v1) }|   (x > v0 too).
// On the degree-ordered copy (id 0 = largest degree) v0 is the cycle's
// highest-degree vertex and every v1 has degree <= deg(v0), so the wedges
// v0 - v1 - x number at most the sum over edges of the smaller endpoint's
// degree.
//
// A root's wedge endpoints x are tallied on chip, never in global memory:
//
//  * c4_light_kernel: a warp per root (roots of degree below the heavy
//    threshold).  Lanes take the root's upper neighbours v1, find where
//    N(v1) rises above v0 and add up the wedges W.  With W <= kWarpWedges
//    the lanes walk their lists into a warp-private open-addressing table in
//    shared memory (key x, count c), then read every slot once, add C(c, 2)
//    and clear it.  A root with more wedges is appended to a deferred list.
//  * c4_root_kernel: a CTA per root, for the heavy roots and the deferred
//    ones, largest degree first.  Segment starts (N(v1) above v0) are found
//    once; with W <= kCtaWedges the wedges go to a CTA-wide table as above,
//    otherwise the ids above v0 are swept in windows of consecutive x whose
//    counters (16-bit pairs, or 32-bit words when a count could reach 2^16)
//    fill the shared-memory region: per window each list advances from its
//    cursor to the window's end (galloping search), the segments are
//    flattened with a block scan so that consecutive threads read
//    consecutive list entries, the counters are incremented with shared
//    atomics, and the window's counters are read, summed as C(c, 2) and
//    cleared before the next window.  Once the wedges left fit the CTA
//    table, the lists' remainders go through the table in one pass (the
//    endpoints crowd the low, high-degree ids: on R-MAT most heavy roots
//    need one window and the table).
//
// Neither kernel waits on another CTA; the deferred list is written by the
// first launch and read by the second, ordered on the stream.
#include <cub/cub.cuh>

#include <algorithm>

#include "engine.hpp"

namespace gat {
namespace {

constexpr int32_t kEmpty = -1;
constexpr int kWarpSlots = 1024;          // per-warp table slots
constexpr int kWarpWedges = kWarpSlots / 2;
constexpr int kLightBlock = 256;          // 8 warps
constexpr int kCtaSlots = 16384;          // CTA table slots (128 KB)
constexpr int kCtaWedges = kCtaSlots / 2;
constexpr int kCtaBits = 14;               // log2(kCtaSlots)
static_assert((1 << kCtaBits) == kCtaSlots, "table size is a power of two");
constexpr int kRegionBytes = 196608;      // counters / table region (192 KB)
constexpr int kRegionWords = kRegionBytes / 4;
static_assert(kCtaSlots * 8 <= kRegionBytes, "table fits in the region");

__device__ __forceinline__ unsigned long long pairs_of(unsigned long long c) {
    return c * (c - 1) / 2;
}

// First index i of the sorted a[0, n) with a[i] > x (one thread alone).
__device__ __forceinline__ int32_t upper_index(const int32_t *a, int32_t n, int32_t x) {
    int32_t lo = 0;
    while (n > 0) {
        const int32_t h = n >> 1;
        const bool right = a[lo + h] <= x;
        lo = right ? lo + h + 1 : lo;
        n = right ? n - h - 1 : h;
    }
    return lo;
}

// First index k in [lo, n) with a[k] >= x, galloping from lo (a short
// advance costs one or two loads).
__device__ __forceinline__ int32_t gallop_lower(const int32_t *a, int32_t lo, int32_t n,
                                                int32_t x) {
    if (lo >= n || a[lo] >= x) return lo;
    int32_t below = lo, step = 1;  // a[below] < x
    while (true) {
        const int32_t probe = below + step;
        if (probe >= n || a[probe] >= x) {
            int32_t l = below + 1, len = min(probe, n) - l;
            while (len > 0) {
                const int32_t h = len >> 1;
                const bool right = a[l + h] < x;
                l = right ? l + h + 1 : l;
                len = right ? len - h - 1 : h;
            }
            return l;
        }
        below = probe;
        step <<= 1;
    }
}

__device__ __forceinline__ unsigned slot_of(int32_t x, int bits) {
    return ((unsigned)x * 0x9E3779B1u) >> (32 - bits);
}

// Adds one occurrence of x to an open-addressing table of 2^bits slots that
// is never more than half full.  The probe is bounded by the table size (it
// cannot run out by construction; running out would flag an error).
__device__ __forceinline__ void table_add(int32_t *key, uint32_t *cnt, int bits, int32_t x,
                                          unsigned long long *error) {
    const unsigned mask = (1u << bits) - 1u;
    unsigned h = slot_of(x, bits);
    for (unsigned probes = 0; probes <= mask; probes++) {
        const int32_t k = reinterpret_cast<volatile int32_t *>(key)[h];
        if (k == x) {
            atomicAdd(&cnt[h], 1u);
            return;
        }
        if (k == kEmpty) {
            const int32_t old = atomicCAS(&key[h], kEmpty, x);
            if (old == kEmpty || old == x) {
                atomicAdd(&cnt[h], 1u);
                return;
            }
        }
        h = (h + 1) & mask;
    }
    atomicOr(error, GAT_DEVERR_TABLE);
}

struct LightArgs {
    const int64_t *off;
    const int32_t *adj;
    const int64_t *lo_off;
    int64_t v_begin, v_end;
    DevCounters *ctr;
    C4Aux *aux;
    int32_t *deferred;
};

// A warp per root of [v_begin, v_end), roots handed out one at a time.
constexpr size_t kLightSmem = size_t(kLightBlock / 32) * kWarpSlots * 8;

template <bool STATS>
__global__ void __launch_bounds__(kLightBlock) c4_light_kernel(const LightArgs a) {
    extern __shared__ __align__(16) unsigned char lsmem[];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    int32_t *key = reinterpret_cast<int32_t *>(lsmem) + w * 2 * kWarpSlots;
    uint32_t *cnt = reinterpret_cast<uint32_t *>(key + kWarpSlots);
    for (int i = lane; i < kWarpSlots; i += 32) {
        key[i] = kEmpty;
        cnt[i] = 0;
    }
    __syncwarp();
    unsigned long long part = 0, bytes = 0;
    for (;;) {
        unsigned long long r = 0;
        if (lane == 0) r = atomicAdd(&a.aux->light_cursor, 1ull);
        r = __shfl_sync(0xffffffffu, r, 0);
        const int64_t v0 = a.v_begin + (int64_t)r;
        if (v0 >= a.v_end) break;
        const int64_t o0 = a.off[v0];
        const int32_t d0 = (int32_t)(a.off[v0 + 1] - o0);
        const int32_t lo0 = (int32_t)(a.lo_off[v0 + 1] - a.lo_off[v0]);
        if (d0 - lo0 < 2) continue;  // a cycle needs two neighbours above v0
        // wedges of this root: sum over upper neighbours of |N(v1) above v0|
        int32_t wl = 0;
        for (int i = lo0 + lane; i < d0; i += 32) {
            const int32_t v1 = a.adj[o0 + i];
            const int64_t o1 = a.off[v1];
            const int32_t d1 = (int32_t)(a.off[v1 + 1] - o1);
            wl += d1 - upper_index(a.adj + o1, d1, (int32_t)v0);
        }
        int32_t W = wl;
        for (int o = 16; o > 0; o >>= 1) W += __shfl_xor_sync(0xffffffffu, W, o);
        if (W > kWarpWedges) {
            if (lane == 0) {
                const unsigned long long at = atomicAdd(&a.aux->deferred_count, 1ull);
                a.deferred[at] = (int32_t)v0;
            }
            continue;
        }
        if (W < 2) continue;
        for (int i = lo0 + lane; i < d0; i += 32) {
            const int32_t v1 = a.adj[o0 + i];
            const int64_t o1 = a.off[v1];
            const int32_t d1 = (int32_t)(a.off[v1 + 1] - o1);
            for (int32_t k = upper_index(a.adj + o1, d1, (int32_t)v0); k < d1; k++)
                table_add(key, cnt, 10, a.adj[o1 + k], &a.ctr->error);
            if (STATS) bytes += 20;
        }
        if (STATS) bytes += 4ull * (unsigned)wl;
        __syncwarp();
        for (int i = lane; i < kWarpSlots; i += 32) {
            if (key[i] != kEmpty) {
                part += pairs_of(cnt[i]);
                key[i] = kEmpty;
                cnt[i] = 0;
            }
        }
        __syncwarp();
    }
    for (int o = 16; o > 0; o >>= 1) {
        part += __shfl_xor_sync(0xffffffffu, part, o);
        if (STATS) bytes += __shfl_xor_sync(0xffffffffu, bytes, o);
    }
    if (lane == 0) {
        atomicAdd(&a.ctr->result, part);
        if (STATS) atomicAdd(&a.ctr->bytes, bytes);
    }
}

struct RootArgs {
    const int64_t *off;
    const int32_t *adj;
    const int64_t *lo_off;
    int32_t V;
    int64_t heavy_begin, heavy_end;  // roots taken directly, in id order
    DevCounters *ctr;
    C4Aux *aux;
    const int32_t *deferred;         // then these (count in aux)
    int32_t *cursors;                // per CTA: max_degree list positions
    int64_t cursor_stride;
};

template <int BLOCK>
struct RootSmem {
    typedef cub::BlockScan<int32_t, BLOCK> Scan;
    typedef cub::BlockReduce<long long, BLOCK> Reduce;
    int64_t seg_base[BLOCK];   // absolute index of the segment's first entry
    int32_t pref[BLOCK + 1];   // exclusive prefix of segment lengths
    union {
        typename Scan::TempStorage scan;
        typename Reduce::TempStorage reduce;
    } tmp;
    int64_t root;
    long long total;
};

// Shared memory the root kernel needs: the counter region plus its state.
template <int BLOCK>
constexpr size_t root_smem_bytes() {
    return size_t(kRegionBytes) + sizeof(RootSmem<BLOCK>);
}

// Flattens this group's segments (thread t: seg_base, len) and calls
// f(x) for every entry, consecutive threads on consecutive entries.
template <int BLOCK, class F>
__device__ __forceinline__ int32_t expand_group(RootSmem<BLOCK> &S, const int32_t *adj,
                                                int64_t base, int32_t len, F &&f) {
    int32_t pre, total;
    __syncthreads();  // pref / seg_base of the previous group are consumed
    typename RootSmem<BLOCK>::Scan(S.tmp.scan).ExclusiveSum(len, pre, total);
    S.pref[threadIdx.x] = pre;
    S.seg_base[threadIdx.x] = base;
    if (threadIdx.x == 0) S.pref[BLOCK] = total;
    __syncthreads();
    // Each warp takes one contiguous block of the flattened entries, its
    // lanes on consecutive entries (coalesced reads), so a lane's next entry
    // is 32 further on.  The segment holding entry j is the last s with
    // pref[s] <= j; it only moves forward, so the lane gallops from its
    // previous segment (one comparison while the segment lasts) and narrows
    // the last step by bisection.
    constexpr int kWarps = BLOCK / 32;
    const int32_t per = (total + kWarps - 1) / kWarps;
    const int32_t jb = (int32_t)(threadIdx.x >> 5) * per;
    const int32_t je = min(total, jb + per);
    int32_t lo = 0;
    // Four entries per step: their list loads are all issued before the
    // first update uses one, so each lane has four loads in flight.
    constexpr int kUnroll = 4;
    for (int32_t j0 = jb + (int32_t)(threadIdx.x & 31); j0 < je; j0 += 32 * kUnroll) {
        int32_t xs[kUnroll];
#pragma unroll
        for (int u = 0; u < kUnroll; u++) {
            const int32_t j = j0 + 32 * u;
            xs[u] = 0;
            if (j >= je) continue;
            int32_t step = 1;
            while (lo + step < BLOCK && S.pref[lo + step] <= j) {
                lo += step;
                step <<= 1;
            }
            int32_t n = min(lo + step, BLOCK) - lo;
            while (n > 1) {
                const int32_t h = n >> 1;
                if (S.pref[lo + h] <= j) {
                    lo += h;
                    n -= h;
                } else {
                    n = h;
                }
            }
            xs[u] = __ldg(adj + S.seg_base[lo] + (j - S.pref[lo]));
        }
#pragma unroll
        for (int u = 0; u < kUnroll; u++)
            if (j0 + 32 * u < je) f(xs[u]);
    }
    return total;
}

// A CTA per root: heavy roots [heavy_begin, heavy_end) first, then the
// deferred ones.  WIDE: 32-bit window counters (a count may reach 2^16).
template <int BLOCK, bool WIDE, bool STATS>
__global__ void __launch_bounds__(BLOCK, 1) c4_root_kernel(const RootArgs a) {
    extern __shared__ __align__(16) unsigned char smem[];
    uint32_t *region = reinterpret_cast<uint32_t *>(smem);
    RootSmem<BLOCK> &S = *reinterpret_cast<RootSmem<BLOCK> *>(smem + kRegionBytes);
    int32_t *tkey = reinterpret_cast<int32_t *>(smem);
    uint32_t *tcnt = region + kCtaSlots;
    constexpr int kPerWord = WIDE ? 1 : 2;
    constexpr int32_t kWindow = kRegionWords * kPerWord;  // ids per window
    // the region starts as an empty table; the windows clear it back
    for (int i = threadIdx.x; i < kCtaSlots; i += BLOCK) {
        tkey[i] = kEmpty;
        tcnt[i] = 0;
    }
    int32_t *cur = a.cursors + (int64_t)blockIdx.x * a.cursor_stride;
    const int64_t nheavy = a.heavy_end - a.heavy_begin;
    unsigned long long part = 0, bytes = 0;
    for (;;) {
        __syncthreads();
        if (threadIdx.x == 0) {
            const int64_t i = (int64_t)atomicAdd(&a.aux->root_cursor, 1ull);
            const int64_t nd = (int64_t)*reinterpret_cast<volatile unsigned long long *>(
                &a.aux->deferred_count);
            S.root = i < nheavy ? a.heavy_begin + i : (i - nheavy < nd ? a.deferred[i - nheavy] : -1);
        }
        __syncthreads();
        const int64_t v0 = S.root;
        if (v0 < 0) break;
        const int64_t o0 = a.off[v0];
        const int32_t d0 = (int32_t)(a.off[v0 + 1] - o0);
        const int32_t lo0 = (int32_t)(a.lo_off[v0 + 1] - a.lo_off[v0]);
        const int32_t dp = d0 - lo0;
        if (dp < 2) continue;
        const int32_t *U = a.adj + o0 + lo0;
        const int ngroups = (dp + BLOCK - 1) / BLOCK;
        // Segment starts; one group's positions stay in registers, more go
        // to the CTA's cursor array.
        int64_t my_o1 = 0;
        int32_t my_pos = 0, my_end = 0;
        long long wl = 0;
        for (int g = 0; g < ngroups; g++) {
            const int i = g * BLOCK + threadIdx.x;
            if (i < dp) {
                const int32_t v1 = U[i];
                const int64_t o1 = a.off[v1];
                const int32_t d1 = (int32_t)(a.off[v1 + 1] - o1);
                const int32_t s1 = upper_index(a.adj + o1, d1, (int32_t)v0);
                wl += d1 - s1;
                if (ngroups == 1) {
                    my_o1 = o1;
                    my_pos = s1;
                    my_end = d1;
                } else {
                    cur[i] = s1;
                }
            }
        }
        const long long W =
            typename RootSmem<BLOCK>::Reduce(S.tmp.reduce).Sum(wl);
        if (threadIdx.x == 0) S.total = W;
        __syncthreads();
        const long long Wall = S.total;
        if (Wall < 2) continue;
        if (STATS && threadIdx.x == 0) bytes += 4ull * (unsigned long long)Wall + 20ull * dp;
        if (Wall <= kCtaWedges) {
            // CTA table
            for (int g = 0; g < ngroups; g++) {
                const int i = g * BLOCK + threadIdx.x;
                int64_t base = 0;
                int32_t len = 0;
                if (i < dp) {
                    if (ngroups == 1) {
                        base = my_o1 + my_pos;
                        len = my_end - my_pos;
                    } else {
                        const int32_t v1 = U[i];
                        const int64_t o1 = a.off[v1];
                        base = o1 + cur[i];
                        len = (int32_t)(a.off[v1 + 1] - o1) - cur[i];
                    }
                }
                expand_group<BLOCK>(S, a.adj, base, len, [&](int32_t x) {
                    table_add(tkey, tcnt, kCtaBits, x, &a.ctr->error);
                });
            }
            __syncthreads();
            for (int s = threadIdx.x; s < kCtaSlots; s += BLOCK) {
                if (tkey[s] != kEmpty) {
                    part += pairs_of(tcnt[s]);
                    tkey[s] = kEmpty;
                    tcnt[s] = 0;
                }
            }
            continue;
        }
        // Windows of kWindow consecutive ids above v0.  The region holds a
        // (cleared) table, whose empty keys are -1: clear it to zero first.
        __syncthreads();
        for (int i = threadIdx.x; i < kRegionWords; i += BLOCK) region[i] = 0u;
        long long left = Wall;
        for (int64_t xlo = v0 + 1; xlo < a.V && left > 0; xlo += kWindow) {
            if (left <= kCtaWedges) {
                // The rest fits the CTA table (wedge endpoints crowd the low,
                // high-degree ids, so this is usually after the first
                // window): one pass over every list's remainder.
                __syncthreads();
                for (int i = threadIdx.x; i < kCtaSlots; i += BLOCK) {
                    tkey[i] = kEmpty;
                    tcnt[i] = 0;
                }
                for (int g = 0; g < ngroups; g++) {
                    const int i = g * BLOCK + threadIdx.x;
                    int64_t base = 0;
                    int32_t len = 0;
                    if (i < dp) {
                        if (ngroups == 1) {
                            base = my_o1 + my_pos;
                            len = my_end - my_pos;
                        } else {
                            const int32_t v1 = U[i];
                            const int64_t o1 = a.off[v1];
                            base = o1 + cur[i];
                            len = (int32_t)(a.off[v1 + 1] - o1) - cur[i];
                        }
                    }
                    expand_group<BLOCK>(S, a.adj, base, len, [&](int32_t x) {
                        table_add(tkey, tcnt, kCtaBits, x, &a.ctr->error);
                    });
                }
                __syncthreads();
                for (int s = threadIdx.x; s < kCtaSlots; s += BLOCK) {
                    if (tkey[s] != kEmpty) {
                        part += pairs_of(tcnt[s]);
                        tkey[s] = kEmpty;
                        tcnt[s] = 0;
                    }
                }
                break;
            }
            const int32_t xhi = (int32_t)(xlo + kWindow < (int64_t)a.V ? xlo + kWindow : (int64_t)a.V);
            int32_t in_window = 0;
            for (int g = 0; g < ngroups; g++) {
                const int i = g * BLOCK + threadIdx.x;
                int64_t base = 0;
                int32_t len = 0;
                if (i < dp) {
                    if (ngroups == 1) {
                        const int32_t e = gallop_lower(a.adj + my_o1, my_pos, my_end, xhi);
                        base = my_o1 + my_pos;
                        len = e - my_pos;
                        my_pos = e;
                    } else {
                        const int32_t v1 = U[i];
                        const int64_t o1 = a.off[v1];
                        const int32_t d1 = (int32_t)(a.off[v1 + 1] - o1);
                        const int32_t p = cur[i];
                        const int32_t e = gallop_lower(a.adj + o1, p, d1, xhi);
                        base = o1 + p;
                        len = e - p;
                        cur[i] = e;
                    }
                }
                const int32_t xl = (int32_t)xlo;
                in_window += expand_group<BLOCK>(S, a.adj, base, len, [&](int32_t x) {
                    const int32_t r = x - xl;
                    if (WIDE)
                        atomicAdd(&region[r], 1u);
                    else
                        atomicAdd(&region[r >> 1], 1u << ((r & 1) << 4));
                });
            }
            __syncthreads();
            if (in_window > 0) {
                const int words = (xhi - (int32_t)xlo + kPerWord - 1) / kPerWord;
                for (int i = threadIdx.x; i < words; i += BLOCK) {
                    const uint32_t c = region[i];
                    if (c) {
                        part += WIDE ? pairs_of(c) : pairs_of(c & 0xFFFFu) + pairs_of(c >> 16);
                        region[i] = 0u;
                    }
                }
            }
            left -= in_window;
        }
        // leave the region an empty table again
        __syncthreads();
        for (int i = threadIdx.x; i < kCtaSlots; i += BLOCK) {
            tkey[i] = kEmpty;
            tcnt[i] = 0;
        }
    }
    typedef cub::BlockReduce<unsigned long long, BLOCK> R2;
    __syncthreads();
    const unsigned long long tot =
        R2(*reinterpret_cast<typename R2::TempStorage *>(&S.tmp)).Sum(part);
    if (threadIdx.x == 0) {
        atomicAdd(&a.ctr->result, tot);
        if (STATS) atomicAdd(&a.ctr->bytes, bytes);
    }
}

constexpr int kRootBlock = 1024;

template <bool WIDE, bool STATS>
cudaError_t launch_root(const RootArgs &a, int grid, cudaStream_t st) {
    const size_t smem = root_smem_bytes<kRootBlock>();
    cudaError_t e = cudaFuncSetAttribute(c4_root_kernel<kRootBlock, WIDE, STATS>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    c4_root_kernel<kRootBlock, WIDE, STATS><<<grid, kRootBlock, smem, st>>>(a);
    return cudaGetLastError();
}

template <bool WIDE, bool STATS>
int root_occupancy() {
    const size_t smem = root_smem_bytes<kRootBlock>();
    if (cudaFuncSetAttribute(c4_root_kernel<kRootBlock, WIDE, STATS>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) !=
        cudaSuccess)
        return 0;
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(
            &n, c4_root_kernel<kRootBlock, WIDE, STATS>, kRootBlock, smem) != cudaSuccess)
        return 0;
    return n;
}

template <bool STATS>
cudaError_t light_attr() {
    return cudaFuncSetAttribute(c4_light_kernel<STATS>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kLightSmem);
}

template <bool STATS>
int light_occupancy() {
    int n = 0;
    if (light_attr<STATS>() != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, c4_light_kernel<STATS>, kLightBlock,
                                                      kLightSmem) != cudaSuccess)
        return 0;
    return n;
}

}  // namespace

int c4_light_blocks_per_sm(bool stats) {
    return stats ? light_occupancy<true>() : light_occupancy<false>();
}

int c4_root_blocks_per_sm(bool wide, bool stats) {
    if (wide) return stats ? root_occupancy<true, true>() : root_occupancy<true, false>();
    return stats ? root_occupancy<false, true>() : root_occupancy<false, false>();
}

cudaError_t launch_c4(const C4Launch &L, cudaStream_t st) {
    const DevGraphView &g = L.g;
    cudaError_t e;
    if ((e = cudaMemsetAsync(L.ctr, 0, sizeof(DevCounters), st)) != cudaSuccess ||
        (e = cudaMemsetAsync(L.aux, 0, sizeof(C4Aux), st)) != cudaSuccess)
        return e;
    const int64_t lb = std::max(L.v_begin, L.heavy_end), le = L.v_end;
    if (lb < le) {
        LightArgs la{g.off, g.adj, g.lo_off, lb, le, L.ctr, L.aux, L.deferred};
        if ((e = L.stats ? light_attr<true>() : light_attr<false>()) != cudaSuccess) return e;
        if (L.stats)
            c4_light_kernel<true><<<L.light_grid, kLightBlock, kLightSmem, st>>>(la);
        else
            c4_light_kernel<false><<<L.light_grid, kLightBlock, kLightSmem, st>>>(la);
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    RootArgs ra{g.off, g.adj, g.lo_off, g.V, L.v_begin, std::min(L.v_end, L.heavy_end),
                L.ctr, L.aux, L.deferred, L.cursors, L.cursor_stride};
    if (ra.heavy_end < ra.heavy_begin) ra.heavy_end = ra.heavy_begin;
    // 16-bit counters hold any c(v0, x) <= the largest degree when it is below 2^16
    const bool wide = g.max_degree >= 65536;
    if (wide)
        e = L.stats ? launch_root<true, true>(ra, L.root_grid, st)
                    : launch_root<true, false>(ra, L.root_grid, st);
    else
        e = L.stats ? launch_root<false, true>(ra, L.root_grid, st)
                    : launch_root<false, false>(ra, L.root_grid, st);
    return e;
}

}  // namespace gat
