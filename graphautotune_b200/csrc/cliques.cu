// Exact k-clique count (4 <= k <= 7) by bit-matrix induced subgraphs (sm_100a).
//
// On the degree-ordered copy (id 0 = largest degree) every k-clique is
// counted once, at its largest id v0 (its member of smallest degree).  The
// other members lie in L = N<(v0) = {u in N(v0) : u < v0}: the first lo(v0)
// entries of v0's sorted row, which the orientation keeps short (at most
// 668 on R-MAT 2^20 with 16M edges although the largest degree is 64,337).
// With L sorted, the subgraph induced on L is a bit matrix R: row i has bit
// j (j < i) set iff L[j] is a neighbour of L[i].  A k-clique at v0 is then a
// (k-1)-clique of R taken in decreasing index order:
//
//   k = 4:  sum_i  sum_{j in R_i}  |R_i & R_j|
//   k = 5:  sum_i  sum_{j in R_i}  sum_{l in R_i & R_j}  |R_i & R_j & R_l|
//
// and so on; the innermost level is a popcount, never an enumeration.  The
// exact schedule plan of K_k (all restrictions v_b < v_a, level-1 units
// v1 < v0) counts the same cliques at the same roots, so root ranges and
// shards agree between the two paths.
//
// Two kernels split the roots by lo(v0):
//  * clique_warp_kernel: a warp per root with lo(v0) <= kWarpD (rows of at
//    most two words, in the warp's slice of shared memory);
//  * clique_cta_kernel: a CTA per larger root.  v0's list is staged into
//    shared memory by one bulk copy (cp.async.bulk, completion on an
//    mbarrier, waits bounded); the matrix is in shared memory when it fits
//    and in a per-CTA slice of global scratch otherwise (lo(v0) up to 2048).
//
// Building row i intersects N<(L[i]) with L[0, i).  Three ways, chosen per
// row by their cost:
//  * L[i] has a hub bitmap: lanes take j and test bit L[j] of that row (one
//    load each); the warp's ballot is one word of R_i;
//  * scan: lanes read the part of N<(L[i]) inside [L[0], L[i-1]] with
//    128-bit non-coherent loads (ld.global.nc.v4) and find each element in
//    L[0, i) by binary search in shared memory (shared atomicOr sets the bit);
//  * probe: when that part is much longer than i, lanes take j and
//    binary-search L[j] in it; the ballot is one word of R_i.
// Counting gives lanes one candidate each: the set bits of the current mask
// are compacted into a per-warp queue (ballot + popc), and each lane adds
// popc(mask & R_q) over the words below its candidate q.  Levels between
// the first and the last are walked by the whole warp (the AND of the masks
// kept per warp in shared memory).
//
// Neither kernel waits on another CTA.  The only inter-CTA traffic is the
// root cursors and the total.
#include <algorithm>

#include "engine.hpp"

namespace gat {
namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kMaxD = kCliqueMaxLower;  // longest lower list (64 words a row)
constexpr int kMaxWords = kMaxD / 32;
constexpr int kWarpD = 64;              // roots up to this go to the warp kernel
constexpr int kWarpPitch = 3;           // row pitch of the warp kernel's matrix
constexpr int kWarpThreads = 256;
constexpr int kCtaThreads = kCliqueCtaThreads;
constexpr int kCtaWarps = kCtaThreads / 32;
constexpr int kRowSmemWords = 22 * 1024;  // 88 KB of matrix rows in shared memory
constexpr int kQueue = 64;
constexpr int kRootChunk = 32;            // root ids per cursor grab
constexpr unsigned kWaitLimit = 1u << 24;  // mbarrier polls before giving up

__device__ __forceinline__ int words_below(int q) { return (q + 31) >> 5; }

// Row pitch for a root with d lower neighbours: words of the longest row,
// made odd so lanes reading rows of different candidates hit different banks.
__host__ __device__ __forceinline__ int row_pitch(int d) { return ((d + 31) >> 5) | 1; }

__device__ __forceinline__ unsigned lanemask_lt() {
    unsigned m;
    asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
    return m;
}

__device__ __forceinline__ int4 ldg_nc_v4(const int32_t *p) {
    int4 v;
    asm volatile("ld.global.nc.v4.s32 {%0, %1, %2, %3}, [%4];"
                 : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
                 : "l"(p));
    return v;
}

__device__ __forceinline__ int ceil_log2(int x) { return x <= 1 ? 1 : 32 - __clz(x - 1); }

// First index i of the sorted a[0, n) with a[i] >= x; the whole warp
// cooperates (32-ary search) and every lane gets the result.
__device__ __forceinline__ int warp_lower(const int32_t *a, int n, int32_t x, int lane) {
    int lo = 0, hi = n;
    while (hi - lo > 32) {
        const int p = lo + (int)(((long long)(lane + 1) * (hi - lo)) / 33);
        const int c = __popc(__ballot_sync(kFull, a[p] < x));
        const int plo = __shfl_sync(kFull, p, c > 0 ? c - 1 : 0);
        const int phi = __shfl_sync(kFull, p, c < 32 ? c : 31);
        lo = c > 0 ? plo + 1 : lo;
        hi = c < 32 ? phi : hi;
    }
    const bool less = lo + lane < hi && a[lo + lane] < x;
    return lo + __popc(__ballot_sync(kFull, less));
}

// Index of x in the sorted s[0, n) (shared memory), or -1.
__device__ __forceinline__ int find_in(const int32_t *s, int n, int32_t x) {
    if (n <= 0) return -1;
    int lo = 0, len = n;
    while (len > 1) {
        const int h = len >> 1;
        lo = (s[lo + h] <= x) ? lo + h : lo;
        len -= h;
    }
    return s[lo] == x ? lo : -1;
}

// Membership of x in the sorted global list b[0, n): branch-free search.
__device__ __forceinline__ bool contains(const int32_t *b, int n, int32_t x) {
    if (n <= 0) return false;
    int lo = 0, len = n;
    while (len > 1) {
        const int h = len >> 1;
        lo = (__ldg(b + lo + h) <= x) ? lo + h : lo;
        len -= h;
    }
    return __ldg(b + lo) == x;
}

struct CliqueArgs {
    const int64_t *off;
    const int32_t *adj;  // rows padded: 4 readable ints past the last entry
    const int64_t *lo_off;
    const int32_t *hub_slot;  // null: no bitmaps
    const uint32_t *bitmaps;
    int64_t bitmap_words;
    int64_t v_begin, v_end;   // roots holding the units [u_begin, u_end)
    int64_t u_begin, u_end;   // level-1 units (v0, L[i]) numbered by lo_off
    DevCounters *ctr;
    CliqueAux *aux;
    uint32_t *rows;       // CTA kernel: per-CTA matrix for roots too large for
    int64_t rows_stride;  // shared memory (null when none is)
};

__device__ __forceinline__ int32_t lower_degree(const CliqueArgs &a, int64_t v) {
    return (int32_t)(a.lo_off[v + 1] - a.lo_off[v]);
}

// Rows [*r0, *r1) of root v0 (d rows) are units of this launch: unit
// lo_off[v0] + i is (v0, L[i]), and its cliques are row i's.
__device__ __forceinline__ void unit_rows(const CliqueArgs &a, int64_t v0, int d, int *r0,
                                          int *r1) {
    const int64_t lb = a.lo_off[v0];
    *r0 = (int)max((int64_t)0, a.u_begin - lb);
    *r1 = (int)min((int64_t)d, a.u_end - lb);
}

// Words [0, words_below(i)) of R_i = { j < i : L[j] in N(L[i]) }.  One warp.
// STATS adds the intersection's list bytes 4 (|part of N<(L[i])| + i).
template <bool STATS>
__device__ void build_row(const CliqueArgs &a, const int32_t *L, int i, uint32_t *Ri, int lane,
                          unsigned long long &bytes) {
    const int nw = words_below(i);
    if (nw == 0) return;
    const int32_t u = L[i];
    const int hs = a.hub_slot != nullptr ? __ldg(a.hub_slot + u) : -1;
    if (hs >= 0) {
        const uint32_t *bm = a.bitmaps + (int64_t)hs * a.bitmap_words;
        for (int w = 0; w < nw; w++) {
            const int j = (w << 5) + lane;
            bool f = false;
            if (j < i) {
                const int32_t y = L[j];
                f = (__ldg(bm + (y >> 5)) >> (y & 31)) & 1u;
            }
            const unsigned word = __ballot_sync(kFull, f);
            if (lane == 0) Ri[w] = word;
        }
        if (STATS && lane == 0) bytes += 8ull * (unsigned)i;
        return;
    }
    const int64_t o = a.off[u];
    const int32_t nu = lower_degree(a, u);
    const int32_t *N = a.adj + o;
    // only N<(u) inside [L[0], L[i-1]] can meet L[0, i)
    const int s = warp_lower(N, nu, L[0], lane);
    const int e = s + warp_lower(N + s, nu - s, L[i - 1] + 1, lane);
    const int ns = e - s;
    if (STATS && lane == 0) bytes += 4ull * (unsigned)(ns + i);
    if ((long long)i * ceil_log2(ns + 1) * 8 < ns) {
        // probe: few candidates against a long list
        for (int w = 0; w < nw; w++) {
            const int j = (w << 5) + lane;
            const bool f = j < i && contains(N + s, ns, L[j]);
            const unsigned word = __ballot_sync(kFull, f);
            if (lane == 0) Ri[w] = word;
        }
        return;
    }
    for (int w = lane; w < nw; w += 32) Ri[w] = 0u;
    __syncwarp();
    // scan [o + s, o + e) in aligned 4-entry groups
    const int64_t gs = o + s, ge = o + e;
    for (int64_t q = (gs & ~3ll) + 4 * lane; q < ge; q += 128) {
        const int4 v = ldg_nc_v4(a.adj + q);
        const int32_t xs[4] = {v.x, v.y, v.z, v.w};
#pragma unroll
        for (int t = 0; t < 4; t++) {
            if (q + t < gs || q + t >= ge) continue;
            const int j = find_in(L, i, xs[t]);
            if (j >= 0) atomicOr(Ri + (j >> 5), 1u << (j & 31));
        }
    }
    __syncwarp();
}

// sum over w < n of popc(m[w] & r[w])
__device__ __forceinline__ unsigned pop_and(const uint32_t *m, const uint32_t *r, int n) {
    unsigned c = 0;
    for (int w = 0; w < n; w++) c += __popc(m[w] & r[w]);
    return c;
}

// The last level: lanes take the set bits q of m[0, nw) and add
// popc(m & R_q) over R_q's words.  Q: the warp's queue (kQueue entries).
__device__ unsigned long long last_level(const uint32_t *m, int nw, const uint32_t *R, int pitch,
                                         int32_t *Q, int lane, unsigned long long &words) {
    unsigned long long c = 0;
    int nq = 0;
    for (int w = 0; w < nw; w++) {
        const uint32_t x = m[w];
        if (x == 0u) continue;
        if ((x >> lane) & 1u) Q[nq + __popc(x & lanemask_lt())] = (w << 5) + lane;
        nq += __popc(x);
        if (nq >= 32) {
            __syncwarp();
            const int q = Q[lane];
            const int n = words_below(q);
            c += pop_and(m, R + (int64_t)q * pitch, n);
            words += (unsigned)n;
            const int rest = nq - 32;
            const int32_t moved = lane < rest ? Q[32 + lane] : 0;
            __syncwarp();
            if (lane < rest) Q[lane] = moved;
            nq = rest;
            __syncwarp();
        }
    }
    __syncwarp();
    if (lane < nq) {
        const int q = Q[lane];
        const int n = words_below(q);
        c += pop_and(m, R + (int64_t)q * pitch, n);
        words += (unsigned)n;
    }
    __syncwarp();
    return c;
}

// Cliques continuing from mask m[0, nw) with DEPTH more levels walked by the
// whole warp before the last one.  stack: DEPTH buffers of kMaxWords words.
template <int DEPTH>
__device__ unsigned long long walk(const uint32_t *m, int nw, const uint32_t *R, int pitch,
                                   uint32_t *stack, int32_t *Q, int lane,
                                   unsigned long long &words) {
    if constexpr (DEPTH == 0) {
        return last_level(m, nw, R, pitch, Q, lane, words);
    } else {
        unsigned long long c = 0;
        for (int w = 0; w < nw; w++) {
            uint32_t x = m[w];
            while (x != 0u) {
                const int j = (w << 5) + __ffs(x) - 1;
                x &= x - 1;
                const int n2 = words_below(j);
                const uint32_t *Rj = R + (int64_t)j * pitch;
                unsigned any = 0;
                for (int t = lane; t < n2; t += 32) {
                    const uint32_t y = m[t] & Rj[t];
                    stack[t] = y;
                    any |= y;
                }
                words += (unsigned)(lane < n2 ? (n2 - lane + 31) / 32 : 0);
                // a mask with no bits cannot continue
                if (__any_sync(kFull, any != 0u)) {
                    __syncwarp();
                    c += walk<DEPTH - 1>(stack, n2, R, pitch, stack + kMaxWords, Q, lane, words);
                }
                __syncwarp();
            }
        }
        return c;
    }
}

// The 4-clique's last level spans rows: queue entries are (i, q) pairs, so a
// row with few bits does not leave lanes idle.
struct PairQueue {
    int32_t *Q;  // kQueue entries: i << 11 | q   (i, q < 2048)
    int n = 0;
};

__device__ __forceinline__ void pairs_push_row(PairQueue &pq, const uint32_t *R, int pitch, int i,
                                               int lane, unsigned long long &c,
                                               unsigned long long &words) {
    const uint32_t *Ri = R + (int64_t)i * pitch;
    const int nw = words_below(i);
    for (int w = 0; w < nw; w++) {
        const uint32_t x = Ri[w];
        if (x == 0u) continue;
        if ((x >> lane) & 1u) pq.Q[pq.n + __popc(x & lanemask_lt())] = (i << 11) | ((w << 5) + lane);
        pq.n += __popc(x);
        if (pq.n >= 32) {
            __syncwarp();
            const int32_t e = pq.Q[lane];
            const int q = e & 2047;
            const int n = words_below(q);
            c += pop_and(R + (int64_t)(e >> 11) * pitch, R + (int64_t)q * pitch, n);
            words += (unsigned)n;
            const int rest = pq.n - 32;
            const int32_t moved = lane < rest ? pq.Q[32 + lane] : 0;
            __syncwarp();
            if (lane < rest) pq.Q[lane] = moved;
            pq.n = rest;
            __syncwarp();
        }
    }
}

__device__ __forceinline__ void pairs_flush(PairQueue &pq, const uint32_t *R, int pitch, int lane,
                                            unsigned long long &c, unsigned long long &words) {
    __syncwarp();
    if (lane < pq.n) {
        const int32_t e = pq.Q[lane];
        const int q = e & 2047;
        const int n = words_below(q);
        c += pop_and(R + (int64_t)(e >> 11) * pitch, R + (int64_t)q * pitch, n);
        words += (unsigned)n;
    }
    pq.n = 0;
    __syncwarp();
}

// Cliques of R with their first member at row i (K >= 5).
template <int K>
__device__ __forceinline__ unsigned long long count_row(const uint32_t *R, int pitch, int i,
                                                        uint32_t *stack, int32_t *Q, int lane,
                                                        unsigned long long &words) {
    return walk<K - 4>(R + (int64_t)i * pitch, words_below(i), R, pitch, stack, Q, lane, words);
}

__device__ __forceinline__ void flush_totals(const CliqueArgs &a, unsigned long long c,
                                             unsigned long long bytes, bool stats, int lane) {
    for (int o = 16; o > 0; o >>= 1) {
        c += __shfl_xor_sync(kFull, c, o);
        if (stats) bytes += __shfl_xor_sync(kFull, bytes, o);
    }
    if (lane == 0) {
        if (c) atomicAdd(&a.ctr->result, c);
        if (stats && bytes) atomicAdd(&a.ctr->bytes, bytes);
    }
}

// ---------------------------------------------------------------- warp kernel

template <int K>
struct WarpSmem {
    int32_t L[kWarpD];
    uint32_t R[kWarpD * kWarpPitch];
    uint32_t stack[(K > 4 ? K - 4 : 1) * kMaxWords];
    int32_t Q[kQueue];
};

// A warp per root v0 of [v_begin, v_end) with K-1 <= lo(v0) <= kWarpD; root
// ids are handed out kRootChunk at a time.
template <int K, bool STATS>
__global__ void __launch_bounds__(kWarpThreads) clique_warp_kernel(const CliqueArgs a) {
    extern __shared__ __align__(16) unsigned char wsmem[];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    WarpSmem<K> &S = reinterpret_cast<WarpSmem<K> *>(wsmem)[wid];
    unsigned long long c = 0, bytes = 0, words = 0;
    PairQueue pq;
    pq.Q = S.Q;
    for (;;) {
        unsigned long long r0 = 0;
        if (lane == 0) r0 = atomicAdd(&a.aux->warp_cursor, (unsigned long long)kRootChunk);
        r0 = __shfl_sync(kFull, r0, 0);
        const int64_t base = a.v_begin + (int64_t)r0;
        if (base >= a.v_end) break;
        const int64_t v = base + lane;
        const int32_t dl = v < a.v_end ? lower_degree(a, v) : 0;
        unsigned mine = __ballot_sync(kFull, dl >= K - 1 && dl <= kWarpD);
        while (mine != 0u) {
            const int r = __ffs(mine) - 1;
            mine &= mine - 1;
            const int64_t v0 = base + r;
            const int d = __shfl_sync(kFull, dl, r);
            int r0, r1;
            unit_rows(a, v0, d, &r0, &r1);
            r0 = max(r0, K - 2);  // row i needs K-2 members below it
            if (r0 >= r1) continue;
            const int pitch = row_pitch(d);
            const int32_t *src = a.adj + a.off[v0];
            for (int t = lane; t < r1; t += 32) S.L[t] = __ldg(src + t);
            if (STATS && lane == 0) bytes += 4ull * (unsigned)r1;
            __syncwarp();
            for (int i = 1; i < r1; i++) build_row<STATS>(a, S.L, i, S.R + i * pitch, lane, bytes);
            __syncwarp();
            if constexpr (K == 4) {
                for (int i = r0; i < r1; i++) pairs_push_row(pq, S.R, pitch, i, lane, c, words);
                pairs_flush(pq, S.R, pitch, lane, c, words);
            } else {
                for (int i = r0; i < r1; i++)
                    c += count_row<K>(S.R, pitch, i, S.stack, S.Q, lane, words);
            }
        }
    }
    if (STATS) bytes += 8ull * words;
    flush_totals(a, c, bytes, STATS, lane);
}

// ----------------------------------------------------------------- CTA kernel

__device__ __forceinline__ unsigned smem_u32(const void *p) {
    return (unsigned)__cvta_generic_to_shared(p);
}

template <int K>
struct CtaSmem {
    alignas(16) int32_t Lbuf[kMaxD + 8];  // v0's list, staged from 16-byte boundaries
    alignas(16) uint32_t R[kRowSmemWords];
    uint32_t stack[kCtaWarps][(K > 4 ? K - 4 : 1) * kMaxWords];
    int32_t Q[kCtaWarps][kQueue];
    alignas(8) unsigned long long bar;
    int32_t roots[kRootChunk];
    int nroots;
    int next_build, next_count;
    int abort;
};

// Bulk copy of src[0, n_ints) (16-byte aligned, n_ints a multiple of 4) into
// shared memory, completion counted on the mbarrier.  One thread.
__device__ __forceinline__ void bulk_stage(void *dst, const int32_t *src, int n_ints,
                                           unsigned long long *bar) {
    const unsigned bytes = (unsigned)n_ints * 4u;
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)),
                 "r"(bytes)
                 : "memory");
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
            "r"(smem_u32(dst)),
        "l"(src), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ bool mbar_test(unsigned long long *bar, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Polls the mbarrier phase at most `limit` times.
__device__ __forceinline__ bool mbar_wait(unsigned long long *bar, unsigned parity,
                                          unsigned limit) {
    for (unsigned t = 0; t < limit; t++)
        if (mbar_test(bar, parity)) return true;
    return false;
}

template <int K>
constexpr size_t cta_smem_bytes() {
    return sizeof(CtaSmem<K>);
}

// A CTA per root v0 of [v_begin, v_end) with lo(v0) > kWarpD.
template <int K, bool STATS>
__global__ void __launch_bounds__(kCtaThreads) clique_cta_kernel(const CliqueArgs a) {
    extern __shared__ __align__(16) unsigned char csmem[];
    CtaSmem<K> &S = *reinterpret_cast<CtaSmem<K> *>(csmem);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    unsigned long long c = 0, bytes = 0, words = 0;
    unsigned phase = 0;
    if (threadIdx.x == 0) {
        asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&S.bar)) : "memory");
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        S.abort = 0;
    }
    __syncthreads();
    uint32_t *grows = a.rows != nullptr ? a.rows + (int64_t)blockIdx.x * a.rows_stride : nullptr;
    PairQueue pq;
    pq.Q = S.Q[wid];
    for (;;) {
        if (wid == 0) {
            unsigned long long r0 = 0;
            if (lane == 0) r0 = atomicAdd(&a.aux->cta_cursor, (unsigned long long)kRootChunk);
            r0 = __shfl_sync(kFull, r0, 0);
            const int64_t v = a.v_begin + (int64_t)r0 + lane;
            const bool big = (int64_t)r0 < a.v_end - a.v_begin && v < a.v_end &&
                             lower_degree(a, v) > kWarpD;
            const unsigned m = __ballot_sync(kFull, big);
            if (big) S.roots[__popc(m & lanemask_lt())] = (int32_t)v;
            if (lane == 0) S.nroots = (int64_t)r0 < a.v_end - a.v_begin ? __popc(m) : -1;
        }
        __syncthreads();
        const int nroots = S.nroots;
        // every warp has read the chunk before warp 0 may refill it
        __syncthreads();
        if (nroots < 0) break;
        bool aborted = false;
        for (int r = 0; r < nroots; r++) {
            const int64_t v0 = S.roots[r];
            const int64_t o0 = a.off[v0];
            const int d = lower_degree(a, v0);
            const int pitch = row_pitch(d);
            uint32_t *R = (int64_t)d * pitch <= kRowSmemWords ? S.R : grows;
            if (d > kMaxD || R == nullptr) {
                // the host sizes the row scratch for the graph's longest list
                if (threadIdx.x == 0) atomicOr(&a.ctr->error, GAT_DEVERR_SCRATCH);
                continue;
            }
            // stage L = adj[o0, o0 + d) from the 16-byte boundary below it
            const int64_t a0 = o0 & ~3ll, a1 = (o0 + d + 3) & ~3ll;
            const int32_t *L = S.Lbuf + (o0 - a0);
            if (threadIdx.x == 0) {
                asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                bulk_stage(S.Lbuf, a.adj + a0, (int)(a1 - a0), &S.bar);
            }
            const bool ok = mbar_wait(&S.bar, phase, kWaitLimit);
            phase ^= 1u;
            if (__syncthreads_or(!ok)) {
                // the copy did not complete: report, let it land, stop
                if (threadIdx.x == 0) {
                    atomicOr(&a.ctr->error, GAT_DEVERR_WAIT);
                    mbar_wait(&S.bar, phase ^ 1u, kWaitLimit);
                }
                aborted = true;
                break;
            }
            if (STATS && threadIdx.x == 0) bytes += 4ull * (unsigned)d;
            if (threadIdx.x == 0) {
                S.next_build = kCtaWarps;
                S.next_count = kCtaWarps;
            }
            // rows below r1 are built; rows [r0, r1) are counted
            int r0, r1;
            unit_rows(a, v0, d, &r0, &r1);
            r0 = max(r0, K - 2);
            __syncthreads();
            for (int i = wid;;) {
                if (i >= r1) break;
                build_row<STATS>(a, L, i, R + (int64_t)i * pitch, lane, bytes);
                int nx = 0;
                if (lane == 0) nx = atomicAdd(&S.next_build, 1);
                i = __shfl_sync(kFull, nx, 0);
            }
            __syncthreads();
            for (int i = r0 + wid;;) {
                if (i >= r1) break;
                if constexpr (K == 4)
                    pairs_push_row(pq, R, pitch, i, lane, c, words);
                else
                    c += count_row<K>(R, pitch, i, S.stack[wid], S.Q[wid], lane, words);
                int nx = 0;
                if (lane == 0) nx = atomicAdd(&S.next_count, 1);
                i = r0 + __shfl_sync(kFull, nx, 0);
            }
            if constexpr (K == 4) pairs_flush(pq, R, pitch, lane, c, words);
            __syncthreads();
        }
        if (aborted) break;
    }
    if (STATS) bytes += 8ull * words;
    flush_totals(a, c, bytes, STATS, lane);
}

template <int K, bool STATS>
cudaError_t launch_k(const CliqueArgs &a, int warp_grid, int cta_grid, cudaStream_t st) {
    cudaError_t e;
    const size_t ws = sizeof(WarpSmem<K>) * (kWarpThreads / 32);
    if ((e = cudaFuncSetAttribute(clique_warp_kernel<K, STATS>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ws)) !=
        cudaSuccess)
        return e;
    clique_warp_kernel<K, STATS><<<warp_grid, kWarpThreads, ws, st>>>(a);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    const size_t cs = cta_smem_bytes<K>();
    if ((e = cudaFuncSetAttribute(clique_cta_kernel<K, STATS>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize, (int)cs)) !=
        cudaSuccess)
        return e;
    clique_cta_kernel<K, STATS><<<cta_grid, kCtaThreads, cs, st>>>(a);
    return cudaGetLastError();
}

template <int K, bool STATS>
void occupancy_k(int &warp_occ, int &cta_occ) {
    warp_occ = cta_occ = 0;
    const size_t ws = sizeof(WarpSmem<K>) * (kWarpThreads / 32);
    const size_t cs = cta_smem_bytes<K>();
    if (cudaFuncSetAttribute(clique_warp_kernel<K, STATS>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)ws) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&warp_occ, clique_warp_kernel<K, STATS>,
                                                      kWarpThreads, ws) != cudaSuccess)
        warp_occ = 0;
    if (cudaFuncSetAttribute(clique_cta_kernel<K, STATS>,
                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)cs) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&cta_occ, clique_cta_kernel<K, STATS>,
                                                      kCtaThreads, cs) != cudaSuccess)
        cta_occ = 0;
}

}  // namespace

int64_t clique_rows_words(int32_t max_lower) {
    const int64_t need = (int64_t)max_lower * row_pitch(max_lower);
    return need <= kRowSmemWords ? 0 : need;
}

void clique_blocks_per_sm(int k, bool stats, int *warp_occ, int *cta_occ) {
    int w = 0, c = 0;
    switch (k * 2 + (stats ? 1 : 0)) {
        case 8: occupancy_k<4, false>(w, c); break;
        case 9: occupancy_k<4, true>(w, c); break;
        case 10: occupancy_k<5, false>(w, c); break;
        case 11: occupancy_k<5, true>(w, c); break;
        case 12: occupancy_k<6, false>(w, c); break;
        case 13: occupancy_k<6, true>(w, c); break;
        case 14: occupancy_k<7, false>(w, c); break;
        case 15: occupancy_k<7, true>(w, c); break;
        default: break;
    }
    *warp_occ = w;
    *cta_occ = c;
}

cudaError_t launch_clique(const CliqueLaunch &L, cudaStream_t st) {
    const DevGraphView &g = L.g;
    if (g.lo_off == nullptr) return cudaErrorInvalidValue;
    cudaError_t e;
    if ((e = cudaMemsetAsync(L.ctr, 0, sizeof(DevCounters), st)) != cudaSuccess ||
        (e = cudaMemsetAsync(L.aux, 0, sizeof(CliqueAux), st)) != cudaSuccess)
        return e;
    CliqueArgs a{g.off, g.adj, g.lo_off, g.hub_slot, g.bitmaps, g.bitmap_words,
                 L.v_begin, L.v_end, L.u_begin, L.u_end, L.ctr, L.aux, L.rows, L.rows_stride};
    if (L.v_end <= L.v_begin) return cudaSuccess;
    switch (L.k * 2 + (L.stats ? 1 : 0)) {
        case 8: return launch_k<4, false>(a, L.warp_grid, L.cta_grid, st);
        case 9: return launch_k<4, true>(a, L.warp_grid, L.cta_grid, st);
        case 10: return launch_k<5, false>(a, L.warp_grid, L.cta_grid, st);
        case 11: return launch_k<5, true>(a, L.warp_grid, L.cta_grid, st);
        case 12: return launch_k<6, false>(a, L.warp_grid, L.cta_grid, st);
        case 13: return launch_k<6, true>(a, L.warp_grid, L.cta_grid, st);
        case 14: return launch_k<7, false>(a, L.warp_grid, L.cta_grid, st);
        case 15: return launch_k<7, true>(a, L.warp_grid, L.cta_grid, st);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace gat
