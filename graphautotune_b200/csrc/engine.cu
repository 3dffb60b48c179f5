// The pattern-counting search kernel for sm_100a.
//
// Work decomposition.  The reference expands whole BFS levels from the host
// (engine/engine.cuh:232-319): one prepare kernel, a cub scan, a device->host
// copy and a stream sync per (level, chunk), storing max-degree ints per unit
// per prefix.  Here one persistent launch does the whole search:
//
//  * The level-1 units (v0, v1) are the work queue.  They are numbered by
//    CSR entry (or, when the plan bounds v1 < v0, by entry among each row's
//    lower neighbours) and handed out in chunks through one atomic cursor,
//    which balances power-law rows across the grid.
//  * A tile of G lanes (G = the reference's threads_per_warp knob) owns one
//    unit at a time and walks levels 2 .. basic-1 depth-first; its state
//    (embedding, per-level candidate cursor, per-prefix set descriptor) lives
//    in shared memory.  Sets that later levels intersect with are written to
//    a per-tile scratch slot of max-degree ints; only one chain of sets per
//    tile is live, so scratch is tiles x slots x max_degree, not
//    units x prefixes x max_degree.
//  * Set intersection is tile-cooperative: each lane takes elements of the
//    shorter sorted list and searches the longer one (branch-free binary
//    search, or a linear scan below the set_search_type threshold); stored
//    outputs are compacted in order with ballot + popc.  Bounds from the
//    symmetry-breaking conditions truncate both inputs first (lower_bound,
//    G-ary when G >= 8).
//  * At the last enumerated level the inclusion-exclusion value of the unit
//    is formed from the IEP set sizes and added to a per-tile int64
//    accumulator; each tile adds it to the global total once at exit.
//
// The kernel has no waits on other CTAs: the only inter-CTA interaction is
// atomicAdd on the cursor and the totals.
#include <cub/cub.cuh>

#include <algorithm>
#include <climits>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <string>

#include "../../include/gat.h"
#include "engine.hpp"

namespace gat {
namespace {

constexpr int32_t kInf = INT32_MAX;

struct TileSmem {
    int32_t v[GAT_MAX_VERTICES];
    int32_t cnt[GAT_MAX_VERTICES];
    int32_t pos[GAT_MAX_VERTICES];
    int32_t sl[GAT_MAX_PREFIX];
    int32_t owner[GAT_MAX_PREFIX];  // ALIAS sets: the vertex whose list it is
    int32_t pad[2];
    const int32_t *src[GAT_MAX_VERTICES];
    const int32_t *sp[GAT_MAX_PREFIX];
};

struct SearchArgs {
    const GatPlan *plan;
    const int64_t *off;
    const int32_t *adj;
    const int64_t *lo_off;
    int32_t V;
    int32_t cap;
    int64_t task_begin;  // first level-1 unit of this launch
    int64_t num_tasks;   // one past the last
    DevCounters *ctr;
    int32_t *scratch;
    int64_t scratch_stride;
    int32_t chunk;
    int32_t linear_below;
    const int32_t *hub_slot;   // null: no bitmaps
    const uint32_t *bitmaps;
    int64_t bitmap_words;
};

// One job of a batched launch: a plan on a graph, over the level-1 units
// [task_begin, num_tasks) (ctr, scratch and chunk of `args` are unused; the
// batch supplies them).
struct BatchJob {
    SearchArgs args;
};

template <int G>
struct Tile {
    unsigned mask;
    int lane;
    int base;
    __device__ __forceinline__ Tile() {
        const int wl = threadIdx.x & 31;
        lane = wl & (G - 1);
        base = wl - lane;
        mask = (G == 32) ? 0xffffffffu : (((1u << G) - 1u) << base);
    }
    __device__ __forceinline__ void sync() const { __syncwarp(mask); }
    __device__ __forceinline__ unsigned ballot(bool p) const {
        const unsigned b = __ballot_sync(mask, p);
        return G == 32 ? b : ((b >> base) & ((1u << G) - 1u));
    }
    template <class T>
    __device__ __forceinline__ T bcast(T x, int src) const {
        return __shfl_sync(mask, x, src, G);
    }
    template <class T>
    __device__ __forceinline__ T sum(T x) const {
#pragma unroll
        for (int o = G / 2; o > 0; o >>= 1) x += __shfl_xor_sync(mask, x, o, G);
        return x;
    }
};

__device__ __forceinline__ int32_t min_of(const TileSmem &S, unsigned m) {
    int32_t r = kInf;
    while (m) {
        const int j = __ffs(m) - 1;
        m &= m - 1;
        r = min(r, S.v[j]);
    }
    return r;
}

// First index i in a[0, n) with a[i] >= x (lower) or a[i] > x (upper),
// computed identically on every lane of the tile.
template <int G, bool UPPER, class T>
__device__ __forceinline__ int tile_bound(const Tile<G> &t, const T *a, int n,
                                          T x) {
    if (G < 8) {
        int lo = 0, len = n;
        while (len > 0) {
            const int h = len >> 1;
            const T y = a[lo + h];
            const bool go = UPPER ? (y <= x) : (y < x);
            if (go) {
                lo += h + 1;
                len -= h + 1;
            } else {
                len = h;
            }
        }
        return lo;
    }
    int lo = 0, hi = n;
    while (hi - lo > G) {
        const int p = lo + (int)(((long long)(t.lane + 1) * (hi - lo)) / (G + 1));
        const T y = a[p];
        const bool less = UPPER ? (y <= x) : (y < x);
        const int c = __popc(t.ballot(less));
        const int plo = t.bcast(p, c > 0 ? c - 1 : 0);
        const int phi = t.bcast(p, c < G ? c : G - 1);
        const int nlo = c > 0 ? plo + 1 : lo;
        const int nhi = c < G ? phi : hi;
        lo = nlo;
        hi = nhi;
    }
    bool less = false;
    if (lo + t.lane < hi) {
        const T y = a[lo + t.lane];
        less = UPPER ? (y <= x) : (y < x);
    }
    return lo + __popc(t.ballot(less));
}

// Membership of x in the sorted list b[0, nb): branch-free binary search
// (largest element <= x), or a linear scan for short lists.
__device__ __forceinline__ bool contains(const int32_t *b, int nb, int32_t x,
                                         int linear_below) {
    if (nb <= 0) return false;
    if (nb < linear_below) {
        for (int i = 0; i < nb; i++) {
            const int32_t y = b[i];
            if (y >= x) return y == x;
        }
        return false;
    }
    int lo = 0, len = nb;
    while (len > 1) {
        const int h = len >> 1;
        lo = (b[lo + h] <= x) ? lo + h : lo;
        len -= h;
    }
    return b[lo] == x;
}

// Merge-based intersection for balanced pairs: binary search costs
// |A| log |B| probes, a merge |A| + |B| steps.  Lane l of the tile owns the
// block [l |A| / G, (l + 1) |A| / G) of the shorter list A, finds where the
// block starts in B by one binary search and walks both lists from there, so
// every common element is found once, by the lane owning it in A.
__device__ __forceinline__ bool merge_pays(int shorter, int longer) {
    int lg = 1;
    while ((1 << lg) < longer + 1) lg++;
    return (long long)shorter * lg > 2ll * (shorter + longer);
}

// First i in a[0, n) with a[i] >= x (one lane alone).
__device__ __forceinline__ int lower_index(const int32_t *a, int n, int32_t x) {
    int lo = 0;
    while (n > 0) {
        const int h = n >> 1;
        const bool right = a[lo + h] < x;
        lo = right ? lo + h + 1 : lo;
        n = right ? n - h - 1 : h;
    }
    return lo;
}

// Common elements of a[i0, i1) and b[j, nb) (both sorted), in order: f(x)
// for each.  One lane alone.
template <class F>
__device__ __forceinline__ void merge_walk(const int32_t *a, int i0, int i1, const int32_t *b,
                                           int nb, F &&f) {
    if (i0 >= i1) return;
    int i = i0, j = lower_index(b, nb, a[i0]);
    while (i < i1 && j < nb) {
        const int32_t x = a[i], y = b[j];
        if (x == y) f(x);
        i += x <= y ? 1 : 0;
        j += y <= x ? 1 : 0;
    }
}

template <int G>
__device__ __forceinline__ int merge_count(const Tile<G> &t, const int32_t *a, int na,
                                           const int32_t *b, int nb, const TileSmem &S,
                                           unsigned excl) {
    const int i0 = (int)((long long)na * t.lane / G), i1 = (int)((long long)na * (t.lane + 1) / G);
    int c = 0;
    merge_walk(a, i0, i1, b, nb, [&](int32_t x) {
        bool ok = true;
        unsigned m = excl;
        while (m) {
            const int j = __ffs(m) - 1;
            m &= m - 1;
            ok &= (S.v[j] != x);
        }
        c += ok ? 1 : 0;
    });
    return t.sum(c);
}

// Stored merge: a counting walk, an exclusive scan of the lanes' counts,
// and a writing walk (outputs in order, at most `cap` kept).
template <int G>
__device__ __forceinline__ int merge_store(const Tile<G> &t, const int32_t *a, int na,
                                           const int32_t *b, int nb, int32_t *out, int cap) {
    const int i0 = (int)((long long)na * t.lane / G), i1 = (int)((long long)na * (t.lane + 1) / G);
    int c = 0;
    merge_walk(a, i0, i1, b, nb, [&](int32_t) { c++; });
    int at = c;
#pragma unroll
    for (int o = 1; o < G; o <<= 1) {
        const int y = __shfl_up_sync(t.mask, at, o, G);
        if (t.lane >= o) at += y;
    }
    const int total = t.bcast(at, G - 1);
    at -= c;
    merge_walk(a, i0, i1, b, nb, [&](int32_t x) {
        if (at < cap) out[at] = x;
        at++;
    });
    return total;
}

template <int G>
__device__ __forceinline__ int isect_count(const Tile<G> &t, const int32_t *a,
                                           int na, const int32_t *b, int nb,
                                           const TileSmem &S, unsigned excl,
                                           int linear_below) {
    if (na > nb) {
        const int32_t *tp = a;
        a = b;
        b = tp;
        const int tn = na;
        na = nb;
        nb = tn;
    }
    if (G > 1 && nb >= linear_below && merge_pays(na, nb))
        return merge_count(t, a, na, b, nb, S, excl);
    int c = 0;
    for (int i = t.lane; i < na; i += G) {
        const int32_t x = a[i];
        bool ok = contains(b, nb, x, linear_below);
        unsigned m = excl;
        while (m) {
            const int j = __ffs(m) - 1;
            m &= m - 1;
            ok &= (S.v[j] != x);
        }
        c += ok ? 1 : 0;
    }
    return t.sum(c);
}

// Stored outputs keep at most `cap` elements (the scratch slot's size); the
// returned length is the full intersection size, so a caller sees an
// overflow as a length above cap.
template <int G>
__device__ __forceinline__ int isect_store(const Tile<G> &t, const int32_t *a,
                                           int na, const int32_t *b, int nb,
                                           int32_t *out, int linear_below, int cap) {
    if (na > nb) {
        const int32_t *tp = a;
        a = b;
        b = tp;
        const int tn = na;
        na = nb;
        nb = tn;
    }
    if (G > 1 && nb >= linear_below && merge_pays(na, nb))
        return merge_store(t, a, na, b, nb, out, cap);
    int n = 0;
    for (int base = 0; base < na; base += G) {
        const int i = base + t.lane;
        bool f = false;
        int32_t x = 0;
        if (i < na) {
            x = a[i];
            f = contains(b, nb, x, linear_below);
        }
        const unsigned m = t.ballot(f);
        const int at = n + __popc(m & ((1u << t.lane) - 1u));
        if (f && at < cap) out[at] = x;
        n += __popc(m);
    }
    return n;
}

// Intersections against a hub bitmap: every element of the probe list (a
// sorted list whose elements are all below the bitmap owner's truncation
// bound) costs one read of the owner's row instead of a binary search.
__device__ __forceinline__ bool bit_set(const uint32_t *row, int32_t x) {
    return (__ldg(row + (x >> 5)) >> (x & 31)) & 1u;
}

template <int G>
__device__ __forceinline__ int bitmap_count(const Tile<G> &t, const int32_t *probe,
                                            int np, const uint32_t *row,
                                            const TileSmem &S, unsigned excl) {
    int c = 0;
    for (int i = t.lane; i < np; i += G) {
        const int32_t x = probe[i];
        bool ok = bit_set(row, x);
        unsigned m = excl;
        while (m) {
            const int j = __ffs(m) - 1;
            m &= m - 1;
            ok &= (S.v[j] != x);
        }
        c += ok ? 1 : 0;
    }
    return t.sum(c);
}

template <int G>
__device__ __forceinline__ int bitmap_store(const Tile<G> &t, const int32_t *probe,
                                            int np, const uint32_t *row,
                                            int32_t *out, int cap) {
    int n = 0;
    for (int base = 0; base < np; base += G) {
        const int i = base + t.lane;
        bool f = false;
        int32_t x = 0;
        if (i < np) {
            x = probe[i];
            f = bit_set(row, x);
        }
        const unsigned m = t.ballot(f);
        const int at = n + __popc(m & ((1u << t.lane) - 1u));
        if (f && at < cap) out[at] = x;
        n += __popc(m);
    }
    return n;
}

__device__ __forceinline__ int ceil_log2(int x) {
    return x <= 1 ? 1 : 32 - __clz(x - 1);
}

// |{u in N(v) : u < T}|.  Cut at v itself it is v's lower degree, one read
// of the lower-neighbour offsets (rows are sorted); otherwise a search.
template <int G>
__device__ __forceinline__ int32_t cut_neighbours(const Tile<G> &t, const SearchArgs &a,
                                                  int32_t v, const int32_t *nb, int32_t dv,
                                                  int32_t T) {
    if (T == kInf) return dv;
    if (T == v && a.lo_off != nullptr) return (int32_t)(a.lo_off[v + 1] - a.lo_off[v]);
    return tile_bound<G, false>(t, nb, dv, T);
}

// Builds every prefix set that ends at level k for candidate v.  `cand_idx`
// is v's position in the list it was drawn from (the loop set of level k),
// or -1: that list cut at v is exactly its first cand_idx elements.
template <int G, bool STATS>
__device__ void level_sets(const Tile<G> &t, TileSmem &S, const GatPlan &P,
                           const SearchArgs &a, int k, int32_t v, bool collided,
                           int32_t *scratch, unsigned long long &bytes, int cand_idx = -1) {
    const int64_t o = a.off[v];
    const int32_t *nb = a.adj + o;
    const int32_t dv = (int32_t)(a.off[v + 1] - o);
    const int pe = P.l_pbegin[k + 1];
    const int hub_v = (a.hub_slot != nullptr) ? a.hub_slot[v] : -1;
    for (int p = P.l_pbegin[k]; p < pe; p++) {
        const int kind = P.p_kind[p];
        const int32_t *ptr = S.sp[p];
        int32_t len = 0;
        int32_t owner = -1;
        if (!collided) {
            const int32_t T = min_of(S, P.p_trunc[p]);
            if (kind == GAT_SET_ALIAS) {
                ptr = nb;
                owner = v;
                len = cut_neighbours(t, a, v, nb, dv, T);
            } else {
                const int f = P.p_father[p];
                const int32_t *fp = S.sp[f];
                int32_t fl = S.sl[f];
                // F is already cut at its own bound; cut again only when this
                // set's bound is a different expression.  When F is the list
                // v was drawn from and the bound is v, the cut is v's index.
                if (T != kInf) {
                    if (cand_idx >= 0 && T == v && f == P.l_loop[k])
                        fl = min(fl, cand_idx);
                    else if (P.p_trunc[p] != P.p_trunc[f])
                        fl = tile_bound<G, false>(t, fp, fl, T);
                }
                // Cheapest way to intersect: probe F into v's bitmap, probe
                // N(v) into the bitmap of F's owner, or binary-search the
                // shorter list in the longer one.  Probe lists are cut at T,
                // which is at most F's own bound, so a bit found in the
                // owner's full row is a member of F.  Probing F into v's row
                // when F is no longer than N(v) needs no cut of N(v) at all.
                const int owner_f = S.owner[f];
                const int hub_f =
                    (a.hub_slot != nullptr && owner_f >= 0) ? a.hub_slot[owner_f] : -1;
                const uint32_t *row = nullptr;
                const int32_t *probe = nullptr;
                int np = 0;
                int32_t nl = dv;
                if (hub_v >= 0 && fl <= dv) {
                    row = a.bitmaps + (int64_t)hub_v * a.bitmap_words;
                    probe = fp;
                    np = fl;
                    if (STATS) nl = cut_neighbours(t, a, v, nb, dv, T);
                } else {
                    nl = cut_neighbours(t, a, v, nb, dv, T);
                    const int shorter = min(nl, fl), longer = max(nl, fl);
                    const long long bs_cost = (long long)shorter * ceil_log2(longer + 1);
                    if (hub_v >= 0 && (long long)fl <= bs_cost &&
                        (hub_f < 0 || fl <= nl)) {
                        row = a.bitmaps + (int64_t)hub_v * a.bitmap_words;
                        probe = fp;
                        np = fl;
                    } else if (hub_f >= 0 && (long long)nl <= bs_cost) {
                        row = a.bitmaps + (int64_t)hub_f * a.bitmap_words;
                        probe = nb;
                        np = nl;
                    }
                }
                if (STATS && t.lane == 0) bytes += 4ull * (unsigned)(nl + fl);
                if (kind == GAT_SET_STORE) {
                    int32_t *out = scratch + (int64_t)P.p_slot[p] * a.cap;
                    len = row ? bitmap_store(t, probe, np, row, out, a.cap)
                              : isect_store(t, nb, nl, fp, fl, out, a.linear_below, a.cap);
                    if (len > a.cap) {
                        // The slot is smaller than the set (a caller stated a
                        // maximum degree below the graph's): the count is
                        // void, and the set is cut so no access leaves it.
                        if (t.lane == 0 && a.ctr != nullptr)
                            atomicOr(&a.ctr->error, GAT_DEVERR_SCRATCH);
                        len = a.cap;
                    }
                    ptr = out;
                    if (STATS && t.lane == 0) bytes += 4ull * (unsigned)len;
                } else {
                    len = row ? bitmap_count(t, probe, np, row, S, P.p_excl[p])
                              : isect_count(t, nb, nl, fp, fl, S, P.p_excl[p],
                                            a.linear_below);
                }
            }
        }
        if (t.lane == 0) {
            S.sp[p] = ptr;
            S.sl[p] = len;
            S.owner[p] = owner;
        }
        t.sync();
    }
}

template <int G>
__device__ __forceinline__ void setup_level(const Tile<G> &t, TileSmem &S,
                                            const GatPlan &P, int k) {
    const int lp = P.l_loop[k];
    const int32_t *ptr = S.sp[lp];
    const int32_t len = S.sl[lp];
    const int32_t B = min_of(S, P.l_bound[k]);
    const int32_t cnt = (B == kInf) ? len : tile_bound<G, false>(t, ptr, len, B);
    if (t.lane == 0) {
        S.src[k] = ptr;
        S.cnt[k] = cnt;
        S.pos[k] = 0;
    }
    t.sync();
}

// Inclusion-exclusion value of the current unit (valid on lane 0).  The
// slot values live in lane 0's local memory (only lane 0 forms the terms),
// which keeps the per-tile shared state small enough for 256 one-lane tiles
// per CTA.
template <int G>
__device__ long long iep_value(const Tile<G> &t, TileSmem &S, const GatPlan &P,
                               int linear_below) {
    const int basic = P.basic;
    long long vals[GAT_MAX_PREFIX];
    for (int x = 0; x < P.iep_num; x++) {
        const int p = P.iep_prefix[x];
        long long val;
        if (P.p_kind[p] == GAT_SET_COUNT) {
            val = S.sl[p];
        } else {
            const int32_t *ptr = S.sp[p];
            int32_t len = S.sl[p];
            const int32_t B = min_of(S, P.iep_bound[x]);
            if (B != kInf) len = tile_bound<G, false>(t, ptr, len, B);
            const unsigned m = P.iep_sub[x];
            int hit = 0;
            for (int j = t.lane; j < basic; j += G)
                if ((m >> j) & 1u) hit += contains(ptr, len, S.v[j], linear_below);
            hit = t.sum(hit);
            val = (long long)len - hit;
        }
        if (t.lane == 0) vals[x] = val;
    }
    unsigned long long local = 0, cur = 1;
    if (t.lane == 0) {
        int last = -1;
        for (int g = 0; g < P.num_terms; g++) {
            const unsigned long long v = (unsigned long long)vals[P.t_slot[g]];
            cur = (g == last + 1) ? v : cur * v;
            if (P.t_close[g]) {
                last = g;
                local += cur * (unsigned long long)(long long)P.t_coef[g];
            }
        }
    }
    return (long long)local;
}

// One lane alone: first i in a[0, n) with a[i] >= x.
__device__ __forceinline__ int lower_serial(const int32_t *a, int n, int32_t x) {
    int lo = 0;
    while (n > 0) {
        const int h = n >> 1;
        const bool right = a[lo + h] < x;
        lo = right ? lo + h + 1 : lo;
        n = right ? n - h - 1 : h;
    }
    return lo;
}

__device__ __forceinline__ int32_t cut_serial(const SearchArgs &a, int32_t v,
                                              const int32_t *nb, int32_t dv, int32_t T) {
    if (T == kInf) return dv;
    if (T == v && a.lo_off != nullptr) return (int32_t)(a.lo_off[v + 1] - a.lo_off[v]);
    return lower_serial(nb, dv, T);
}

// y equals one of the levels in `ex` (bit k stands for the lane's candidate).
__device__ __forceinline__ bool excluded(const TileSmem &S, unsigned ex, int k, int32_t cand,
                                         int32_t y) {
    bool r = ((ex >> k) & 1u) && y == cand;
    unsigned m = ex & ~(1u << k);
    while (m) {
        const int j = __ffs(m) - 1;
        m &= m - 1;
        r |= (S.v[j] == y);
    }
    return r;
}

// Last level with one candidate per lane (plans with lane_last set).  Every
// set of level k = basic-1 is either a count |N(cand) n F| whose father F
// belongs to an earlier level or N(cand) itself, so nothing of level k has to
// be stored: lane i takes candidates i, i+G, ... of the level's loop list and
// forms that level's sets and the unit's IEP value alone (IEP slots of
// earlier levels are read from the tile's state).  No shared-memory writes,
// no syncs, and no idle lanes when the lists are shorter than the tile.  Each
// set and each IEP value is formed exactly as level_sets and iep_value form
// it for that candidate (same bounds, exclusions and bitmap-or-search
// choice).  Returns the sum of the candidates' IEP values on every lane.
// The candidates are src[i] for i in [i0, i1): the level's loop list (k >= 2),
// or, at k = 1, the slice of N(v0) that holds the chunk's level-1 units.
template <int G, bool STATS>
__device__ unsigned long long lane_last_level(const Tile<G> &t, const TileSmem &S,
                                              const GatPlan &P, const SearchArgs &a, int k,
                                              unsigned long long &bytes, const int32_t *src,
                                              int i0, int i1) {
    const unsigned kbit = 1u << k;
    const int loop = P.l_loop[k];
    const int pb = P.l_pbegin[k], pe = P.l_pbegin[k + 1];
    unsigned long long sum = 0, by = 0;
    long long lv[8];   // level-k sets: count, or cut length of N(cand)
    long long val[8];  // IEP slots
    for (int i = i0 + t.lane; i < i1; i += G) {
        const int32_t cand = src[i];
        bool hit = false;
        unsigned dm = P.l_distinct[k];
        while (dm) {
            const int j = __ffs(dm) - 1;
            dm &= dm - 1;
            hit |= (S.v[j] == cand);
        }
        // Exact plans skip a colliding candidate; reference plans keep it
        // with every level-k set empty.
        if (hit && !P.collide_clear) continue;
        const int64_t o = a.off[cand];
        const int32_t *nb = a.adj + o;
        const int32_t dv = (int32_t)(a.off[cand + 1] - o);
        const int hub_v = (a.hub_slot != nullptr) ? a.hub_slot[cand] : -1;
        for (int p = pb; p < pe; p++) {
            if (hit) {
                lv[p - pb] = 0;
                continue;
            }
            const unsigned tm = P.p_trunc[p];
            int32_t T = min_of(S, tm & ~kbit);
            if (tm & kbit) T = min(T, cand);
            if (P.p_kind[p] == GAT_SET_ALIAS) {
                lv[p - pb] = cut_serial(a, cand, nb, dv, T);
                continue;
            }
            const int f = P.p_father[p];
            const int32_t *fp = S.sp[f];
            int32_t fl = S.sl[f];
            if (T != kInf) {
                if (T == cand && f == loop)
                    fl = min(fl, i);
                else if (tm != P.p_trunc[f])
                    fl = lower_serial(fp, fl, T);
            }
            const int owner_f = S.owner[f];
            const int hub_f =
                (a.hub_slot != nullptr && owner_f >= 0) ? a.hub_slot[owner_f] : -1;
            const uint32_t *row = nullptr;
            const int32_t *probe = nullptr;
            int np = 0;
            int32_t nl = dv;
            if (hub_v >= 0 && fl <= dv) {
                row = a.bitmaps + (int64_t)hub_v * a.bitmap_words;
                probe = fp;
                np = fl;
                if (STATS) nl = cut_serial(a, cand, nb, dv, T);
            } else {
                nl = cut_serial(a, cand, nb, dv, T);
                const int shorter = min(nl, fl), longer = max(nl, fl);
                const long long bs_cost = (long long)shorter * ceil_log2(longer + 1);
                if (hub_v >= 0 && (long long)fl <= bs_cost && (hub_f < 0 || fl <= nl)) {
                    row = a.bitmaps + (int64_t)hub_v * a.bitmap_words;
                    probe = fp;
                    np = fl;
                } else if (hub_f >= 0 && (long long)nl <= bs_cost) {
                    row = a.bitmaps + (int64_t)hub_f * a.bitmap_words;
                    probe = nb;
                    np = nl;
                }
            }
            if (STATS) by += 4ull * (unsigned)(nl + fl);
            const unsigned ex = P.p_excl[p];
            int c = 0;
            if (row) {
                for (int e = 0; e < np; e++) {
                    const int32_t y = probe[e];
                    c += (bit_set(row, y) && !excluded(S, ex, k, cand, y)) ? 1 : 0;
                }
            } else {
                const int32_t *sa = nl <= fl ? nb : fp;
                const int32_t *lb = nl <= fl ? fp : nb;
                const int ns = min(nl, fl), nlong = max(nl, fl);
                if (nlong >= a.linear_below && merge_pays(ns, nlong)) {
                    merge_walk(sa, 0, ns, lb, nlong, [&](int32_t y) {
                        c += excluded(S, ex, k, cand, y) ? 0 : 1;
                    });
                } else {
                    for (int e = 0; e < ns; e++) {
                        const int32_t y = sa[e];
                        c += (contains(lb, nlong, y, a.linear_below) &&
                              !excluded(S, ex, k, cand, y))
                                 ? 1
                                 : 0;
                    }
                }
            }
            lv[p - pb] = c;
        }
        for (int x = 0; x < P.iep_num; x++) {
            const int p = P.iep_prefix[x];
            const bool here = P.p_level[p] == k;
            if (P.p_kind[p] == GAT_SET_COUNT) {
                val[x] = here ? lv[p - pb] : (long long)S.sl[p];
                continue;
            }
            const int32_t *ptr = here ? nb : S.sp[p];
            int32_t len = here ? (int32_t)lv[p - pb] : S.sl[p];
            const unsigned bm = P.iep_bound[x];
            int32_t B = min_of(S, bm & ~kbit);
            if (bm & kbit) B = min(B, cand);
            if (B != kInf) len = lower_serial(ptr, len, B);
            const unsigned m = P.iep_sub[x];
            int h = 0;
            for (int j = 0; j < P.basic; j++)
                if ((m >> j) & 1u)
                    h += contains(ptr, len, j == k ? cand : S.v[j], a.linear_below) ? 1 : 0;
            val[x] = (long long)len - h;
        }
        unsigned long long local = 0, cur = 1;
        int last = -1;
        for (int g = 0; g < P.num_terms; g++) {
            const unsigned long long v = (unsigned long long)val[P.t_slot[g]];
            cur = (g == last + 1) ? v : cur * v;
            if (P.t_close[g]) {
                last = g;
                local += cur * (unsigned long long)(long long)P.t_coef[g];
            }
        }
        sum += local;
    }
    if (STATS) {
        by = t.sum(by);
        if (t.lane == 0) bytes += by;
    }
    return t.sum(sum);
}

// The lane path pays when the candidates fill at least half the tile, or
// outnumber the elements of the longest father list (the cooperative path
// would then leave most lanes idle on every candidate).
template <int G>
__device__ __forceinline__ bool lane_worth(const TileSmem &S, const GatPlan &P, int k,
                                           int32_t cnt) {
    if (2 * cnt >= G) return true;
    int32_t fmax = 0;
    for (int p = P.l_pbegin[k]; p < P.l_pbegin[k + 1]; p++)
        if (P.p_kind[p] == GAT_SET_COUNT) fmax = max(fmax, S.sl[P.p_father[p]]);
    return cnt >= fmax;
}

// Runs the level-1 units [start, end) of one job: each unit (v0, v1) is the
// start of a depth-first walk over levels 2 .. basic-1.  Lane 0 of the tile
// accumulates the units' IEP values in `acc`.
// ALL_ENTRIES: units are numbered by CSR entry even when the plan bounds
// v1 < v0, and the units that break the bound are skipped here (no
// lower-neighbour offset table needed); used by the allocation-free path.
template <int G, bool STATS, bool ALL_ENTRIES>
__device__ __forceinline__ void run_units(const Tile<G> &t, TileSmem &S, const GatPlan &P,
                                          const SearchArgs &a, int64_t start, int64_t end,
                                          int32_t *scratch, unsigned long long &acc,
                                          unsigned long long &bytes) {
    const int basic = P.basic;
    const int64_t *task_off = (!ALL_ENTRIES && P.level1_bounded) ? a.lo_off : a.off;
    int32_t row = tile_bound<G, true, int64_t>(t, task_off, a.V + 1, start) - 1;
    int32_t cur_v0 = -1;
    for (int64_t tk = start; tk < end; tk++) {
        while (task_off[row + 1] <= tk) row++;
        const int32_t v0 = row;
        const int32_t v1 = a.adj[a.off[v0] + (tk - task_off[v0])];
        if (ALL_ENTRIES && P.level1_bounded && v1 >= v0) continue;
        if (v0 != cur_v0) {
            if (t.lane == 0) S.v[0] = v0;
            t.sync();
            level_sets<G, STATS>(t, S, P, a, 0, v0, false, scratch, bytes);
            cur_v0 = v0;
        }
        if (!ALL_ENTRIES && basic == 2 && P.lane_last) {
            // Two-level plan: the lanes take this row's units of the chunk.
            const int64_t row_end = min(end, task_off[v0 + 1]);
            const int i0 = (int)(tk - task_off[v0]), i1 = (int)(row_end - task_off[v0]);
            if (lane_worth<G>(S, P, 1, i1 - i0)) {
                const unsigned long long r = lane_last_level<G, STATS>(
                    t, S, P, a, 1, bytes, a.adj + a.off[v0], i0, i1);
                if (t.lane == 0) acc += r;
                tk = row_end - 1;
                continue;
            }
        }
        if (t.lane == 0) S.v[1] = v1;
        t.sync();
        level_sets<G, STATS>(t, S, P, a, 1, v1, false, scratch, bytes,
                             (int)(tk - task_off[v0]));
        if (basic == 2) {
            const long long r = iep_value(t, S, P, a.linear_below);
            if (t.lane == 0) acc += (unsigned long long)r;
            t.sync();
            continue;
        }
        setup_level(t, S, P, 2);
        if (basic == 3 && P.lane_last && lane_worth<G>(S, P, 2, S.cnt[2])) {
            const unsigned long long r =
                lane_last_level<G, STATS>(t, S, P, a, 2, bytes, S.src[2], 0, S.cnt[2]);
            if (t.lane == 0) acc += r;
            continue;
        }
        int k = 2;
        while (k >= 2) {
            if (S.pos[k] >= S.cnt[k]) {
                k--;
                continue;
            }
            const int32_t cand = S.src[k][S.pos[k]];
            bool hit = false;
            unsigned dm = P.l_distinct[k];
            while (dm) {
                const int j = __ffs(dm) - 1;
                dm &= dm - 1;
                hit |= (S.v[j] == cand);
            }
            t.sync();
            if (t.lane == 0) S.pos[k]++;
            if (hit && !P.collide_clear) {
                t.sync();
                continue;
            }
            if (t.lane == 0) S.v[k] = cand;
            t.sync();
            level_sets<G, STATS>(t, S, P, a, k, cand, hit, scratch, bytes, S.pos[k] - 1);
            if (k == basic - 1) {
                const long long r = iep_value(t, S, P, a.linear_below);
                if (t.lane == 0) acc += (unsigned long long)r;
                t.sync();
                continue;
            }
            setup_level(t, S, P, k + 1);
            if (k + 1 == basic - 1 && P.lane_last && lane_worth<G>(S, P, k + 1, S.cnt[k + 1])) {
                const unsigned long long r = lane_last_level<G, STATS>(
                    t, S, P, a, k + 1, bytes, S.src[k + 1], 0, S.cnt[k + 1]);
                if (t.lane == 0) acc += r;
                continue;
            }
            k++;
        }
    }
}

template <int G, bool STATS, bool ALL_ENTRIES = false>
__global__ void __launch_bounds__(256)
    search_kernel(const SearchArgs a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const Tile<G> t;
    const int tiles_per_block = blockDim.x / G;
    const int tile_in_block = threadIdx.x / G;
    TileSmem &S = reinterpret_cast<TileSmem *>(smem_raw)[tile_in_block];
    const GatPlan &P = *a.plan;
    int32_t *scratch =
        a.scratch + ((int64_t)blockIdx.x * tiles_per_block + tile_in_block) *
                        a.scratch_stride;
    unsigned long long acc = 0, bytes = 0;
    for (;;) {
        unsigned long long start = 0;
        if (t.lane == 0)
            start = (unsigned long long)a.task_begin +
                    atomicAdd(&a.ctr->cursor, (unsigned long long)a.chunk);
        start = t.bcast(start, 0);
        if (start >= (unsigned long long)a.num_tasks) break;
        const int64_t end = min((int64_t)start + a.chunk, a.num_tasks);
        run_units<G, STATS, ALL_ENTRIES>(t, S, P, a, (int64_t)start, end, scratch, acc,
                                         bytes);
    }
    if (t.lane == 0) {
        atomicAdd(&a.ctr->result, acc);
        if (STATS) atomicAdd(&a.ctr->bytes, bytes);
    }
}

// Many (pattern, graph) jobs in one persistent launch.  Job j owns the
// virtual unit range [vstart[j], vstart[j] + its units rounded up to a whole
// chunk), so a chunk never straddles two jobs; one atomic cursor walks the
// concatenated ranges.  A tile adds its running total to the job's result
// whenever it moves to another job, and at exit.
template <int G>
__global__ void __launch_bounds__(256)
    batch_kernel(const BatchJob *__restrict__ jobs, const int64_t *__restrict__ vstart,
                 int32_t num_jobs, int64_t vtotal, int32_t chunk,
                 unsigned long long *cursor, unsigned long long *results,
                 int32_t *scratch_all, int64_t scratch_stride) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    const Tile<G> t;
    const int tiles_per_block = blockDim.x / G;
    const int tile_in_block = threadIdx.x / G;
    TileSmem &S = reinterpret_cast<TileSmem *>(smem_raw)[tile_in_block];
    int32_t *scratch =
        scratch_all + ((int64_t)blockIdx.x * tiles_per_block + tile_in_block) * scratch_stride;
    unsigned long long acc = 0, bytes = 0;
    int cur_job = -1;
    for (;;) {
        unsigned long long vs = 0;
        if (t.lane == 0) vs = atomicAdd(cursor, (unsigned long long)chunk);
        vs = t.bcast(vs, 0);
        if (vs >= (unsigned long long)vtotal) break;
        const int j = tile_bound<G, true, int64_t>(t, vstart, num_jobs, (int64_t)vs) - 1;
        const BatchJob &job = jobs[j];
        const int64_t start = job.args.task_begin + ((int64_t)vs - vstart[j]);
        if (start >= job.args.num_tasks) continue;  // padding of the job's last chunk
        if (j != cur_job) {
            if (t.lane == 0 && cur_job >= 0 && acc) atomicAdd(&results[cur_job], acc);
            acc = 0;
            cur_job = j;
        }
        const int64_t end = min(start + chunk, job.args.num_tasks);
        run_units<G, false, false>(t, S, *job.args.plan, job.args, start, end, scratch, acc,
                                   bytes);
    }
    if (t.lane == 0 && cur_job >= 0 && acc) atomicAdd(&results[cur_job], acc);
}

template <int G, bool STATS>
cudaError_t launch_one(const SearchArgs &a, int grid, int block,
                       cudaStream_t stream) {
    const size_t smem = size_t(block / G) * sizeof(TileSmem);
    // Set on every launch: the attribute belongs to the current device's
    // context, and a process may count on several devices or reset one.
    cudaError_t e = cudaFuncSetAttribute(
        search_kernel<G, STATS>, cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
    if (e != cudaSuccess) return e;
    search_kernel<G, STATS><<<grid, block, smem, stream>>>(a);
    return cudaGetLastError();
}

template <bool STATS>
cudaError_t dispatch(const SearchArgs &a, int tile, int grid, int block,
                     cudaStream_t s) {
    switch (tile) {
        case 1: return launch_one<1, STATS>(a, grid, block, s);
        case 2: return launch_one<2, STATS>(a, grid, block, s);
        case 4: return launch_one<4, STATS>(a, grid, block, s);
        case 8: return launch_one<8, STATS>(a, grid, block, s);
        case 16: return launch_one<16, STATS>(a, grid, block, s);
        case 32: return launch_one<32, STATS>(a, grid, block, s);
        default: return cudaErrorInvalidValue;
    }
}

template <int G, bool STATS>
int occupancy(int block) {
    int n = 0;
    const size_t smem = size_t(block / G) * sizeof(TileSmem);
    cudaFuncSetAttribute(search_kernel<G, STATS>,
                         cudaFuncAttributeMaxDynamicSharedMemorySize, 227 * 1024);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(
            &n, search_kernel<G, STATS>, block, smem) != cudaSuccess)
        return 0;
    return n;
}

// One CTA per hub (grid-stride over hubs): sets bit x of the hub's row for
// every neighbour x.  Rows are ceil(V/32) words and every x < V.
__global__ void __launch_bounds__(256)
    hub_bitmap_kernel(const int64_t *off, const int32_t *adj, const int32_t *hubs,
                      int32_t nhubs, int64_t words, uint32_t *bitmaps) {
    for (int h = blockIdx.x; h < nhubs; h += gridDim.x) {
        const int32_t v = hubs[h];
        uint32_t *row = bitmaps + (int64_t)h * words;
        for (int64_t i = off[v] + threadIdx.x; i < off[v + 1]; i += blockDim.x) {
            const int32_t x = adj[i];
            atomicOr(row + (x >> 5), 1u << (x & 31));
        }
    }
}

}  // namespace

cudaError_t build_hub_bitmaps(const int64_t *off, const int32_t *adj,
                              const int32_t *hubs, int32_t nhubs, int64_t words,
                              uint32_t *bitmaps, cudaStream_t stream) {
    if (nhubs <= 0) return cudaSuccess;
    const int grid = nhubs < 4096 ? nhubs : 4096;
    hub_bitmap_kernel<<<grid, 256, 0, stream>>>(off, adj, hubs, nhubs, words, bitmaps);
    return cudaGetLastError();
}

size_t tile_smem_bytes() { return sizeof(TileSmem); }

size_t batch_job_bytes() { return sizeof(BatchJob); }

void batch_fill_job(void *dst, const GatPlan *d_plan, const GatPlan &h_plan,
                    const DevGraphView &g, int linear_below, bool use_bitmaps, int shard,
                    int num_shards) {
    BatchJob j{};
    SearchArgs &a = j.args;
    a.plan = d_plan;
    a.off = g.off;
    a.adj = g.adj;
    a.lo_off = g.lo_off;
    a.V = g.V;
    a.cap = g.max_degree > 0 ? g.max_degree : 1;
    const int64_t total = h_plan.level1_bounded ? g.lo_total : g.E;
    a.task_begin = num_shards > 0 ? total * shard / num_shards : 0;
    a.num_tasks = num_shards > 0 ? total * (shard + 1) / num_shards : total;
    a.linear_below = linear_below;
    const bool hubs = use_bitmaps && g.bitmaps != nullptr && g.hub_slot != nullptr;
    a.hub_slot = hubs ? g.hub_slot : nullptr;
    a.bitmaps = hubs ? g.bitmaps : nullptr;
    a.bitmap_words = hubs ? g.bitmap_words : 0;
    std::memcpy(dst, &j, sizeof(j));
}

int64_t batch_job_tasks(const void *job) {
    const SearchArgs &a = reinterpret_cast<const BatchJob *>(job)->args;
    return a.num_tasks - a.task_begin;
}

namespace {
template <int G>
cudaError_t batch_launch_g(const BatchJob *jobs, const int64_t *vstart, int32_t num_jobs,
                           int64_t vtotal, int grid, int block, int chunk,
                           unsigned long long *cursor, unsigned long long *results,
                           int32_t *scratch, int64_t stride, cudaStream_t st) {
    // The shared-memory attribute is set by batch_blocks_per_sm, which callers
    // run first (outside any stream capture).
    const size_t smem = size_t(block / G) * sizeof(TileSmem);
    batch_kernel<G><<<grid, block, smem, st>>>(jobs, vstart, num_jobs, vtotal, chunk, cursor,
                                               results, scratch, stride);
    return cudaGetLastError();
}
template <int G>
int batch_occ(int block) {
    int n = 0;
    const size_t smem = size_t(block / G) * sizeof(TileSmem);
    cudaFuncSetAttribute(batch_kernel<G>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                         227 * 1024);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, batch_kernel<G>, block, smem) !=
        cudaSuccess)
        return 0;
    return n;
}
}  // namespace

int batch_blocks_per_sm(int tile, int block) {
    switch (tile) {
        case 1: return batch_occ<1>(block);
        case 2: return batch_occ<2>(block);
        case 4: return batch_occ<4>(block);
        case 8: return batch_occ<8>(block);
        case 16: return batch_occ<16>(block);
        case 32: return batch_occ<32>(block);
        default: return 0;
    }
}

cudaError_t launch_batch(const void *d_jobs, const int64_t *d_vstart, int32_t num_jobs,
                         int64_t vtotal, int tile, int grid, int block, int chunk,
                         unsigned long long *d_cursor, unsigned long long *d_results,
                         int32_t *scratch, int64_t stride, cudaStream_t st) {
    const BatchJob *jobs = reinterpret_cast<const BatchJob *>(d_jobs);
#define GAT_BL(G)                                                                        \
    return batch_launch_g<G>(jobs, d_vstart, num_jobs, vtotal, grid, block, chunk, d_cursor, \
                             d_results, scratch, stride, st)
    switch (tile) {
        case 1: GAT_BL(1);
        case 2: GAT_BL(2);
        case 4: GAT_BL(4);
        case 8: GAT_BL(8);
        case 16: GAT_BL(16);
        case 32: GAT_BL(32);
        default: return cudaErrorInvalidValue;
    }
#undef GAT_BL
}

int blocks_per_sm(int tile, int block, bool stats) {
#define GAT_OCC(G) \
    return stats ? occupancy<G, true>(block) : occupancy<G, false>(block)
    switch (tile) {
        case 1: GAT_OCC(1);
        case 2: GAT_OCC(2);
        case 4: GAT_OCC(4);
        case 8: GAT_OCC(8);
        case 16: GAT_OCC(16);
        case 32: GAT_OCC(32);
        default: return 0;
    }
#undef GAT_OCC
}

int64_t tile_scratch_ints(const GatPlan &plan, int32_t max_degree) {
    return int64_t(plan.num_store) * int64_t(max_degree > 0 ? max_degree : 1);
}

cudaError_t launch_search(const GatPlan *d_plan, const GatPlan &h_plan,
                          const DevGraphView &g, const LaunchShape &shape,
                          int32_t *scratch, int64_t scratch_stride,
                          DevCounters *counters, bool stats,
                          cudaStream_t stream) {
    cudaError_t e = cudaMemsetAsync(counters, 0, sizeof(DevCounters), stream);
    if (e != cudaSuccess) return e;
    SearchArgs a;
    a.plan = d_plan;
    a.off = g.off;
    a.adj = g.adj;
    a.lo_off = g.lo_off;
    a.V = g.V;
    a.cap = g.max_degree > 0 ? g.max_degree : 1;
    a.task_begin = shape.task_begin;
    a.num_tasks = shape.task_end >= 0 ? shape.task_end
                                      : (h_plan.level1_bounded ? g.lo_total : g.E);
    a.ctr = counters;
    a.scratch = scratch;
    a.scratch_stride = scratch_stride;
    a.chunk = shape.chunk > 0 ? shape.chunk : 1;
    a.linear_below = shape.linear_below;
    const bool hubs = shape.use_bitmaps && g.bitmaps != nullptr && g.hub_slot != nullptr;
    a.hub_slot = hubs ? g.hub_slot : nullptr;
    a.bitmaps = hubs ? g.bitmaps : nullptr;
    a.bitmap_words = hubs ? g.bitmap_words : 0;
    return stats ? dispatch<true>(a, shape.tile, shape.grid, shape.block, stream)
                 : dispatch<false>(a, shape.tile, shape.grid, shape.block, stream);
}

}  // namespace gat

// ------------------------------------------------- allocation-free counting
//
// Every CUDA context that loads this library holds this array until the
// process exits.  Layout: [0, 256) counters, [256, 2048) the device plan,
// [2048, end) per-tile scratch for the stored prefix sets.  Host code must not
// use the array's name as an address: its device address is obtained once
// per device with cudaGetSymbolAddress and passed to the kernels.
static __device__ __align__(256) unsigned char
    gat_noalloc_scratch[GAT_NOALLOC_SCRATCH_BYTES];

namespace gat {
namespace {

constexpr size_t kNoAllocPlanOffset = 256;
constexpr size_t kNoAllocScratchOffset = 2048;
static_assert(sizeof(DevCounters) <= kNoAllocPlanOffset, "counters fit");
static_assert(kNoAllocPlanOffset + sizeof(GatPlan) <= kNoAllocScratchOffset, "plan fits");

std::mutex g_noalloc_mu;
unsigned char *g_noalloc_base[256] = {};  // per device ordinal

// Writes the plan into the static array from the launch's own parameter
// block, so no host buffer has to outlive the call.
__global__ void noalloc_store_plan(const GatPlan plan, GatPlan *dst) {
    constexpr int kWords = int(sizeof(GatPlan) / sizeof(uint32_t));
    static_assert(sizeof(GatPlan) % sizeof(uint32_t) == 0, "plan is whole words");
    const uint32_t *src = reinterpret_cast<const uint32_t *>(&plan);
    uint32_t *out = reinterpret_cast<uint32_t *>(dst);
    for (int i = threadIdx.x; i < kWords; i += blockDim.x) out[i] = src[i];
}

__global__ void noalloc_finish(const DevCounters *c, long long divisor, long long *out) {
    if (threadIdx.x == 0 && blockIdx.x == 0) {
        const long long raw = (long long)c->result;
        const bool ok = c->error == 0 && divisor > 0 && raw % divisor == 0;
        *out = ok ? raw / divisor : LLONG_MIN;
    }
}

template <int G>
cudaError_t noalloc_launch(const SearchArgs &a, int block, int max_grid, int sms,
                           cudaStream_t stream) {
    const size_t smem = size_t(block / G) * sizeof(TileSmem);
    cudaError_t e = cudaFuncSetAttribute(search_kernel<G, false, true>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         227 * 1024);
    if (e != cudaSuccess) return e;
    int occ = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, search_kernel<G, false, true>,
                                                      block, smem);
    if (e != cudaSuccess) return e;
    if (occ < 1) return cudaErrorInvalidConfiguration;
    int grid = sms * occ;
    if (max_grid > 0 && grid > max_grid) grid = max_grid;
    search_kernel<G, false, true><<<grid, block, smem, stream>>>(a);
    return cudaGetLastError();
}

}  // namespace

int count_noalloc(const GatPlan &plan, const int64_t *d_off, const int32_t *d_adj,
                  int32_t V, int64_t E, int32_t max_degree, const LaunchShape &shape,
                  long long *d_count, cudaStream_t stream, std::string *err) {
    auto bad = [&](int code, const std::string &m) {
        if (err) *err = m;
        return code;
    };
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return bad(GAT_ERR_CUDA, cudaGetErrorString(e));
    if (dev < 0 || dev >= 256) return bad(GAT_ERR_CUDA, "device ordinal out of range");
    unsigned char *base = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_noalloc_mu);
        if (!g_noalloc_base[dev]) {
            void *p = nullptr;
            e = cudaGetSymbolAddress(&p, gat_noalloc_scratch);
            if (e != cudaSuccess)
                return bad(GAT_ERR_CUDA, std::string("cudaGetSymbolAddress: ") +
                                             cudaGetErrorString(e));
            g_noalloc_base[dev] = static_cast<unsigned char *>(p);
        }
        base = g_noalloc_base[dev];
    }
    const int tile = shape.tile, block = shape.block;
    const int64_t cap = max_degree > 0 ? max_degree : 1;
    const int64_t stride = int64_t(plan.num_store) * cap;
    const int64_t per_block = int64_t(block / tile) * stride * int64_t(sizeof(int32_t));
    const int64_t avail = int64_t(GAT_NOALLOC_SCRATCH_BYTES) - int64_t(kNoAllocScratchOffset);
    int max_grid = 0;
    if (plan.num_store > 0) {
        if (per_block > avail)
            return bad(GAT_ERR_MEMORY,
                       "one CTA needs " + std::to_string(per_block) +
                           " bytes of set scratch (tiles x stored sets x max degree x 4); "
                           "the static scratch holds " + std::to_string(avail));
        max_grid = (int)std::min<int64_t>(avail / per_block, 1 << 20);
    }
    int sms = 0;
    e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return bad(GAT_ERR_CUDA, cudaGetErrorString(e));
    DevCounters *ctr = reinterpret_cast<DevCounters *>(base);
    GatPlan *dplan = reinterpret_cast<GatPlan *>(base + kNoAllocPlanOffset);
    if ((e = cudaMemsetAsync(ctr, 0, sizeof(DevCounters), stream)) != cudaSuccess)
        return bad(GAT_ERR_CUDA, cudaGetErrorString(e));
    noalloc_store_plan<<<1, 128, 0, stream>>>(plan, dplan);
    if ((e = cudaGetLastError()) != cudaSuccess) return bad(GAT_ERR_CUDA, cudaGetErrorString(e));
    SearchArgs a{};
    a.plan = dplan;
    a.off = d_off;
    a.adj = d_adj;
    a.lo_off = nullptr;
    a.V = V;
    a.cap = (int32_t)cap;
    a.task_begin = 0;
    a.num_tasks = E;
    a.ctr = ctr;
    a.scratch = reinterpret_cast<int32_t *>(base + kNoAllocScratchOffset);
    a.scratch_stride = stride;
    a.chunk = shape.chunk > 0 ? shape.chunk : 1;
    a.linear_below = shape.linear_below;
    a.hub_slot = nullptr;
    a.bitmaps = nullptr;
    a.bitmap_words = 0;
    switch (tile) {
        case 1: e = noalloc_launch<1>(a, block, max_grid, sms, stream); break;
        case 2: e = noalloc_launch<2>(a, block, max_grid, sms, stream); break;
        case 4: e = noalloc_launch<4>(a, block, max_grid, sms, stream); break;
        case 8: e = noalloc_launch<8>(a, block, max_grid, sms, stream); break;
        case 16: e = noalloc_launch<16>(a, block, max_grid, sms, stream); break;
        case 32: e = noalloc_launch<32>(a, block, max_grid, sms, stream); break;
        default: return bad(GAT_ERR_CONFIG, "threads_per_warp must be 1, 2, 4, 8, 16 or 32");
    }
    if (e != cudaSuccess) return bad(GAT_ERR_CUDA, cudaGetErrorString(e));
    noalloc_finish<<<1, 32, 0, stream>>>(ctr, (long long)plan.divisor, d_count);
    e = cudaGetLastError();
    if (e != cudaSuccess) return bad(GAT_ERR_CUDA, cudaGetErrorString(e));
    return GAT_OK;
}

}  // namespace gat
