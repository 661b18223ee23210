// Device-side pieces of the counting DFS shared by the counting kernels:
// per-warp stack state, sorted-set intersections (warp-cooperative binary
// search and merge path, per-lane galloping), the IEP formula and the
// per-warp DFS context (Ctx).  Included by count.cu and noalloc.cu; every
// translation unit gets its own copy (internal linkage).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "internal.hpp"

namespace gi {
namespace {


constexpr int kWarpsPerBlock = 4;
constexpr int kBlockThreads = kWarpsPerBlock * 32;
constexpr int kTaskChunk = GI_TASK_CHUNK;
constexpr unsigned kFull = 0xffffffffu;

// Counter slots in gi_graph::d_counters; kQueue.. kQueue+3 are the handoff
// queue's head, tail, idle-warp and exited-warp counters.
enum : int { kSum = 0, kCursor = 1, kBytes = 2, kTasks = 3, kTimeout = 4, kChunks = 5, kQueue = 6, kLost = 10 };
constexpr int kCounterSlots = 16;

struct WarpState {
    const uint32_t *set_ptr[GI_MAX_PREFIX];
    int32_t set_size[GI_MAX_PREFIX];
    int32_t hub[GI_MAX_PREFIX];        // row in the graph's hub bitmaps when the set is a hub's list, else -1
    int32_t src[GI_MAX_PREFIX];        // v when the set is N(v) itself (an alias), else -1
    uint32_t emb_mask[GI_MAX_PREFIX];  // leaf level: which emb[0, D) lie in each earlier set
    uint32_t emb[GI_MAX_PATTERN + 1];
    int32_t cursor[GI_MAX_PATTERN + 1];
    int32_t end[GI_MAX_PATTERN + 1];
    uint32_t minv[GI_MAX_PATTERN + 1];
};

// Work donation: a warp with a long loop range hands the upper half to an
// idle warp through a queue in device memory.  An item is the partial
// embedding emb[0, depth) and a range [lo, hi) of depth's loop set; the taker
// rebuilds the prefix sets from the embedding (the same sets, built the same
// way) and runs the range.
struct Handoff {
    uint32_t emb[GI_MAX_PATTERN];
    int32_t depth;
    int32_t lo;
    int32_t hi;
    int32_t job;     // the batch job the range belongs to (0 for single counts)
    uint32_t ready;  // == the launch's epoch once the item is written
};

// Adjacency bitmaps of the graph's highest-degree vertices (hubs): row r
// has bit x set when x is a neighbour of the r-th hub, so a membership test
// against a hub's list is one load instead of a search.  Every vertex of
// degree >= min_degree is a hub and row[v] gives its row (row[] is read only
// for such vertices).  n == 0 (the default): no bitmaps, searches only.
struct HubIndex {
    const uint32_t *bits = nullptr;
    const int32_t *row = nullptr;
    int64_t words = 0;  // 32-bit words per row
    int32_t min_degree = 0x7fffffff;
};

// The graph's hub bitmaps as the DFS reads them (none when it has no hubs).
inline HubIndex hubs_of(const gi_graph *g) {
    HubIndex h;
    if (g->n_hubs > 0) {
        h.bits = g->d_hub_bits;
        h.row = g->d_hub_row;
        h.words = g->hub_words;
        h.min_degree = g->hub_min_degree;
    }
    return h;
}

__device__ __forceinline__ bool hub_test(const HubIndex &H, int r, uint32_t x) {
    return (__ldg(&H.bits[static_cast<int64_t>(r) * H.words + (x >> 5)]) >> (x & 31)) & 1u;
}

// Adjacency hash sets (graph.cu): vertex v of degree >= min_degree has the
// table slots[off[v] .. off[v+1]) of a power-of-two size, holding N(v) by
// linear probing from the multiplicative hash; empty slots are 0xffffffff.
struct HashIndex {
    const uint32_t *slots = nullptr;
    const int64_t *off = nullptr;
    int32_t min_degree = 0x7fffffff;
};

inline HashIndex hashes_of(const gi_graph *g) {
    HashIndex h;
    if (g->hash_slots > 0) {
        h.slots = g->d_hash;
        h.off = g->d_hash_off;
        h.min_degree = g->hash_min_degree;
    }
    return h;
}

// v's table and log2 of its size, or nullptr when v (degree deg) has none.
__device__ __forceinline__ const uint32_t *hash_table(const HashIndex &H, uint32_t v, int deg, int &bits) {
    if (deg < H.min_degree) return nullptr;
    const int64_t a = __ldg(&H.off[v]), b = __ldg(&H.off[v + 1]);
    bits = __ffsll(b - a) - 1;
    return H.slots + a;
}

__device__ __forceinline__ bool hash_contains(const uint32_t *t, int bits, uint32_t x) {
    const uint32_t mask = (1u << bits) - 1u;
    uint32_t s = (x * 2654435769u) >> (32 - bits);
    for (uint32_t k = 0; k <= mask; ++k) {
        const uint32_t y = __ldg(&t[s]);
        if (y == x) return true;
        if (y == 0xffffffffu) return false;
        s = (s + 1) & mask;
    }
    return false;
}

// Row of v's bitmap, or -1 when v (degree deg) is not a hub.
__device__ __forceinline__ int hub_row_of(const HubIndex &H, uint32_t v, int deg) {
    return deg >= H.min_degree ? __ldg(&H.row[v]) : -1;
}

struct HandoffQueue {
    Handoff *items = nullptr;       // nullptr: donation off
    unsigned long long cap = 0;
    unsigned long long *ctr = nullptr;  // [0] head, [1] tail, [2] idle warps, [3] exited warps
    uint32_t epoch = 0;
    uint32_t v_cnt = 0;  // items naming a vertex >= v_cnt are rejected
    int32_t job = 0;     // batches: the job being counted, and its count of
    unsigned long long *job_left = nullptr;  // outstanding work items (a donation adds one)
};

// Smallest ranges worth handing off: leaf candidates (lane-parallel) and
// intermediate-level candidates (each a whole subtree).
#ifndef GI_LEAF_HANDOFF_MIN
#define GI_LEAF_HANDOFF_MIN 64
#endif
constexpr int kLeafHandoffMin = GI_LEAF_HANDOFF_MIN;
constexpr int kMidHandoffMin = 4;

__device__ __forceinline__ unsigned long long globaltimer() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %globaltimer;" : "=l"(t));
    return t;
}

// First index in b[0, nb) whose value is >= x.
__device__ __forceinline__ int lower_bound_u32(const uint32_t *b, int nb, uint32_t x) {
    int lo = 0, len = nb;
    while (len > 0) {
        const int half = len >> 1;
        if (b[lo + half] < x) {
            lo += half + 1;
            len -= half + 1;
        } else {
            len = half;
        }
    }
    return lo;
}

__device__ __forceinline__ bool contains_u32(const uint32_t *b, int nb, uint32_t x) {
    const int i = lower_bound_u32(b, nb, x);
    return i < nb && b[i] == x;
}

// Two sorted, duplicate-free lists are "skewed" when the larger is at least
// this many times the smaller: then binary search of the smaller's elements
// beats merging.
constexpr int kSkew = 8;

// Merge path: the position (i, d - i) where the merge of a and b (a first on
// ties) has emitted d elements.
__device__ __forceinline__ int merge_split(const uint32_t *a, int na, const uint32_t *b, int nb, int d) {
    int lo = max(0, d - nb), hi = min(d, na);
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (a[mid] <= b[d - mid - 1])
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo;
}

// This lane's slice [d0, d1) of the merge of a and b: matches (a element
// equal to the b element it is merged against), also those below bound.
// When out is given the matches are written there in order.
__device__ __forceinline__ void merge_slice(const uint32_t *a, int na, const uint32_t *b, int nb, int d0, int d1,
                                            uint32_t bound, int &tot, int &bel, uint32_t *out) {
    int i = merge_split(a, na, b, nb, d0);
    int j = d0 - i;
    int t = 0, u = 0;
    for (int d = d0; d < d1; ++d) {
        if (i < na && (j >= nb || a[i] <= b[j])) {
            const uint32_t x = a[i];
            if (j < nb && x == b[j]) {
                if (out) out[t] = x;
                ++t;
                u += x < bound;
            }
            ++i;
        } else {
            ++j;
        }
    }
    tot = t;
    bel = u;
}

// Warp-cooperative |a ∩ b| (out == nullptr) or a ∩ b written to out in
// sorted order.  Skewed pairs: the smaller set is spread over the lanes and
// each lane binary-searches the larger one.  Balanced pairs: merge path,
// 32 equal slices of the merged sequence, one per lane; with an output the
// slices are counted, scanned and merged again to write.
__device__ __forceinline__ int warp_intersect(const uint32_t *a, int na, const uint32_t *b, int nb, uint32_t *out,
                                              int lane) {
    if (na > nb) {
        const uint32_t *t = a;
        a = b;
        b = t;
        const int tn = na;
        na = nb;
        nb = tn;
    }
    if (na == 0) return 0;
    if (nb >= kSkew * na || na + nb <= 64) {
        int count = 0;
        for (int base = 0; base < na; base += 32) {
            const int i = base + lane;
            bool found = false;
            uint32_t x = 0;
            if (i < na) {
                x = a[i];
                found = contains_u32(b, nb, x);
            }
            const unsigned m = __ballot_sync(kFull, found);
            if (out && found) out[count + __popc(m & ((1u << lane) - 1u))] = x;
            count += __popc(m);
        }
        return count;
    }
    const int total = na + nb;
    const int per = (total + 31) >> 5;
    const int d0 = min(lane * per, total), d1 = min(d0 + per, total);
    int t, u;
    merge_slice(a, na, b, nb, d0, d1, 0u, t, u, nullptr);
    int incl = t;
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(kFull, incl, o);
        if (lane >= o) incl += y;
    }
    const int count = __shfl_sync(kFull, incl, 31);
    if (out && t) merge_slice(a, na, b, nb, d0, d1, 0u, t, u, out + (incl - t));
    return count;
}

// Warp-cooperative |a ∩ b| and |a ∩ b ∩ [0, bound)| (warp-uniform results).
// With need_total false both lists are first cut at bound.
__device__ __forceinline__ void warp_count2(const uint32_t *a, int na, const uint32_t *b, int nb, uint32_t bound,
                                            bool need_total, int lane, int &total, int &below) {
    if (!need_total) {
        na = lower_bound_u32(a, na, bound);
        nb = lower_bound_u32(b, nb, bound);
    }
    if (na > nb) {
        const uint32_t *t = a;
        a = b;
        b = t;
        const int tn = na;
        na = nb;
        nb = tn;
    }
    int t = 0, u = 0;
    if (na > 0) {
        if (nb >= kSkew * na) {
            for (int i = lane; i < na; i += 32) {
                const uint32_t x = a[i];
                if (contains_u32(b, nb, x)) {
                    ++t;
                    u += x < bound;
                }
            }
        } else {
            const int all = na + nb;
            const int per = (all + 31) >> 5;
            const int d0 = min(lane * per, all), d1 = min(d0 + per, all);
            merge_slice(a, na, b, nb, d0, d1, bound, t, u, nullptr);
        }
    }
    for (int o = 16; o; o >>= 1) {
        t += __shfl_xor_sync(kFull, t, o);
        u += __shfl_xor_sync(kFull, u, o);
    }
    total = t;
    below = need_total ? u : t;
}

// First index in b[lo, nb) whose value is >= x, galloping forward from lo
// (cost grows with the log of the distance moved).
__device__ __forceinline__ int gallop_u32(const uint32_t *b, int lo, int nb, uint32_t x) {
    int step = 1, hi = lo;
    while (hi < nb && b[hi] < x) {
        lo = hi + 1;
        hi += step;
        step <<= 1;
    }
    hi = min(hi, nb);
    return lo + lower_bound_u32(b + lo, hi - lo, x);
}

// One lane: |a ∩ b| and |a ∩ b ∩ [0, bound)|.  With need_total false both
// lists are first cut at bound and only the second number is computed.  The
// smaller list is walked in order, galloping through the larger one.
__device__ __forceinline__ void lane_intersect(const uint32_t *a, int na, const uint32_t *b, int nb, uint32_t bound,
                                               bool need_total, int &total, int &below) {
    if (!need_total) {
        na = lower_bound_u32(a, na, bound);
        nb = lower_bound_u32(b, nb, bound);
    }
    if (na > nb) {
        const uint32_t *t = a;
        a = b;
        b = t;
        const int tn = na;
        na = nb;
        nb = tn;
    }
    int tot = 0, bel = 0, lo = 0;
    for (int i = 0; i < na && lo < nb; ++i) {
        const uint32_t x = a[i];
        lo = gallop_u32(b, lo, nb, x);
        if (lo < nb && b[lo] == x) {
            ++tot;
            bel += x < bound;
            ++lo;
        }
    }
    total = tot;
    below = need_total ? bel : tot;
}

// Membership tests for the counting helpers below: a hub's bitmap row, or
// an adjacency hash set.
struct HubTest {
    const HubIndex &H;
    int r;
    __device__ __forceinline__ bool operator()(uint32_t x) const { return hub_test(H, r, x); }
};
struct HashTest {
    const uint32_t *t;
    int bits;
    __device__ __forceinline__ bool operator()(uint32_t x) const { return hash_contains(t, bits, x); }
};

// One lane: |a ∩ T| and |a ∩ T ∩ [0, bound)| for a membership test T, one
// test per element of a; with need_total false only elements below bound
// are tested.  Loads are issued four at a time.
template <class Test>
__device__ __forceinline__ void lane_count_member(const Test &test, const uint32_t *a, int na, uint32_t bound,
                                                  bool need_total, int &total, int &below) {
    int tot = 0, bel = 0;
    int i = 0;
    for (; i + 4 <= na; i += 4) {
        const uint32_t x0 = a[i], x1 = a[i + 1], x2 = a[i + 2], x3 = a[i + 3];
        if (!need_total && x0 >= bound) {
            na = i;  // sorted: nothing further is below bound
            break;
        }
        const bool h0 = test(x0), h1 = test(x1), h2 = test(x2), h3 = test(x3);
        tot += h0 + h1 + h2 + h3;
        bel += (h0 && x0 < bound) + (h1 && x1 < bound) + (h2 && x2 < bound) + (h3 && x3 < bound);
    }
    for (; i < na; ++i) {
        const uint32_t x = a[i];
        if (!need_total && x >= bound) break;
        const bool h = test(x);
        tot += h;
        bel += h && x < bound;
    }
    total = need_total ? tot : bel;
    below = bel;
}

// Warp-cooperative |a ∩ T| and |a ∩ T ∩ [0, bound)| (warp-uniform).
template <class Test>
__device__ __forceinline__ void warp_count_member(const Test &test, const uint32_t *a, int na, uint32_t bound,
                                                  bool need_total, int lane, int &total, int &below) {
    if (!need_total) na = lower_bound_u32(a, na, bound);
    int t = 0, u = 0;
    for (int i = lane; i < na; i += 32) {
        const uint32_t x = a[i];
        if (test(x)) {
            ++t;
            u += x < bound;
        }
    }
    for (int o = 16; o; o >>= 1) {
        t += __shfl_xor_sync(kFull, t, o);
        u += __shfl_xor_sync(kFull, u, o);
    }
    total = need_total ? t : u;
    below = u;
}

// Warp-cooperative a ∩ N(h) written to out in a's (sorted) order, or only
// its size when out is nullptr.
__device__ __forceinline__ int warp_intersect_hub(const HubIndex &H, int r, const uint32_t *a, int na, uint32_t *out,
                                                  int lane) {
    int count = 0;
    for (int base = 0; base < na; base += 32) {
        const int i = base + lane;
        uint32_t x = 0;
        bool found = false;
        if (i < na) {
            x = a[i];
            found = hub_test(H, r, x);
        }
        const unsigned m = __ballot_sync(kFull, found);
        if (out && found) out[count + __popc(m & ((1u << lane) - 1u))] = x;
        count += __popc(m);
    }
    return count;
}

// Steps a lane would spend intersecting lists of sizes x and y: the smaller
// times the log of the size ratio.
__device__ __forceinline__ int lane_cost(int x, int y) {
    const int lo = min(x, y), hi = max(x, y);
    if (lo == 0) return 0;
    return lo * (33 - __clz(hi / lo + 1));
}

// A leaf candidate costlier than DevPlan::lane_budget for one lane goes to the
// whole warp; GI_LANE_BUDGET (experiments) overrides every plan's value.
#ifdef GI_LANE_BUDGET
constexpr int kLaneBudgetOverride = GI_LANE_BUDGET;
#else
constexpr int kLaneBudgetOverride = -1;
#endif

// How many of emb[0, d) occur in s[0, n), warp-cooperative.
__device__ __forceinline__ int warp_count_embedded(const uint32_t *s, int n, const WarpState &w, int d, int lane) {
    const bool hit = lane < d && n > 0 && contains_u32(s, n, w.emb[lane]);
    return __popc(__ballot_sync(kFull, hit));
}

// Bit u set when emb[u] (u < d) occurs in s[0, n), warp-cooperative.
__device__ __forceinline__ uint32_t warp_embedded_mask(const uint32_t *s, int n, const WarpState &w, int d, int lane) {
    const bool hit = lane < d && n > 0 && contains_u32(s, n, w.emb[lane]);
    return __ballot_sync(kFull, hit);
}

// Vertex-induced filter: x must not be adjacent to an embedded vertex whose
// pattern position is not adjacent to position d (reference
// gpu/function/pattern_matching.cuh:145-206, src/graph.cpp:195-232).
__device__ __forceinline__ bool anti_adjacent(const DevPlan &P, const WarpState &w, int d, uint32_t x,
                                              const int64_t *__restrict__ vertex,
                                              const uint32_t *__restrict__ edge) {
    for (int u = 0; u < d; ++u) {
        if (P.adj[u * P.n + d]) continue;
        const uint32_t e = w.emb[u];
        const int64_t l = __ldg(&vertex[e]);
        const int deg = static_cast<int>(__ldg(&vertex[e + 1]) - l);
        if (contains_u32(edge + l, deg, x)) return true;
    }
    return false;
}

__device__ __forceinline__ unsigned long long warp_sum(unsigned long long x) {
    for (int o = 16; o; o >>= 1) x += __shfl_xor_sync(kFull, x, o);
    return x;
}

// IEP formula (reference src/graph.cpp:474-492): products of the answers
// of each partition's blocks, times the partition's signed coefficient.
__device__ __forceinline__ unsigned long long iep_combine(const DevPlan &P, const int *ans) {
    unsigned long long acc = 0, val = 0;
    int last_pos = -1;
#pragma unroll 1
    for (int pos = 0; pos < P.iep_nterms; ++pos) {
        const long long a = ans[P.iep_pos[pos]];
        if (pos == last_pos + 1)
            val = static_cast<unsigned long long>(a);
        else if (val != 0)
            val = val * static_cast<unsigned long long>(a);
        if (P.iep_flag[pos]) {
            last_pos = pos;
            acc += val * static_cast<unsigned long long>(static_cast<long long>(P.iep_coef[pos]));
        }
    }
    return acc;
}

// One sorted list of a pair, with the structures that answer membership
// in it: a hub's bitmap row (hub >= 0) or an adjacency hash set (hash).
struct ListRef {
    const uint32_t *p;
    int n;
    int hub;
    const uint32_t *hash;
    int hash_bits;
};

// Membership of x in a target coded as flat_count codes it: code >= 0 a
// sorted list tgt[0, code); -1 a bitmap row; <= -2 a hash set of -2 - code
// bits.
__device__ __forceinline__ bool member_of(int code, const uint32_t *tgt, uint32_t x) {
    if (code >= 0) return contains_u32(tgt, code, x);
    if (code == -1) return ((__ldg(&tgt[x >> 5]) >> (x & 31)) & 1u) != 0;
    return hash_contains(tgt, -2 - code, x);
}

// Warp-cooperative a ∩ T for a membership target T (member_of), written to
// out in a's (sorted) order, or only its size when out is nullptr.
__device__ __forceinline__ int warp_intersect_probe(const uint32_t *a, int na, int code, const uint32_t *tgt,
                                                    uint32_t *out, int lane) {
    int count = 0;
    for (int base = 0; base < na; base += 32) {
        const int i = base + lane;
        uint32_t x = 0;
        bool found = false;
        if (i < na) {
            x = a[i];
            found = member_of(code, tgt, x);
        }
        const unsigned m = __ballot_sync(kFull, found);
        if (out && found) out[count + __popc(m & ((1u << lane) - 1u))] = x;
        count += __popc(m);
    }
    return count;
}

// Steps to test one element for membership in l: one bitmap load, about two
// hash-set loads, or a binary search.
__device__ __forceinline__ int member_cost(const ListRef &l) {
    return l.hub >= 0 ? 1 : l.hash ? 2 : 33 - __clz(l.n + 1);
}

// Per lane: |a ∩ b| and |a ∩ b ∩ [0, bound)| for the lane's own pair of
// sorted lists, with the work of all 32 pairs spread evenly over the lanes.
// Each lane's probes are the elements of one list of its pair, tested for
// membership in the other through the other's bitmap row, hash set or, for a
// plain list, binary search; the direction with fewer expected steps is
// taken.  The warp walks the concatenation of all lanes' probes 32 at a
// time: a lane finds the pair owning its probe (binary search over the
// exclusive scan of the probe counts), tests it, and the hit ballots are
// split back to the owners by their probe ranges.  Every lane does one test
// per step whatever the list sizes, and consecutive lanes read consecutive
// elements of a list.  Without need_total only elements below bound are
// probed (tot == bel).  A lane with active false has no probes and gets 0.
// All lanes must call it together.
__device__ __forceinline__ void flat_count(const HubIndex &H, const ListRef &a, const ListRef &b, uint32_t bound,
                                           bool need_total, bool active, int lane, int &tot, int &bel) {
    const uint32_t *probe = a.p, *tgt = b.p;
    int n = 0, code = 0;  // code >= 0: binary search in tgt[0, code); -1: bitmap row; <= -2: hash of -2 - code bits
    if (active) {
        const bool a_in_b = static_cast<int64_t>(a.n) * member_cost(b) <= static_cast<int64_t>(b.n) * member_cost(a);
        const ListRef &pr = a_in_b ? a : b;
        const ListRef &tg = a_in_b ? b : a;
        probe = pr.p;
        n = pr.n;
        if (tg.hub >= 0) {
            tgt = H.bits + static_cast<int64_t>(tg.hub) * H.words;
            code = -1;
        } else if (tg.hash) {
            tgt = tg.hash;
            code = -2 - tg.hash_bits;
        } else {
            tgt = tg.p;
            code = tg.n;
        }
        if (!need_total) n = lower_bound_u32(probe, n, bound);
    }
    int incl = n;
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(kFull, incl, o);
        if (lane >= o) incl += y;
    }
    const int off = incl - n;
    const int total = __shfl_sync(kFull, incl, 31);
    const unsigned long long pa = reinterpret_cast<unsigned long long>(probe);
    const unsigned long long ta = reinterpret_cast<unsigned long long>(tgt);
    int t = 0, u = 0;
    for (int t0 = 0; t0 < total; t0 += 32) {
        const int item = t0 + lane;
        // Owner: the last lane whose probes start at or before item.
        int c = 0;
        for (int step = 16; step; step >>= 1) {
            const int o2 = __shfl_sync(kFull, off, c + step);
            if (o2 <= item) c += step;
        }
        const int k = item - __shfl_sync(kFull, off, c);
        const uint32_t *pc = reinterpret_cast<const uint32_t *>(__shfl_sync(kFull, pa, c));
        const uint32_t *tc = reinterpret_cast<const uint32_t *>(__shfl_sync(kFull, ta, c));
        const int cc = __shfl_sync(kFull, code, c);
        const uint32_t bc = __shfl_sync(kFull, bound, c);
        bool hit = false, below = false;
        if (item < total) {
            const uint32_t x = pc[k];
            if (cc >= 0)
                hit = contains_u32(tc, cc, x);
            else if (cc == -1)
                hit = ((__ldg(&tc[x >> 5]) >> (x & 31)) & 1u) != 0;
            else
                hit = hash_contains(tc, -2 - cc, x);
            below = hit && x < bc;
        }
        const unsigned hm = __ballot_sync(kFull, hit), bm = __ballot_sync(kFull, below);
        const int lo = max(off - t0, 0), hi = min(off + n - t0, 32);
        if (lo < hi) {
            const unsigned rm = (hi == 32 ? kFull : (1u << hi) - 1u) & ~((1u << lo) - 1u);
            t += __popc(hm & rm);
            u += __popc(bm & rm);
        }
    }
    tot = t;
    bel = u;
}

template <bool kBytesOn>
struct Ctx {
    const DevPlan &P;
    const int64_t *__restrict__ vertex;
    const uint32_t *__restrict__ edge;
    uint32_t *slot_base;
    int64_t slot_stride;
    WarpState &w;
    int lane;
    unsigned long long bytes;  // per lane in the leaf level, warp-uniform elsewhere (summed over lanes at the end / 1 lane)
    unsigned long long t_start = 0;
    unsigned long long hard_ns = 0;  // > 0: give up the current work item past this much time
    bool aborted = false;
    HandoffQueue hq{};
    HubIndex hubs{};
    HashIndex hashes{};

    // Offers [lo, hi) of depth d's loop to an idle warp (warp-uniform);
    // true when it was queued and is no longer this warp's to do.
    __device__ __forceinline__ bool donate(int d, int lo, int hi) {
        int ok = 0;
        if (d < 2 || d >= P.stop || lo < 0 || hi <= lo) return false;  // not a handoff range
        if (lane == 0 && *(volatile unsigned long long *)&hq.ctr[2] > 0) {
            const unsigned long long slot = atomicAdd(&hq.ctr[1], 1ull);
            if (slot < hq.cap) {
                Handoff &h = hq.items[slot];
                for (int u = 0; u < d; ++u) h.emb[u] = w.emb[u];
                h.depth = d;
                h.lo = lo;
                h.hi = hi;
                h.job = hq.job;
                if (hq.job_left) atomicAdd(&hq.job_left[hq.job], 1ull);
                __threadfence();
                *(volatile uint32_t *)&h.ready = hq.epoch;
                ok = 1;
            }
        }
        return __shfl_sync(kFull, ok, 0) != 0;
    }

    // Warp-uniform: true once the hard time limit has passed (lane 0's
    // clock decides for the warp).
    __device__ __forceinline__ bool out_of_time() {
        if (!hard_ns) return false;
        unsigned long long now = 0;
        if (lane == 0) now = globaltimer();
        now = __shfl_sync(kFull, now, 0);
        if (now - t_start > hard_ns) aborted = true;
        return aborted;
    }

    // Builds every prefix whose last member is position d, with v placed at d.
    // Returns false when a prefix reaches its break size (no completion can
    // use it), mirroring the reference prune (src/graph.cpp:535-545).
    __device__ __forceinline__ bool build_chain(int d, uint32_t v, bool account = true) {
        const int64_t l = __ldg(&vertex[v]);
        const int deg = static_cast<int>(__ldg(&vertex[v + 1]) - l);
        const uint32_t *nb = edge + l;
        const int hv = hub_row_of(hubs, v, deg);  // v's own bitmap row, or -1
        for (int p = P.last[d]; p != -1; p = P.next[p]) {
            int size;
            const int f = P.father[p];
            if (f == -1) {
                if (lane == 0) {
                    w.set_ptr[p] = nb;
                    w.hub[p] = hv;
                    w.src[p] = static_cast<int32_t>(v);
                }
                size = deg;
                if (kBytesOn && account && lane == 0) bytes += 16;
            } else {
                const uint32_t *fs = w.set_ptr[f];
                const int fn = w.set_size[f];
                const int hf = w.hub[f];
                // A hub's list on either side: test the other list's elements
                // against its bitmap.
                const bool by_f = hf >= 0 && fn >= deg, by_v = !by_f && hv >= 0;
                uint32_t *out = P.mode[p] == kMaterialize ? slot_base + static_cast<int64_t>(P.slot[p]) * slot_stride
                                                          : nullptr;
                int bf = 0, bv = 0;
                const int sf = w.src[f];
                const uint32_t *tf = by_f || by_v || sf < 0 ? nullptr : hash_table(hashes, sf, fn, bf);
                const uint32_t *tv = by_f || by_v ? nullptr : hash_table(hashes, v, deg, bv);
                // A hash set on either side: probe the other list through it
                // when that takes fewer steps than merging.
                const int64_t via_v = tv ? 2ll * fn : INT64_MAX, via_f = tf ? 2ll * deg : INT64_MAX;
                if (by_f)
                    size = warp_intersect_hub(hubs, hf, nb, deg, out, lane);
                else if (by_v)
                    size = warp_intersect_hub(hubs, hv, fs, fn, out, lane);
                else if (min(via_v, via_f) < static_cast<int64_t>(fn) + deg)
                    size = via_v <= via_f ? warp_intersect_probe(fs, fn, -2 - bv, tv, out, lane)
                                          : warp_intersect_probe(nb, deg, -2 - bf, tf, out, lane);
                else
                    size = warp_intersect(fs, fn, nb, deg, out, lane);
                if (lane == 0) {
                    if (out) w.set_ptr[p] = out;
                    w.hub[p] = -1;
                    w.src[p] = -1;
                }
                if (kBytesOn && account && lane == 0) bytes += 4ull * (fn + deg + (out ? size : 0));
            }
            if (lane == 0) w.set_size[p] = size;
            __syncwarp();
            if (size == P.break_size[p]) return false;
        }
        return true;
    }

    __device__ __forceinline__ uint32_t min_vertex(int d) const {
        uint32_t m = 0xffffffffu;
        for (int i = P.restrict_last[d]; i != -1; i = P.restrict_next[i]) m = min(m, w.emb[P.restrict_index[i]]);
        return m;
    }

    // Last position without an IEP tail, warp-cooperative: candidates below
    // the restriction bound that are not already embedded (reference
    // src/graph.cpp:496-519).
    __device__ __forceinline__ unsigned long long last_level(int d) {
        const int ls = P.loop_set[d];
        const uint32_t *s = w.set_ptr[ls];
        const int n = w.set_size[ls];
        if (n <= 0) return 0;
        const uint32_t bound_v = min_vertex(d);
        const int bound = lower_bound_u32(s, n, bound_v);
        if (kBytesOn && lane == 0) bytes += 4ull * bound;
        if (bound <= 0) return 0;
        if (!P.vertex_induced) return static_cast<unsigned long long>(bound - warp_count_embedded(s, bound, w, d, lane));
        unsigned long long c = 0;
        for (int base = 0; base < bound; base += 32) {
            const int i = base + lane;
            bool ok = false;
            if (i < bound) {
                const uint32_t x = s[i];
                ok = true;
                for (int u = 0; u < d; ++u) ok = ok && w.emb[u] != x;
                ok = ok && !anti_adjacent(P, w, d, x, vertex, edge);
            }
            c += __popc(__ballot_sync(kFull, ok));
        }
        return c;
    }

    // IEP tail at position d = n - k, warp-cooperative (reference
    // src/graph.cpp:456-493, gpu/function/pattern_matching.cuh:110-139).
    __device__ __forceinline__ unsigned long long iep_tail(int d) {
        if (w.set_size[P.loop_set[d]] <= 0) return 0;
        int ans[GI_MAX_IEP_SETS];
#pragma unroll 1
        for (int i = 0; i < P.iep_nsets; ++i) {
            const int p = P.iep_set[i];
            const int sz = w.set_size[p];
            if (P.iep_set_flag[i]) {
                ans[i] = sz - P.iep_set_coef[i];
            } else {
                ans[i] = sz - warp_count_embedded(w.set_ptr[p], sz, w, d, lane);
                if (kBytesOn && lane == 0) bytes += 4ull * sz;
            }
        }
        return iep_combine(P, ans);
    }

    // One candidate v at the leaf-parent depth D: the prefixes it would build
    // (sizes only), the break-size prune, then the last-level count or the
    // IEP formula.  kWarp = false: this lane alone, no warp-synchronous
    // operation; kWarp = true: the whole warp with merge-path counts, every
    // lane computing the same (warp-uniform) result.  emb[0, D) and the
    // emb_mask of every earlier set are warp-shared.
    template <bool kWarp>
    __device__ __forceinline__ unsigned long long leaf_eval(int D, uint32_t v) {
        const int64_t l = __ldg(&vertex[v]);
        const int dv = static_cast<int>(__ldg(&vertex[v + 1]) - l);
        const uint32_t *nv = edge + l;
        const int hv = hub_row_of(hubs, v, dv);
        uint32_t mask_nv = 0;  // emb[u] in N(v)
        if (kWarp) {
            mask_nv = __ballot_sync(kFull, lane < D && (hv >= 0 ? hub_test(hubs, hv, w.emb[lane])
                                                              : contains_u32(nv, dv, w.emb[lane])));
        } else {
            for (int u = 0; u < D; ++u)
                mask_nv |= static_cast<uint32_t>(hv >= 0 ? hub_test(hubs, hv, w.emb[u]) : contains_u32(nv, dv, w.emb[u]))
                           << u;
        }
        const bool count_here = !kWarp || lane == 0;  // who adds the bytes
        const int stop = P.stop;
        const int L = P.loop_set[stop];
        const bool last_level = P.iep_k == 0;
        // Restriction bound of the last position (may involve v itself).
        uint32_t bound = 0xffffffffu;
        if (last_level)
            for (int i = P.restrict_last[stop]; i != -1; i = P.restrict_next[i]) {
                const int idx = P.restrict_index[i];
                bound = min(bound, idx == D ? v : w.emb[idx]);
            }
        int size[GI_MAX_PREFIX];
        uint32_t mask[GI_MAX_PREFIX];
        int below_L = 0;
        unsigned long long b = 0;
        for (int p = P.last[D]; p != -1; p = P.next[p]) {
            const int f = P.father[p];
            if (f == -1) {
                size[p] = dv;
                mask[p] = mask_nv;
                if (kBytesOn) b += 16;
                below_L = p == L ? lower_bound_u32(nv, dv, bound) : below_L;
            } else {
                const uint32_t *fs = w.set_ptr[f];
                const int fn = w.set_size[f];
                // L's own prune is implied by its count (a set that holds only
                // embedded vertices counts zero), so L alone may stop at bound.
                const bool need_total = kBytesOn || !(last_level && p == L);
                const int hf = w.hub[f];
                int tot, bel;
                // A hash set on either side (when no bitmap serves): probe
                // the other list through it if that takes fewer steps.
                int bf = 0, bv = 0;
                const uint32_t *tf = nullptr, *tv = nullptr;
                if (!(hf >= 0 && fn >= dv) && hv < 0) {
                    if (w.src[f] >= 0) tf = hash_table(hashes, static_cast<uint32_t>(w.src[f]), fn, bf);
                    tv = hash_table(hashes, v, dv, bv);
                }
                const int merge_steps = kWarp ? (fn + dv + 31) / 32 : lane_cost(fn, dv);
                const int via_v = tv ? 2 * fn / (kWarp ? 32 : 1) : 0x7fffffff;
                const int via_f = tf ? 2 * dv / (kWarp ? 32 : 1) : 0x7fffffff;
                if (hf >= 0 && fn >= dv) {
                    if (kWarp)
                        warp_count_member(HubTest{hubs, hf}, nv, dv, bound, need_total, lane, tot, bel);
                    else
                        lane_count_member(HubTest{hubs, hf}, nv, dv, bound, need_total, tot, bel);
                } else if (hv >= 0) {
                    if (kWarp)
                        warp_count_member(HubTest{hubs, hv}, fs, fn, bound, need_total, lane, tot, bel);
                    else
                        lane_count_member(HubTest{hubs, hv}, fs, fn, bound, need_total, tot, bel);
                } else if (min(via_v, via_f) < merge_steps) {
                    const bool probe_f = via_v <= via_f;  // fs's elements into N(v)'s set
                    const HashTest test{probe_f ? tv : tf, probe_f ? bv : bf};
                    if (kWarp)
                        warp_count_member(test, probe_f ? fs : nv, probe_f ? fn : dv, bound, need_total, lane, tot,
                                          bel);
                    else
                        lane_count_member(test, probe_f ? fs : nv, probe_f ? fn : dv, bound, need_total, tot, bel);
                } else if (kWarp) {
                    warp_count2(fs, fn, nv, dv, bound, need_total, lane, tot, bel);
                } else {
                    lane_intersect(fs, fn, nv, dv, bound, need_total, tot, bel);
                }
                size[p] = tot;
                if (p == L) below_L = bel;
                mask[p] = w.emb_mask[f] & mask_nv;
                if (kBytesOn) b += 4ull * (fn + dv + (P.mode[p] == kSizeOnly ? 0 : tot));
                if (!need_total) continue;
            }
            if (size[p] == P.break_size[p]) {
                if (kBytesOn && count_here) bytes += b;
                return 0;
            }
        }
        unsigned long long contrib = 0;
        if (last_level) {
            const bool in_chain = P.pdepth[L] == D;
            int below;
            uint32_t m;
            bool v_in = false;
            if (in_chain) {
                below = below_L;
                m = mask[L];
            } else {
                const uint32_t *s = w.set_ptr[L];
                const int n = w.set_size[L];
                if (n <= 0) {
                    if (kBytesOn && count_here) bytes += b;
                    return 0;
                }
                below = lower_bound_u32(s, n, bound);
                m = w.emb_mask[L];
                v_in = v < bound && contains_u32(s, below, v);
            }
            if (kBytesOn) b += 4ull * below;
            int emb_below = v_in ? 1 : 0;
            for (int u = 0; u < D; ++u) emb_below += ((m >> u) & 1u) && w.emb[u] < bound;
            contrib = static_cast<unsigned long long>(below - emb_below);
        } else {
            const int ls = L;  // loop set of the IEP depth: empty means no completion
            const int ls_size = P.pdepth[ls] == D ? size[ls] : w.set_size[ls];
            if (ls_size > 0) {
                int ans[GI_MAX_IEP_SETS];
#pragma unroll 1
                for (int i = 0; i < P.iep_nsets; ++i) {
                    const int q = P.iep_set[i];
                    const bool in_chain = P.pdepth[q] == D;
                    const int sz = in_chain ? size[q] : w.set_size[q];
                    if (P.iep_set_flag[i]) {
                        ans[i] = sz - P.iep_set_coef[i];
                    } else {
                        // |S - emb[0, D]|: v itself is in S only for earlier sets.
                        const uint32_t m = in_chain ? mask[q] : w.emb_mask[q];
                        int c = __popc(m & ((1u << D) - 1u));
                        if (!in_chain && contains_u32(w.set_ptr[q], sz, v)) ++c;
                        ans[i] = sz - c;
                        if (kBytesOn) b += 4ull * sz;
                    }
                }
                contrib = iep_combine(P, ans);
            }
        }
        if (kBytesOn && count_here) bytes += b;
        return contrib;
    }

    // Leaf-parent depth D: every candidate of the loop set in [i0, i1) below
    // the restriction bound, one per lane; a candidate whose intersections
    // would keep one lane busy for more than the plan's lane budget (hub
    // against hub) is handed to the whole warp instead.  Returns the warp's sum.
    __device__ unsigned long long leaf_level(int D, int i0, int i1) {
        const int ls = P.loop_set[D];
        const uint32_t *s = w.set_ptr[ls];
        const int ns = w.set_size[ls];
        i1 = min(i1, lower_bound_u32(s, ns, w.minv[D]));
        if (i0 >= i1) return 0;
        // Which embedded vertices each earlier set holds (fathers of the
        // leaf chain, IEP sets and the last loop set built before D).
        for (int q = 0; q < P.total_prefix; ++q) {
            if (P.pdepth[q] >= D) continue;
            const uint32_t m = warp_embedded_mask(w.set_ptr[q], w.set_size[q], w, D, lane);
            if (lane == 0) w.emb_mask[q] = m;
        }
        __syncwarp();
        unsigned long long acc = 0;
        for (int base = i0; base < i1; base += 32) {
            if (out_of_time()) break;
            if (hq.items && i1 - base >= 2 * (P.leaf_handoff > 0 ? P.leaf_handoff : kLeafHandoffMin)) {
                const int mid = base + ((i1 - base) / 2 + 31) / 32 * 32;
                if (mid < i1 && donate(D, mid, i1)) i1 = mid;
            }
            const int i = base + lane;
            uint32_t v = 0;
            bool heavy = false;
            if (i < i1) {
                v = s[i];
                bool used = false;
                for (int u = 0; u < D; ++u) used |= w.emb[u] == v;
                if (!used && !(P.vertex_induced && anti_adjacent(P, w, D, v, vertex, edge))) {
                    const int dv = static_cast<int>(__ldg(&vertex[v + 1]) - __ldg(&vertex[v]));
                    const bool v_hub = dv >= hubs.min_degree;
                    const bool v_hash = dv >= hashes.min_degree;
                    int cost = 0;
                    for (int p = P.last[D]; p != -1; p = P.next[p]) {
                        const int f = P.father[p];
                        if (f < 0) continue;
                        const int fn = w.set_size[f];
                        // bitmap tests: one step per element of the other
                        // list; hash-set probes about two
                        const bool f_hash = w.src[f] >= 0 && fn >= hashes.min_degree;
                        int c = w.hub[f] >= 0 && fn >= dv ? dv : v_hub ? fn : lane_cost(fn, dv);
                        if (v_hash) c = min(c, 2 * fn);
                        if (f_hash) c = min(c, 2 * dv);
                        cost += c;
                    }
                    heavy = cost > (kLaneBudgetOverride >= 0 ? kLaneBudgetOverride : P.lane_budget);
                    if (!heavy) acc += leaf_eval<false>(D, v);
                }
            }
            unsigned todo = __ballot_sync(kFull, heavy);
            while (todo) {
                const int src = __ffs(todo) - 1;
                todo &= todo - 1;
                const unsigned long long c = leaf_eval<true>(D, __shfl_sync(kFull, v, src));
                if (lane == 0) acc += c;
            }
        }
        return warp_sum(acc);
    }

    // One candidate per lane at the leaf-parent depth D, the probes of all
    // 32 candidates' intersections spread evenly over the lanes (flat_count).
    // For each prefix p of D's chain, in chain order (so the break-size prune
    // still skips later prefixes), every live lane's pair (S_father(p), N(v))
    // is counted at once; then each lane closes its candidate with the
    // last-level count or the IEP formula.  `early` describes the sets built
    // before depth D and the embedding emb[0, D) for this lane: warp-shared
    // for D >= 2 (EarlyShared), the lane's own first-level edge for D = 1
    // (EarlyEdge).  The counts, prunes and byte accounting are those of
    // leaf_eval; so is the result.  Returns this lane's contribution; `passed`
    // tells whether the candidate passed its chain's break-size prunes.
    template <class Early>
    __device__ __forceinline__ unsigned long long flat_eval(int D, uint32_t v, bool alive, const Early &early,
                                                           bool &passed) {
        const int stop = P.stop;
        const int L = P.loop_set[stop];
        const bool last_level = P.iep_k == 0;
        int64_t l = 0;
        int dv = 0, hv = -1, hv_bits = 0;
        const uint32_t *hv_hash = nullptr;
        uint32_t bound = 0xffffffffu, mask_nv = 0;
        if (alive) {
            l = __ldg(&vertex[v]);
            dv = static_cast<int>(__ldg(&vertex[v + 1]) - l);
            hv = hub_row_of(hubs, v, dv);
            hv_hash = hash_table(hashes, v, dv, hv_bits);
            if (last_level)
                for (int r = P.restrict_last[stop]; r != -1; r = P.restrict_next[r]) {
                    const int idx = P.restrict_index[r];
                    bound = min(bound, idx == D ? v : early.emb(idx));
                }
            if (Early::kFirstEdge) {
                mask_nv = 1u;  // v = v1 and emb[0] = v0 are the ends of an edge
            } else {
                for (int u = 0; u < D; ++u) {
                    const uint32_t x = early.emb(u);
                    const bool in = hv >= 0 ? hub_test(hubs, hv, x)
                                            : hv_hash ? hash_contains(hv_hash, hv_bits, x) : contains_u32(edge + l, dv, x);
                    mask_nv |= static_cast<uint32_t>(in) << u;
                }
            }
        }
        const uint32_t *nv = edge + l;
        int size[GI_MAX_PREFIX];
        uint32_t mask[GI_MAX_PREFIX];
        int below_L = 0;
        unsigned long long b = 0;
        for (int p = P.last[D]; p != -1; p = P.next[p]) {
            const int f = P.father[p];
            if (f == -1) {
                size[p] = dv;
                mask[p] = mask_nv;
                if (kBytesOn && alive) b += 16;
                if (p == L && alive) below_L = lower_bound_u32(nv, dv, bound);
                if (alive && dv == P.break_size[p]) {
                    if (kBytesOn) bytes += b;
                    alive = false;
                }
                continue;
            }
            const uint32_t *fs = early.set_ptr(f);
            const int fn = early.set_size(f);
            const bool need_total = kBytesOn || !(last_level && p == L);
            ListRef fa{fs, fn, early.hub(f), nullptr, 0};
            const int fsrc = early.src(f);
            if (fsrc >= 0) fa.hash = hash_table(hashes, static_cast<uint32_t>(fsrc), fn, fa.hash_bits);
            int tot, bel;
            flat_count(hubs, fa, ListRef{nv, dv, hv, hv_hash, hv_bits}, bound, need_total, alive, lane, tot, bel);
            size[p] = tot;
            if (p == L) below_L = bel;
            mask[p] = early.emb_mask(f) & mask_nv;
            if (kBytesOn && alive) b += 4ull * (fn + dv + (P.mode[p] == kSizeOnly ? 0 : tot));
            if (alive && need_total && tot == P.break_size[p]) {
                if (kBytesOn) bytes += b;
                alive = false;
            }
        }
        passed = alive;
        if (!alive) return 0;
        unsigned long long contrib = 0;
        if (last_level) {
            int below;
            uint32_t m;
            bool v_in = false;
            if (P.pdepth[L] == D) {
                below = below_L;
                m = mask[L];
            } else {
                const uint32_t *sl = early.set_ptr(L);
                const int nl = early.set_size(L);
                if (nl <= 0) {
                    if (kBytesOn) bytes += b;
                    return 0;
                }
                below = lower_bound_u32(sl, nl, bound);
                m = early.emb_mask(L);
                v_in = v < bound && contains_u32(sl, below, v);
            }
            if (kBytesOn) b += 4ull * below;
            int emb_below = v_in ? 1 : 0;
            for (int u = 0; u < D; ++u) emb_below += ((m >> u) & 1u) && early.emb(u) < bound;
            contrib = static_cast<unsigned long long>(below - emb_below);
        } else {
            const int ls_size = P.pdepth[L] == D ? size[L] : early.set_size(L);
            if (ls_size > 0) {
                int ans[GI_MAX_IEP_SETS];
#pragma unroll 1
                for (int j = 0; j < P.iep_nsets; ++j) {
                    const int q = P.iep_set[j];
                    const bool in_chain = P.pdepth[q] == D;
                    const int sz = in_chain ? size[q] : early.set_size(q);
                    if (P.iep_set_flag[j]) {
                        ans[j] = sz - P.iep_set_coef[j];
                    } else {
                        const uint32_t m = in_chain ? mask[q] : early.emb_mask(q);
                        int cnt = __popc(m & ((1u << D) - 1u));
                        if (!in_chain && contains_u32(early.set_ptr(q), sz, v)) ++cnt;
                        ans[j] = sz - cnt;
                        if (kBytesOn) b += 4ull * sz;
                    }
                }
                contrib = iep_combine(P, ans);
            }
        }
        if (kBytesOn) bytes += b;
        return contrib;
    }

    // The sets built before the leaf-parent depth, shared by the warp.
    struct EarlyShared {
        static constexpr bool kFirstEdge = false;
        const WarpState &w;
        __device__ __forceinline__ uint32_t emb(int u) const { return w.emb[u]; }
        __device__ __forceinline__ const uint32_t *set_ptr(int q) const { return w.set_ptr[q]; }
        __device__ __forceinline__ int set_size(int q) const { return w.set_size[q]; }
        __device__ __forceinline__ int hub(int q) const { return w.hub[q]; }
        __device__ __forceinline__ int src(int q) const { return w.src[q]; }
        __device__ __forceinline__ uint32_t emb_mask(int q) const { return w.emb_mask[q]; }
    };

    // Leaf-parent depth D >= 2, 32 candidates of the loop set at a time
    // (flat_eval).  Returns the warp's sum.
    __device__ unsigned long long leaf_level_flat(int D, int i0, int i1) {
        const int ls = P.loop_set[D];
        const uint32_t *s = w.set_ptr[ls];
        const int ns = w.set_size[ls];
        i1 = min(i1, lower_bound_u32(s, ns, w.minv[D]));
        if (i0 >= i1) return 0;
        for (int q = 0; q < P.total_prefix; ++q) {
            if (P.pdepth[q] >= D) continue;
            const uint32_t m = warp_embedded_mask(w.set_ptr[q], w.set_size[q], w, D, lane);
            if (lane == 0) w.emb_mask[q] = m;
        }
        __syncwarp();
        const EarlyShared early{w};
        unsigned long long acc = 0;
        for (int base = i0; base < i1; base += 32) {
            if (out_of_time()) break;
            if (hq.items && i1 - base >= 2 * (P.leaf_handoff > 0 ? P.leaf_handoff : kLeafHandoffMin)) {
                const int mid = base + ((i1 - base) / 2 + 31) / 32 * 32;
                if (mid < i1 && donate(D, mid, i1)) i1 = mid;
            }
            const int i = base + lane;
            uint32_t v = 0;
            bool alive = false;
            if (i < i1) {
                v = s[i];
                bool used = false;
                for (int u = 0; u < D; ++u) used |= w.emb[u] == v;
                alive = !used && !(P.vertex_induced && anti_adjacent(P, w, D, v, vertex, edge));
            }
            bool passed;
            acc += flat_eval(D, v, alive, early, passed);
        }
        return warp_sum(acc);
    }

    // The sets of depth 0 for a lane's own first-level edge (v0, v1): every
    // depth-0 prefix is N(v0), which holds v1 and not v0.
    struct EarlyEdge {
        static constexpr bool kFirstEdge = true;
        uint32_t v0;
        const uint32_t *n0;
        int d0, h0;
        __device__ __forceinline__ uint32_t emb(int) const { return v0; }
        __device__ __forceinline__ const uint32_t *set_ptr(int) const { return n0; }
        __device__ __forceinline__ int set_size(int) const { return d0; }
        __device__ __forceinline__ int hub(int) const { return h0; }
        __device__ __forceinline__ int src(int) const { return static_cast<int>(v0); }
        __device__ __forceinline__ uint32_t emb_mask(int) const { return 0u; }
    };

    // Plans whose DFS ends at depth 2 (P.flat_first): the 32 first-level
    // edges of a chunk, one per lane, evaluated as leaf candidates v1 at
    // depth 1 below their own v0 (flat_eval).  Returns the warp's sum;
    // `passed` counts the edges that passed the depth-1 prunes.
    __device__ unsigned long long first_level_flat(uint32_t v0, uint32_t v1, bool valid, unsigned long long &passed) {
        EarlyEdge early{v0, edge, 0, -1};
        if (valid) {
            const int64_t l0 = __ldg(&vertex[v0]);
            early.n0 = edge + l0;
            early.d0 = static_cast<int>(__ldg(&vertex[v0 + 1]) - l0);
            early.h0 = hub_row_of(hubs, v0, early.d0);
        }
        bool ok = false;
        const unsigned long long c = flat_eval(1, v1, valid, early, ok);
        passed = __popc(__ballot_sync(kFull, ok));
        return warp_sum(c);
    }

    __device__ __forceinline__ unsigned long long leaf_run(int D, int i0, int i1) {
        return P.leaf_flat ? leaf_level_flat(D, i0, i1) : leaf_level(D, i0, i1);
    }

    // The DFS below the first two positions for depth-2 candidates [lo, hi);
    // returns the subtask's sum (warp-uniform).
    __device__ unsigned long long dfs(int lo, int hi) { return dfs_from(2, lo, hi); }

    // The DFS from depth `base` (>= 2, emb[0, base) and their prefix sets in
    // place) over loop indices [lo, hi) of that depth.
    __device__ unsigned long long dfs_from(int base, int lo, int hi) {
        const int stop = P.stop;
        const int leaf = P.leaf_depth;
        unsigned long long acc = 0;
        if (lane == 0) {
            w.cursor[base] = lo;
            w.end[base] = hi;
            w.minv[base] = min_vertex(base);
        }
        __syncwarp();
        if (leaf == base) return leaf_run(base, lo, hi);
        int d = base;
        while (true) {
            if (out_of_time()) break;
            if (d == stop) {
                acc += P.iep_k > 0 ? iep_tail(d) : last_level(d);
                --d;
                if (d < base) break;
                continue;
            }
            if (d == leaf) {
                acc += leaf_run(d, 0, 0x7fffffff);
                --d;
                if (d < base) break;
                continue;
            }
            const int ls = P.loop_set[d];
            const uint32_t *s = w.set_ptr[ls];
            int ns = min(w.set_size[ls], w.end[d]);
            const uint32_t bound = w.minv[d];
            int i = w.cursor[d];
            bool descended = false;
            while (i < ns) {
                if (hq.items && ns - i >= 2 * (P.mid_handoff > 0 ? P.mid_handoff : kMidHandoffMin)) {
                    const int mid = i + (ns - i + 1) / 2;
                    if (donate(d, mid, ns)) {
                        ns = mid;
                        if (lane == 0) w.end[d] = mid;
                        __syncwarp();
                    }
                }
                const uint32_t v = s[i++];
                if (v >= bound) {
                    i = ns;
                    break;
                }
                bool used = false;
                for (int u = 0; u < d; ++u) used |= w.emb[u] == v;
                if (used) continue;
                if (P.vertex_induced && anti_adjacent(P, w, d, v, vertex, edge)) continue;
                if (!build_chain(d, v)) continue;
                if (lane == 0) {
                    w.cursor[d] = i;
                    w.emb[d] = v;
                }
                __syncwarp();
                ++d;
                if (lane == 0) {
                    w.cursor[d] = 0;
                    w.end[d] = 0x7fffffff;
                    w.minv[d] = min_vertex(d);
                }
                __syncwarp();
                descended = true;
                break;
            }
            if (descended) continue;
            --d;
            if (d < base) break;
        }
        return acc;
    }

    // Runs a handed-off item: rebuilds the prefix sets of emb[0, depth) (no
    // byte accounting: the donor already counted them) and the range.
    // The item is read through L2 (ld.global.cg): it was written by another
    // SM after this launch began.
    // Returns false (and counts nothing) for an item that fails its checks.
    __device__ bool run_handoff(const Handoff *h, unsigned long long &out) {
        const int D = __ldcg(&h->depth);
        const int lo = __ldcg(&h->lo), hi = __ldcg(&h->hi);
        out = 0;
        if (D < 2 || D >= P.stop || lo < 0 || hi < lo) return false;
        const uint32_t x = lane < D ? __ldcg(&h->emb[lane]) : 0u;
        if (__any_sync(kFull, lane < D && x >= hq.v_cnt)) return false;
        if (lane < D) w.emb[lane] = x;
        __syncwarp();
        // Depth 0 is built unconditionally, as the chunk path does; deeper
        // chains passed their break-size prune when the donor built them.
        build_chain(0, w.emb[0], false);
        for (int j = 1; j < D; ++j)
            if (!build_chain(j, w.emb[j], false)) return true;
        out = dfs_from(D, lo, hi);
        return true;
    }
};

constexpr unsigned kTakerSpins = 1u << 20;  // empty polls of ~2 us before an idle warp leaves
constexpr unsigned kReadySpins = 1u << 22;  // polls of a claimed item's ready flag

// A warp out of chunks takes handed-off ranges from hq until every warp is
// idle or gone and the queue is empty; run(slot) counts item `slot` (its
// ready flag seen) and returns false when the item fails its checks.  Waits
// are bounded: an idle warp gives up after kTakerSpins empty polls (items
// still queued then are drained by the warps that queued them, which poll
// before they leave), and a taken item whose ready flag never appears is
// reported.  A warp that timed out only marks itself gone.  Returns true
// when an item was lost (never published, or rejected).
template <class Run>
__device__ bool take_handoffs(const HandoffQueue &hq, bool timed_out, int lane, Run &&run) {
    unsigned long long *qc = hq.ctr;  // head, tail, idle, exited
    if (timed_out) {
        if (lane == 0) atomicAdd(&qc[3], 1ull);  // gone
        return false;
    }
    bool lost = false;
    const unsigned long long total = static_cast<unsigned long long>(gridDim.x) * kWarpsPerBlock;
    if (lane == 0) atomicAdd(&qc[2], 1ull);
    unsigned spins = 0;
    while (true) {
        long long slot = -1;
        int quit = 0;
        if (lane == 0) {
            const unsigned long long h = *(volatile unsigned long long *)&qc[0];
            const unsigned long long t = *(volatile unsigned long long *)&qc[1];
            if (h < (t < hq.cap ? t : hq.cap)) {
                atomicAdd(&qc[2], ~0ull);  // busy unless the claim fails
                if (atomicCAS(&qc[0], h, h + 1) == h)
                    slot = static_cast<long long>(h);
                else
                    atomicAdd(&qc[2], 1ull);
            } else {
                const unsigned long long idle = *(volatile unsigned long long *)&qc[2];
                const unsigned long long gone = *(volatile unsigned long long *)&qc[3];
                if (idle + gone >= total || ++spins > kTakerSpins)
                    quit = 1;
                else
                    __nanosleep(2000);
            }
        }
        slot = __shfl_sync(kFull, slot, 0);
        if (__shfl_sync(kFull, quit, 0)) break;
        if (slot < 0) continue;
        int ready = 0;
        if (lane == 0) {
            for (unsigned k = 0; k < kReadySpins && !ready; ++k) {
                ready = *(volatile uint32_t *)&hq.items[slot].ready == hq.epoch;
                if (!ready) __nanosleep(64);
            }
            __threadfence();
        }
        if (!(__shfl_sync(kFull, ready, 0) && slot < static_cast<long long>(hq.cap) && run(slot))) lost = true;
        if (lane == 0) atomicAdd(&qc[2], 1ull);
        spins = 0;
    }
    if (lane == 0) {
        atomicAdd(&qc[2], ~0ull);
        atomicAdd(&qc[3], 1ull);
    }
    return lost;
}

}  // namespace
}  // namespace gi
