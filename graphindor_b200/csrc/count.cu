// Pattern counting: the edge-parallel DFS with warp-cooperative sorted-set
// intersections, a lane-parallel leaf level and the inclusion-exclusion
// (IEP) tail.
//
// Reference path replaced: gpu_pattern_matching (reference
// gpu/src/gpu_pattern_matching.cuh:14-104) -> GPU_pattern_matching_func
// (gpu/function/pattern_matching.cuh:212-288) -> build_vertex_set /
// intersection2 / unordered_subtraction_size (gpu/component/
// gpu_vertex_set.cuh:67-248) and the IEP tail (pattern_matching.cuh:110-139).
// Result semantics are those of the reference CPU path (src/graph.cpp:
// 305-566), which the reference GPU path also computes.
//
// Design (sm_100a):
//  * work items are subtasks: a first-level directed edge (v0, v1) plus a
//    range of at most kSplit candidates of the depth-2 loop.  A pre-pass
//    bounds each edge's depth-2 loop by degrees, a cub scan turns the bounds
//    into subtask offsets, and the persistent grid claims 32 subtasks per
//    atomic (interleaved across shards), each lane mapping its subtask to an
//    edge by binary search over the offsets.  Hub edges thus spread over
//    many warps instead of pinning one;
//  * levels 2 .. stop-2 run warp-cooperatively: S_father ∩ N(v) has each
//    lane binary-search one element of the smaller set in the larger, with
//    __ballot_sync / __popc compaction into the warp's scratch slot;
//  * level stop-1 (the leaf parent) runs one candidate per lane: each lane
//    counts |S_father ∩ N(v)| for the prefixes that candidate would build,
//    applies the break-size prune, then evaluates the last-level count or
//    the IEP formula for its candidate — sizes only, nothing materialised;
//  * per-warp stack state lives in shared memory, written by lane 0 and
//    published with __syncwarp; all counting is modulo 2^64.
#include <cuda_runtime.h>
#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <cstdio>
#include <cstring>

#include "internal.hpp"

namespace gi {

int cuda_fail(cudaError_t e, const char *what);

namespace {

constexpr int kWarpsPerBlock = 4;
constexpr int kBlockThreads = kWarpsPerBlock * 32;
constexpr int kTaskChunk = GI_TASK_CHUNK;
constexpr unsigned kFull = 0xffffffffu;

// Counter slots in gi_graph::d_counters.
enum : int { kSum = 0, kCursor = 1, kBytes = 2, kTasks = 3, kTimeout = 4, kChunks = 5 };

struct WarpState {
    const uint32_t *set_ptr[GI_MAX_PREFIX];
    int32_t set_size[GI_MAX_PREFIX];
    uint32_t emb_mask[GI_MAX_PREFIX];  // leaf level: which emb[0, D) lie in each earlier set
    uint32_t emb[GI_MAX_PATTERN + 1];
    int32_t cursor[GI_MAX_PATTERN + 1];
    int32_t end[GI_MAX_PATTERN + 1];
    uint32_t minv[GI_MAX_PATTERN + 1];
};

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

// Steps a lane would spend intersecting lists of sizes x and y: the smaller
// times the log of the size ratio.
__device__ __forceinline__ int lane_cost(int x, int y) {
    const int lo = min(x, y), hi = max(x, y);
    if (lo == 0) return 0;
    return lo * (33 - __clz(hi / lo + 1));
}

// A leaf candidate costlier than this for one lane goes to the whole warp.
constexpr int kLaneBudget = 2048;

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
        for (int p = P.last[d]; p != -1; p = P.next[p]) {
            int size;
            const int f = P.father[p];
            if (f == -1) {
                if (lane == 0) w.set_ptr[p] = nb;
                size = deg;
                if (kBytesOn && account && lane == 0) bytes += 16;
            } else {
                const uint32_t *fs = w.set_ptr[f];
                const int fn = w.set_size[f];
                if (P.mode[p] == kMaterialize) {
                    uint32_t *out = slot_base + static_cast<int64_t>(P.slot[p]) * slot_stride;
                    size = warp_intersect(fs, fn, nb, deg, out, lane);
                    if (lane == 0) w.set_ptr[p] = out;
                    if (kBytesOn && lane == 0) bytes += 4ull * (fn + deg + size);
                } else {
                    size = warp_intersect(fs, fn, nb, deg, nullptr, lane);
                    if (kBytesOn && lane == 0) bytes += 4ull * (fn + deg);
                }
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
        uint32_t mask_nv = 0;  // emb[u] in N(v)
        if (kWarp) {
            mask_nv = __ballot_sync(kFull, lane < D && contains_u32(nv, dv, w.emb[lane]));
        } else {
            for (int u = 0; u < D; ++u) mask_nv |= static_cast<uint32_t>(contains_u32(nv, dv, w.emb[u])) << u;
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
                int tot, bel;
                if (kWarp)
                    warp_count2(fs, fn, nv, dv, bound, need_total, lane, tot, bel);
                else
                    lane_intersect(fs, fn, nv, dv, bound, need_total, tot, bel);
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
    // would keep one lane busy for more than kLaneBudget steps (hub against
    // hub) is handed to the whole warp instead.  Returns the warp's sum.
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
            const int i = base + lane;
            uint32_t v = 0;
            bool heavy = false;
            if (i < i1) {
                v = s[i];
                bool used = false;
                for (int u = 0; u < D; ++u) used |= w.emb[u] == v;
                if (!used && !(P.vertex_induced && anti_adjacent(P, w, D, v, vertex, edge))) {
                    const int dv = static_cast<int>(__ldg(&vertex[v + 1]) - __ldg(&vertex[v]));
                    int cost = 0;
                    for (int p = P.last[D]; p != -1; p = P.next[p])
                        if (P.father[p] >= 0) cost += lane_cost(w.set_size[P.father[p]], dv);
                    heavy = cost > kLaneBudget;
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

    // The DFS below the first two positions for depth-2 candidates [lo, hi);
    // returns the subtask's sum (warp-uniform).
    __device__ unsigned long long dfs(int lo, int hi) {
        const int stop = P.stop;
        const int leaf = P.leaf_depth;
        unsigned long long acc = 0;
        if (lane == 0) {
            w.cursor[2] = lo;
            w.end[2] = hi;
            w.minv[2] = min_vertex(2);
        }
        __syncwarp();
        if (leaf == 2) return leaf_level(2, lo, hi);
        int d = 2;
        while (true) {
            if (out_of_time()) break;
            if (d == stop) {
                acc += P.iep_k > 0 ? iep_tail(d) : last_level(d);
                --d;
                if (d < 2) break;
                continue;
            }
            if (d == leaf) {
                acc += leaf_level(d, 0, 0x7fffffff);
                --d;
                if (d < 2) break;
                continue;
            }
            const int ls = P.loop_set[d];
            const uint32_t *s = w.set_ptr[ls];
            const int ns = min(w.set_size[ls], w.end[d]);
            const uint32_t bound = w.minv[d];
            int i = w.cursor[d];
            bool descended = false;
            while (i < ns) {
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
            if (d < 2) break;
        }
        return acc;
    }
};

// Subtasks per edge: a degree bound on the depth-2 loop set, cut into
// pieces of `split` candidates; 0 for edges the depth-1 restriction drops.
__global__ void split_count_kernel(const __grid_constant__ DevPlan P, const int64_t *__restrict__ vertex,
                                   const uint32_t *__restrict__ edge, const uint32_t *__restrict__ edge_from,
                                   int64_t e_cnt, int split, int64_t *__restrict__ counts) {
    const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < e_cnt; i += stride) {
        const uint32_t v0 = edge_from[i], v1 = edge[i];
        if (P.first_restricted && v0 <= v1) {
            counts[i] = 0;
            continue;
        }
        const int64_t d0 = vertex[v0 + 1] - vertex[v0], d1 = vertex[v1 + 1] - vertex[v1];
        const int64_t b = P.loop2_kind == 0 ? d0 : P.loop2_kind == 1 ? d1 : min(d0, d1);
        const int64_t pieces = (b + split - 1) / split;
        counts[i] = pieces > 0 ? pieces : 1;
    }
}

template <bool kBytesOn>
__global__ void __launch_bounds__(kBlockThreads)
    dfs_count_kernel(const __grid_constant__ DevPlan P, const int64_t *__restrict__ vertex,
                     const uint32_t *__restrict__ edge, const uint32_t *__restrict__ edge_from, int64_t e_cnt,
                     const int64_t *__restrict__ offsets, int64_t n_tasks, int split, uint32_t *scratch,
                     int64_t slot_stride, unsigned long long *counters, unsigned long long budget_ns, int64_t shard,
                     int64_t num_shards, int64_t n_chunks, int64_t perm_a, int64_t perm_b,
                     unsigned long long hard_ns) {
    __shared__ WarpState states[kWarpsPerBlock];
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    const int64_t gwarp = static_cast<int64_t>(blockIdx.x) * kWarpsPerBlock + wib;
    WarpState &w = states[wib];
    Ctx<kBytesOn> c{P, vertex, edge, scratch + gwarp * P.n_slots * slot_stride, slot_stride, w, lane, 0ull};
    unsigned long long sum = 0, tasks = 0, chunks = 0;
    bool timed_out = false;
    const unsigned long long t_start = globaltimer();
    c.t_start = t_start;
    c.hard_ns = hard_ns;
    while (true) {
        // Claim the next chunk of kTaskChunk consecutive work items of this
        // shard: slot shard + j * num_shards (the reference's static
        // interleave, gpu/src/gpu_pattern_matching_static_task.cuh:63),
        // mapped through the bijection slot -> (slot * perm_a + perm_b) mod
        // n_chunks when a sampled count wants a pseudo-random order.
        unsigned long long j = 0;
        int stop = 0;
        if (lane == 0) {
            j = atomicAdd(&counters[kCursor], 1ull);
            if (budget_ns && globaltimer() - t_start > budget_ns) {
                timed_out = true;
                stop = 1;
            }
        }
        j = __shfl_sync(kFull, j, 0);
        stop = __shfl_sync(kFull, stop, 0);
        const int64_t slot = shard + static_cast<int64_t>(j) * num_shards;
        if (stop || slot >= n_chunks) break;
        const int64_t chunk = perm_a ? static_cast<int64_t>(
                                           (static_cast<unsigned long long>(slot) * static_cast<unsigned long long>(perm_a) +
                                            static_cast<unsigned long long>(perm_b)) %
                                           static_cast<unsigned long long>(n_chunks))
                                     : slot;
        const int64_t base = chunk * kTaskChunk;
        const int64_t t = base + lane;
        bool valid = t < n_tasks;
        int64_t e = t;
        int lo = 0;
        if (valid && offsets) {
            // Edge of subtask t: the last e with offsets[e] <= t.
            int64_t a = 0, len = e_cnt + 1;
            while (len > 0) {
                const int64_t half = len >> 1;
                if (offsets[a + half] <= t) {
                    a += half + 1;
                    len -= half + 1;
                } else {
                    len = half;
                }
            }
            e = a - 1;
            lo = static_cast<int>((t - offsets[e]) * split);
        }
        uint32_t v0 = 0, v1 = 0;
        if (valid) {
            v0 = __ldg(&edge_from[e]);
            v1 = __ldg(&edge[e]);
            // Depth-1 restriction (reference gpu/src/gpu_pattern_matching.cuh:77).
            if (!offsets && P.first_restricted && v0 <= v1) valid = false;
        }
        unsigned todo = __ballot_sync(kFull, valid);
        unsigned long long chunk_sum = 0, chunk_tasks = 0;
        while (todo) {
            const int src = __ffs(todo) - 1;
            todo &= todo - 1;
            const uint32_t a = __shfl_sync(kFull, v0, src);
            const uint32_t b = __shfl_sync(kFull, v1, src);
            const int sub_lo = __shfl_sync(kFull, lo, src);
            if (lane == 0) {
                w.emb[0] = a;
                w.emb[1] = b;
            }
            __syncwarp();
            // Depth 0 is accounted per start vertex on the host; depth 1 once
            // per edge (the first of its subtasks).
            c.build_chain(0, a, false);
            const bool first = sub_lo == 0;
            const unsigned long long before = c.bytes;
            if (!c.build_chain(1, b)) {
                if (kBytesOn && !first) c.bytes = before;
                continue;
            }
            if (kBytesOn && !first) c.bytes = before;
            chunk_tasks += first;
            chunk_sum += c.dfs(sub_lo, offsets ? sub_lo + split : 0x7fffffff);
            if (c.aborted) break;
        }
        // A chunk cut short by the hard limit is dropped whole, so the
        // counted chunks stay a sample of complete work items.
        if (c.aborted) {
            timed_out = true;
            break;
        }
        sum += chunk_sum;
        tasks += chunk_tasks;
        ++chunks;
    }
    const unsigned long long lane_bytes = kBytesOn ? warp_sum(c.bytes) : 0;
    if (lane == 0) {
        atomicAdd(&counters[kSum], sum);
        atomicAdd(&counters[kTasks], tasks);
        atomicAdd(&counters[kChunks], chunks);
        if (kBytesOn) atomicAdd(&counters[kBytes], lane_bytes);
        if (timed_out) atomicExch(&counters[kTimeout], 1ull);
    }
}

}  // namespace

// Ensures the graph's scratch can hold `bytes`; caller holds g->mu.
int ensure_scratch(gi_graph *g, size_t bytes) {
    if (g->scratch_bytes >= bytes) return GI_OK;
    cudaFree(g->d_scratch);
    g->d_scratch = nullptr;
    g->scratch_bytes = 0;
    cudaError_t e = cudaMalloc(&g->d_scratch, bytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return cuda_fail(e, "scratch allocation");
    }
    g->scratch_bytes = bytes;
    return GI_OK;
}

// Candidates of the depth-2 loop per subtask: one lane each when depth 2 is
// the leaf level, one warp at a time otherwise.
static int split_size(const DevPlan &P) { return P.leaf_depth == 2 ? 256 : 32; }

// Builds the subtask offsets for the plan's depth-2 split; returns the
// number of subtasks.  Caller holds g->mu.
static int build_split(gi_graph *g, const DevPlan &P, cudaStream_t st, int split, int64_t *n_tasks) {
    cudaError_t e;
    const size_t n = static_cast<size_t>(g->e_cnt) + 1;
    if (!g->d_offsets) {
        if ((e = cudaMalloc(&g->d_offsets, 2 * n * sizeof(int64_t))) != cudaSuccess) {
            g->d_offsets = nullptr;
            return cuda_fail(e, "split offsets allocation");
        }
    }
    int64_t *counts = g->d_offsets + n;
    size_t need = 0;
    cub::DeviceScan::ExclusiveSum(nullptr, need, counts, g->d_offsets, static_cast<int64_t>(n), st);
    if (need > g->scan_tmp_bytes) {
        cudaFree(g->d_scan_tmp);
        g->d_scan_tmp = nullptr;
        if ((e = cudaMalloc(&g->d_scan_tmp, need)) != cudaSuccess) return cuda_fail(e, "scan workspace");
        g->scan_tmp_bytes = need;
    }
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, g->device);
    if ((e = cudaMemsetAsync(counts + g->e_cnt, 0, sizeof(int64_t), st)) != cudaSuccess) return cuda_fail(e, "memset");
    split_count_kernel<<<sms * 16, 256, 0, st>>>(P, g->d_vertex, reinterpret_cast<const uint32_t *>(g->d_edge),
                                                  g->d_edge_from, g->e_cnt, split, counts);
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "split count kernel");
    size_t tmp = g->scan_tmp_bytes;
    if ((e = cub::DeviceScan::ExclusiveSum(g->d_scan_tmp, tmp, counts, g->d_offsets, static_cast<int64_t>(n), st)) !=
        cudaSuccess)
        return cuda_fail(e, "split scan");
    int64_t total = 0;
    if ((e = cudaMemcpyAsync(&total, g->d_offsets + g->e_cnt, sizeof(total), cudaMemcpyDeviceToHost, st)) !=
            cudaSuccess ||
        (e = cudaStreamSynchronize(st)) != cudaSuccess)
        return cuda_fail(e, "split total");
    *n_tasks = total;
    return GI_OK;
}

// Runs the counting kernel for one plan on one graph (or one shard of it).
// budget_ms = 0 means no budget.
int count_impl(gi_graph *g, const DevPlan &P, cudaStream_t st, uint64_t *raw_sum, gi_stats *stats,
               double budget_ms, int64_t shard, int64_t num_shards) {
    int prev = 0;
    cudaGetDevice(&prev);
    if (prev != g->device) cudaSetDevice(g->device);
    int sms = 148, blocks_per_sm = 1;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, g->device);
    const bool bytes_on = stats && stats->count_bytes;
    cudaError_t e;
    if (bytes_on)
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks_per_sm, dfs_count_kernel<true>, kBlockThreads, 0);
    else
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks_per_sm, dfs_count_kernel<false>, kBlockThreads, 0);
    if (e != cudaSuccess) return cuda_fail(e, "occupancy query");
    const int blocks = sms * std::max(1, blocks_per_sm);
    const int64_t warps = static_cast<int64_t>(blocks) * kWarpsPerBlock;
    const int64_t stride = std::max<int64_t>(g->max_isect, 1);
    const size_t need = static_cast<size_t>(warps) * std::max(P.n_slots, 1) * stride * sizeof(uint32_t);
    int st_code = ensure_scratch(g, need);
    if (st_code != GI_OK) return st_code;
    cudaEvent_t t0, tm, t1;
    cudaEventCreate(&t0);
    cudaEventCreate(&tm);
    cudaEventCreate(&t1);
    cudaEventRecord(t0, st);
    // Split the depth-2 loop when the plan has one; otherwise a work item is
    // an edge.
    const bool use_split = P.loop2_kind >= 0 && g->e_cnt > 0;
    const int split = split_size(P);
    int64_t n_tasks = g->e_cnt;
    int launches = 0;
    if (use_split) {
        st_code = build_split(g, P, st, split, &n_tasks);
        if (st_code != GI_OK) {
            cudaEventDestroy(t0);
            cudaEventDestroy(tm);
            cudaEventDestroy(t1);
            return st_code;
        }
        launches += 1;  // split count (the scan is cub's)
    }
    if ((e = cudaMemsetAsync(g->d_counters, 0, 8 * sizeof(unsigned long long), st)) != cudaSuccess)
        return cuda_fail(e, "counter reset");
    // Work budget: each warp stops claiming work once %globaltimer has
    // advanced budget_ns past its own start, and the call reports
    // GI_ETIMEOUT.  No wait in the kernel depends on another warp.  A
    // sampled count (allow_partial) visits the chunks in a pseudo-random
    // order and drops chunks still running at three times the budget.
    const unsigned long long budget_ns = budget_ms > 0 ? static_cast<unsigned long long>(budget_ms * 1e6) : 0ull;
    const bool partial = budget_ns && stats && stats->allow_partial;
    const int64_t *offs = use_split ? g->d_offsets : nullptr;
    const int64_t n_chunks = (n_tasks + kTaskChunk - 1) / kTaskChunk;
    int64_t perm_a = 0, perm_b = 0;
    if (partial && n_chunks > 1) {
        perm_a = static_cast<int64_t>(2654435761ull % static_cast<unsigned long long>(n_chunks));
        auto gcd = [](int64_t x, int64_t y) {
            while (y) {
                const int64_t t = x % y;
                x = y;
                y = t;
            }
            return x;
        };
        if (perm_a == 0) perm_a = 1;
        while (gcd(perm_a, n_chunks) != 1) perm_a = perm_a % (n_chunks - 1) + 1;
        perm_b = n_chunks / 3;
    }
    const unsigned long long hard_ns = partial ? 3ull * budget_ns : 0ull;
    cudaEventRecord(tm, st);
    if (bytes_on)
        dfs_count_kernel<true><<<blocks, kBlockThreads, 0, st>>>(
            P, g->d_vertex, reinterpret_cast<const uint32_t *>(g->d_edge), g->d_edge_from, g->e_cnt, offs, n_tasks,
            split, static_cast<uint32_t *>(g->d_scratch), stride, g->d_counters, budget_ns, shard, num_shards, n_chunks,
            perm_a, perm_b, hard_ns);
    else
        dfs_count_kernel<false><<<blocks, kBlockThreads, 0, st>>>(
            P, g->d_vertex, reinterpret_cast<const uint32_t *>(g->d_edge), g->d_edge_from, g->e_cnt, offs, n_tasks,
            split, static_cast<uint32_t *>(g->d_scratch), stride, g->d_counters, budget_ns, shard, num_shards, n_chunks,
            perm_a, perm_b, hard_ns);
    launches += 1;
    e = cudaGetLastError();
    cudaEventRecord(t1, st);
    unsigned long long host[8] = {0};
    if (e == cudaSuccess) e = cudaMemcpyAsync(host, g->d_counters, sizeof(host), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    float ms = 0.f, prep = 0.f;
    if (e == cudaSuccess) {
        cudaEventElapsedTime(&prep, t0, tm);
        cudaEventElapsedTime(&ms, tm, t1);
    }
    cudaEventDestroy(t0);
    cudaEventDestroy(tm);
    cudaEventDestroy(t1);
    if (e != cudaSuccess) return cuda_fail(e, "counting kernel");
    if (host[kTimeout] && !partial) return fail(GI_ETIMEOUT, "count exceeded its device time budget");
    *raw_sum = host[kSum];
    if (stats) {
        stats->chunks_done += static_cast<int64_t>(host[kChunks]);
        stats->chunks_total += n_chunks > shard ? (n_chunks - shard + num_shards - 1) / num_shards : 0;
        stats->kernel_ms += ms;
        stats->prep_ms += prep;
        stats->raw_sum = host[kSum];
        stats->tasks += host[kTasks];
        if (bytes_on) stats->alg_bytes += host[kBytes];
        stats->grid_blocks = blocks;
        stats->block_threads = kBlockThreads;
        stats->kernel_launches += launches;
    }
    if (prev != g->device) cudaSetDevice(prev);
    return GI_OK;
}

}  // namespace gi

using namespace gi;

static void reset_stats(gi_stats *stats, double &budget) {
    budget = 0.0;
    if (!stats) return;
    const int cb = stats->count_bytes;
    const int partial = stats->allow_partial;
    budget = stats->budget_ms;
    std::memset(stats, 0, sizeof(*stats));
    stats->count_bytes = cb;
    stats->budget_ms = budget;
    stats->allow_partial = partial;
}

extern "C" int gi_count(const gi_graph *cg, const gi_plan *p, gi_stream stream, uint64_t *out_count,
                        gi_stats *stats) {
    if (!cg || !p || !out_count) return fail(GI_EINVAL, "NULL argument");
    gi_graph *g = const_cast<gi_graph *>(cg);
    std::lock_guard<std::mutex> lock(g->mu);
    uint64_t raw = 0;
    double budget = 0.0;
    reset_stats(stats, budget);
    const int st = count_impl(g, p->dev, static_cast<cudaStream_t>(stream), &raw, stats, budget, 0, 1);
    if (st != GI_OK) return st;
    if (stats && stats->count_bytes) {
        // Depth-0 aliases are built once per start vertex on the reference
        // CPU path; account for them the same way.
        int chain0 = 0;
        for (int q = p->dev.last[0]; q != -1; q = p->dev.next[q]) ++chain0;
        stats->alg_bytes += 16ull * chain0 * static_cast<uint64_t>(g->v_cnt);
    }
    const uint64_t red = static_cast<uint64_t>(p->sched->get_count_divisor());
    *out_count = red ? raw / red : raw;
    return GI_OK;
}

extern "C" int gi_count_shard(const gi_graph *cg, const gi_plan *p, int32_t shard, int32_t num_shards,
                              gi_stream stream, uint64_t *raw_sum, gi_stats *stats) {
    if (!cg || !p || !raw_sum) return fail(GI_EINVAL, "NULL argument");
    if (num_shards < 1 || shard < 0 || shard >= num_shards) return fail(GI_EINVAL, "shard out of range");
    gi_graph *g = const_cast<gi_graph *>(cg);
    std::lock_guard<std::mutex> lock(g->mu);
    double budget = 0.0;
    reset_stats(stats, budget);
    return count_impl(g, p->dev, static_cast<cudaStream_t>(stream), raw_sum, stats, budget, shard, num_shards);
}
