// Pattern counting: the edge-parallel DFS with warp-cooperative sorted-set
// intersections and the inclusion-exclusion (IEP) tail.
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
//  * persistent grid, one warp per first-level task (a directed edge
//    (v0, v1) = (edge_from[i], edge[i])); a warp claims 32 consecutive edges
//    with one atomic, filters them with one ballot and walks the survivors;
//  * the DFS is iterative; per-warp stack state (embedding, loop cursors,
//    set pointers and sizes) lives in shared memory and is written by lane 0
//    then published with __syncwarp;
//  * S_father ∩ N(v): each lane takes one element of the smaller set and
//    binary-searches the larger, matches are compacted with __ballot_sync /
//    __popc into the warp's scratch slot, or only counted when the plan needs
//    the size alone;
//  * |S - embedding| and the last-level count test the (at most six)
//    embedded vertices in parallel, one per lane;
//  * all counting is modulo 2^64, as the reference GPU path.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstring>

#include "internal.hpp"

namespace gi {

int cuda_fail(cudaError_t e, const char *what);

namespace {

constexpr int kWarpsPerBlock = 4;
constexpr int kBlockThreads = kWarpsPerBlock * 32;
constexpr int kTaskChunk = 32;
constexpr unsigned kFull = 0xffffffffu;

// Counter slots in gi_graph::d_counters.
enum : int { kSum = 0, kCursor = 1, kBytes = 2, kTasks = 3, kTimeout = 4 };

struct WarpState {
    const uint32_t *set_ptr[GI_MAX_PREFIX];
    int32_t set_size[GI_MAX_PREFIX];
    uint32_t emb[GI_MAX_PATTERN + 1];
    int32_t cursor[GI_MAX_PATTERN + 1];
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

// Warp-cooperative |a ∩ b| (out == nullptr) or a ∩ b written to out in
// sorted order.  The smaller set is spread over the lanes; each lane
// binary-searches the larger set.
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

// How many of emb[0, d) occur in s[0, n).
__device__ __forceinline__ int warp_count_embedded(const uint32_t *s, int n, const WarpState &w, int d, int lane) {
    const bool hit = lane < d && n > 0 && contains_u32(s, n, w.emb[lane]);
    return __popc(__ballot_sync(kFull, hit));
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

template <bool kBytesOn>
struct Ctx {
    const DevPlan &P;
    const int64_t *__restrict__ vertex;
    const uint32_t *__restrict__ edge;
    uint32_t *slot_base;
    int64_t slot_stride;
    WarpState &w;
    int lane;
    unsigned long long bytes;

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
                if (kBytesOn && account) bytes += 16;
            } else {
                const uint32_t *fs = w.set_ptr[f];
                const int fn = w.set_size[f];
                if (P.mode[p] == kMaterialize) {
                    uint32_t *out = slot_base + static_cast<int64_t>(P.slot[p]) * slot_stride;
                    size = warp_intersect(fs, fn, nb, deg, out, lane);
                    if (lane == 0) w.set_ptr[p] = out;
                    if (kBytesOn) bytes += 4ull * (fn + deg + size);
                } else {
                    size = warp_intersect(fs, fn, nb, deg, nullptr, lane);
                    if (kBytesOn) bytes += 4ull * (fn + deg);
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

    // Last position without an IEP tail: candidates below the restriction
    // bound that are not already embedded (reference src/graph.cpp:496-519).
    __device__ __forceinline__ unsigned long long last_level(int d) {
        const int ls = P.loop_set[d];
        const uint32_t *s = w.set_ptr[ls];
        const int n = w.set_size[ls];
        if (n <= 0) return 0;
        const uint32_t bound_v = min_vertex(d);
        const int bound = lower_bound_u32(s, n, bound_v);
        if (kBytesOn) bytes += 4ull * bound;
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

    // IEP tail at position d = n - k (reference src/graph.cpp:456-493,
    // gpu/function/pattern_matching.cuh:110-139).
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
                if (kBytesOn) bytes += 4ull * sz;
            }
        }
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

    // The DFS below the first two positions; returns the task's sum.
    __device__ unsigned long long dfs() {
        const int n = P.n;
        const int stop = P.iep_k > 0 ? n - P.iep_k : n - 1;  // depth handled in closed form
        unsigned long long acc = 0;
        int d = 2;
        if (lane == 0) {
            w.cursor[2] = 0;
            w.minv[2] = min_vertex(2);
        }
        __syncwarp();
        while (true) {
            if (d == stop) {
                acc += P.iep_k > 0 ? iep_tail(d) : last_level(d);
                --d;
                if (d < 2) break;
                continue;
            }
            const int ls = P.loop_set[d];
            const uint32_t *s = w.set_ptr[ls];
            const int ns = w.set_size[ls];
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

template <bool kBytesOn>
__global__ void __launch_bounds__(kBlockThreads)
    dfs_count_kernel(const __grid_constant__ DevPlan P, const int64_t *__restrict__ vertex,
                     const uint32_t *__restrict__ edge, const uint32_t *__restrict__ edge_from, int64_t e_cnt,
                     uint32_t *scratch, int64_t slot_stride, unsigned long long *counters,
                     unsigned long long budget_ns, int64_t shard, int64_t num_shards) {
    __shared__ WarpState states[kWarpsPerBlock];
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    const int64_t gwarp = static_cast<int64_t>(blockIdx.x) * kWarpsPerBlock + wib;
    WarpState &w = states[wib];
    Ctx<kBytesOn> c{P, vertex, edge, scratch + gwarp * P.n_slots * slot_stride, slot_stride, w, lane, 0ull};
    unsigned long long sum = 0, tasks = 0;
    bool timed_out = false;
    const unsigned long long t_start = globaltimer();
    while (true) {
        // Claim the next chunk of kTaskChunk consecutive edges of this shard:
        // chunk shard + j * num_shards (the reference's static interleave,
        // gpu/src/gpu_pattern_matching_static_task.cuh:63).
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
        const int64_t base = (shard + static_cast<int64_t>(j) * num_shards) * kTaskChunk;
        if (stop || base >= e_cnt) break;
        const int64_t idx = static_cast<int64_t>(base) + lane;
        bool valid = idx < e_cnt;
        uint32_t v0 = 0, v1 = 0;
        if (valid) {
            v0 = __ldg(&edge_from[idx]);
            v1 = __ldg(&edge[idx]);
            // Depth-1 restriction (reference gpu/src/gpu_pattern_matching.cuh:77).
            if (P.first_restricted && v0 <= v1) valid = false;
        }
        unsigned todo = __ballot_sync(kFull, valid);
        while (todo) {
            const int j = __ffs(todo) - 1;
            todo &= todo - 1;
            const uint32_t a = __shfl_sync(kFull, v0, j);
            const uint32_t b = __shfl_sync(kFull, v1, j);
            if (lane == 0) {
                w.emb[0] = a;
                w.emb[1] = b;
            }
            __syncwarp();
            c.build_chain(0, a, false);  // depth 0 is accounted per start vertex on the host
            if (!c.build_chain(1, b)) continue;
            ++tasks;
            sum += c.dfs();
        }
    }
    if (lane == 0) {
        atomicAdd(&counters[kSum], sum);
        atomicAdd(&counters[kTasks], tasks);
        if (kBytesOn) atomicAdd(&counters[kBytes], c.bytes);
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

// Runs the counting kernel for one plan on one graph.  deadline_ms = 0 means
// no budget.
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
    if ((e = cudaMemsetAsync(g->d_counters, 0, 8 * sizeof(unsigned long long), st)) != cudaSuccess)
        return cuda_fail(e, "counter reset");
    // Work budget: each warp stops claiming tasks once %globaltimer has
    // advanced budget_ns past its own start, and the call reports
    // GI_ETIMEOUT.  No wait in the kernel depends on another warp.
    const unsigned long long budget_ns =
        budget_ms > 0 ? static_cast<unsigned long long>(budget_ms * 1e6) : 0ull;
    cudaEvent_t t0, t1;
    cudaEventCreate(&t0);
    cudaEventCreate(&t1);
    cudaEventRecord(t0, st);
    if (bytes_on)
        dfs_count_kernel<true><<<blocks, kBlockThreads, 0, st>>>(P, g->d_vertex, reinterpret_cast<const uint32_t *>(g->d_edge),
                                                                 g->d_edge_from, g->e_cnt,
                                                                 static_cast<uint32_t *>(g->d_scratch), stride,
                                                                 g->d_counters, budget_ns, shard, num_shards);
    else
        dfs_count_kernel<false><<<blocks, kBlockThreads, 0, st>>>(P, g->d_vertex, reinterpret_cast<const uint32_t *>(g->d_edge),
                                                                  g->d_edge_from, g->e_cnt,
                                                                  static_cast<uint32_t *>(g->d_scratch), stride,
                                                                  g->d_counters, budget_ns, shard, num_shards);
    e = cudaGetLastError();
    cudaEventRecord(t1, st);
    unsigned long long host[8] = {0};
    if (e == cudaSuccess) e = cudaMemcpyAsync(host, g->d_counters, sizeof(host), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    float ms = 0.f;
    if (e == cudaSuccess) cudaEventElapsedTime(&ms, t0, t1);
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    if (e != cudaSuccess) return cuda_fail(e, "counting kernel");
    if (host[kTimeout]) return fail(GI_ETIMEOUT, "count exceeded its device time budget");
    *raw_sum = host[kSum];
    if (stats) {
        stats->kernel_ms += ms;
        stats->raw_sum = host[kSum];
        stats->tasks += host[kTasks];
        if (bytes_on) stats->alg_bytes += host[kBytes];
        stats->grid_blocks = blocks;
        stats->block_threads = kBlockThreads;
        stats->kernel_launches += 1;
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
    budget = stats->budget_ms;
    std::memset(stats, 0, sizeof(*stats));
    stats->count_bytes = cb;
    stats->budget_ms = budget;
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
