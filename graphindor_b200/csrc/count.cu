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

#include "dfs_device.cuh"
#include "internal.hpp"

namespace gi {

int cuda_fail(cudaError_t e, const char *what);

namespace {

// Subtasks per edge: a degree bound on the depth-2 loop set, cut into
// pieces of `split` candidates; 0 for edges the depth-1 restriction drops.
// With edge_step > 1 only the edges i with i % edge_step == edge_offset get
// subtasks (an edge subset).
__global__ void split_count_kernel(const __grid_constant__ DevPlan P, const int64_t *__restrict__ vertex,
                                   const uint32_t *__restrict__ edge, const uint32_t *__restrict__ edge_from,
                                   int64_t e_cnt, int split, int64_t edge_step, int64_t edge_offset,
                                   int64_t *__restrict__ counts) {
    const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < e_cnt; i += stride) {
        const uint32_t v0 = edge_from[i], v1 = edge[i];
        if ((P.first_restricted && v0 <= v1) || (edge_step > 1 && i % edge_step != edge_offset)) {
            counts[i] = 0;
            continue;
        }
        const int64_t d0 = vertex[v0 + 1] - vertex[v0], d1 = vertex[v1 + 1] - vertex[v1];
        const int64_t b = P.loop2_kind == 0 ? d0 : P.loop2_kind == 1 ? d1 : min(d0, d1);
        const int64_t pieces = (b + split - 1) / split;
        counts[i] = pieces > 0 ? pieces : 1;
    }
}

// kMinBlocks: resident blocks per SM the register allocation is held to.
// Deep plans (six or more pattern vertices) spend their time in long chains
// of dependent loads and gain from the extra resident warps despite some
// spilling (R-MAT scale 22: prism 1.6x, 6-cycle+chord 1.6x faster at 16
// blocks); shallower plans run best with the unconstrained allocation.
constexpr unsigned long long kHandoffCap = 1ull << 20;

template <bool kBytesOn, int kMinBlocks>
__global__ void __launch_bounds__(kBlockThreads, kMinBlocks)
    dfs_count_kernel(const __grid_constant__ DevPlan P, const int64_t *__restrict__ vertex,
                     const uint32_t *__restrict__ edge, const uint32_t *__restrict__ edge_from, int64_t e_cnt,
                     const int64_t *__restrict__ offsets, int64_t n_tasks, int split, uint32_t *scratch,
                     int64_t slot_stride, unsigned long long *counters, unsigned long long budget_ns, int64_t shard,
                     int64_t num_shards, int64_t n_chunks, int64_t perm_a, int64_t perm_b,
                     unsigned long long hard_ns, unsigned long long max_claims, Handoff *hitems,
                     unsigned long long hcap, uint32_t hepoch, uint32_t v_cnt, int64_t edge_step,
                     int64_t edge_offset, HubIndex hubs, HashIndex hashes) {
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
    c.hubs = hubs;
    c.hashes = hashes;
    if (hitems) {
        c.hq.items = hitems;
        c.hq.cap = hcap;
        c.hq.ctr = counters + kQueue;
        c.hq.epoch = hepoch;
        c.hq.v_cnt = v_cnt;
    }
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
            if (max_claims && j >= max_claims) {
                stop = 1;  // a fixed sample: the first max_claims chunks of the order
            } else if (budget_ns && globaltimer() - t_start > budget_ns) {
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
        int64_t e = edge_offset + t * edge_step;  // without the split, work item t is the t-th edge of the subset
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
        if (P.flat_first) {
            // The DFS ends at depth 2: the chunk's edges are one flat leaf.
            chunk_sum = c.first_level_flat(v0, v1, valid, chunk_tasks);
            todo = 0;
        }
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
    // Out of chunks: take handed-off ranges (take_handoffs).
    bool lost = false;
    const bool warp_timed_out = __shfl_sync(kFull, timed_out ? 1 : 0, 0) != 0;
    if (hitems)
        lost = take_handoffs(c.hq, warp_timed_out, lane, [&](long long slot) {
            unsigned long long part = 0;
            if (!c.run_handoff(&hitems[slot], part)) return false;
            sum += part;
            return true;
        });
    const unsigned long long lane_bytes = kBytesOn ? warp_sum(c.bytes) : 0;
    if (lane == 0) {
        if (lost) atomicAdd(&counters[kLost], 1ull);
        atomicAdd(&counters[kSum], sum);
        atomicAdd(&counters[kTasks], tasks);
        atomicAdd(&counters[kChunks], chunks);
        if (kBytesOn) atomicAdd(&counters[kBytes], lane_bytes);
        if (timed_out) atomicExch(&counters[kTimeout], 1ull);
    }
}

}  // namespace

// Ensures the graph's scratch can hold `bytes`; caller holds g->mu.  A
// growing scratch at least doubles (when the device has the room), so that
// the plans of a workload, each needing a few more sets than the last, cost
// few reallocations: each is a device-wide cudaFree and a cudaMalloc of up to
// gigabytes.
int ensure_scratch(gi_graph *g, size_t bytes) {
    if (g->scratch_bytes >= bytes) return GI_OK;
    cudaFree(g->d_scratch);
    g->d_scratch = nullptr;
    const size_t doubled = std::max(bytes, 2 * g->scratch_bytes);
    g->scratch_bytes = 0;
    cudaError_t e = doubled > bytes ? cudaMalloc(&g->d_scratch, doubled) : cudaErrorMemoryAllocation;
    size_t got = doubled;
    if (e != cudaSuccess) {
        cudaGetLastError();
        g->d_scratch = nullptr;
        e = cudaMalloc(&g->d_scratch, bytes);
        got = bytes;
    }
    if (e != cudaSuccess) {
        cudaGetLastError();
        g->d_scratch = nullptr;
        return cuda_fail(e, "scratch allocation");
    }
    g->scratch_bytes = got;
    return GI_OK;
}

// Candidates of the depth-2 loop per subtask: one lane each when depth 2 is
// the leaf level, one warp at a time otherwise.
#ifndef GI_SPLIT_LEAF2
#define GI_SPLIT_LEAF2 256
#endif
#ifndef GI_SPLIT_DEEP
#define GI_SPLIT_DEEP 32
#endif
static int split_size(const DevPlan &P) {
    if (P.split > 0) return P.split;
    return P.leaf_depth == 2 ? GI_SPLIT_LEAF2 : GI_SPLIT_DEEP;
}

// Builds the subtask offsets for the plan's depth-2 split; returns the
// number of subtasks.  Caller holds g->mu.
static int build_split(gi_graph *g, const DevPlan &P, cudaStream_t st, int split, int64_t edge_step,
                       int64_t edge_offset, int64_t *n_tasks) {
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
                                                  g->d_edge_from, g->e_cnt, split, edge_step, edge_offset,
                                                  counts);
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

using DfsKernel = decltype(&dfs_count_kernel<false, 1>);

// The instantiation for a plan: byte counting on or off, and the occupancy
// target (the plan's variant, else by pattern size).
DfsKernel pick_dfs_kernel(bool bytes_on, const DevPlan &P) {
    const bool deep = P.occupancy ? P.occupancy >= 16 : P.n >= 6;
    if (bytes_on) return deep ? dfs_count_kernel<true, 16> : dfs_count_kernel<true, 1>;
    return deep ? dfs_count_kernel<false, 16> : dfs_count_kernel<false, 1>;
}

int count_tri_edge(gi_graph *g, const DevPlan &P, cudaStream_t st, int64_t edge_step, int64_t edge_offset,
                   int64_t shard, int64_t num_shards, uint64_t *raw_sum, gi_stats *stats);

// Runs the counting kernel for one plan on one graph (or one shard of it).
// budget_ms = 0 means no budget.
int count_impl(gi_graph *g, const DevPlan &plan, cudaStream_t st, uint64_t *raw_sum, gi_stats *stats,
               double budget_ms, int64_t shard, int64_t num_shards) {
    DeviceGuard device(g->device);
    const DevPlan P = plan_for_graph(plan, g->max_degree);
    int sms = 148, blocks_per_sm = 1;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, g->device);
    const bool bytes_on = stats && stats->count_bytes;
    // Edge subset: the directed edges e with e % edge_step == edge_offset.
    const int64_t edge_step = stats && stats->edge_step > 1 ? stats->edge_step : 1;
    const int64_t edge_offset = edge_step > 1 ? stats->edge_offset : 0;
    if (edge_offset < 0 || edge_offset >= edge_step) return fail(GI_EINVAL, "edge_offset outside [0, edge_step)");
    // The edge-triangle path (tri_edge.cu) for plans that allow it, except
    // for the instrumented, time-budgeted-sample and fixed-sample modes.
    if (P.tri_edge && P.tri_ok && !bytes_on && !(stats && (stats->allow_partial || stats->sample_chunks > 0)))
        return count_tri_edge(g, P, st, edge_step, edge_offset, shard, num_shards, raw_sum, stats);
    cudaError_t e;
    const auto kernel = pick_dfs_kernel(bytes_on, P);
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks_per_sm, kernel, kBlockThreads, 0);
    if (e != cudaSuccess) return cuda_fail(e, "occupancy query");
    const int blocks = sms * std::max(1, blocks_per_sm);
    const int64_t warps = static_cast<int64_t>(blocks) * kWarpsPerBlock;
    const int64_t stride = std::max<int64_t>(g->max_isect, 1);
    const size_t need = static_cast<size_t>(warps) * std::max(P.n_slots, 1) * stride * sizeof(uint32_t);
    int st_code = ensure_scratch(g, need);
    if (st_code != GI_OK) return st_code;
    ScopedEvents ev(3);
    cudaEvent_t t0 = static_cast<cudaEvent_t>(ev[0]), tm = static_cast<cudaEvent_t>(ev[1]),
                t1 = static_cast<cudaEvent_t>(ev[2]);
    if (!t0 || !tm || !t1) return fail(GI_ECUDA, "timing event creation failed");
    cudaEventRecord(t0, st);
    // Split the depth-2 loop when the plan has one; otherwise a work item is
    // an edge of the subset.
    const bool use_split = P.loop2_kind >= 0 && g->e_cnt > 0;
    const int split = split_size(P);
    int64_t n_tasks = g->e_cnt > edge_offset ? (g->e_cnt - edge_offset + edge_step - 1) / edge_step : 0;
    int launches = 0;
    if (use_split) {
        st_code = build_split(g, P, st, split, edge_step, edge_offset, &n_tasks);
        if (st_code != GI_OK) return st_code;
        launches += 1;  // split count (the scan is cub's)
    }
    if ((e = cudaMemsetAsync(g->d_counters, 0, kCounterSlots * sizeof(unsigned long long), st)) != cudaSuccess)
        return cuda_fail(e, "counter reset");
    // Work budget: each warp stops claiming work once %globaltimer has
    // advanced budget_ns past its own start, and the call reports
    // GI_ETIMEOUT.  No wait in the kernel depends on another warp.  A
    // sampled count (allow_partial) visits the chunks in a pseudo-random
    // order and drops chunks still running at three times the budget.
    // A fixed sample (sample_chunks) visits the same pseudo-random order and
    // stops claiming after that many chunks, each counted to completion.
    const unsigned long long budget_ns = budget_ms > 0 ? static_cast<unsigned long long>(budget_ms * 1e6) : 0ull;
    const bool partial = budget_ns && stats && stats->allow_partial;
    const unsigned long long max_claims =
        stats && stats->sample_chunks > 0 ? static_cast<unsigned long long>(stats->sample_chunks) : 0ull;
    const int64_t *offs = use_split ? g->d_offsets : nullptr;
    const int64_t n_chunks = (n_tasks + kTaskChunk - 1) / kTaskChunk;
    int64_t perm_a = 0, perm_b = 0;
    if ((partial || max_claims) && n_chunks > 1) {
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
    // Work donation, except in time-budgeted samples (whose dropped chunks
    // must take their handed-off ranges with them).
    Handoff *hitems = nullptr;
    if (!hard_ns) {
        if (!g->d_handoff) {
            if ((e = cudaMalloc(&g->d_handoff, kHandoffCap * sizeof(Handoff))) != cudaSuccess ||
                (e = cudaMemsetAsync(g->d_handoff, 0, kHandoffCap * sizeof(Handoff), st)) != cudaSuccess) {
                cudaFree(g->d_handoff);
                g->d_handoff = nullptr;
                return cuda_fail(e, "handoff queue allocation");
            }
        }
        hitems = static_cast<Handoff *>(g->d_handoff);
        if (++g->handoff_epoch == 0) ++g->handoff_epoch;
    }
    cudaEventRecord(tm, st);
    kernel<<<blocks, kBlockThreads, 0, st>>>(P, g->d_vertex, reinterpret_cast<const uint32_t *>(g->d_edge),
                                             g->d_edge_from, g->e_cnt, offs, n_tasks, split,
                                             static_cast<uint32_t *>(g->d_scratch), stride, g->d_counters, budget_ns,
                                             shard, num_shards, n_chunks, perm_a, perm_b, hard_ns, max_claims,
                                             hitems, kHandoffCap, g->handoff_epoch,
                                             static_cast<uint32_t>(g->v_cnt), edge_step, edge_offset,
                                             hubs_of(g), hashes_of(g));
    launches += 1;
    e = cudaGetLastError();
    cudaEventRecord(t1, st);
    unsigned long long host[kCounterSlots] = {0};
    if (e == cudaSuccess) e = cudaMemcpyAsync(host, g->d_counters, sizeof(host), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return cuda_fail(e, "counting kernel");
    float ms = 0.f, prep = 0.f;
    cudaEventElapsedTime(&prep, t0, tm);
    cudaEventElapsedTime(&ms, tm, t1);
    if (host[kLost]) return fail(GI_ECUDA, "a handed-off work item was never published");
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
    return GI_OK;
}

}  // namespace gi

using namespace gi;

static void reset_stats(gi_stats *stats, double &budget) {
    budget = 0.0;
    if (!stats) return;
    const int cb = stats->count_bytes;
    const int partial = stats->allow_partial;
    const int64_t sample = stats->sample_chunks;
    const int64_t step = stats->edge_step, offset = stats->edge_offset;
    budget = stats->budget_ms;
    std::memset(stats, 0, sizeof(*stats));
    stats->edge_step = step;
    stats->edge_offset = offset;
    stats->count_bytes = cb;
    stats->budget_ms = budget;
    stats->allow_partial = partial;
    stats->sample_chunks = sample;
}

extern "C" int gi_count(const gi_graph *cg, const gi_plan *p, gi_stream stream, uint64_t *out_count,
                        gi_stats *stats) {
    if (!cg || !p || !out_count) return fail(GI_EINVAL, "NULL argument");
    gi_graph *g = const_cast<gi_graph *>(cg);
    std::lock_guard<std::mutex> lock(g->mu);
    uint64_t raw = 0;
    double budget = 0.0;
    reset_stats(stats, budget);
    if (stats) {  // samples are a gi_count_shard feature; a whole count is whole
        stats->allow_partial = 0;
        stats->sample_chunks = 0;
        stats->edge_step = 0;
        stats->edge_offset = 0;
    }
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
