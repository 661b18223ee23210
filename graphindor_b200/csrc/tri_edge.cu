// Edge-triangle counting: a pattern-specialized path for plans whose DFS ends
// at depth 2 in an inclusion-exclusion tail over the sets N(v0), N(v1) and
// N(v0) ∩ N(v1) only (the diamond, and "books": k triangles sharing an edge).
//
// For such a plan the contribution of a first-level edge (v0, v1) depends on
// three numbers: d(v0), d(v1) and t = |N(v0) ∩ N(v1)|, the triangles on the
// edge (reference gpu/function/pattern_matching.cuh:110-139 evaluates the
// same formula from set sizes).  The general kernel computes t by one
// intersection per edge, and for a hub pair that intersection is long.  Here
// every triangle is listed once on the degree-oriented DAG (arcs from lower
// to higher (degree, id)), so the lists intersected are out-lists of at most
// sqrt(2m) entries, and each triangle adds one to the counts of its three
// arcs.  A second kernel then evaluates the plan's break-size prunes and IEP
// formula for every first-level task of the count (edge subset and shard as
// the general kernel defines them) from (d(v0), d(v1), t).  The raw sum is
// the general kernel's; the arc counts are recomputed by every count.
#include <cuda_runtime.h>

#include <algorithm>

#include "dfs_device.cuh"
#include "internal.hpp"

namespace gi {

int cuda_fail(cudaError_t e, const char *what);
int oriented_graph(gi_graph *g, int orientation, cudaStream_t st, gi_graph **out);

namespace {

// A warp per arc u -> v of the oriented DAG: the common out-neighbours w of
// u and v, each a triangle (u, v, w) whose arcs u->v, u->w and v->w get one
// count each.  The smaller out-list's elements are searched in the larger.
__global__ void tri_arc_kernel(const int64_t *__restrict__ ov, const int32_t *__restrict__ oe,
                               const uint32_t *__restrict__ ofrom, int64_t arcs, unsigned int *__restrict__ t) {
    const int lane = threadIdx.x & 31;
    const int64_t warp = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = (static_cast<int64_t>(gridDim.x) * blockDim.x) >> 5;
    for (int64_t a = warp; a < arcs; a += nwarps) {
        const uint32_t u = ofrom[a], v = static_cast<uint32_t>(oe[a]);
        int64_t pa = ov[u], pb = ov[v];
        int na = static_cast<int>(ov[u + 1] - pa), nb = static_cast<int>(ov[v + 1] - pb);
        if (na == 0 || nb == 0) continue;
        if (na > nb) {
            const int64_t tp = pa;
            pa = pb;
            pb = tp;
            const int tn = na;
            na = nb;
            nb = tn;
        }
        const uint32_t *b = reinterpret_cast<const uint32_t *>(oe + pb);
        int found = 0;
        for (int i = lane; i < na; i += 32) {
            const uint32_t w = static_cast<uint32_t>(oe[pa + i]);
            const int j = lower_bound_u32(b, nb, w);
            if (j < nb && b[j] == w) {
                atomicAdd(&t[pa + i], 1u);
                atomicAdd(&t[pb + j], 1u);
                ++found;
            }
        }
        for (int o = 16; o; o >>= 1) found += __shfl_xor_sync(kFull, found, o);
        if (lane == 0 && found) atomicAdd(&t[a], static_cast<unsigned>(found));
    }
}

// Index of the arc of the undirected edge {x, y} in the oriented DAG.
__device__ __forceinline__ int64_t arc_of(const int64_t *__restrict__ vertex, const int64_t *__restrict__ ov,
                                          const int32_t *__restrict__ oe, uint32_t x, uint32_t y) {
    const int64_t dx = vertex[x + 1] - vertex[x], dy = vertex[y + 1] - vertex[y];
    const bool x_first = dx < dy || (dx == dy && x < y);
    const uint32_t tail = x_first ? x : y, head = x_first ? y : x;
    const int64_t p = ov[tail];
    const int n = static_cast<int>(ov[tail + 1] - p);
    return p + lower_bound_u32(reinterpret_cast<const uint32_t *>(oe + p), n, head);
}

// A thread per first-level task of the count: the task's edge (the t-th
// directed edge of the subset), its chunk's shard, the depth-1 restriction,
// the chain-1 break-size prunes and the IEP formula from (d0, d1, t).
__global__ void tri_eval_kernel(const __grid_constant__ DevPlan P, const int64_t *__restrict__ vertex,
                                const uint32_t *__restrict__ edge, const uint32_t *__restrict__ edge_from,
                                const int64_t *__restrict__ ov, const int32_t *__restrict__ oe,
                                const unsigned int *__restrict__ t, int64_t n_tasks, int64_t edge_step,
                                int64_t edge_offset, int64_t shard, int64_t num_shards,
                                unsigned long long *__restrict__ counters) {
    const int lane = threadIdx.x & 31;
    unsigned long long sum = 0, tasks = 0;
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < n_tasks;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        if ((i / kTaskChunk) % num_shards != shard) continue;
        const int64_t e = edge_offset + i * edge_step;
        const uint32_t v0 = edge_from[e], v1 = edge[e];
        if (P.first_restricted && v0 <= v1) continue;
        const int d0 = static_cast<int>(vertex[v0 + 1] - vertex[v0]);
        const int d1 = static_cast<int>(vertex[v1 + 1] - vertex[v1]);
        const int tri = static_cast<int>(t[arc_of(vertex, ov, oe, v0, v1)]);
        // Sizes of the sets: depth 0 is N(v0); at depth 1 an alias is N(v1),
        // anything else N(v0) ∩ N(v1).
        auto size_of = [&](int q) { return P.pdepth[q] == 0 ? d0 : P.father[q] == -1 ? d1 : tri; };
        bool pruned = false;
        for (int p = P.last[1]; p != -1; p = P.next[p])
            if (size_of(p) == P.break_size[p]) pruned = true;
        if (pruned) continue;
        ++tasks;
        if (size_of(P.loop_set[2]) <= 0) continue;
        int ans[GI_MAX_IEP_SETS];
        for (int k = 0; k < P.iep_nsets; ++k) {
            const int q = P.iep_set[k];
            const int sz = size_of(q);
            // Embedded vertices in the set: v1 lies in N(v0), v0 in N(v1),
            // neither in N(v0) ∩ N(v1).
            const int emb = P.pdepth[q] == 0 || P.father[q] == -1 ? 1 : 0;
            ans[k] = P.iep_set_flag[k] ? sz - P.iep_set_coef[k] : sz - emb;
        }
        sum += iep_combine(P, ans);
    }
    sum = warp_sum(sum);
    tasks = warp_sum(tasks);
    if (lane == 0) {
        if (sum) atomicAdd(&counters[kSum], sum);
        if (tasks) atomicAdd(&counters[kTasks], tasks);
    }
}

}  // namespace

// Raw sum of plan P over the edge subset and shard, by edge-triangle counts.
// Caller holds g->mu and has checked P.tri_ok.
int count_tri_edge(gi_graph *g, const DevPlan &P, cudaStream_t st, int64_t edge_step, int64_t edge_offset,
                   int64_t shard, int64_t num_shards, uint64_t *raw_sum, gi_stats *stats) {
    gi_graph *o = nullptr;
    int rc = oriented_graph(g, 1, st, &o);
    if (rc != GI_OK) return rc;
    cudaError_t e;
    if (g->tri_arc_cap < o->e_cnt) {
        cudaFree(g->d_tri_arc);
        g->d_tri_arc = nullptr;
        g->tri_arc_cap = 0;
        if ((e = cudaMalloc(&g->d_tri_arc, std::max<int64_t>(o->e_cnt, 1) * sizeof(unsigned int))) != cudaSuccess)
            return cuda_fail(e, "arc triangle counts");
        g->tri_arc_cap = std::max<int64_t>(o->e_cnt, 1);
    }
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, g->device);
    ScopedEvents ev(2);
    cudaEvent_t t0 = static_cast<cudaEvent_t>(ev[0]), t1 = static_cast<cudaEvent_t>(ev[1]);
    if (!t0 || !t1) return fail(GI_ECUDA, "timing event creation failed");
    cudaEventRecord(t0, st);
    unsigned int *t = static_cast<unsigned int *>(g->d_tri_arc);
    if ((e = cudaMemsetAsync(t, 0, std::max<int64_t>(o->e_cnt, 1) * sizeof(unsigned int), st)) != cudaSuccess ||
        (e = cudaMemsetAsync(g->d_counters, 0, kCounterSlots * sizeof(unsigned long long), st)) != cudaSuccess)
        return cuda_fail(e, "triangle count reset");
    if (o->e_cnt > 0)
        tri_arc_kernel<<<sms * 16, 256, 0, st>>>(o->d_vertex, o->d_edge, o->d_edge_from, o->e_cnt, t);
    const int64_t n_tasks = g->e_cnt > edge_offset ? (g->e_cnt - edge_offset + edge_step - 1) / edge_step : 0;
    if (n_tasks > 0)
        tri_eval_kernel<<<sms * 8, 256, 0, st>>>(P, g->d_vertex, reinterpret_cast<const uint32_t *>(g->d_edge),
                                                 g->d_edge_from, o->d_vertex, o->d_edge, t, n_tasks, edge_step,
                                                 edge_offset, shard, num_shards, g->d_counters);
    e = cudaGetLastError();
    cudaEventRecord(t1, st);
    unsigned long long host[kCounterSlots] = {0};
    if (e == cudaSuccess) e = cudaMemcpyAsync(host, g->d_counters, sizeof(host), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) return cuda_fail(e, "edge-triangle count");
    float ms = 0.f;
    cudaEventElapsedTime(&ms, t0, t1);
    *raw_sum = host[kSum];
    if (stats) {
        const int64_t n_chunks = (n_tasks + kTaskChunk - 1) / kTaskChunk;
        stats->chunks_done += n_chunks > shard ? (n_chunks - shard + num_shards - 1) / num_shards : 0;
        stats->chunks_total = stats->chunks_done;
        stats->kernel_ms += ms;
        stats->raw_sum = host[kSum];
        stats->tasks += host[kTasks];
        stats->grid_blocks = sms * 8;
        stats->block_threads = 256;
        stats->kernel_launches += o->e_cnt > 0 ? 2 : 1;
    }
    return GI_OK;
}

}  // namespace gi
