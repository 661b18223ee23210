// k-clique and motif counting entry points.
//
// gi_clique_count: the graph is oriented into a DAG on the device, then the
// clique plan (Schedule_IEP(adj_mat, k): every position adjacent to every
// earlier one, no restrictions, no IEP) runs through the counting kernel
// over the DAG's edges — or, for the degree orientation, the per-vertex
// bitmap kernels of kclique.cu.  orientation 0 keeps u -> v when v < u (reference
// reduce_edges_for_clique, src/graph.cpp:710-735, used by gpu/gpu_clique.cu
// :585 and src/clique_test.cpp:73); orientation 1 keeps u -> v when
// (deg u, u) < (deg v, v) (reference degree_orientation_init,
// src/graph.cpp:821-859, used by gpu/gpu_kclique.cu:535).
//
// gi_motif_count: one plan per connected k-vertex pattern in MotifGenerator
// order, each Schedule_IEP(p, valid, 1, 1, true, v, e, tri) and counted on
// the graph (reference gpu/gpu_mc.cu:93-112).
#include <cuda_runtime.h>
#include <cub/device/device_scan.cuh>

#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "internal.hpp"

namespace gi {

int cuda_fail(cudaError_t e, const char *what);
int count_impl(gi_graph *g, const DevPlan &P, cudaStream_t st, uint64_t *raw_sum, gi_stats *stats, double budget_ms,
               int64_t shard, int64_t num_shards);
void graph_free(gi_graph *g);
int kclique_bitmap(gi_graph *o, int k, cudaStream_t st, uint64_t *out, gi_stats *stats);
int kclique_pivot(gi_graph *o, int kmax, cudaStream_t st, uint64_t *counts, gi_stats *stats);
int kclique_max_bitmap_degree();

namespace {

__device__ __forceinline__ bool keep_arc(int orientation, uint32_t u, uint32_t v, const int64_t *vertex) {
    if (orientation == 0) return v < u;
    const int64_t du = vertex[u + 1] - vertex[u], dv = vertex[v + 1] - vertex[v];
    return du < dv || (du == dv && u < v);
}

// Warp per vertex: out-degree of the oriented graph.
__global__ void oriented_degree_kernel(const int64_t *__restrict__ vertex, const int32_t *__restrict__ edge,
                                       int32_t v_cnt, int orientation, int64_t *__restrict__ deg) {
    const int lane = threadIdx.x & 31;
    const int64_t warp = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = (static_cast<int64_t>(gridDim.x) * blockDim.x) >> 5;
    for (int64_t v = warp; v < v_cnt; v += nwarps) {
        int c = 0;
        for (int64_t j = vertex[v] + lane; j < vertex[v + 1]; j += 32)
            c += keep_arc(orientation, static_cast<uint32_t>(v), static_cast<uint32_t>(edge[j]), vertex);
        for (int o = 16; o; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
        if (lane == 0) deg[v] = c;
    }
}

// Warp per vertex: copies the kept arcs (order preserved, so lists stay
// sorted) and fills edge_from.
__global__ void oriented_fill_kernel(const int64_t *__restrict__ vertex, const int32_t *__restrict__ edge,
                                     int32_t v_cnt, int orientation, const int64_t *__restrict__ out_vertex,
                                     int32_t *__restrict__ out_edge, uint32_t *__restrict__ out_from) {
    const int lane = threadIdx.x & 31;
    const int64_t warp = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = (static_cast<int64_t>(gridDim.x) * blockDim.x) >> 5;
    for (int64_t v = warp; v < v_cnt; v += nwarps) {
        int64_t w = out_vertex[v];
        for (int64_t base = vertex[v]; base < vertex[v + 1]; base += 32) {
            const int64_t j = base + lane;
            bool k = false;
            int32_t x = 0;
            if (j < vertex[v + 1]) {
                x = edge[j];
                k = keep_arc(orientation, static_cast<uint32_t>(v), static_cast<uint32_t>(x), vertex);
            }
            const unsigned m = __ballot_sync(0xffffffffu, k);
            if (k) {
                const int64_t at = w + __popc(m & ((1u << lane) - 1u));
                out_edge[at] = x;
                out_from[at] = static_cast<uint32_t>(v);
            }
            w += __popc(m);
        }
    }
}

}  // namespace

// Builds (once) and caches the oriented DAG of g.  Caller holds g->mu.
int oriented_graph(gi_graph *g, int orientation, cudaStream_t st, gi_graph **out) {
    if (g->oriented[orientation]) {
        *out = g->oriented[orientation];
        return GI_OK;
    }
    auto *o = new (std::nothrow) gi_graph;
    if (!o) return fail(GI_ENOMEM, "out of host memory");
    o->device = g->device;
    o->v_cnt = g->v_cnt;
    o->tri_cnt = g->tri_cnt;
    cudaError_t e;
    int64_t *deg = nullptr;
    void *tmp = nullptr;
    size_t tmp_bytes = 0;
    const size_t vb = sizeof(int64_t) * (static_cast<size_t>(g->v_cnt) + 1);
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, g->device);
    auto bail = [&](cudaError_t err, const char *what) {
        cudaFree(deg);
        cudaFree(tmp);
        graph_free(o);
        return cuda_fail(err, what);
    };
    if ((e = cudaMalloc(&deg, vb)) != cudaSuccess) return bail(e, "orientation allocation");
    if ((e = cudaMalloc(&o->d_vertex, vb)) != cudaSuccess) return bail(e, "orientation allocation");
    if ((e = cudaMemsetAsync(deg + g->v_cnt, 0, sizeof(int64_t), st)) != cudaSuccess) return bail(e, "memset");
    oriented_degree_kernel<<<sms * 8, 256, 0, st>>>(g->d_vertex, g->d_edge, g->v_cnt, orientation, deg);
    if ((e = cudaGetLastError()) != cudaSuccess) return bail(e, "orientation degrees");
    cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, deg, o->d_vertex, g->v_cnt + 1, st);
    if ((e = cudaMalloc(&tmp, tmp_bytes)) != cudaSuccess) return bail(e, "scan workspace");
    if ((e = cub::DeviceScan::ExclusiveSum(tmp, tmp_bytes, deg, o->d_vertex, g->v_cnt + 1, st)) != cudaSuccess)
        return bail(e, "orientation scan");
    int64_t arcs = 0;
    if ((e = cudaMemcpyAsync(&arcs, o->d_vertex + g->v_cnt, sizeof(arcs), cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
        (e = cudaStreamSynchronize(st)) != cudaSuccess)
        return bail(e, "orientation size");
    o->e_cnt = arcs;
    const size_t eb = sizeof(int32_t) * static_cast<size_t>(arcs > 0 ? arcs : 1);
    if ((e = cudaMalloc(&o->d_edge, eb)) != cudaSuccess || (e = cudaMalloc(&o->d_edge_from, eb)) != cudaSuccess ||
        (e = cudaMalloc(&o->d_counters, 16 * sizeof(unsigned long long))) != cudaSuccess)
        return bail(e, "oriented graph allocation");
    oriented_fill_kernel<<<sms * 8, 256, 0, st>>>(g->d_vertex, g->d_edge, g->v_cnt, orientation, o->d_vertex,
                                                  o->d_edge, o->d_edge_from);
    std::vector<int64_t> hv(static_cast<size_t>(g->v_cnt) + 1);
    if ((e = cudaGetLastError()) != cudaSuccess ||
        (e = cudaMemcpyAsync(hv.data(), o->d_vertex, vb, cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
        (e = cudaStreamSynchronize(st)) != cudaSuccess)
        return bail(e, "orientation fill");
    cudaFree(deg);
    cudaFree(tmp);
    int64_t a = 0, b = 0;
    for (int32_t v = 0; v < g->v_cnt; ++v) {
        const int64_t d = hv[v + 1] - hv[v];
        if (d > a) {
            b = a;
            a = d;
        } else if (d > b) {
            b = d;
        }
    }
    o->max_degree = static_cast<int32_t>(a);
    // Sets below the first level are intersections with some out-list, so
    // the largest out-degree bounds them.
    o->max_isect = static_cast<int32_t>(a);
    g->oriented[orientation] = o;
    *out = o;
    return GI_OK;
}

namespace {

std::string clique_adj(int k) {
    std::string s(static_cast<size_t>(k) * k, '1');
    for (int i = 0; i < k; ++i) s[i * k + i] = '0';
    return s;
}

}  // namespace

}  // namespace gi

using namespace gi;

extern "C" int gi_clique_count(const gi_graph *cg, int k, int orientation, gi_stream stream, uint64_t *out_count,
                               gi_stats *stats) {
    if (!cg || !out_count) return fail(GI_EINVAL, "NULL argument");
    if (k < 3 || k > GI_MAX_PATTERN) return fail(GI_EINVAL, "clique size must be between 3 and 7");
    if (orientation != 0 && orientation != 1) return fail(GI_EINVAL, "orientation must be 0 or 1");
    gi_graph *g = const_cast<gi_graph *>(cg);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    std::lock_guard<std::mutex> lock(g->mu);
    gi_plan *plan = nullptr;
    const std::string adj = clique_adj(k);
    int rc = gi_plan_create_induced(k, adj.c_str(), &plan);
    if (rc != GI_OK) return rc;
    std::unique_ptr<gi_plan> hold(plan);
    gi_graph *o = nullptr;
    if ((rc = oriented_graph(g, orientation, st, &o)) != GI_OK) return rc;
    double budget = 0;
    if (stats) {
        const int cb = stats->count_bytes;
        budget = stats->budget_ms;
        std::memset(stats, 0, sizeof(*stats));
        stats->count_bytes = cb;
        stats->budget_ms = budget;
    }
    uint64_t raw = 0;
    if (o->e_cnt == 0) {
        *out_count = 0;
        return GI_OK;
    }
    std::lock_guard<std::mutex> lock2(o->mu);
    // Degree orientation: per-vertex bitmaps (kclique.cu) unless an
    // out-degree is too large for them or the caller asked for a work budget
    // or byte accounting, which only the general kernel provides.
    if (orientation == 1 && o->max_degree <= kclique_max_bitmap_degree() && budget <= 0 &&
        !(stats && stats->count_bytes)) {
        rc = kclique_bitmap(o, k, st, out_count, stats);
        if (rc != GI_ENOMEM) return rc;  // bitmaps too large for free memory: general kernel below
    }
    rc = count_impl(o, plan->dev, st, &raw, stats, budget, 0, 1);
    if (rc != GI_OK) return rc;
    *out_count = raw;  // redundancy is 1 for the clique plan (reference gpu/gpu_clique.cu:628)
    return GI_OK;
}

extern "C" int gi_clique_counts_pivot(const gi_graph *cg, int kmax, gi_stream stream, uint64_t *counts,
                                      gi_stats *stats) {
    if (!cg || !counts) return fail(GI_EINVAL, "NULL argument");
    if (kmax < 1 || kmax > GI_MAX_PATTERN) return fail(GI_EINVAL, "kmax must be between 1 and 7");
    gi_graph *g = const_cast<gi_graph *>(cg);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    std::lock_guard<std::mutex> lock(g->mu);
    gi_graph *o = nullptr;
    int rc = oriented_graph(g, 1, st, &o);
    if (rc != GI_OK) return rc;
    if (stats) std::memset(stats, 0, sizeof(*stats));
    if (o->max_degree > kclique_max_bitmap_degree())
        return fail(GI_ENOTSUP, "an out-degree of the degree-oriented graph exceeds the bitmap limit");
    std::lock_guard<std::mutex> lock2(o->mu);
    rc = kclique_pivot(o, kmax, st, counts, stats);
    if (rc == GI_ENOMEM) return fail(GI_ENOMEM, "k-clique bitmaps do not fit in half the free device memory");
    return rc;
}

extern "C" int gi_motif_count(const gi_graph *cg, int k, gi_stream stream, uint64_t *out_counts, int cap,
                              gi_stats *stats) {
    if (!cg || !out_counts) return fail(GI_EINVAL, "NULL argument");
    const int m = gi_motif_num(k);
    if (m < 0) return fail(GI_EINVAL, "motif size must be between 3 and 7");
    if (cap < m) return fail(GI_EINVAL, "out_counts too small");
    std::vector<char> adj(static_cast<size_t>(m) * k * k);
    int rc = gi_motif_patterns(k, adj.data(), m);
    if (rc != GI_OK) return rc;
    gi_stats total{};
    if (stats) {
        total.count_bytes = stats->count_bytes;
        total.budget_ms = stats->budget_ms;
    }
    for (int i = 0; i < m; ++i) {
        std::string a(adj.data() + static_cast<size_t>(i) * k * k, static_cast<size_t>(k) * k);
        gi_plan *plan = nullptr;
        rc = gi_plan_create(k, a.c_str(), cg->v_cnt, cg->e_cnt, cg->tri_cnt, 1, 1, &plan);
        if (rc != GI_OK) return rc;
        std::unique_ptr<gi_plan> hold(plan);
        gi_stats one{};
        one.count_bytes = total.count_bytes;
        one.budget_ms = total.budget_ms;
        rc = gi_count(cg, plan, stream, &out_counts[i], &one);
        if (rc != GI_OK) return rc;
        total.kernel_ms += one.kernel_ms;
        total.tasks += one.tasks;
        total.alg_bytes += one.alg_bytes;
        total.kernel_launches += one.kernel_launches;
        total.grid_blocks = one.grid_blocks;
        total.block_threads = one.block_threads;
    }
    if (stats) *stats = total;
    return GI_OK;
}
