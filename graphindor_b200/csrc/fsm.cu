// MNI support of labeled patterns on the GPU.
//
// The reference gives one warp to one labeled pattern and enumerates every
// embedding from every start vertex of the first label, inserting the
// matched vertices of each pattern vertex into per-warp bit vectors until
// the minimum image count reaches min_support (reference
// gpu/gpu_fsm.cu:315-574).  The decision it makes — frequent or not — only
// depends on the image sets: pattern vertex i's image set is the set of
// graph vertices v with label(i) for which some embedding maps i to v.  This
// kernel decides membership in those sets directly: one lane takes one
// (labeled pattern, pattern vertex i, candidate v) and runs a depth-first
// search rooted at i = v that stops at the first complete embedding.  Lanes
// of a warp take 32 consecutive candidates of one (pattern, vertex) pair;
// per pair a hit count and a miss count decide early: the pair is done once
// hits reach min_support, and the labeled pattern is infrequent as soon as
// some pair can no longer reach it (candidates - misses < min_support).
//
// Work order: the pairs are sorted by their number of 32-candidate chunks
// (descending) and the chunk sequence runs round by round — the first chunk
// of every pair, then the second chunk of every pair that has one, ... — so
// that early exits cut the later chunks.  Vertices of a label are stored by
// descending degree, so early chunks hold the hubs, where embeddings are
// likeliest.  The whole labeled structure (bucket index and edges) is read
// through L2; no wait in the kernel depends on another warp.
#include <cuda_runtime.h>

#include <algorithm>
#include <numeric>
#include <vector>

#include "fsm.hpp"
#include "internal.hpp"

namespace gi {

int cuda_fail(cudaError_t e, const char *what);

namespace {

constexpr int kFsmBlock = 128;
constexpr int kFsmWarps = kFsmBlock / 32;
constexpr unsigned kAll = 0xffffffffu;

__device__ __forceinline__ bool in_sorted(const uint32_t *__restrict__ a, uint32_t lo, uint32_t end, uint32_t x) {
    uint32_t hi = end;
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (a[mid] < x)
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo < end && a[lo] == x;
}

// Is there an embedding of the labeled pattern `lab` (by pattern vertex)
// that maps pattern vertex `root` to graph vertex v?
__device__ bool embeds(const FsmDevPattern &P, const uint32_t *__restrict__ bucket, const uint32_t *__restrict__ edge,
                       const uint8_t *lab, int root, uint32_t v, int64_t l_cnt) {
    const int n = P.n;
    // Cheap filter: v needs, for every label, at least as many neighbours
    // with that label as the root has pattern neighbours with it.
    const uint8_t nm = P.adj_mask[root];
    for (int q = 0; q < n; ++q) {
        if (!((nm >> q) & 1)) continue;
        int need = 0;
        for (int q2 = 0; q2 < n; ++q2) need += ((nm >> q2) & 1) && lab[q2] == lab[q];
        const int64_t b = static_cast<int64_t>(v) * l_cnt + lab[q];
        if (static_cast<int64_t>(bucket[b + 1]) - static_cast<int64_t>(bucket[b]) < need) return false;
    }
    uint32_t m[GI_MAX_PATTERN];   // matched graph vertex per step
    uint32_t cur[GI_MAX_PATTERN];  // position in the anchor bucket per step
    uint32_t end[GI_MAX_PATTERN];
    uint8_t anc[GI_MAX_PATTERN];   // anchor step per step
    uint8_t sl[GI_MAX_PATTERN];    // label per step
    for (int t = 0; t < n; ++t) sl[t] = lab[P.order[root][t]];
    m[0] = v;
    // Sets up step t: iterate the smallest bucket among its parents.
    auto setup = [&](int t) {
        const uint8_t par = P.parents[root][t];
        uint32_t best = 0xffffffffu;
        for (int u = 0; u < t; ++u) {
            if (!((par >> u) & 1)) continue;
            const int64_t b = static_cast<int64_t>(m[u]) * l_cnt + sl[t];
            const uint32_t lo = bucket[b], hi = bucket[b + 1];
            if (hi - lo < best) {
                best = hi - lo;
                anc[t] = static_cast<uint8_t>(u);
                cur[t] = lo;
                end[t] = hi;
            }
        }
    };
    int t = 1;
    setup(1);
    while (true) {
        if (cur[t] >= end[t]) {
            if (t == 1) return false;
            --t;
            ++cur[t];
            continue;
        }
        const uint32_t w = edge[cur[t]];
        bool ok = true;
        for (int u = 0; u < t && ok; ++u)
            if (sl[u] == sl[t] && m[u] == w) ok = false;
        const uint8_t par = P.parents[root][t];
        for (int u = 0; u < t && ok; ++u) {
            if (!((par >> u) & 1) || u == anc[t]) continue;
            const int64_t b = static_cast<int64_t>(m[u]) * l_cnt + sl[t];
            ok = in_sorted(edge, bucket[b], bucket[b + 1], w);
        }
        if (!ok) {
            ++cur[t];
            continue;
        }
        m[t] = w;
        if (t == n - 1) return true;
        ++t;
        setup(t);
    }
}

__global__ void __launch_bounds__(kFsmBlock)
    fsm_support_kernel(const __grid_constant__ FsmDevPattern P, const uint32_t *__restrict__ bucket,
                       const uint32_t *__restrict__ edge, const uint32_t *__restrict__ label_start,
                       const uint8_t *__restrict__ labels, const uint32_t *__restrict__ pairs,
                       const int64_t *__restrict__ round_start, int n_rounds, int64_t n_tasks, unsigned *hits,
                       unsigned *misses, unsigned *dead, unsigned long long *counters) {
    const int lane = threadIdx.x & 31;
    const int n = P.n;
    unsigned long long checked = 0;
    while (true) {
        unsigned long long t = 0;
        if (lane == 0) t = atomicAdd(&counters[0], 1ull);
        t = __shfl_sync(kAll, t, 0);
        if (t >= static_cast<unsigned long long>(n_tasks)) break;
        // Round k: the largest k with round_start[k] <= t.
        int lo = 0, hi = n_rounds;
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (round_start[mid] <= static_cast<int64_t>(t))
                lo = mid;
            else
                hi = mid;
        }
        const int k = lo;
        const uint32_t pair = pairs[static_cast<int64_t>(t) - round_start[k]];
        const uint32_t job = pair / n;
        const int root = static_cast<int>(pair % n);
        int skip = 0;
        if (lane == 0) skip = *(volatile unsigned *)&dead[job] || *(volatile unsigned *)&hits[pair] >= P.min_support;
        if (__shfl_sync(kAll, skip, 0)) continue;
        const uint8_t *lab = labels + static_cast<int64_t>(job) * n;
        const int l = lab[root];
        const uint32_t first = label_start[l], last = label_start[l + 1];
        const uint32_t v = first + static_cast<uint32_t>(k) * 32u + lane;
        const bool valid = v < last;
        const bool hit = valid && embeds(P, bucket, edge, lab, root, v, P.l_cnt);
        const unsigned hit_mask = __ballot_sync(kAll, hit);
        const unsigned valid_mask = __ballot_sync(kAll, valid);
        if (lane == 0) {
            checked += __popc(valid_mask);
            const unsigned nh = __popc(hit_mask), nm = __popc(valid_mask) - nh;
            if (nh) atomicAdd(&hits[pair], nh);
            if (nm) {
                const unsigned missed = atomicAdd(&misses[pair], nm) + nm;
                if (static_cast<int64_t>(last - first) - missed < P.min_support) atomicExch(&dead[job], 1u);
            }
        }
    }
    if (lane == 0 && checked) atomicAdd(&counters[1], checked);
}

struct DeviceBuffer {
    void *p = nullptr;
    ~DeviceBuffer() {
        if (p) cudaFree(p);
    }
};

}  // namespace

int fsm_upload(gi_labeled_graph *g) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
    g->device = dev;
    const size_t eb = std::max<size_t>(g->edge.size(), 1) * sizeof(uint32_t);
    const size_t bb = g->bucket.size() * sizeof(uint32_t);
    const size_t lb = g->label_start.size() * sizeof(uint32_t);
    if ((e = cudaMalloc(&g->d_edge, eb)) != cudaSuccess) return cuda_fail(e, "labeled edge allocation");
    if ((e = cudaMalloc(&g->d_bucket, bb)) != cudaSuccess) return cuda_fail(e, "bucket allocation");
    if ((e = cudaMalloc(&g->d_label_start, lb)) != cudaSuccess) return cuda_fail(e, "label start allocation");
    if (!g->edge.empty() &&
        (e = cudaMemcpy(g->d_edge, g->edge.data(), g->edge.size() * sizeof(uint32_t), cudaMemcpyHostToDevice)) !=
            cudaSuccess)
        return cuda_fail(e, "labeled edge upload");
    if ((e = cudaMemcpy(g->d_bucket, g->bucket.data(), bb, cudaMemcpyHostToDevice)) != cudaSuccess)
        return cuda_fail(e, "bucket upload");
    if ((e = cudaMemcpy(g->d_label_start, g->label_start.data(), lb, cudaMemcpyHostToDevice)) != cudaSuccess)
        return cuda_fail(e, "label start upload");
    return GI_OK;
}

void fsm_free(gi_labeled_graph *g) {
    int prev = 0;
    cudaGetDevice(&prev);
    if (prev != g->device) cudaSetDevice(g->device);
    if (g->d_edge) cudaFree(g->d_edge);
    if (g->d_bucket) cudaFree(g->d_bucket);
    if (g->d_label_start) cudaFree(g->d_label_start);
    g->d_edge = g->d_bucket = g->d_label_start = nullptr;
    if (prev != g->device) cudaSetDevice(prev);
}

int fsm_support(gi_labeled_graph *g, const FsmDevPattern &P, const std::vector<uint8_t> &labels, int64_t n_jobs,
                void *stream, std::vector<uint8_t> &frequent, FsmRunStats &rs) {
    const int n = P.n;
    const int64_t n_pairs = n_jobs * n;
    if (n_pairs >= (int64_t(1) << 32)) return fail(GI_EOVERFLOW, "too many labeled patterns");
    int prev = 0;
    cudaGetDevice(&prev);
    if (prev != g->device) cudaSetDevice(g->device);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    // Pairs by descending chunk count; round k holds the pairs with more
    // than k chunks.
    std::vector<uint32_t> chunks(n_pairs);
    for (int64_t p = 0; p < n_pairs; ++p) {
        const int l = labels[p];
        const uint32_t size = g->label_start[l + 1] - g->label_start[l];
        chunks[p] = (size + 31) / 32;
    }
    std::vector<uint32_t> order(n_pairs);
    std::iota(order.begin(), order.end(), 0u);
    std::stable_sort(order.begin(), order.end(), [&](uint32_t a, uint32_t b) { return chunks[a] > chunks[b]; });
    const uint32_t max_chunks = n_pairs ? chunks[order[0]] : 0;
    std::vector<int64_t> round_start(max_chunks + 1, 0);
    {
        int64_t acc = 0, cnt = n_pairs;  // the pairs with more than k chunks are a prefix of `order`
        for (uint32_t k = 0; k < max_chunks; ++k) {
            while (cnt > 0 && chunks[order[cnt - 1]] <= k) --cnt;
            round_start[k] = acc;
            acc += cnt;
        }
        round_start[max_chunks] = acc;
    }
    const int64_t n_tasks = round_start[max_chunks];
    // One device block: labels | pairs | round_start | hits | misses | dead | counters.
    auto align = [](size_t x) { return (x + 255) & ~size_t(255); };
    const size_t b_lab = align(labels.size());
    const size_t b_pairs = align(n_pairs * sizeof(uint32_t));
    const size_t b_rounds = align((max_chunks + 1) * sizeof(int64_t));
    const size_t b_hits = align(n_pairs * sizeof(unsigned));
    const size_t b_dead = align(n_jobs * sizeof(unsigned));
    const size_t b_cnt = align(2 * sizeof(unsigned long long));
    const size_t total = b_lab + b_pairs + b_rounds + 2 * b_hits + b_dead + b_cnt;
    DeviceBuffer buf;
    cudaError_t e = cudaMalloc(&buf.p, total);
    if (e != cudaSuccess) {
        if (prev != g->device) cudaSetDevice(prev);
        return cuda_fail(e, "fsm work allocation");
    }
    char *base = static_cast<char *>(buf.p);
    uint8_t *d_lab = reinterpret_cast<uint8_t *>(base);
    uint32_t *d_pairs = reinterpret_cast<uint32_t *>(base + b_lab);
    int64_t *d_rounds = reinterpret_cast<int64_t *>(base + b_lab + b_pairs);
    unsigned *d_hits = reinterpret_cast<unsigned *>(base + b_lab + b_pairs + b_rounds);
    unsigned *d_miss = reinterpret_cast<unsigned *>(base + b_lab + b_pairs + b_rounds + b_hits);
    unsigned *d_dead = reinterpret_cast<unsigned *>(base + b_lab + b_pairs + b_rounds + 2 * b_hits);
    unsigned long long *d_cnt =
        reinterpret_cast<unsigned long long *>(base + b_lab + b_pairs + b_rounds + 2 * b_hits + b_dead);
    int sms = 148, per_sm = 1;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, g->device);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fsm_support_kernel, kFsmBlock, 0);
    const int64_t want = (n_tasks + kFsmWarps - 1) / kFsmWarps;
    const int blocks = static_cast<int>(std::max<int64_t>(1, std::min<int64_t>(want, int64_t(sms) * std::max(per_sm, 1))));
    cudaEvent_t t0, t1;
    cudaEventCreate(&t0);
    cudaEventCreate(&t1);
    std::vector<unsigned> hits(n_pairs), dead(n_jobs);
    unsigned long long counters[2] = {0, 0};
    if ((e = cudaMemcpyAsync(d_lab, labels.data(), labels.size(), cudaMemcpyHostToDevice, st)) == cudaSuccess &&
        (e = cudaMemcpyAsync(d_pairs, order.data(), n_pairs * sizeof(uint32_t), cudaMemcpyHostToDevice, st)) ==
            cudaSuccess &&
        (e = cudaMemcpyAsync(d_rounds, round_start.data(), (max_chunks + 1) * sizeof(int64_t), cudaMemcpyHostToDevice,
                             st)) == cudaSuccess &&
        (e = cudaMemsetAsync(d_hits, 0, 2 * b_hits + b_dead + b_cnt, st)) == cudaSuccess) {
        cudaEventRecord(t0, st);
        if (n_tasks > 0)
            fsm_support_kernel<<<blocks, kFsmBlock, 0, st>>>(P, g->d_bucket, g->d_edge, g->d_label_start, d_lab,
                                                             d_pairs, d_rounds, static_cast<int>(max_chunks), n_tasks,
                                                             d_hits, d_miss, d_dead, d_cnt);
        e = cudaGetLastError();
        cudaEventRecord(t1, st);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(hits.data(), d_hits, n_pairs * sizeof(unsigned), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(dead.data(), d_dead, n_jobs * sizeof(unsigned), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaMemcpyAsync(counters, d_cnt, sizeof(counters), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    }
    float ms = 0.f;
    if (e == cudaSuccess) cudaEventElapsedTime(&ms, t0, t1);
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    if (prev != g->device) cudaSetDevice(prev);
    if (e != cudaSuccess) return cuda_fail(e, "fsm support kernel");
    rs.kernel_ms += ms;
    rs.candidates += static_cast<int64_t>(counters[1]);
    rs.launches += n_tasks > 0 ? 1 : 0;
    frequent.assign(n_jobs, 0);
    for (int64_t j = 0; j < n_jobs; ++j) {
        bool ok = !dead[j];
        for (int i = 0; i < n && ok; ++i) ok = hits[j * n + i] >= static_cast<uint64_t>(P.min_support);
        frequent[j] = ok ? 1 : 0;
    }
    return GI_OK;
}

}  // namespace gi
