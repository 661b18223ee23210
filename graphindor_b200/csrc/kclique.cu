// k-clique counting on the degree-oriented DAG with per-vertex adjacency
// bitmaps (reference gpu/gpu_kclique.cu:199-469, k_clique_counting :471-546).
//
// Every k-clique has exactly one lowest vertex u in the DAG order, and its
// other k-1 vertices form a (k-1)-clique of the DAG induced on N+(u).  For
// each u with at least two out-neighbours a bitmap holds that induced DAG —
// row i has bit j when N+(u)[j] is an out-neighbour of N+(u)[i] — and the
// (k-1)-cliques are counted by AND-ing rows along a depth-first search with a
// popcount at the last level.
//
// The reference builds the bitmaps on the host and gives each vertex one
// block, a thread per row.  Here:
//   - kc_build_kernel builds every bitmap on the device, once per graph (they
//     do not depend on k and are kept on the graph handle): a warp per vertex
//     fills each row either by reading N+(v_i) coalesced and searching the
//     vertex's list (kept in shared memory), or — when N+(v_i) is much longer
//     than the list — by searching each list entry in N+(v_i) and assembling
//     32-bit words with __ballot_sync;
//   - kc_count_kernel makes the rows themselves (one per DAG arc) the work
//     items, claimed 32 at a time, so a hub's rows spread over the whole GPU
//     instead of one block: rows of at most four words run one per lane;
//     longer rows run one per warp, a lane holding every 32nd word of the
//     current set, so each step is warp-uniform.
// Graphs whose out-degree exceeds kclique_max_bitmap_degree(), or whose
// bitmaps would not fit in half the free device memory, use the general
// counting kernel on the DAG instead (clique_motif.cu).
#include <cuda_runtime.h>
#include <cub/device/device_scan.cuh>

#include <algorithm>
#include <vector>

#include "internal.hpp"
#include "pivot.cuh"

namespace gi {

int cuda_fail(cudaError_t e, const char *what);

namespace {

constexpr unsigned kFull = 0xffffffffu;
constexpr int kBlock = 128;
constexpr int kWarps = kBlock / 32;
constexpr int kLaneWords = 4;                   // rows of <= 128 bits run one per lane
constexpr int kMaxLevels = GI_MAX_PATTERN - 2;  // set levels below a row (k <= 7)
constexpr int kWarpWpl = 4;                     // words per lane in the warp search (rows <= 4096 bits)
constexpr int kListCap = 1024;                  // list entries kept in shared memory per warp

enum Counter { kSum = 0, kCursor = 1, kBuildCursor = 2 };

// Bitmap words of vertex v: d * ceil(d/32) when d >= 2.
__global__ void kc_words_kernel(const int64_t *__restrict__ vertex, int32_t v_cnt, int64_t *__restrict__ words) {
    for (int64_t v = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; v <= v_cnt;
         v += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        if (v == v_cnt) {
            words[v] = 0;
            continue;
        }
        const int64_t d = vertex[v + 1] - vertex[v];
        words[v] = d >= 2 ? d * ((d + 31) >> 5) : 0;
    }
}

template <class T>
__device__ __forceinline__ int find_pos(const T *list, int n, int32_t x) {
    int lo = 0, hi = n;
    while (lo < hi) {
        const int mid = (lo + hi) >> 1;
        if (list[mid] < x)
            lo = mid + 1;
        else
            hi = mid;
    }
    return (lo < n && list[lo] == x) ? lo : -1;
}

__global__ void __launch_bounds__(kBlock)
    kc_build_kernel(const int64_t *__restrict__ vertex, const int32_t *__restrict__ edge, int32_t v_cnt,
                    const int64_t *__restrict__ off, uint32_t *__restrict__ bitmap, unsigned long long *counters) {
    __shared__ int32_t s_list[kWarps][kListCap];
    __shared__ uint32_t s_row[kWarps][kWarpWpl * 32];
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5;
    while (true) {
        unsigned long long u = 0;
        if (lane == 0) u = atomicAdd(&counters[kBuildCursor], 1ull);
        u = __shfl_sync(kFull, u, 0);
        if (u >= static_cast<unsigned long long>(v_cnt)) break;
        const int64_t b = vertex[u];
        const int d = static_cast<int>(vertex[u + 1] - b);
        if (d < 2) continue;
        const int W = (d + 31) >> 5;
        const int32_t *list = edge + b;
        if (d <= kListCap) {
            for (int j = lane; j < d; j += 32) s_list[wib][j] = list[j];
            __syncwarp();
            list = s_list[wib];
        }
        uint32_t *out = bitmap + off[u];
        for (int i = 0; i < d; ++i) {
            const int32_t v = list[i];
            const int64_t vb = vertex[v], ve = vertex[v + 1];
            const int dv = static_cast<int>(ve - vb);
            uint32_t *row = out + static_cast<int64_t>(i) * W;
            if (dv <= 8 * d) {
                // Scan N+(v), search the list.
                for (int w = lane; w < W; w += 32) s_row[wib][w] = 0;
                __syncwarp();
                for (int64_t p = vb + lane; p < ve; p += 32) {
                    const int j = find_pos(list, d, edge[p]);
                    if (j >= 0) atomicOr(&s_row[wib][j >> 5], 1u << (j & 31));
                }
                __syncwarp();
                for (int w = lane; w < W; w += 32) row[w] = s_row[wib][w];
                __syncwarp();
            } else {
                // Search each list entry in N+(v).
                for (int w = 0; w < W; ++w) {
                    const int j = w * 32 + lane;
                    const bool hit = j < d && find_pos(edge + vb, dv, list[j]) >= 0;
                    const unsigned m = __ballot_sync(kFull, hit);
                    if (lane == 0) row[w] = m;
                }
            }
        }
        __syncwarp();
    }
}

// (k-1)-cliques below row i, one lane, rows of W <= 4 words: levels = k-3
// AND steps, the last a popcount.
__device__ unsigned long long lane_cliques(const uint32_t *__restrict__ rows, int W, int i, int levels) {
    uint32_t S[kMaxLevels][kLaneWords];
    int wi[kMaxLevels];
    uint32_t rem[kMaxLevels];
    unsigned long long acc = 0;
    for (int w = 0; w < W; ++w) S[0][w] = rows[i * W + w];
    if (levels == 0) {
        for (int w = 0; w < W; ++w) acc += __popc(S[0][w]);
        return acc;
    }
    int t = 0;
    wi[0] = 0;
    rem[0] = S[0][0];
    while (t >= 0) {
        while (rem[t] == 0 && ++wi[t] < W) rem[t] = S[t][wi[t]];
        if (rem[t] == 0) {
            --t;
            continue;
        }
        const int j = wi[t] * 32 + __ffs(rem[t]) - 1;
        rem[t] &= rem[t] - 1;
        const uint32_t *r = rows + j * W;
        if (t + 1 == levels) {
            for (int w = 0; w < W; ++w) acc += __popc(S[t][w] & r[w]);
        } else {
            uint32_t any = 0;
            for (int w = 0; w < W; ++w) any |= (S[t + 1][w] = S[t][w] & r[w]);
            if (any) {
                ++t;
                wi[t] = 0;
                rem[t] = S[t][0];
            }
        }
    }
    return acc;
}

// The same for one row of W <= 128 words, warp-cooperative: lane l holds
// words l, l+32, l+64, l+96 of each set.  Returns this lane's share.
__device__ unsigned long long warp_cliques(const uint32_t *__restrict__ rows, int W, int i, int levels, int lane) {
    uint32_t S[kMaxLevels][kWarpWpl];
    int wi[kMaxLevels];
    uint32_t rem[kMaxLevels];
    unsigned long long acc = 0;
#pragma unroll
    for (int s = 0; s < kWarpWpl; ++s) {
        const int w = lane + 32 * s;
        S[0][s] = w < W ? rows[static_cast<int64_t>(i) * W + w] : 0u;
    }
    if (levels == 0) {
#pragma unroll
        for (int s = 0; s < kWarpWpl; ++s) acc += __popc(S[0][s]);
        return acc;
    }
    // Word w of level t, broadcast from lane w % 32 (slot w / 32).
    auto word = [&](int t, int w) {
        uint32_t mine = 0;
#pragma unroll
        for (int s = 0; s < kWarpWpl; ++s)
            if (s == (w >> 5)) mine = S[t][s];
        return __shfl_sync(kFull, mine, w & 31);
    };
    int t = 0;
    wi[0] = 0;
    rem[0] = word(0, 0);
    while (t >= 0) {
        while (rem[t] == 0 && ++wi[t] < W) rem[t] = word(t, wi[t]);
        if (rem[t] == 0) {
            --t;
            continue;
        }
        const int j = wi[t] * 32 + __ffs(rem[t]) - 1;
        rem[t] &= rem[t] - 1;
        const uint32_t *r = rows + static_cast<int64_t>(j) * W;
        if (t + 1 == levels) {
#pragma unroll
            for (int s = 0; s < kWarpWpl; ++s) {
                const int w = lane + 32 * s;
                if (w < W) acc += __popc(S[t][s] & r[w]);
            }
        } else {
            uint32_t any = 0;
#pragma unroll
            for (int s = 0; s < kWarpWpl; ++s) {
                const int w = lane + 32 * s;
                S[t + 1][s] = w < W ? (S[t][s] & r[w]) : 0u;
                any |= S[t + 1][s];
            }
            if (__any_sync(kFull, any != 0)) {
                ++t;
                wi[t] = 0;
                rem[t] = word(t, 0);
            }
        }
    }
    return acc;
}

// Work item = DAG arc e = (u -> N+(u)[i]), i.e. row i of u's bitmap.
__global__ void __launch_bounds__(kBlock)
    kc_count_kernel(const int64_t *__restrict__ vertex, const uint32_t *__restrict__ edge_from, int64_t e_cnt,
                    const int64_t *__restrict__ off, const uint32_t *__restrict__ bitmap, int k,
                    unsigned long long *counters) {
    const int lane = threadIdx.x & 31;
    const int levels = k - 3;
    unsigned long long acc = 0;
    while (true) {
        unsigned long long c = 0;
        if (lane == 0) c = atomicAdd(&counters[kCursor], 1ull);
        c = __shfl_sync(kFull, c, 0);
        const int64_t base = static_cast<int64_t>(c) * 32;
        if (base >= e_cnt) break;
        const int64_t e = base + lane;
        int W = 0, i = 0;
        int64_t rows_at = 0;
        if (e < e_cnt) {
            const uint32_t u = edge_from[e];
            const int64_t b = vertex[u];
            const int d = static_cast<int>(vertex[u + 1] - b);
            if (d >= k - 1) {
                W = (d + 31) >> 5;
                i = static_cast<int>(e - b);
                rows_at = off[u];
            }
        }
        if (W > 0 && W <= kLaneWords) acc += lane_cliques(bitmap + rows_at, W, i, levels);
        unsigned wide = __ballot_sync(kFull, W > kLaneWords);
        while (wide) {
            const int src = __ffs(wide) - 1;
            wide &= wide - 1;
            const int Ws = __shfl_sync(kFull, W, src);
            const int is = __shfl_sync(kFull, i, src);
            const int64_t rs = __shfl_sync(kFull, rows_at, src);
            acc += warp_cliques(bitmap + rs, Ws, is, levels, lane);
        }
    }
    for (int o = 16; o; o >>= 1) acc += __shfl_xor_sync(kFull, acc, o);
    if (lane == 0 && acc) atomicAdd(&counters[kSum], acc);
}

// Clique-tree pivoting (pivot.cuh): a warp per root vertex, claimed one at a
// time in the order of `roots` (largest out-degree first, so that the
// heaviest searches start early); counters [0] root cursor, [1] stack
// overflow, [2 + k] k-cliques.
__global__ void __launch_bounds__(kBlock)
    kc_pivot_kernel(const int64_t *__restrict__ vertex, int32_t v_cnt, const int32_t *__restrict__ roots,
                    const int64_t *__restrict__ off, const uint32_t *__restrict__ bitmap, int kmax,
                    const uint64_t *__restrict__ binom, pivot::Layout L, uint32_t *scratch,
                    unsigned long long *counters) {
    const int lane = threadIdx.x & 31;
    const int64_t warp = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    uint32_t *mine = scratch + warp * L.words();
    const pivot::WarpLanes wp{lane};
    uint64_t acc[pivot::kMaxK + 1] = {};
    bool ok = true;
    while (true) {
        unsigned long long c = 0;
        if (lane == 0) c = atomicAdd(&counters[0], 1ull);
        c = __shfl_sync(kFull, c, 0);
        if (c >= static_cast<unsigned long long>(v_cnt)) break;
        const int64_t v = roots[c];
        const int d = static_cast<int>(vertex[v + 1] - vertex[v]);
        if (d > L.dmax) {  // the layout is sized by the largest out-degree
            ok = false;
            break;
        }
        const uint32_t *D = d >= 2 ? bitmap + off[v] : nullptr;
        if (!pivot::count_root(wp, D, d, kmax, binom, L, mine, acc)) {
            ok = false;
            break;
        }
    }
    if (lane == 0) {
        if (!ok) atomicExch(&counters[1], 1ull);
        for (int k = 0; k <= kmax; ++k)
            if (acc[k]) atomicAdd(&counters[2 + k], static_cast<unsigned long long>(acc[k]));
    }
}

}  // namespace

int kclique_max_bitmap_degree() { return 32 * 32 * kWarpWpl; }

// Builds (once) the bitmaps of DAG o.  Returns GI_ENOMEM, recording nothing,
// when they would take more than half of the free device memory.
static int ensure_bitmaps(gi_graph *o, cudaStream_t st, float *ms, int *launches) {
    if (o->d_bitmap) return GI_OK;
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, o->device);
    const size_t vb = sizeof(int64_t) * (static_cast<size_t>(o->v_cnt) + 1);
    cudaError_t e;
    int64_t *words = nullptr;
    void *tmp = nullptr;
    size_t tmp_bytes = 0;
    auto bail = [&](cudaError_t err, const char *what) {
        cudaFree(words);
        cudaFree(tmp);
        cudaFree(o->d_bitmap_off);
        o->d_bitmap_off = nullptr;
        return cuda_fail(err, what);
    };
    if ((e = cudaMalloc(&words, vb)) != cudaSuccess) return bail(e, "bitmap sizes");
    if ((e = cudaMalloc(&o->d_bitmap_off, vb)) != cudaSuccess) return bail(e, "bitmap offsets");
    kc_words_kernel<<<sms * 8, 256, 0, st>>>(o->d_vertex, o->v_cnt, words);
    cub::DeviceScan::ExclusiveSum(nullptr, tmp_bytes, words, o->d_bitmap_off, o->v_cnt + 1, st);
    if ((e = cudaMalloc(&tmp, tmp_bytes)) != cudaSuccess) return bail(e, "bitmap scan workspace");
    if ((e = cub::DeviceScan::ExclusiveSum(tmp, tmp_bytes, words, o->d_bitmap_off, o->v_cnt + 1, st)) !=
        cudaSuccess)
        return bail(e, "bitmap scan");
    int64_t total = 0;
    if ((e = cudaMemcpyAsync(&total, o->d_bitmap_off + o->v_cnt, sizeof(total), cudaMemcpyDeviceToHost, st)) !=
            cudaSuccess ||
        (e = cudaStreamSynchronize(st)) != cudaSuccess)
        return bail(e, "bitmap size");
    cudaFree(words);
    cudaFree(tmp);
    words = nullptr;
    tmp = nullptr;
    size_t free_b = 0, total_b = 0;
    cudaMemGetInfo(&free_b, &total_b);
    const size_t bytes = static_cast<size_t>(std::max<int64_t>(total, 1)) * sizeof(uint32_t);
    if (bytes > free_b / 2) {
        cudaFree(o->d_bitmap_off);
        o->d_bitmap_off = nullptr;
        return GI_ENOMEM;
    }
    if ((e = cudaMalloc(&o->d_bitmap, bytes)) != cudaSuccess) return bail(e, "bitmap allocation");
    unsigned long long *ctr = o->d_counters;
    cudaEvent_t t0, t1;
    cudaEventCreate(&t0);
    cudaEventCreate(&t1);
    cudaEventRecord(t0, st);
    int per_sm = 1;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kc_build_kernel, kBlock, 0);
    if ((e = cudaMemsetAsync(ctr, 0, 8 * sizeof(unsigned long long), st)) == cudaSuccess) {
        kc_build_kernel<<<sms * std::max(per_sm, 1), kBlock, 0, st>>>(o->d_vertex, o->d_edge, o->v_cnt,
                                                                      o->d_bitmap_off, o->d_bitmap, ctr);
        e = cudaGetLastError();
    }
    cudaEventRecord(t1, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    float m = 0.f;
    if (e == cudaSuccess) cudaEventElapsedTime(&m, t0, t1);
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    if (e != cudaSuccess) {
        cudaFree(o->d_bitmap);
        o->d_bitmap = nullptr;
        return bail(e, "bitmap build");
    }
    o->bitmap_words = total;
    *ms += m;
    *launches += 3;  // sizes, scan, build
    return GI_OK;
}

// k-cliques of the degree-oriented DAG `o` (out-lists sorted), 3 <= k <= 7,
// when its largest out-degree is at most kclique_max_bitmap_degree().
// Returns GI_ENOMEM without counting when the bitmaps do not fit.
int kclique_bitmap(gi_graph *o, int k, cudaStream_t st, uint64_t *out, gi_stats *stats) {
    float build_ms = 0.f;
    int launches = 0;
    int rc = ensure_bitmaps(o, st, &build_ms, &launches);
    if (rc != GI_OK) return rc;
    int sms = 148, per_sm = 1;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, o->device);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kc_count_kernel, kBlock, 0);
    const int blocks = sms * std::max(per_sm, 1);
    unsigned long long *ctr = o->d_counters;
    cudaEvent_t t0, t1;
    cudaEventCreate(&t0);
    cudaEventCreate(&t1);
    cudaError_t e;
    cudaEventRecord(t0, st);
    if ((e = cudaMemsetAsync(ctr, 0, 8 * sizeof(unsigned long long), st)) == cudaSuccess) {
        kc_count_kernel<<<blocks, kBlock, 0, st>>>(o->d_vertex, o->d_edge_from, o->e_cnt, o->d_bitmap_off,
                                                   o->d_bitmap, k, ctr);
        e = cudaGetLastError();
    }
    cudaEventRecord(t1, st);
    unsigned long long host[8] = {0};
    if (e == cudaSuccess) e = cudaMemcpyAsync(host, ctr, sizeof(host), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    float ms = 0.f;
    if (e == cudaSuccess) cudaEventElapsedTime(&ms, t0, t1);
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    if (e != cudaSuccess) return cuda_fail(e, "k-clique count kernel");
    *out = host[kSum];
    if (stats) {
        stats->kernel_ms = ms + build_ms;
        stats->prep_ms = build_ms;
        stats->raw_sum = host[kSum];
        stats->tasks = static_cast<uint64_t>(o->e_cnt);
        stats->kernel_launches = launches + 1;
        stats->grid_blocks = blocks;
        stats->block_threads = kBlock;
    }
    return GI_OK;
}

// Counts of every clique size 1..kmax (kmax <= 7) of the degree-oriented DAG
// `o` at once by clique-tree pivoting: counts[k] = k-cliques (counts[0] = 0).
// Stack levels start at 64 and grow (up to the largest out-degree + 2) when a
// search is deeper; the workers' scratch is held to about 1 GiB.
int kclique_pivot(gi_graph *o, int kmax, cudaStream_t st, uint64_t *counts, gi_stats *stats) {
    float build_ms = 0.f;
    int launches = 0;
    int rc = ensure_bitmaps(o, st, &build_ms, &launches);
    if (rc != GI_OK) return rc;
    int sms = 148, per_sm = 1;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, o->device);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kc_pivot_kernel, kBlock, 0);
    pivot::Layout L;
    L.dmax = std::max<int64_t>(o->max_degree, 1);
    L.wmax = std::max<int64_t>((L.dmax + 31) / 32, 1);
    const int64_t max_levels = L.dmax + 2;
    L.levels = std::min<int64_t>(64, max_levels);
    // Roots by out-degree, largest first (counting sort on the host; ties in
    // id order), built once and kept on the DAG next to its bitmaps.
    if (!o->d_roots) {
        int32_t *d_roots = nullptr;
        std::vector<int64_t> hv(static_cast<size_t>(o->v_cnt) + 1);
        cudaError_t e = cudaMemcpyAsync(hv.data(), o->d_vertex, hv.size() * sizeof(int64_t), cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return cuda_fail(e, "out-degrees for the root order");
        // Bucket of v: L.dmax - out-degree, clamped into [0, L.dmax].
        auto bucket = [&](int32_t v) {
            const int64_t d = hv[v + 1] - hv[v];
            return static_cast<size_t>(L.dmax - std::min<int64_t>(std::max<int64_t>(d, 0), L.dmax));
        };
        std::vector<int64_t> start(static_cast<size_t>(L.dmax) + 2, 0);
        for (int32_t v = 0; v < o->v_cnt; ++v) ++start[bucket(v) + 1];
        for (size_t i = 1; i < start.size(); ++i) start[i] += start[i - 1];
        std::vector<int32_t> order(static_cast<size_t>(o->v_cnt));
        for (int32_t v = 0; v < o->v_cnt; ++v) order[static_cast<size_t>(start[bucket(v)]++)] = v;
        if ((e = cudaMalloc(&d_roots, order.size() * sizeof(int32_t) + sizeof(int32_t))) != cudaSuccess)
            return cuda_fail(e, "root order");
        if ((e = cudaMemcpyAsync(d_roots, order.data(), order.size() * sizeof(int32_t), cudaMemcpyHostToDevice, st)) !=
                cudaSuccess ||
            (e = cudaStreamSynchronize(st)) != cudaSuccess) {
            cudaFree(d_roots);
            return cuda_fail(e, "root order");
        }
        o->d_roots = d_roots;
    }
    const int32_t *d_roots = o->d_roots;
    float total_ms = 0.f;
    while (true) {
        const size_t per_warp = static_cast<size_t>(L.words()) * sizeof(uint32_t);
        const int64_t fit = std::max<int64_t>(1, (int64_t(1) << 30) / static_cast<int64_t>(per_warp) / kWarps);
        const int blocks = static_cast<int>(std::min<int64_t>(static_cast<int64_t>(sms) * std::max(per_sm, 1), fit));
        uint32_t *scratch = nullptr;
        uint64_t *binom = nullptr;
        unsigned long long *ctr = nullptr;
        cudaError_t e = cudaMalloc(&scratch, per_warp * static_cast<size_t>(blocks) * kWarps);
        const int64_t rows = L.levels + 1;
        std::vector<uint64_t> hb(static_cast<size_t>(rows) * pivot::kBinomCols, 0);
        for (int64_t q = 0; q < rows; ++q)
            for (int j = 0; j < pivot::kBinomCols; ++j)
                hb[q * pivot::kBinomCols + j] =
                    j == 0 ? 1 : (q == 0 ? 0 : hb[(q - 1) * pivot::kBinomCols + j - 1] + hb[(q - 1) * pivot::kBinomCols + j]);
        if (e == cudaSuccess) e = cudaMalloc(&binom, hb.size() * sizeof(uint64_t));
        if (e == cudaSuccess) e = cudaMalloc(&ctr, 16 * sizeof(unsigned long long));
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(binom, hb.data(), hb.size() * sizeof(uint64_t), cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess) e = cudaMemsetAsync(ctr, 0, 16 * sizeof(unsigned long long), st);
        cudaEvent_t t0 = nullptr, t1 = nullptr;
        unsigned long long host[16] = {0};
        float ms = 0.f;
        if (e == cudaSuccess) {
            cudaEventCreate(&t0);
            cudaEventCreate(&t1);
            cudaEventRecord(t0, st);
            kc_pivot_kernel<<<blocks, kBlock, 0, st>>>(o->d_vertex, o->v_cnt, d_roots, o->d_bitmap_off,
                                                       o->d_bitmap, kmax, binom, L, scratch, ctr);
            e = cudaGetLastError();
            cudaEventRecord(t1, st);
            if (e == cudaSuccess) e = cudaMemcpyAsync(host, ctr, sizeof(host), cudaMemcpyDeviceToHost, st);
            if (e == cudaSuccess) e = cudaStreamSynchronize(st);
            if (e == cudaSuccess) cudaEventElapsedTime(&ms, t0, t1);
            cudaEventDestroy(t0);
            cudaEventDestroy(t1);
        }
        cudaFree(scratch);
        cudaFree(binom);
        cudaFree(ctr);
        if (e != cudaSuccess) return cuda_fail(e, "clique-tree pivoting kernel");
        ++launches;
        total_ms += ms;
        if (host[1] == 0) {
            counts[0] = 0;
            for (int k = 1; k <= kmax; ++k) counts[k] = host[2 + k];
            if (stats) {
                stats->kernel_ms = total_ms + build_ms;
                stats->prep_ms = build_ms;
                stats->raw_sum = counts[kmax];
                stats->tasks = static_cast<uint64_t>(o->v_cnt);
                stats->kernel_launches = launches;
                stats->grid_blocks = blocks;
                stats->block_threads = kBlock;
            }
            return GI_OK;
        }
        if (L.levels >= max_levels) {
            return fail(GI_EOVERFLOW, "clique-tree pivoting: search deeper than its stack");
        }
        L.levels = std::min<int64_t>(L.levels * 4, max_levels);
    }
}

}  // namespace gi

