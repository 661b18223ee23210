// Graph handles: CSR upload with on-device validation, .g file I/O.
//
// The .g layout follows the reference loader (reference
// src/dataloader.cpp:21-124); the device-side CSR replaces the copies made by
// PatternMatchingDeviceContext::init (reference
// gpu/function/pattern_matching.cuh:18-81), including the edge_from array
// (there built on the host at :27-31, here by a kernel).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <functional>
#include <cstring>
#include <new>
#include <vector>

#include "internal.hpp"

namespace gi {

namespace {

struct GHeader {
    int32_t v_cnt;
    int32_t pad;
    int64_t e_cnt;
    uint32_t max_intersection_size;
    uint32_t checksum;
    int64_t tri_cnt;
};
static_assert(sizeof(GHeader) == 32, "the .g header is 32 bytes");

uint32_t header_word_sum(const GHeader &h) {
    uint32_t w[8];
    std::memcpy(w, &h, sizeof(w));
    uint32_t s = 0;
    for (uint32_t x : w) s += x;
    return s;
}

// One warp per vertex: writes edge_from for the vertex's adjacency range and
// flags out-of-range ids, self-loops and unsorted or duplicate neighbours.
__global__ void build_edge_from_kernel(const int64_t *__restrict__ vertex, const int32_t *__restrict__ edge,
                                       uint32_t *__restrict__ edge_from, int32_t v_cnt, int *bad) {
    const int lane = threadIdx.x & 31;
    const int64_t warp = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = (static_cast<int64_t>(gridDim.x) * blockDim.x) >> 5;
    for (int64_t v = warp; v < v_cnt; v += nwarps) {
        const int64_t l = vertex[v], r = vertex[v + 1];
        bool err = r < l;
        for (int64_t j = l + lane; j < r; j += 32) {
            const int32_t x = edge[j];
            edge_from[j] = static_cast<uint32_t>(v);
            if (x < 0 || x >= v_cnt || x == v) err = true;
            if (j + 1 < r && edge[j + 1] <= x) err = true;
        }
        if (__any_sync(0xffffffffu, err) && lane == 0) atomicExch(bad, 1);
    }
}

// Block r: the bitmap row of hub ids[r] (bits zeroed before) and its entry
// in the row index.
__global__ void build_hub_bits_kernel(const int64_t *__restrict__ vertex, const int32_t *__restrict__ edge,
                                      const int32_t *__restrict__ ids, int64_t words, uint32_t *__restrict__ bits,
                                      int32_t *__restrict__ row) {
    const int r = blockIdx.x;
    const int32_t h = ids[r];
    if (threadIdx.x == 0) row[h] = r;
    uint32_t *b = bits + static_cast<int64_t>(r) * words;
    for (int64_t j = vertex[h] + threadIdx.x; j < vertex[h + 1]; j += blockDim.x) {
        const uint32_t x = static_cast<uint32_t>(edge[j]);
        atomicOr(&b[x >> 5], 1u << (x & 31));
    }
}

}  // namespace

// Hub bitmaps: the counting DFS tests membership in a hub's adjacency list
// with one load.  Hubs are all vertices of degree >= T, T the smallest value
// >= kHubMinDegree for which their bitmaps fit the budget: kHubBitmapBytes,
// at most a sixteenth of the device's free memory.  Measured on the B200 (R-MAT
// scale 22, the six-pattern workload): 64 MiB 3.69 s per step, 1 GiB 2.93 s,
// 4 GiB 2.39 s.
int cuda_fail(cudaError_t e, const char *what);

constexpr size_t kHubBitmapBytes = size_t(4) << 30;
constexpr int32_t kHubMinDegree = 256;

// The bitmap budget in bytes and the smallest hub degree: the defaults
// above, or GI_HUB_BITMAP_MB / GI_HUB_MIN_DEGREE from the environment
// (tuning; 0 MB turns the bitmaps off).
static void hub_limits(size_t &bytes, int32_t &min_degree) {
    bytes = kHubBitmapBytes;
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) == cudaSuccess) bytes = std::min(bytes, free_b / 16);
    min_degree = kHubMinDegree;
    if (const char *s = std::getenv("GI_HUB_BITMAP_MB")) bytes = static_cast<size_t>(std::strtoull(s, nullptr, 10)) << 20;
    if (const char *s = std::getenv("GI_HUB_MIN_DEGREE")) min_degree = std::max(1, std::atoi(s));
}

static int build_hubs(gi_graph *g, const int64_t *vertex, cudaStream_t st) {
    size_t budget = 0;
    int32_t min_degree = 0;
    hub_limits(budget, min_degree);
    const int64_t words = (static_cast<int64_t>(g->v_cnt) + 31) / 32;
    const int64_t max_hubs = static_cast<int64_t>(budget / (static_cast<size_t>(words) * sizeof(uint32_t)));
    if (max_hubs < 1 || g->max_degree < min_degree) return GI_OK;
    std::vector<int32_t> big;
    for (int32_t v = 0; v < g->v_cnt; ++v) {
        const int64_t d = vertex[v + 1] - vertex[v];
        if (d >= min_degree) big.push_back(static_cast<int32_t>(d));
    }
    int32_t T = min_degree;
    if (static_cast<int64_t>(big.size()) > max_hubs) {
        std::nth_element(big.begin(), big.begin() + max_hubs, big.end(), std::greater<int32_t>());
        T = big[static_cast<size_t>(max_hubs)] + 1;  // the (max_hubs+1)-th largest degree is left out
    }
    std::vector<int32_t> ids;
    for (int32_t v = 0; v < g->v_cnt; ++v)
        if (vertex[v + 1] - vertex[v] >= T) ids.push_back(v);
    if (ids.empty()) return GI_OK;
    int32_t *d_ids = nullptr;
    cudaError_t e;
    const size_t bits_bytes = ids.size() * static_cast<size_t>(words) * sizeof(uint32_t);
    if ((e = cudaMalloc(&g->d_hub_bits, bits_bytes)) != cudaSuccess ||
        (e = cudaMalloc(&g->d_hub_row, sizeof(int32_t) * static_cast<size_t>(g->v_cnt))) != cudaSuccess ||
        (e = cudaMalloc(&d_ids, sizeof(int32_t) * ids.size())) != cudaSuccess) {
        cudaFree(d_ids);
        return cuda_fail(e, "hub bitmap allocation");
    }
    if ((e = cudaMemcpyAsync(d_ids, ids.data(), sizeof(int32_t) * ids.size(), cudaMemcpyHostToDevice, st)) ==
            cudaSuccess &&
        (e = cudaMemsetAsync(g->d_hub_bits, 0, bits_bytes, st)) == cudaSuccess &&
        (e = cudaMemsetAsync(g->d_hub_row, 0xff, sizeof(int32_t) * static_cast<size_t>(g->v_cnt), st)) == cudaSuccess) {
        build_hub_bits_kernel<<<static_cast<unsigned>(ids.size()), 256, 0, st>>>(g->d_vertex, g->d_edge, d_ids, words,
                                                                               g->d_hub_bits, g->d_hub_row);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);  // d_ids is freed next
    cudaFree(d_ids);
    if (e != cudaSuccess) return cuda_fail(e, "hub bitmap build");
    g->n_hubs = static_cast<int32_t>(ids.size());
    g->hub_min_degree = T;
    g->hub_words = words;
    return GI_OK;
}

// Per-vertex hash sets of adjacency lists: a membership test against N(v) in
// one or two loads instead of a binary search of log2 d(v) dependent loads.
// Every vertex of degree >= T gets a table of next_pow2(2 d(v)) slots (load
// at most 1/2, linear probing); T is the smallest value >= kHashMinDegree
// for which all tables fit the budget (GI_HASH_MB, default kHashBytes;
// GI_HASH_MIN_DEGREE overrides kHashMinDegree).  Off by default: with the
// default hub bitmaps they did not shorten the six-pattern workload at R-MAT
// scale 22 on the B200 (2.385 s per step with 4 GiB of them, 2.386 s without)
// and cost 100 ms of upload; they pay where the bitmap budget is small
// (64 MiB of bitmaps: 3.57 s with them, 3.69 s without).
constexpr size_t kHashBytes = 0;
constexpr int32_t kHashMinDegree = 32;

int64_t hash_capacity(int64_t deg) {
    int64_t c = 2;
    while (c < 2 * deg) c <<= 1;
    return c;
}

namespace {
// A warp per table vertex: inserts its neighbours (duplicate-free) by
// linear probing from the multiplicative hash slot.
__global__ void build_hash_kernel(const int64_t *__restrict__ vertex, const int32_t *__restrict__ edge,
                                  const int32_t *__restrict__ ids, int32_t n_ids, const int64_t *__restrict__ off,
                                  uint32_t *__restrict__ slots) {
    const int lane = threadIdx.x & 31;
    const int64_t warp = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = (static_cast<int64_t>(gridDim.x) * blockDim.x) >> 5;
    for (int64_t i = warp; i < n_ids; i += nwarps) {
        const int32_t v = ids[i];
        uint32_t *t = slots + off[v];
        const uint32_t cap = static_cast<uint32_t>(off[v + 1] - off[v]);
        const int bits = __ffs(cap) - 1;
        for (int64_t j = vertex[v] + lane; j < vertex[v + 1]; j += 32) {
            const uint32_t x = static_cast<uint32_t>(edge[j]);
            uint32_t s = (x * 2654435769u) >> (32 - bits);
            for (uint32_t k = 0; k < cap; ++k) {
                if (atomicCAS(&t[s], 0xffffffffu, x) == 0xffffffffu) break;
                s = (s + 1) & (cap - 1);
            }
        }
    }
}
}  // namespace

static int build_hash(gi_graph *g, const int64_t *vertex, cudaStream_t st) {
    size_t budget = kHashBytes;
    int32_t min_degree = kHashMinDegree;
    if (const char *s = std::getenv("GI_HASH_MB")) budget = static_cast<size_t>(std::strtoull(s, nullptr, 10)) << 20;
    if (const char *s = std::getenv("GI_HASH_MIN_DEGREE")) min_degree = std::max(1, std::atoi(s));
    if (budget == 0 || g->max_degree < min_degree) return GI_OK;
    // The smallest threshold whose tables fit the budget.
    std::vector<std::pair<int32_t, int64_t>> big;  // (degree, table slots), largest degree first
    for (int32_t v = 0; v < g->v_cnt; ++v) {
        const int64_t d = vertex[v + 1] - vertex[v];
        if (d >= min_degree) big.emplace_back(static_cast<int32_t>(d), hash_capacity(d));
    }
    std::sort(big.begin(), big.end(), [](const auto &a, const auto &b) { return a.first > b.first; });
    int64_t total = 0;
    int32_t T = min_degree;
    for (size_t i = 0; i < big.size(); ++i) {
        if (static_cast<size_t>(total + big[i].second) * sizeof(uint32_t) > budget) {
            T = big[i].first + 1;  // this degree and all below are left out
            break;
        }
        total += big[i].second;
    }
    if (T > g->max_degree) return GI_OK;
    std::vector<int64_t> off(static_cast<size_t>(g->v_cnt) + 1, 0);
    std::vector<int32_t> ids;
    for (int32_t v = 0; v < g->v_cnt; ++v) {
        const int64_t d = vertex[v + 1] - vertex[v];
        const bool has = d >= T;
        off[v + 1] = off[v] + (has ? hash_capacity(d) : 0);
        if (has) ids.push_back(v);
    }
    const int64_t slots = off[g->v_cnt];
    int32_t *d_ids = nullptr;
    cudaError_t e;
    if ((e = cudaMalloc(&g->d_hash, static_cast<size_t>(slots) * sizeof(uint32_t))) != cudaSuccess ||
        (e = cudaMalloc(&g->d_hash_off, off.size() * sizeof(int64_t))) != cudaSuccess ||
        (e = cudaMalloc(&d_ids, ids.size() * sizeof(int32_t))) != cudaSuccess) {
        cudaFree(d_ids);
        return cuda_fail(e, "hash table allocation");
    }
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, g->device);
    if ((e = cudaMemcpyAsync(g->d_hash_off, off.data(), off.size() * sizeof(int64_t), cudaMemcpyHostToDevice, st)) ==
            cudaSuccess &&
        (e = cudaMemcpyAsync(d_ids, ids.data(), ids.size() * sizeof(int32_t), cudaMemcpyHostToDevice, st)) ==
            cudaSuccess &&
        (e = cudaMemsetAsync(g->d_hash, 0xff, static_cast<size_t>(slots) * sizeof(uint32_t), st)) == cudaSuccess) {
        build_hash_kernel<<<sms * 8, 256, 0, st>>>(g->d_vertex, g->d_edge, d_ids, static_cast<int32_t>(ids.size()),
                                                   g->d_hash_off, g->d_hash);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);  // d_ids is freed next
    cudaFree(d_ids);
    if (e != cudaSuccess) return cuda_fail(e, "hash table build");
    g->hash_min_degree = T;
    g->hash_slots = slots;
    return GI_OK;
}

void cost_model_graph_features(const int64_t *vertex, int32_t v_cnt, int64_t tri_cnt, float *out);

int cuda_fail(cudaError_t e, const char *what) {
    char buf[256];
    std::snprintf(buf, sizeof(buf), "%s: %s", what, cudaGetErrorString(e));
    return fail(e == cudaErrorMemoryAllocation ? GI_ENOMEM : GI_ECUDA, buf);
}

DeviceGuard::DeviceGuard(int device) : device_(device) {
    cudaGetDevice(&prev_);
    if (prev_ != device_) cudaSetDevice(device_);
}

DeviceGuard::~DeviceGuard() {
    if (prev_ >= 0 && prev_ != device_) cudaSetDevice(prev_);
}

ScopedEvents::ScopedEvents(int n) : n_(n < 4 ? n : 4) {
    for (int i = 0; i < n_; ++i) {
        cudaEvent_t e = nullptr;
        if (cudaEventCreate(&e) != cudaSuccess) {
            cudaGetLastError();
            e = nullptr;
        }
        ev_[i] = e;
    }
}

ScopedEvents::~ScopedEvents() {
    for (int i = 0; i < n_; ++i)
        if (ev_[i]) cudaEventDestroy(static_cast<cudaEvent_t>(ev_[i]));
}

void graph_free(gi_graph *g) {
    if (!g) return;
    for (auto *o : g->oriented) graph_free(o);
    int prev = 0;
    cudaGetDevice(&prev);
    cudaSetDevice(g->device);
    cudaFree(g->d_vertex);
    cudaFree(g->d_edge);
    cudaFree(g->d_edge_from);
    cudaFree(g->d_scratch);
    cudaFree(g->d_counters);
    cudaFree(g->d_offsets);
    cudaFree(g->d_scan_tmp);
    cudaFree(g->d_handoff);
    cudaFree(g->d_bitmap);
    cudaFree(g->d_bitmap_off);
    cudaFree(g->d_roots);
    cudaFree(g->d_hub_bits);
    cudaFree(g->d_hub_row);
    cudaFree(g->d_hash);
    cudaFree(g->d_hash_off);
    cudaFree(g->d_tri_arc);
    cudaSetDevice(prev);
    delete g;
}

// Degree statistics on the host offsets: max degree and the second-largest
// degree (the reference's max_intersection_size).
static void degree_stats(const int64_t *vertex, int32_t v_cnt, int32_t &mx, int32_t &second) {
    int64_t a = 0, b = 0;
    for (int32_t v = 0; v < v_cnt; ++v) {
        const int64_t d = vertex[v + 1] - vertex[v];
        if (d > a) {
            b = a;
            a = d;
        } else if (d > b) {
            b = d;
        }
    }
    mx = static_cast<int32_t>(a);
    second = static_cast<int32_t>(b);
}

int graph_create_impl(const int64_t *vertex, const int32_t *edge, int32_t v_cnt, int64_t e_cnt, int64_t tri_cnt,
                      cudaStream_t st, gi_graph **out) {
    if (!out) return fail(GI_EINVAL, "out is NULL");
    *out = nullptr;
    if (v_cnt < 2 || e_cnt < 0 || !vertex || (e_cnt > 0 && !edge))
        return fail(GI_EINVAL, "graph needs v_cnt >= 2, e_cnt >= 0 and both arrays");
    if (e_cnt >= (int64_t(1) << 40)) return fail(GI_EOVERFLOW, "e_cnt too large");
    if (vertex[0] != 0 || vertex[v_cnt] != e_cnt) return fail(GI_EINVAL, "vertex[0] must be 0 and vertex[v_cnt] e_cnt");
    // Offsets must be non-decreasing so that every adjacency range the
    // device reads lies inside edge[0, e_cnt).
    for (int32_t v = 0; v < v_cnt; ++v)
        if (vertex[v + 1] < vertex[v]) return fail(GI_EINVAL, "vertex offsets must be non-decreasing");
    auto *g = new (std::nothrow) gi_graph;
    if (!g) return fail(GI_ENOMEM, "out of host memory");
    cudaGetDevice(&g->device);
    g->v_cnt = v_cnt;
    g->e_cnt = e_cnt;
    g->tri_cnt = tri_cnt;
    degree_stats(vertex, v_cnt, g->max_degree, g->max_isect);
    cost_model_graph_features(vertex, v_cnt, tri_cnt, g->graph_features);
    cudaError_t e;
    const size_t vb = sizeof(int64_t) * (static_cast<size_t>(v_cnt) + 1);
    const size_t eb = sizeof(int32_t) * static_cast<size_t>(e_cnt > 0 ? e_cnt : 1);
    int *d_bad = nullptr;
    if ((e = cudaMalloc(&g->d_vertex, vb)) != cudaSuccess ||
        (e = cudaMalloc(&g->d_edge, eb)) != cudaSuccess ||
        (e = cudaMalloc(&g->d_edge_from, eb)) != cudaSuccess ||
        (e = cudaMalloc(&g->d_counters, 16 * sizeof(unsigned long long))) != cudaSuccess) {
        graph_free(g);
        return cuda_fail(e, "graph allocation");
    }
    d_bad = reinterpret_cast<int *>(g->d_counters + 15);
    if ((e = cudaMemcpyAsync(g->d_vertex, vertex, vb, cudaMemcpyHostToDevice, st)) != cudaSuccess ||
        (e_cnt > 0 && (e = cudaMemcpyAsync(g->d_edge, edge, sizeof(int32_t) * e_cnt, cudaMemcpyHostToDevice, st)) != cudaSuccess) ||
        (e = cudaMemsetAsync(g->d_counters, 0, 16 * sizeof(unsigned long long), st)) != cudaSuccess) {
        graph_free(g);
        return cuda_fail(e, "graph upload");
    }
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, g->device);
    build_edge_from_kernel<<<sms * 8, 256, 0, st>>>(g->d_vertex, g->d_edge, g->d_edge_from, v_cnt, d_bad);
    int bad = 0;
    if ((e = cudaGetLastError()) != cudaSuccess ||
        (e = cudaMemcpyAsync(&bad, d_bad, sizeof(int), cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
        (e = cudaStreamSynchronize(st)) != cudaSuccess) {
        graph_free(g);
        return cuda_fail(e, "graph validation");
    }
    if (bad) {
        graph_free(g);
        return fail(GI_EINVAL, "adjacency lists must be sorted, duplicate-free, in range and without self-loops");
    }
    int hub_status = build_hubs(g, vertex, st);
    if (hub_status == GI_OK) hub_status = build_hash(g, vertex, st);
    if (hub_status != GI_OK) {
        graph_free(g);
        return hub_status;
    }
    *out = g;
    return GI_OK;
}

}  // namespace gi

using namespace gi;

extern "C" {

int gi_graph_create(const int64_t *vertex, const int32_t *edge, int32_t v_cnt, int64_t e_cnt, int64_t tri_cnt,
                    gi_stream stream, gi_graph **out) {
    return graph_create_impl(vertex, edge, v_cnt, e_cnt, tri_cnt, static_cast<cudaStream_t>(stream), out);
}

int gi_graph_destroy(gi_graph *g) {
    graph_free(g);
    return GI_OK;
}

int gi_graph_get_info(const gi_graph *g, gi_graph_info *o) {
    if (!g || !o) return fail(GI_EINVAL, "NULL argument");
    o->v_cnt = g->v_cnt;
    o->e_cnt = g->e_cnt;
    o->tri_cnt = g->tri_cnt;
    o->max_degree = g->max_degree;
    o->max_intersection_size = g->max_isect;
    o->n_hubs = g->n_hubs;
    o->hub_min_degree = g->hub_min_degree;
    o->hash_min_degree = g->hash_min_degree;
    o->hash_slots = g->hash_slots;
    return GI_OK;
}

int gi_g_write(const char *path, const int64_t *vertex, const int32_t *edge, int32_t v_cnt, int64_t e_cnt,
               uint32_t max_isect, int64_t tri_cnt) {
    if (!path || !vertex || (e_cnt > 0 && !edge) || v_cnt < 1 || e_cnt < 0) return fail(GI_EINVAL, "bad arguments");
    GHeader h{};
    h.v_cnt = v_cnt;
    h.e_cnt = e_cnt;
    h.max_intersection_size = max_isect;
    h.tri_cnt = tri_cnt;
    h.checksum = 0;
    h.checksum = 0u - header_word_sum(h);
    FILE *f = std::fopen(path, "wb");
    if (!f) return fail(GI_EIO, std::string("cannot create ") + path);
    bool ok = std::fwrite(&h, sizeof(h), 1, f) == 1 &&
              std::fwrite(vertex, sizeof(int64_t), static_cast<size_t>(v_cnt) + 1, f) == static_cast<size_t>(v_cnt) + 1 &&
              (e_cnt == 0 || std::fwrite(edge, sizeof(int32_t), static_cast<size_t>(e_cnt), f) == static_cast<size_t>(e_cnt));
    ok = (std::fclose(f) == 0) && ok;
    return ok ? GI_OK : fail(GI_EIO, std::string("short write to ") + path);
}

int gi_g_read_header(const char *path, int32_t *v_cnt, int64_t *e_cnt, uint32_t *max_isect, int64_t *tri_cnt) {
    if (!path) return fail(GI_EINVAL, "path is NULL");
    FILE *f = std::fopen(path, "rb");
    if (!f) return fail(GI_EIO, std::string("cannot open ") + path);
    GHeader h{};
    const bool ok = std::fread(&h, sizeof(h), 1, f) == 1;
    std::fclose(f);
    if (!ok) return fail(GI_EIO, "bad header");
    if (header_word_sum(h) != 0) return fail(GI_EIO, "checksum != 0");
    if (h.v_cnt < 1 || h.e_cnt < 0) return fail(GI_EIO, "header sizes out of range");
    if (v_cnt) *v_cnt = h.v_cnt;
    if (e_cnt) *e_cnt = h.e_cnt;
    if (max_isect) *max_isect = h.max_intersection_size;
    if (tri_cnt) *tri_cnt = h.tri_cnt;
    return GI_OK;
}

int gi_g_read(const char *path, int64_t *vertex, int32_t *edge, int32_t v_cap, int64_t e_cap) {
    int32_t v = 0;
    int64_t e = 0;
    int st = gi_g_read_header(path, &v, &e, nullptr, nullptr);
    if (st != GI_OK) return st;
    if (!vertex || (e > 0 && !edge) || v_cap < v || e_cap < e) return fail(GI_EINVAL, "buffers too small");
    FILE *f = std::fopen(path, "rb");
    if (!f) return fail(GI_EIO, std::string("cannot open ") + path);
    std::fseek(f, sizeof(GHeader), SEEK_SET);
    const bool ok = std::fread(vertex, sizeof(int64_t), static_cast<size_t>(v) + 1, f) == static_cast<size_t>(v) + 1 &&
                    (e == 0 || std::fread(edge, sizeof(int32_t), static_cast<size_t>(e), f) == static_cast<size_t>(e));
    std::fclose(f);
    return ok ? GI_OK : fail(GI_EIO, "failed to load vertexes or edges");
}

int gi_graph_load_g(const char *path, gi_graph **out) {
    if (!out) return fail(GI_EINVAL, "out is NULL");
    *out = nullptr;
    int32_t v = 0;
    int64_t e = 0, tri = 0;
    int st = gi_g_read_header(path, &v, &e, nullptr, &tri);
    if (st != GI_OK) return st;
    std::vector<int64_t> vertex;
    std::vector<int32_t> edge;
    try {
        vertex.resize(static_cast<size_t>(v) + 1);
        edge.resize(static_cast<size_t>(e > 0 ? e : 1));
    } catch (const std::bad_alloc &) {
        return fail(GI_ENOMEM, "out of host memory");
    }
    st = gi_g_read(path, vertex.data(), edge.data(), v, e);
    if (st != GI_OK) return st;
    return graph_create_impl(vertex.data(), edge.data(), v, e, tri, nullptr, out);
}

}  // extern "C"
