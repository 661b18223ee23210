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
// >= kHubMinDegree for which their bitmaps fit kHubBitmapBytes.
int cuda_fail(cudaError_t e, const char *what);

constexpr size_t kHubBitmapBytes = size_t(64) << 20;
constexpr int32_t kHubMinDegree = 256;

// The bitmap budget in bytes and the smallest hub degree: the defaults
// above, or GI_HUB_BITMAP_MB / GI_HUB_MIN_DEGREE from the environment
// (tuning; 0 MB turns the bitmaps off).
static void hub_limits(size_t &bytes, int32_t &min_degree) {
    bytes = kHubBitmapBytes;
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
    const int hub_status = build_hubs(g, vertex, st);
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
