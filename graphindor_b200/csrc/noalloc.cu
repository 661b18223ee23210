// gi_count_noalloc: the pattern count without any allocation.
//
// Some callers cannot allocate device memory at the point where they want a
// count: an application whose framework owns the GPU's memory through its
// own pool, a serving loop that must not pay cudaMalloc's latency or its
// implicit device synchronisation, or a plug-in host whose rules forbid
// allocations inside a request.  They hand over the CSR they already hold
// and a small result buffer; every byte of working memory this entry point
// needs comes from one fixed device array declared below, so it calls no
// cudaMalloc, no cudaFree and no allocating library routine.
//
// The counting DFS is the same device code as gi_count (dfs_device.cuh),
// run with one work item per directed edge; the source vertex of an edge is
// found by binary search over the offsets, so no edge_from array is needed.
#include <cuda_runtime.h>

#include <cstring>
#include <mutex>

#include "dfs_device.cuh"
#include "internal.hpp"

namespace gi {

int cuda_fail(cudaError_t e, const char *what);

namespace {

constexpr size_t kScratchBytes = GI_NOALLOC_SCRATCH_BYTES;
constexpr size_t kHeaderBytes = 256;  // counters and graph statistics, then the warps' slots

// The working memory of gi_count_noalloc on every device that loads this
// code.  Every call shares it and it keeps the last call's contents.
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

struct Header {
    unsigned long long counters[8];  // kSum, kCursor, ... as in count.cu
    int32_t bad;                     // malformed CSR seen
    int32_t max_degree;
    int32_t second_degree;           // largest degree below max_degree
    int32_t max_degree_vertices;     // vertices whose degree is max_degree
};
static_assert(sizeof(Header) <= kHeaderBytes, "header must fit its reserved bytes");

// Device address of g_noalloc_scratch per device, taken once per device
// with that device current (host code must not use the symbol itself).
constexpr int kMaxDevices = 64;
unsigned char *g_scratch_ptr[kMaxDevices] = {nullptr};
std::mutex g_setup_mu;

int scratch_address(int device, unsigned char **out) {
    if (device < 0 || device >= kMaxDevices) return fail(GI_ENOTSUP, "device index out of range");
    std::lock_guard<std::mutex> lock(g_setup_mu);
    if (!g_scratch_ptr[device]) {
        void *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return cuda_fail(e, "cudaGetSymbolAddress of the no-alloc scratch");
        g_scratch_ptr[device] = static_cast<unsigned char *>(p);
    }
    *out = g_scratch_ptr[device];
    return GI_OK;
}

// Warp per vertex: offsets in range and non-decreasing, adjacency sorted,
// duplicate-free, in range, without self-loops; the largest degree.
__global__ void noalloc_check_kernel(const int64_t *__restrict__ vertex, const int32_t *__restrict__ edge,
                                     int32_t v_cnt, int64_t e_cnt, Header *h) {
    const int lane = threadIdx.x & 31;
    const int64_t warp = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = (static_cast<int64_t>(gridDim.x) * blockDim.x) >> 5;
    for (int64_t v = warp; v < v_cnt; v += nwarps) {
        const int64_t l = vertex[v], r = vertex[v + 1];
        bool err = (v == 0 && l != 0) || (v == v_cnt - 1 && r != e_cnt) || l < 0 || r < l || r > e_cnt;
        if (!__any_sync(0xffffffffu, err)) {
            for (int64_t j = l + lane; j < r; j += 32) {
                const int32_t x = edge[j];
                if (x < 0 || x >= v_cnt || x == v) err = true;
                if (j + 1 < r && edge[j + 1] <= x) err = true;
            }
        }
        if (__any_sync(0xffffffffu, err)) {
            if (lane == 0) atomicExch(&h->bad, 1);
        } else if (lane == 0) {
            atomicMax(&h->max_degree, static_cast<int32_t>(r - l));
        }
    }
}

// Thread per vertex: the second-largest degree (how many vertices reach the
// largest, and the largest degree below it).  Runs after a clean check.
__global__ void noalloc_second_kernel(const int64_t *__restrict__ vertex, int32_t v_cnt, Header *h) {
    const int32_t mx = h->max_degree;
    const int64_t stride = static_cast<int64_t>(gridDim.x) * blockDim.x;
    for (int64_t v = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; v < v_cnt; v += stride) {
        const int32_t d = static_cast<int32_t>(vertex[v + 1] - vertex[v]);
        if (d == mx)
            atomicAdd(&h->max_degree_vertices, 1);
        else
            atomicMax(&h->second_degree, d);
    }
}

// The counting DFS with one work item per directed edge (no depth-2
// split), warp slots carved from the static scratch.
__global__ void __launch_bounds__(kBlockThreads)
    noalloc_count_kernel(const __grid_constant__ DevPlan P, const int64_t *__restrict__ vertex,
                         const uint32_t *__restrict__ edge, int32_t v_cnt, int64_t e_cnt, uint32_t *slots,
                         int64_t slot_stride, Header *h) {
    __shared__ WarpState states[kWarpsPerBlock];
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    const int64_t gwarp = static_cast<int64_t>(blockIdx.x) * kWarpsPerBlock + wib;
    WarpState &w = states[wib];
    Ctx<false> c{P, vertex, edge, slots + gwarp * P.n_slots * slot_stride, slot_stride, w, lane, 0ull};
    unsigned long long sum = 0;
    while (true) {
        unsigned long long j = 0;
        if (lane == 0) j = atomicAdd(&h->counters[kCursor], 1ull);
        j = __shfl_sync(kFull, j, 0);
        const int64_t base = static_cast<int64_t>(j) * kTaskChunk;
        if (base >= e_cnt) break;
        const int64_t t = base + lane;
        bool valid = t < e_cnt;
        uint32_t v0 = 0, v1 = 0;
        if (valid) {
            // Source of edge t: the last vertex whose offset is <= t.
            int64_t a = 0, len = static_cast<int64_t>(v_cnt) + 1;
            while (len > 0) {
                const int64_t half = len >> 1;
                if (vertex[a + half] <= t) {
                    a += half + 1;
                    len -= half + 1;
                } else {
                    len = half;
                }
            }
            v0 = static_cast<uint32_t>(a - 1);
            v1 = edge[t];
            if (P.first_restricted && v0 <= v1) valid = false;
        }
        unsigned todo = __ballot_sync(kFull, valid);
        while (todo) {
            const int src = __ffs(todo) - 1;
            todo &= todo - 1;
            const uint32_t a = __shfl_sync(kFull, v0, src);
            const uint32_t b = __shfl_sync(kFull, v1, src);
            if (lane == 0) {
                w.emb[0] = a;
                w.emb[1] = b;
            }
            __syncwarp();
            c.build_chain(0, a, false);
            if (!c.build_chain(1, b)) continue;
            sum += c.dfs(0, 0x7fffffff);
        }
    }
    if (lane == 0) atomicAdd(&h->counters[kSum], sum);
}

__global__ void noalloc_finish_kernel(const Header *h, unsigned long long divisor, uint64_t *result) {
    const unsigned long long raw = h->counters[kSum];
    result[0] = divisor ? raw / divisor : raw;
    result[1] = raw;
}

}  // namespace

}  // namespace gi

using namespace gi;

extern "C" int gi_count_noalloc(const int64_t *d_vertex, const int32_t *d_edge, int32_t v_cnt, int64_t e_cnt,
                                const gi_plan *p, gi_stream stream, uint64_t *d_result) {
    if (!d_vertex || (e_cnt > 0 && !d_edge) || !p || !d_result) return fail(GI_EINVAL, "NULL argument");
    if (v_cnt < 2 || e_cnt < 0) return fail(GI_EINVAL, "graph needs v_cnt >= 2 and e_cnt >= 0");
    if (e_cnt >= (int64_t(1) << 40)) return fail(GI_EOVERFLOW, "e_cnt too large");
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    int device = 0;
    cudaError_t e = cudaGetDevice(&device);
    if (e != cudaSuccess) return cuda_fail(e, "cudaGetDevice");
    unsigned char *base = nullptr;
    int rc = scratch_address(device, &base);
    if (rc != GI_OK) return rc;
    Header *h = reinterpret_cast<Header *>(base);
    uint32_t *slots = reinterpret_cast<uint32_t *>(base + kHeaderBytes);
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);

    // The header starts at zero on every call (the array keeps the last
    // call's contents).
    if ((e = cudaMemsetAsync(h, 0, kHeaderBytes, st)) != cudaSuccess) return cuda_fail(e, "header reset");
    noalloc_check_kernel<<<sms * 8, 256, 0, st>>>(d_vertex, d_edge, v_cnt, e_cnt, h);
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "graph check");
    Header host{};
    if ((e = cudaMemcpyAsync(&host, h, sizeof(Header), cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
        (e = cudaStreamSynchronize(st)) != cudaSuccess)
        return cuda_fail(e, "graph check");
    if (host.bad)
        return fail(GI_EINVAL, "adjacency lists must be sorted, duplicate-free, in range and without self-loops, "
                               "with non-decreasing offsets from 0 to e_cnt");
    noalloc_second_kernel<<<sms * 8, 256, 0, st>>>(d_vertex, v_cnt, h);
    if ((e = cudaGetLastError()) != cudaSuccess ||
        (e = cudaMemcpyAsync(&host, h, sizeof(Header), cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
        (e = cudaStreamSynchronize(st)) != cudaSuccess)
        return cuda_fail(e, "degree statistics");
    const int64_t stride = std::max<int64_t>(host.max_degree_vertices >= 2 ? host.max_degree : host.second_degree, 1);

    // As many warps as the scratch holds, at most the grid gi_count uses.
    const DevPlan P = plan_for_graph(p->dev, host.max_degree);
    const int64_t per_warp = static_cast<int64_t>(P.n_slots) * stride * static_cast<int64_t>(sizeof(uint32_t));
    const int64_t room = static_cast<int64_t>(kScratchBytes - kHeaderBytes);
    int blocks_per_sm = 1;
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks_per_sm, noalloc_count_kernel, kBlockThreads, 0)) !=
        cudaSuccess)
        return cuda_fail(e, "occupancy query");
    int64_t blocks = static_cast<int64_t>(sms) * std::max(1, blocks_per_sm);
    if (per_warp > 0) blocks = std::min<int64_t>(blocks, room / (per_warp * kWarpsPerBlock));
    if (blocks < 1)
        return fail(GI_EOVERFLOW, "graph and pattern need more than GI_NOALLOC_SCRATCH_BYTES of scratch for one "
                                  "block (4 warps x materialised sets x the second-largest degree x 4 bytes)");
    if (e_cnt > 0)
        noalloc_count_kernel<<<static_cast<unsigned>(blocks), kBlockThreads, 0, st>>>(
            P, d_vertex, reinterpret_cast<const uint32_t *>(d_edge), v_cnt, e_cnt, slots, stride, h);
    noalloc_finish_kernel<<<1, 1, 0, st>>>(h, static_cast<unsigned long long>(p->sched->get_count_divisor()),
                                           d_result);
    if ((e = cudaGetLastError()) != cudaSuccess || (e = cudaStreamSynchronize(st)) != cudaSuccess)
        return cuda_fail(e, "no-alloc count");
    return GI_OK;
}
