// Labeled-graph ingest on the GPU: the renaming and bucketing of the
// reference's labeled loader (reference src/dataloader.cpp:440-620), built by
// kernels and cub sorts instead of host loops.
//
// Result: the same gi_labeled_graph as build_labeled (fsm_host.cpp), with the
// bucketed neighbour lists (edge, bucket, label_start) left on the device for
// the support kernel; gi_labeled_graph_export downloads them when asked.
// The steps, in order:
//   1. upload the CSR and the labels; a kernel checks neighbour ids and
//      counts each vertex's degree without self-loops (duplicates count);
//   2. a segmented sort of a copy of every neighbour list, then a kernel that
//      looks every entry (v, u) up in u's sorted list (symmetry);
//   3. on the host, the labels in first-seen order and the reference's
//      std::sort of (label, maximum degree) pairs — at most 255 labels, so
//      only the O(v) first-seen pass and the O(l log l) sort stay there;
//      the maxima come from a device reduction;
//   4. a stable radix sort of the vertices by (label, -degree) gives the new
//      numbering by (label, -degree, id);
//   5. the new degrees are scanned into offsets, a warp per new vertex writes
//      its renamed neighbours (self-loops dropped, order kept), and a
//      segmented sort orders each list by new id, which is the order by
//      (label, id) because new ids are grouped by label;
//   6. a warp per vertex finds each label's first entry (bucket).
#include <cuda_runtime.h>
#include <cub/device/device_radix_sort.cuh>
#include <cub/device/device_reduce.cuh>
#include <cub/device/device_scan.cuh>
#include <cub/device/device_segmented_sort.cuh>

#include <algorithm>
#include <cstring>
#include <new>
#include <unordered_map>
#include <vector>

#include "fsm.hpp"
#include "internal.hpp"

namespace gi {

int cuda_fail(cudaError_t e, const char *what);

namespace {

constexpr unsigned kAll = 0xffffffffu;

// Degree of each vertex without self-loops; flags out-of-range ids.
__global__ void ingest_degree_kernel(const int64_t *__restrict__ vertex, const int32_t *__restrict__ edge,
                                     int32_t v_cnt, int64_t *__restrict__ degree, int *bad) {
    const int lane = threadIdx.x & 31;
    const int64_t warp = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = (static_cast<int64_t>(gridDim.x) * blockDim.x) >> 5;
    for (int64_t v = warp; v < v_cnt; v += nwarps) {
        int64_t d = 0;
        bool err = false;
        for (int64_t j = vertex[v] + lane; j < vertex[v + 1]; j += 32) {
            const int32_t x = edge[j];
            if (x < 0 || x >= v_cnt) err = true;
            d += x != v;
        }
        for (int o = 16; o; o >>= 1) d += __shfl_xor_sync(kAll, d, o);
        if (__any_sync(kAll, err) && lane == 0) atomicExch(bad, 1);
        if (lane == 0) degree[v] = d;
    }
}

// Every entry (v, u), u != v, must have v in u's sorted list.
__global__ void ingest_symmetry_kernel(const int64_t *__restrict__ vertex, const int32_t *__restrict__ sorted,
                                       int32_t v_cnt, int *bad) {
    const int lane = threadIdx.x & 31;
    const int64_t warp = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = (static_cast<int64_t>(gridDim.x) * blockDim.x) >> 5;
    for (int64_t v = warp; v < v_cnt; v += nwarps) {
        bool err = false;
        for (int64_t j = vertex[v] + lane; j < vertex[v + 1]; j += 32) {
            const int32_t u = sorted[j];
            if (u == v) continue;
            int64_t lo = vertex[u], len = vertex[u + 1] - lo;
            while (len > 0) {
                const int64_t half = len >> 1;
                if (sorted[lo + half] < v) {
                    lo += half + 1;
                    len -= half + 1;
                } else {
                    len = half;
                }
            }
            if (lo >= vertex[u + 1] || sorted[lo] != v) err = true;
        }
        if (__any_sync(kAll, err) && lane == 0) atomicExch(bad, 1);
    }
}

// Per first-seen label: its largest degree; per vertex the radix key
// (label << 32 | ~degree) of the renumbering, with the new label applied.
__global__ void ingest_label_max_kernel(const int32_t *__restrict__ lab, const int64_t *__restrict__ degree,
                                        int32_t v_cnt, unsigned long long *__restrict__ max_deg) {
    for (int64_t v = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; v < v_cnt;
         v += static_cast<int64_t>(gridDim.x) * blockDim.x)
        atomicMax(&max_deg[lab[v]], static_cast<unsigned long long>(degree[v]));
}

__global__ void ingest_key_kernel(const int32_t *__restrict__ lab, const int32_t *__restrict__ rename,
                                  const int64_t *__restrict__ degree, int32_t v_cnt,
                                  unsigned long long *__restrict__ key, int32_t *__restrict__ ids,
                                  unsigned int *__restrict__ freq) {
    for (int64_t v = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; v < v_cnt;
         v += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int32_t l = rename[lab[v]];
        key[v] = (static_cast<unsigned long long>(l) << 32) | (0xffffffffull - static_cast<unsigned long long>(degree[v]));
        ids[v] = static_cast<int32_t>(v);
        atomicAdd(&freq[l], 1u);
    }
}

// rank[i] = old id of new vertex i: new_id, the new labels and new degrees.
__global__ void ingest_renumber_kernel(const int32_t *__restrict__ rank, const int32_t *__restrict__ lab,
                                       const int32_t *__restrict__ rename, const int64_t *__restrict__ degree,
                                       int32_t v_cnt, int32_t *__restrict__ new_id, int32_t *__restrict__ v_label,
                                       int64_t *__restrict__ new_deg) {
    for (int64_t i = static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x; i < v_cnt;
         i += static_cast<int64_t>(gridDim.x) * blockDim.x) {
        const int32_t x = rank[i];
        new_id[x] = static_cast<int32_t>(i);
        v_label[i] = rename[lab[x]];
        new_deg[i] = degree[x];
    }
}

// A warp per new vertex i: the renamed neighbours of old vertex rank[i],
// self-loops dropped, written from new_off[i] in list order.
__global__ void ingest_fill_kernel(const int64_t *__restrict__ vertex, const int32_t *__restrict__ edge,
                                   const int32_t *__restrict__ rank, const int32_t *__restrict__ new_id,
                                   const int64_t *__restrict__ new_off, int32_t v_cnt, uint32_t *__restrict__ out) {
    const int lane = threadIdx.x & 31;
    const int64_t warp = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = (static_cast<int64_t>(gridDim.x) * blockDim.x) >> 5;
    for (int64_t i = warp; i < v_cnt; i += nwarps) {
        const int32_t x = rank[i];
        int64_t pos = new_off[i];
        for (int64_t base = vertex[x]; base < vertex[x + 1]; base += 32) {
            const int64_t j = base + lane;
            int32_t u = x;
            if (j < vertex[x + 1]) u = edge[j];
            const bool keep = u != x;
            const unsigned m = __ballot_sync(kAll, keep);
            if (keep) out[pos + __popc(m & ((1u << lane) - 1u))] = static_cast<uint32_t>(new_id[u]);
            pos += __popc(m);
        }
    }
}

// bucket[u * l_cnt + l] = first entry of u whose neighbour has label >= l,
// i.e. new id >= label_start[l]; a warp per vertex, a lane per label.
__global__ void ingest_bucket_kernel(const int64_t *__restrict__ new_off, const uint32_t *__restrict__ list,
                                     const uint32_t *__restrict__ label_start, int32_t v_cnt, int32_t l_cnt,
                                     uint32_t *__restrict__ bucket) {
    const int lane = threadIdx.x & 31;
    const int64_t warp = (static_cast<int64_t>(blockIdx.x) * blockDim.x + threadIdx.x) >> 5;
    const int64_t nwarps = (static_cast<int64_t>(gridDim.x) * blockDim.x) >> 5;
    for (int64_t u = warp; u < v_cnt; u += nwarps) {
        const int64_t a = new_off[u], b = new_off[u + 1];
        for (int l = lane; l < l_cnt; l += 32) {
            const uint32_t first = label_start[l];
            int64_t lo = a, len = b - a;
            while (len > 0) {
                const int64_t half = len >> 1;
                if (list[lo + half] < first) {
                    lo += half + 1;
                    len -= half + 1;
                } else {
                    len = half;
                }
            }
            bucket[u * l_cnt + l] = static_cast<uint32_t>(lo);
        }
    }
}

// Device buffers of one ingest, freed on every exit path.
struct Buffers {
    std::vector<void *> ptrs;
    ~Buffers() {
        for (void *p : ptrs) cudaFree(p);
    }
    template <class T>
    cudaError_t alloc(T **p, size_t n) {
        *p = nullptr;
        const cudaError_t e = cudaMalloc(reinterpret_cast<void **>(p), std::max<size_t>(n, 1) * sizeof(T));
        if (e == cudaSuccess) ptrs.push_back(*p);
        return e;
    }
    void release(void *p) {  // ownership moves to the graph
        ptrs.erase(std::remove(ptrs.begin(), ptrs.end(), p), ptrs.end());
    }
};

}  // namespace

int labeled_graph_create_device(int32_t v_cnt, const int64_t *vertex, const int32_t *edge, const uint32_t *labels,
                                const int32_t *order, cudaStream_t st, gi_labeled_graph **out) {
    if (!out) return fail(GI_EINVAL, "out is NULL");
    *out = nullptr;
    if (v_cnt < 1 || !vertex || !labels) return fail(GI_EINVAL, "empty labeled graph");
    if (vertex[0] != 0) return fail(GI_EINVAL, "vertex[0] must be 0");
    for (int32_t v = 0; v < v_cnt; ++v)
        if (vertex[v + 1] < vertex[v]) return fail(GI_EINVAL, "vertex offsets decrease");
    const int64_t entries = vertex[v_cnt];
    if (entries > 0 && !edge) return fail(GI_EINVAL, "edge is NULL");
    if (entries >= (int64_t(1) << 31)) return fail(GI_EOVERFLOW, "more than 2^31 - 1 neighbour entries");
    std::vector<int32_t> seq;
    if (order) {
        std::vector<char> seen(v_cnt, 0);
        seq.resize(v_cnt);
        for (int32_t i = 0; i < v_cnt; ++i) {
            if (order[i] < 0 || order[i] >= v_cnt || seen[order[i]]) return fail(GI_EINVAL, "order is not a permutation");
            seen[order[i]] = 1;
            seq[i] = order[i];
        }
    }
    // Labels in first-seen order (host: an O(v) pass over a small map).
    std::unordered_map<uint32_t, int32_t> first;
    std::vector<uint32_t> first_value;
    std::vector<int32_t> tmp_label(v_cnt);
    for (int32_t i = 0; i < v_cnt; ++i) {
        const int32_t v = order ? seq[i] : i;
        auto it = first.find(labels[v]);
        if (it == first.end()) {
            if (first_value.size() >= 255) return fail(GI_ENOTSUP, "more than 255 labels");
            it = first.emplace(labels[v], static_cast<int32_t>(first_value.size())).first;
            first_value.push_back(labels[v]);
        }
        tmp_label[v] = it->second;
    }
    const int32_t l_cnt = static_cast<int32_t>(first_value.size());
    if (static_cast<int64_t>(v_cnt) * l_cnt >= (int64_t(1) << 31))
        return fail(GI_EOVERFLOW, "v_cnt * l_cnt does not fit the bucket index");

    int sms = 148, device = 0;
    cudaGetDevice(&device);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    const int grid = sms * 8;
    Buffers B;
    cudaError_t e;
    int64_t *d_vertex, *d_degree, *d_new_deg, *d_new_off;
    int32_t *d_edge, *d_sorted, *d_lab, *d_rename, *d_ids, *d_ids2, *d_new_id, *d_v_label;
    unsigned long long *d_maxdeg, *d_key, *d_key2;
    unsigned int *d_freq;
    uint32_t *d_list, *d_list2, *d_bucket, *d_label_start;
    int *d_bad;
    const size_t nv = static_cast<size_t>(v_cnt);
    if ((e = B.alloc(&d_vertex, nv + 1)) != cudaSuccess || (e = B.alloc(&d_degree, nv)) != cudaSuccess ||
        (e = B.alloc(&d_edge, static_cast<size_t>(entries))) != cudaSuccess ||
        (e = B.alloc(&d_sorted, static_cast<size_t>(entries))) != cudaSuccess ||
        (e = B.alloc(&d_lab, nv)) != cudaSuccess || (e = B.alloc(&d_bad, 1)) != cudaSuccess)
        return cuda_fail(e, "labeled ingest allocation");
    if ((e = cudaMemcpyAsync(d_vertex, vertex, (nv + 1) * sizeof(int64_t), cudaMemcpyHostToDevice, st)) != cudaSuccess ||
        (entries > 0 &&
         (e = cudaMemcpyAsync(d_edge, edge, entries * sizeof(int32_t), cudaMemcpyHostToDevice, st)) != cudaSuccess) ||
        (e = cudaMemcpyAsync(d_lab, tmp_label.data(), nv * sizeof(int32_t), cudaMemcpyHostToDevice, st)) != cudaSuccess ||
        (e = cudaMemsetAsync(d_bad, 0, sizeof(int), st)) != cudaSuccess)
        return cuda_fail(e, "labeled ingest upload");
    ingest_degree_kernel<<<grid, 256, 0, st>>>(d_vertex, d_edge, v_cnt, d_degree, d_bad);
    int bad = 0;
    if ((e = cudaGetLastError()) != cudaSuccess ||
        (e = cudaMemcpyAsync(&bad, d_bad, sizeof(int), cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
        (e = cudaStreamSynchronize(st)) != cudaSuccess)
        return cuda_fail(e, "degree kernel");
    if (bad) return fail(GI_EINVAL, "neighbour id out of range");
    // Symmetry on sorted copies of the lists.
    size_t tmp_bytes = 0;
    void *d_tmp = nullptr;
    auto grow_tmp = [&](size_t need) -> cudaError_t {
        if (need <= tmp_bytes) return cudaSuccess;
        B.release(d_tmp);
        cudaFree(d_tmp);
        d_tmp = nullptr;
        tmp_bytes = 0;
        const cudaError_t r = cudaMalloc(&d_tmp, need);
        if (r == cudaSuccess) {
            B.ptrs.push_back(d_tmp);
            tmp_bytes = need;
        }
        return r;
    };
    if (entries > 0) {
        size_t need = 0;
        cub::DeviceSegmentedSort::SortKeys(nullptr, need, d_edge, d_sorted, static_cast<int>(entries), v_cnt, d_vertex,
                                           d_vertex + 1, st);
        if ((e = grow_tmp(need)) != cudaSuccess) return cuda_fail(e, "sort workspace");
        if ((e = cub::DeviceSegmentedSort::SortKeys(d_tmp, need, d_edge, d_sorted, static_cast<int>(entries), v_cnt,
                                                    d_vertex, d_vertex + 1, st)) != cudaSuccess)
            return cuda_fail(e, "neighbour sort");
        ingest_symmetry_kernel<<<grid, 256, 0, st>>>(d_vertex, d_sorted, v_cnt, d_bad);
        if ((e = cudaGetLastError()) != cudaSuccess ||
            (e = cudaMemcpyAsync(&bad, d_bad, sizeof(int), cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
            (e = cudaStreamSynchronize(st)) != cudaSuccess)
            return cuda_fail(e, "symmetry kernel");
        if (bad) return fail(GI_EINVAL, "neighbour lists are not symmetric");
    }
    // Directed entries without self-loops.
    int64_t e_cnt = 0;
    {
        int64_t *d_sum = nullptr;
        if ((e = B.alloc(&d_sum, 1)) != cudaSuccess) return cuda_fail(e, "labeled ingest allocation");
        size_t need = 0;
        cub::DeviceReduce::Sum(nullptr, need, d_degree, d_sum, v_cnt, st);
        if ((e = grow_tmp(need)) != cudaSuccess || (e = cub::DeviceReduce::Sum(d_tmp, need, d_degree, d_sum, v_cnt, st)) != cudaSuccess ||
            (e = cudaMemcpyAsync(&e_cnt, d_sum, sizeof(int64_t), cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
            (e = cudaStreamSynchronize(st)) != cudaSuccess)
            return cuda_fail(e, "edge count");
    }
    if (e_cnt >= (int64_t(1) << 32)) return fail(GI_EOVERFLOW, "more than 2^32 - 1 neighbour entries");
    // Label renaming: maxima on the device, the reference's sort on the host.
    if ((e = B.alloc(&d_maxdeg, static_cast<size_t>(l_cnt))) != cudaSuccess ||
        (e = cudaMemsetAsync(d_maxdeg, 0, l_cnt * sizeof(unsigned long long), st)) != cudaSuccess)
        return cuda_fail(e, "label maxima");
    ingest_label_max_kernel<<<grid, 256, 0, st>>>(d_lab, d_degree, v_cnt, d_maxdeg);
    std::vector<unsigned long long> max_deg(l_cnt);
    if ((e = cudaGetLastError()) != cudaSuccess ||
        (e = cudaMemcpyAsync(max_deg.data(), d_maxdeg, l_cnt * sizeof(unsigned long long), cudaMemcpyDeviceToHost,
                             st)) != cudaSuccess ||
        (e = cudaStreamSynchronize(st)) != cudaSuccess)
        return cuda_fail(e, "label maxima");
    // The same std::sort call on the same sequence as the reference (and as
    // build_labeled): it is not stable, so ties resolve only the same way
    // through the same call (reference src/dataloader.cpp:528-536).
    std::vector<std::pair<int, double>> by_deg;
    by_deg.reserve(l_cnt);
    for (int32_t l = 0; l < l_cnt; ++l) by_deg.emplace_back(l, static_cast<double>(max_deg[l]));
    std::sort(by_deg.begin(), by_deg.end(),
              [](const std::pair<int, double> &a, const std::pair<int, double> &b) { return a.second > b.second; });
    std::vector<int32_t> rename(l_cnt);
    for (int32_t i = 0; i < l_cnt; ++i) rename[by_deg[i].first] = i;
    // Renumbering by (label, -degree, id): a stable radix sort of the ids.
    if ((e = B.alloc(&d_rename, static_cast<size_t>(l_cnt))) != cudaSuccess || (e = B.alloc(&d_key, nv)) != cudaSuccess ||
        (e = B.alloc(&d_key2, nv)) != cudaSuccess || (e = B.alloc(&d_ids, nv)) != cudaSuccess ||
        (e = B.alloc(&d_ids2, nv)) != cudaSuccess || (e = B.alloc(&d_freq, static_cast<size_t>(l_cnt))) != cudaSuccess ||
        (e = cudaMemcpyAsync(d_rename, rename.data(), l_cnt * sizeof(int32_t), cudaMemcpyHostToDevice, st)) !=
            cudaSuccess ||
        (e = cudaMemsetAsync(d_freq, 0, l_cnt * sizeof(unsigned int), st)) != cudaSuccess)
        return cuda_fail(e, "renumbering buffers");
    ingest_key_kernel<<<grid, 256, 0, st>>>(d_lab, d_rename, d_degree, v_cnt, d_key, d_ids, d_freq);
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "renumbering keys");
    {
        size_t need = 0;
        cub::DeviceRadixSort::SortPairs(nullptr, need, d_key, d_key2, d_ids, d_ids2, v_cnt, 0, 40, st);
        if ((e = grow_tmp(need)) != cudaSuccess ||
            (e = cub::DeviceRadixSort::SortPairs(d_tmp, need, d_key, d_key2, d_ids, d_ids2, v_cnt, 0, 40, st)) !=
                cudaSuccess)
            return cuda_fail(e, "renumbering sort");
    }
    const int32_t *d_rank = d_ids2;
    if ((e = B.alloc(&d_new_id, nv)) != cudaSuccess || (e = B.alloc(&d_v_label, nv)) != cudaSuccess ||
        (e = B.alloc(&d_new_deg, nv + 1)) != cudaSuccess || (e = B.alloc(&d_new_off, nv + 1)) != cudaSuccess ||
        (e = cudaMemsetAsync(d_new_deg + nv, 0, sizeof(int64_t), st)) != cudaSuccess)
        return cuda_fail(e, "renumbering buffers");
    ingest_renumber_kernel<<<grid, 256, 0, st>>>(d_rank, d_lab, d_rename, d_degree, v_cnt, d_new_id, d_v_label,
                                                 d_new_deg);
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "renumbering");
    {
        size_t need = 0;
        cub::DeviceScan::ExclusiveSum(nullptr, need, d_new_deg, d_new_off, v_cnt + 1, st);
        if ((e = grow_tmp(need)) != cudaSuccess ||
            (e = cub::DeviceScan::ExclusiveSum(d_tmp, need, d_new_deg, d_new_off, v_cnt + 1, st)) != cudaSuccess)
            return cuda_fail(e, "offset scan");
    }
    // Renamed lists, then each sorted by new id.
    if ((e = B.alloc(&d_list, static_cast<size_t>(e_cnt))) != cudaSuccess ||
        (e = B.alloc(&d_list2, static_cast<size_t>(e_cnt))) != cudaSuccess)
        return cuda_fail(e, "bucketed list allocation");
    ingest_fill_kernel<<<grid, 256, 0, st>>>(d_vertex, d_edge, d_rank, d_new_id, d_new_off, v_cnt, d_list);
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "list fill");
    if (e_cnt > 0) {
        size_t need = 0;
        cub::DeviceSegmentedSort::SortKeys(nullptr, need, d_list, d_list2, static_cast<int>(e_cnt), v_cnt, d_new_off,
                                           d_new_off + 1, st);
        if ((e = grow_tmp(need)) != cudaSuccess ||
            (e = cub::DeviceSegmentedSort::SortKeys(d_tmp, need, d_list, d_list2, static_cast<int>(e_cnt), v_cnt,
                                                    d_new_off, d_new_off + 1, st)) != cudaSuccess)
            return cuda_fail(e, "list sort");
    }
    // Label starts (host scan of at most 255 counts), then the buckets.
    std::vector<unsigned int> freq(l_cnt);
    if ((e = cudaMemcpyAsync(freq.data(), d_freq, l_cnt * sizeof(unsigned int), cudaMemcpyDeviceToHost, st)) !=
            cudaSuccess ||
        (e = cudaStreamSynchronize(st)) != cudaSuccess)
        return cuda_fail(e, "label counts");
    std::vector<uint32_t> label_start(l_cnt + 1, 0);
    for (int32_t l = 0; l < l_cnt; ++l) label_start[l + 1] = label_start[l] + freq[l];
    const size_t n_bucket = nv * static_cast<size_t>(l_cnt) + 1;
    if ((e = B.alloc(&d_label_start, static_cast<size_t>(l_cnt) + 1)) != cudaSuccess ||
        (e = B.alloc(&d_bucket, n_bucket)) != cudaSuccess ||
        (e = cudaMemcpyAsync(d_label_start, label_start.data(), (l_cnt + 1) * sizeof(uint32_t), cudaMemcpyHostToDevice,
                             st)) != cudaSuccess)
        return cuda_fail(e, "bucket allocation");
    const uint32_t e32 = static_cast<uint32_t>(e_cnt);
    if ((e = cudaMemcpyAsync(d_bucket + (n_bucket - 1), &e32, sizeof(uint32_t), cudaMemcpyHostToDevice, st)) !=
        cudaSuccess)
        return cuda_fail(e, "bucket end");
    ingest_bucket_kernel<<<grid, 256, 0, st>>>(d_new_off, d_list2, d_label_start, v_cnt, l_cnt, d_bucket);
    if ((e = cudaGetLastError()) != cudaSuccess) return cuda_fail(e, "bucket kernel");
    // The small per-vertex arrays come back to the host; the lists and
    // buckets stay on the device.
    auto *g = new (std::nothrow) gi_labeled_graph;
    if (!g) return fail(GI_ENOMEM, "host allocation");
    g->device = device;
    g->v_cnt = v_cnt;
    g->e_cnt = e_cnt;
    g->l_cnt = l_cnt;
    g->new_id.resize(nv);
    g->v_label.resize(nv);
    g->label_value.resize(l_cnt);
    for (int32_t l = 0; l < l_cnt; ++l) g->label_value[rename[l]] = first_value[l];
    g->label_frequency.resize(l_cnt);
    for (int32_t l = 0; l < l_cnt; ++l) g->label_frequency[l] = freq[l];
    g->label_start = label_start;
    if ((e = cudaMemcpyAsync(g->new_id.data(), d_new_id, nv * sizeof(int32_t), cudaMemcpyDeviceToHost, st)) !=
            cudaSuccess ||
        (e = cudaMemcpyAsync(g->v_label.data(), d_v_label, nv * sizeof(int32_t), cudaMemcpyDeviceToHost, st)) !=
            cudaSuccess ||
        (e = cudaStreamSynchronize(st)) != cudaSuccess) {
        delete g;
        return cuda_fail(e, "renumbering download");
    }
    B.release(d_list2);
    B.release(d_bucket);
    B.release(d_label_start);
    g->d_edge = d_list2;
    g->d_bucket = d_bucket;
    g->d_label_start = d_label_start;
    g->device_built = true;
    *out = g;
    return GI_OK;
}

// Host copies of the lists and buckets of a graph built on the device.
int labeled_graph_download(const gi_labeled_graph *cg) {
    auto *g = const_cast<gi_labeled_graph *>(cg);
    if (!g->device_built || !g->edge.empty() || !g->bucket.empty()) return GI_OK;
    DeviceGuard guard(g->device);
    std::vector<uint32_t> edge(static_cast<size_t>(g->e_cnt)), bucket(static_cast<size_t>(g->v_cnt) * g->l_cnt + 1);
    cudaError_t e;
    if ((!edge.empty() &&
         (e = cudaMemcpy(edge.data(), g->d_edge, edge.size() * sizeof(uint32_t), cudaMemcpyDeviceToHost)) != cudaSuccess) ||
        (e = cudaMemcpy(bucket.data(), g->d_bucket, bucket.size() * sizeof(uint32_t), cudaMemcpyDeviceToHost)) !=
            cudaSuccess)
        return cuda_fail(e, "labeled graph download");
    g->edge = std::move(edge);
    g->bucket = std::move(bucket);
    return GI_OK;
}

}  // namespace gi

extern "C" int gi_labeled_graph_create_device(int32_t v_cnt, const int64_t *vertex, const int32_t *edge,
                                              const uint32_t *labels, const int32_t *order, gi_stream stream,
                                              gi_labeled_graph **out) {
    try {
        return gi::labeled_graph_create_device(v_cnt, vertex, edge, labels, order, static_cast<cudaStream_t>(stream),
                                               out);
    } catch (const std::bad_alloc &) {
        return gi::fail(GI_ENOMEM, "host allocation");
    }
}
