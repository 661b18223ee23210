// Batched counting: many (graph, plan) jobs in one persistent launch.
//
// The reference counts one pattern on one graph per launch (reference
// gpu/gpu_graph.cu:22-51; gpu_mc.cu:93-112 loops over patterns, re-creating
// the device context each time).  Here a batch fixes a list of jobs once; a
// run is one launch of batch_count_kernel, captured in a CUDA graph on the
// first run and replayed afterwards.  The work items are chunks of
// GI_TASK_CHUNK first-level edges of every job, numbered job after job; a
// warp claims the next chunk with one atomic, finds its job by binary search
// over the jobs' chunk offsets, and — when the job changed — copies that
// job's plan from global memory into its own slot of shared memory, which the
// DFS (dfs_device.cuh) then reads.  Per job: the raw sum, and the device time
// (%globaltimer) at which its last chunk finished, relative to the launch's
// first warp.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <new>
#include <vector>

#include "dfs_device.cuh"

namespace gi {

int cuda_fail(cudaError_t e, const char *what);

namespace {

struct BatchJob {
    const int64_t *vertex;
    const uint32_t *edge;
    const uint32_t *edge_from;
    int64_t e_cnt;
    int64_t chunk_begin;  // first chunk of this job in the launch's numbering
    int32_t plan;         // index into the batch's plans
    uint32_t v_cnt;
    HubIndex hubs;        // the graph's hub bitmaps
    HashIndex hashes;     // and adjacency hash sets
};

// Counter slots of a batch: [0] chunk cursor, [1] launch start (min over
// warps), [2, 6) the handoff queue's head, tail, idle and exited warps, [6]
// set when a handed-off item was lost.
constexpr int kBatchCounters = 7;
constexpr unsigned long long kBatchHandoffCap = 1ull << 20;

// The job's plan into the warp's shared slot (when it changed).
__device__ __forceinline__ void enter_job(const DevPlan *__restrict__ plans, const BatchJob &J, int job, int &cur,
                                          DevPlan &P, int lane) {
    if (job == cur) return;
    const int32_t *src = reinterpret_cast<const int32_t *>(&plans[J.plan]);
    int32_t *dst = reinterpret_cast<int32_t *>(&P);
    for (int i = lane; i < static_cast<int>(sizeof(DevPlan) / 4); i += 32) dst[i] = src[i];
    __syncwarp();
    cur = job;
}

// Advances the handoff queue's epoch before each run (captured in the batch's
// CUDA graph, so every replay gets a new one): items published by an earlier
// run never look ready to this one.
__global__ void bump_epoch_kernel(uint32_t *epoch) {
    uint32_t x = *epoch + 1;
    if (x == 0) x = 1;
    *epoch = x;
}

// One of a job's work items is done: the last one records the job's end time.
__device__ __forceinline__ void job_item_done(unsigned long long *job_left, unsigned long long *job_done, int job) {
    if (atomicAdd(&job_left[job], ~0ull) == 1ull) job_done[job] = globaltimer();
}

__global__ void __launch_bounds__(kBlockThreads)
    batch_count_kernel(const DevPlan *__restrict__ plans, const BatchJob *__restrict__ jobs, int n_jobs,
                       int64_t total_chunks, uint32_t *scratch, int64_t slot_stride, int64_t slots_per_warp,
                       unsigned long long *counters, unsigned long long *job_sum, unsigned long long *job_left,
                       unsigned long long *job_done, Handoff *hitems, unsigned long long hcap,
                       const uint32_t *hepoch) {
    __shared__ WarpState states[kWarpsPerBlock];
    __shared__ DevPlan plan_s[kWarpsPerBlock];
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    const int64_t gwarp = static_cast<int64_t>(blockIdx.x) * kWarpsPerBlock + wib;
    WarpState &w = states[wib];
    DevPlan &P = plan_s[wib];
    uint32_t *slots = scratch + gwarp * slots_per_warp * slot_stride;
    if (lane == 0) atomicMin(&counters[1], globaltimer());
    HandoffQueue hq;
    if (hitems) {
        hq.items = hitems;
        hq.cap = hcap;
        hq.ctr = counters + 2;
        hq.epoch = *hepoch;
        hq.job_left = job_left;
    }
    int cur = -1;
    while (true) {
        unsigned long long c = 0;
        if (lane == 0) c = atomicAdd(&counters[0], 1ull);
        c = __shfl_sync(kFull, c, 0);
        if (c >= static_cast<unsigned long long>(total_chunks)) break;
        // The job of chunk c: the last j with jobs[j].chunk_begin <= c.
        int lo = 0, hi = n_jobs;
        while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (jobs[mid].chunk_begin <= static_cast<int64_t>(c))
                lo = mid;
            else
                hi = mid;
        }
        const int job = lo;
        const BatchJob J = jobs[job];
        enter_job(plans, J, job, cur, P, lane);
        Ctx<false> ctx{P, J.vertex, J.edge, slots, slot_stride, w, lane, 0ull};
        ctx.hubs = J.hubs;
        ctx.hashes = J.hashes;
        ctx.hq = hq;
        ctx.hq.job = job;
        ctx.hq.v_cnt = J.v_cnt;
        const int64_t e = (static_cast<int64_t>(c) - J.chunk_begin) * kTaskChunk + lane;
        bool valid = e < J.e_cnt;
        uint32_t v0 = 0, v1 = 0;
        if (valid) {
            v0 = __ldg(&J.edge_from[e]);
            v1 = __ldg(&J.edge[e]);
            // Depth-1 restriction (reference gpu/src/gpu_pattern_matching.cuh:77).
            if (P.first_restricted && v0 <= v1) valid = false;
        }
        unsigned todo = __ballot_sync(kFull, valid);
        unsigned long long chunk_sum = 0;
        if (P.flat_first) {
            unsigned long long passed = 0;
            chunk_sum = ctx.first_level_flat(v0, v1, valid, passed);
            todo = 0;
        }
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
            ctx.build_chain(0, a, false);
            if (!ctx.build_chain(1, b)) continue;
            chunk_sum += ctx.dfs(0, 0x7fffffff);
        }
        if (lane == 0) {
            if (chunk_sum) atomicAdd(&job_sum[job], chunk_sum);
            job_item_done(job_left, job_done, job);
        }
    }
    // Out of chunks: ranges other warps handed off, each counted for its own
    // job (take_handoffs).
    if (hitems) {
        const bool lost = take_handoffs(hq, false, lane, [&](long long slot) {
            const Handoff *h = &hitems[slot];
            const int job = __ldcg(&h->job);
            if (job < 0 || job >= n_jobs) return false;
            const BatchJob J = jobs[job];
            enter_job(plans, J, job, cur, P, lane);
            Ctx<false> ctx{P, J.vertex, J.edge, slots, slot_stride, w, lane, 0ull};
            ctx.hubs = J.hubs;
            ctx.hashes = J.hashes;
            ctx.hq = hq;
            ctx.hq.job = job;
            ctx.hq.v_cnt = J.v_cnt;
            unsigned long long part = 0;
            const bool ok = ctx.run_handoff(h, part);
            if (lane == 0) {
                if (part) atomicAdd(&job_sum[job], part);
                job_item_done(job_left, job_done, job);
            }
            return ok;
        });
        if (lost && lane == 0) atomicExch(&counters[6], 1ull);
    }
}

}  // namespace
}  // namespace gi

using namespace gi;

struct gi_batch {
    int device = 0;
    int n_jobs = 0;
    int64_t total_chunks = 0;
    std::vector<gi_graph *> graphs;
    std::vector<const gi_plan *> plans;  // one per job (plans may repeat)
    std::vector<uint64_t> divisor;       // per job
    std::vector<unsigned long long> chunks;  // per job
    DevPlan *d_plans = nullptr;
    BatchJob *d_jobs = nullptr;
    uint32_t *d_scratch = nullptr;
    unsigned long long *d_ctr = nullptr;  // counters[kBatchCounters] | sum[n] | left[n] | done[n]
    Handoff *d_handoff = nullptr;         // work donation between the batch's warps
    uint32_t *d_epoch = nullptr;          // the queue's epoch, advanced by every run
    unsigned long long *d_init = nullptr; // the values a run starts from (copied in the graph)
    int64_t slot_stride = 1, slots_per_warp = 1;
    int blocks = 0;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaStream_t captured_on = nullptr;
};

static void batch_free(gi_batch *b) {
    if (!b) return;
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    cudaFree(b->d_plans);
    cudaFree(b->d_jobs);
    cudaFree(b->d_scratch);
    cudaFree(b->d_ctr);
    cudaFree(b->d_init);
    cudaFree(b->d_handoff);
    cudaFree(b->d_epoch);
    delete b;
}

extern "C" {

int gi_batch_create(gi_graph *const *graphs, const gi_plan *const *plans, int n_jobs, gi_batch **out) {
    if (!graphs || !plans || !out || n_jobs < 1) return fail(GI_EINVAL, "bad batch arguments");
    *out = nullptr;
    auto *b = new (std::nothrow) gi_batch;
    if (!b) return fail(GI_ENOMEM, "host allocation");
    b->n_jobs = n_jobs;
    b->device = graphs[0] ? graphs[0]->device : 0;
    std::vector<DevPlan> hplans;
    std::vector<BatchJob> hjobs(n_jobs);
    int64_t chunk = 0;
    for (int j = 0; j < n_jobs; ++j) {
        gi_graph *g = graphs[j];
        const gi_plan *p = plans[j];
        if (!g || !p || g->device != b->device) {
            batch_free(b);
            return fail(GI_EINVAL, "every job needs a graph on the batch's device and a plan");
        }
        b->graphs.push_back(g);
        b->plans.push_back(p);
        b->divisor.push_back(static_cast<uint64_t>(p->sched->get_count_divisor()));
        // The autotuner's cached variant for this job's class, if any.
        DevPlan dp = p->dev;
        tuned_plan(g, p->dev, dp);
        hplans.push_back(plan_for_graph(dp, g->max_degree));
        const int64_t nch = (g->e_cnt + kTaskChunk - 1) / kTaskChunk;
        b->chunks.push_back(static_cast<unsigned long long>(nch));
        hjobs[j] = BatchJob{g->d_vertex, reinterpret_cast<const uint32_t *>(g->d_edge), g->d_edge_from, g->e_cnt,
                            chunk, j, static_cast<uint32_t>(g->v_cnt), hubs_of(g), hashes_of(g)};
        chunk += nch;
        b->slot_stride = std::max<int64_t>(b->slot_stride, g->max_isect);
        b->slots_per_warp = std::max<int64_t>(b->slots_per_warp, p->dev.n_slots);
    }
    b->total_chunks = chunk;
    int prev = 0;
    cudaGetDevice(&prev);
    if (prev != b->device) cudaSetDevice(b->device);
    int sms = 148, per_sm = 1;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, b->device);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, batch_count_kernel, kBlockThreads, 0);
    b->blocks = sms * std::max(per_sm, 1);
    const int64_t warps = static_cast<int64_t>(b->blocks) * kWarpsPerBlock;
    const size_t ctr_words = kBatchCounters + 3 * static_cast<size_t>(n_jobs);
    std::vector<unsigned long long> init(ctr_words, 0);
    init[1] = ~0ull;  // launch start: min over warps
    for (int j = 0; j < n_jobs; ++j) init[kBatchCounters + n_jobs + j] = b->chunks[j];
    cudaError_t e;
    if ((e = cudaMalloc(&b->d_plans, sizeof(DevPlan) * n_jobs)) != cudaSuccess ||
        (e = cudaMalloc(&b->d_jobs, sizeof(BatchJob) * n_jobs)) != cudaSuccess ||
        (e = cudaMalloc(&b->d_scratch, sizeof(uint32_t) * warps * b->slots_per_warp * b->slot_stride)) !=
            cudaSuccess ||
        (e = cudaMalloc(&b->d_ctr, sizeof(unsigned long long) * ctr_words)) != cudaSuccess ||
        (e = cudaMalloc(&b->d_init, sizeof(unsigned long long) * ctr_words)) != cudaSuccess ||
        (e = cudaMalloc(&b->d_handoff, sizeof(Handoff) * kBatchHandoffCap)) != cudaSuccess ||
        (e = cudaMemset(b->d_handoff, 0, sizeof(Handoff) * kBatchHandoffCap)) != cudaSuccess ||
        (e = cudaMalloc(&b->d_epoch, sizeof(uint32_t))) != cudaSuccess ||
        (e = cudaMemset(b->d_epoch, 0, sizeof(uint32_t))) != cudaSuccess ||
        (e = cudaMemcpy(b->d_plans, hplans.data(), sizeof(DevPlan) * n_jobs, cudaMemcpyHostToDevice)) !=
            cudaSuccess ||
        (e = cudaMemcpy(b->d_jobs, hjobs.data(), sizeof(BatchJob) * n_jobs, cudaMemcpyHostToDevice)) !=
            cudaSuccess ||
        (e = cudaMemcpy(b->d_init, init.data(), sizeof(unsigned long long) * ctr_words, cudaMemcpyHostToDevice)) !=
            cudaSuccess) {
        if (prev != b->device) cudaSetDevice(prev);
        batch_free(b);
        return cuda_fail(e, "batch allocation");
    }
    if (prev != b->device) cudaSetDevice(prev);
    *out = b;
    return GI_OK;
}

int gi_batch_run(gi_batch *b, gi_stream stream, uint64_t *counts, double *job_ms, gi_stats *stats) {
    if (!b || !counts) return fail(GI_EINVAL, "NULL argument");
    int prev = 0;
    cudaGetDevice(&prev);
    if (prev != b->device) cudaSetDevice(b->device);
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    cudaStream_t cap = st;
    cudaError_t e = cudaSuccess;
    const int n = b->n_jobs;
    const size_t ctr_words = kBatchCounters + 3 * static_cast<size_t>(n);
    // The run as a CUDA graph: reset the counters, then the one launch.  The
    // legacy default stream cannot be captured, so a private stream carries
    // the capture in that case.
    if (!b->exec) {
        if (!st && (e = cudaStreamCreateWithFlags(&cap, cudaStreamNonBlocking)) != cudaSuccess)
            return cuda_fail(e, "capture stream");
        if ((e = cudaStreamBeginCapture(cap, cudaStreamCaptureModeThreadLocal)) == cudaSuccess) {
            cudaMemcpyAsync(b->d_ctr, b->d_init, sizeof(unsigned long long) * ctr_words, cudaMemcpyDeviceToDevice,
                            cap);
            bump_epoch_kernel<<<1, 1, 0, cap>>>(b->d_epoch);
            batch_count_kernel<<<b->blocks, kBlockThreads, 0, cap>>>(
                b->d_plans, b->d_jobs, n, b->total_chunks, b->d_scratch, b->slot_stride, b->slots_per_warp, b->d_ctr,
                b->d_ctr + kBatchCounters, b->d_ctr + kBatchCounters + n, b->d_ctr + kBatchCounters + 2 * n,
                b->d_handoff, kBatchHandoffCap, b->d_epoch);
            e = cudaStreamEndCapture(cap, &b->graph);
        }
        if (e == cudaSuccess) e = cudaGraphInstantiate(&b->exec, b->graph, 0);
        if (!st) cudaStreamDestroy(cap);
        if (e != cudaSuccess) {
            if (prev != b->device) cudaSetDevice(prev);
            return cuda_fail(e, "batch graph capture");
        }
    }
    cudaEvent_t t0, t1;
    cudaEventCreate(&t0);
    cudaEventCreate(&t1);
    std::vector<unsigned long long> host(ctr_words);
    cudaEventRecord(t0, st);
    e = cudaGraphLaunch(b->exec, st);
    cudaEventRecord(t1, st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(host.data(), b->d_ctr, sizeof(unsigned long long) * ctr_words, cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    float ms = 0.f;
    if (e == cudaSuccess) cudaEventElapsedTime(&ms, t0, t1);
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    if (prev != b->device) cudaSetDevice(prev);
    if (e != cudaSuccess) return cuda_fail(e, "batch run");
    if (host[6]) return fail(GI_ECUDA, "a handed-off batch work item was never published");
    const unsigned long long start = host[1];
    for (int j = 0; j < n; ++j) {
        const uint64_t raw = host[kBatchCounters + j];
        counts[j] = b->divisor[j] ? raw / b->divisor[j] : raw;
        if (job_ms) {
            const unsigned long long done = host[kBatchCounters + 2 * n + j];
            job_ms[j] = b->chunks[j] == 0 || done < start ? 0.0 : (done - start) * 1e-6;
        }
    }
    if (stats) {
        const int cb = stats->count_bytes;
        std::memset(stats, 0, sizeof(*stats));
        stats->count_bytes = cb;
        stats->kernel_ms = ms;
        stats->grid_blocks = b->blocks;
        stats->block_threads = kBlockThreads;
        stats->kernel_launches = 1;
        stats->chunks_total = b->total_chunks;
        stats->chunks_done = b->total_chunks;
    }
    return GI_OK;
}

int gi_batch_destroy(gi_batch *b) {
    batch_free(b);
    return GI_OK;
}

}  // extern "C"
