/*
 * graphindor_b200 — C ABI of the B200 pattern-counting engine.
 *
 * The reference (GraphSet) has no library ABI: its surface is the host
 * classes Pattern / Schedule_IEP / Graph and one kernel launch per pattern on
 * a PatternMatchingDeviceContext (reference gpu/function/pattern_matching.cuh:
 * 9-105, gpu/gpu_graph.cu:22-51).  These entry points replace that surface
 * with plain pointers and sizes.  Every function returns a gi_status; none
 * calls exit().  Distinct handles may be used from different threads; a graph
 * handle serialises the counts that run on it.  Counts are uint64 and follow
 * the reference GPU path's arithmetic: the per-embedding sum is taken modulo
 * 2^64 and then divided by the plan's redundancy (reference
 * gpu/gpu_graph.cu:42-44).
 */
#ifndef GRAPHINDOR_B200_GI_H
#define GRAPHINDOR_B200_GI_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GI_MAX_PATTERN 7        /* reference MAX_DEPTH, gpu/function/pattern_matching.cuh:7 */
#define GI_MAX_PREFIX 22        /* n(n-1)/2 + 1 for n = 7 */
#define GI_MAX_IEP_SETS 32      /* distinct IEP sets for a 5-vertex tail */
#define GI_MAX_IEP_TERMS 160    /* blocks over all set partitions of 5 (151) */

typedef enum gi_status {
    GI_OK = 0,
    GI_EINVAL = 1,       /* bad argument, pattern too large, bad adjacency string */
    GI_ENOMEM = 2,       /* host or device allocation failed */
    GI_ECUDA = 3,        /* a CUDA call failed; see gi_last_error() */
    GI_ETIMEOUT = 4,     /* a device work budget ran out before the count finished */
    GI_EOVERFLOW = 5,    /* a size does not fit the engine's index types */
    GI_EIO = 6,          /* file missing, short read, bad .g checksum */
    GI_ENOTSUP = 7,      /* option not supported by this build */
    GI_EDISCONNECTED = 8 /* pattern is not connected (reference throws) */
} gi_status;

typedef struct gi_graph gi_graph;           /* CSR resident on one GPU */
typedef struct gi_plan gi_plan;             /* immutable Schedule_IEP */
typedef struct gi_labeled_graph gi_labeled_graph;
typedef void *gi_stream;                    /* a cudaStream_t; NULL = legacy default stream */

/* Human-readable text of a status, and of the calling thread's last failure. */
const char *gi_status_string(int status);
const char *gi_last_error(void);
int gi_version(void);

/* ------------------------------------------------------------------ graph */

/* Replaces Graph + PatternMatchingDeviceContext::init's CSR upload
 * (reference include/graph.h:12-33, gpu/function/pattern_matching.cuh:18-81).
 * vertex[v_cnt+1] int64 offsets, edge[e_cnt] int32 sorted adjacency, e_cnt =
 * directed entries (twice the undirected edges).  The library copies both
 * arrays to the current device on `stream` and owns the copy.  tri_cnt feeds
 * the analytic planner only. */
int gi_graph_create(const int64_t *vertex, const int32_t *edge, int32_t v_cnt, int64_t e_cnt,
                    int64_t tri_cnt, gi_stream stream, gi_graph **out);
/* Replaces DataLoader::fast_load (reference src/dataloader.cpp:78-124). */
int gi_graph_load_g(const char *path, gi_graph **out);
int gi_graph_destroy(gi_graph *g);

typedef struct gi_graph_info {
    int32_t v_cnt;
    int64_t e_cnt;
    int64_t tri_cnt;
    int32_t max_degree;
    int32_t max_intersection_size; /* second-largest degree (reference src/dataloader.cpp:297-301) */
    int32_t n_hubs;                /* vertices whose adjacency the counting kernels test through a
                                      bitmap: all of degree >= hub_min_degree (their bitmaps are
                                      held to 4 GiB per graph by default, at most a sixteenth of the
                                      free device memory; GI_HUB_BITMAP_MB) */
    int32_t hub_min_degree;
    int32_t hash_min_degree;       /* vertices of at least this degree have an adjacency hash set
                                      (at most 4 GiB per graph by default; GI_HASH_MB) */
    int64_t hash_slots;            /* 32-bit slots of all hash sets */
} gi_graph_info;
int gi_graph_get_info(const gi_graph *g, gi_graph_info *out);

/* --------------------------------------------------------- .g file format */
/* 32-byte header {i32 v_cnt, 4 pad, i64 e_cnt, u32 max_intersection_size,
 * u32 checksum, i64 tri_cnt}; the header's 32-bit words sum to zero
 * (reference src/dataloader.cpp:21-47).  Host only, no GPU needed. */
int gi_g_write(const char *path, const int64_t *vertex, const int32_t *edge, int32_t v_cnt, int64_t e_cnt,
               uint32_t max_intersection_size, int64_t tri_cnt);
int gi_g_read_header(const char *path, int32_t *v_cnt, int64_t *e_cnt, uint32_t *max_intersection_size,
                     int64_t *tri_cnt);
/* Reads the arrays into caller buffers of at least v_cnt+1 / e_cnt entries. */
int gi_g_read(const char *path, int64_t *vertex, int32_t *edge, int32_t v_cap, int64_t e_cap);

/* ------------------------------------------------------------------- plan */

/* Replaces Schedule_IEP(Pattern(n, adj), valid, model, 1, enable_iep, v_cnt,
 * e_cnt, tri_cnt) (reference include/schedule_IEP.h:15-18,
 * src/schedule_IEP.cpp:12-247; gpu/gpu_graph.cu:102).  model 1 = the
 * reference's analytic model, 0 = keep the pattern's own order: both give
 * the reference's plan, and its count, bit for bit.  model 2 = the same
 * analytic model over the candidates whose restriction set is valid (every
 * subgraph passes its restrictions equally often), divided by that exact
 * multiplicity: an exact count even for patterns where the reference's own
 * restriction generator picks an invalid set.  Returns
 * GI_EDISCONNECTED for a disconnected pattern and GI_EINVAL for n outside
 * [3, 7] or an adjacency string shorter than n*n. */
int gi_plan_create(int n, const char *adj, int32_t v_cnt, int64_t e_cnt, int64_t tri_cnt, int model,
                   int enable_iep, gi_plan **out);
/* A candidate schedule given explicitly: order[i] is the pattern vertex at
 * position i; restricts holds n_restricts (first, second) position pairs
 * meaning id(position second) < id(position first).  The count is exact:
 * GI_EINVAL if the restriction set counts some subgraphs more often than
 * others. */
int gi_plan_create_explicit(int n, const char *adj, const int32_t *order, const int32_t *restricts,
                            int n_restricts, int enable_iep, gi_plan **out);
/* Replaces Schedule_IEP(adj_mat, size): vertex-induced, given order, no
 * restrictions, no IEP (reference src/schedule_IEP.cpp:249-290). */
int gi_plan_create_induced(int n, const char *adj, gi_plan **out);
int gi_plan_destroy(gi_plan *p);

/* A POD mirror of the Schedule_IEP arrays (reference include/schedule_IEP.h
 * :30-110).  The iep_vertex_flag / iep_vertex_coef / iep_ans_pos arrays hold
 * the entries the reference reads (the first iep_vertex_id_size /
 * iep_term_count entries of vectors it never clears between candidate
 * orders); *_raw_len give those vectors' full lengths. */
typedef struct gi_plan_desc {
    int32_t size;
    int32_t adj_mat[GI_MAX_PATTERN * GI_MAX_PATTERN];
    int32_t order[GI_MAX_PATTERN];
    int32_t total_prefix_num;
    int32_t basic_prefix_num;
    int32_t father_prefix_id[GI_MAX_PREFIX];
    int32_t last[GI_MAX_PATTERN];
    int32_t next[GI_MAX_PREFIX];
    int32_t loop_set_prefix_id[GI_MAX_PATTERN];
    int32_t break_size[GI_MAX_PREFIX];
    int32_t only_need_size[GI_MAX_PREFIX];
    int32_t prefix_len[GI_MAX_PREFIX];
    int32_t prefix_data[GI_MAX_PREFIX][GI_MAX_PATTERN];
    int32_t total_restrict_num;
    int32_t restrict_last[GI_MAX_PATTERN];
    int32_t restrict_next[GI_MAX_PREFIX];
    int32_t restrict_index[GI_MAX_PREFIX];
    int32_t n_restrict_pairs;
    int32_t restrict_pairs[GI_MAX_PREFIX][2];
    int32_t in_exclusion_optimize_num;
    int32_t iep_vertex_id_size;
    int32_t iep_vertex_id[GI_MAX_IEP_SETS];
    int32_t iep_vertex_flag[GI_MAX_IEP_SETS];
    int32_t iep_vertex_coef[GI_MAX_IEP_SETS];
    int32_t iep_term_count;
    int32_t iep_coef[GI_MAX_IEP_TERMS];
    int32_t iep_flag[GI_MAX_IEP_TERMS];
    int32_t iep_ans_pos[GI_MAX_IEP_TERMS];
    int64_t iep_vertex_flag_raw_len;
    int64_t iep_ans_pos_raw_len;
    int32_t is_vertex_induced;
    int64_t redundancy;
    int32_t k_val;
    int32_t multiplicity;
    double model_cost;
    int32_t iep_tables_rebuilt; /* 1 when the reference's own tables for this plan index
                                   past its IEP set list (an out-of-bounds read there) and
                                   the engine rebuilt them from the same order and
                                   restrictions */
    int64_t count_divisor;      /* the raw sum is divided by this: the redundancy for
                                   reference plans, the exact multiplicity otherwise */
    int32_t exact;              /* 1: the restrictions the DFS applies count every subgraph
                                   exactly count_divisor times, so the count is the true
                                   subgraph count; 0: they do not (the reference's restriction
                                   generator picked an invalid set; the count still equals the
                                   reference's); -1: vertex-induced plan, not checked */
} gi_plan_desc;
int gi_plan_export(const gi_plan *p, gi_plan_desc *out);
/* Full never-cleared vectors: which = 0 vertex_flag, 1 vertex_coef,
 * 2 ans_pos.  Copies up to cap entries, returns the length in *len. */
int gi_plan_export_raw(const gi_plan *p, int which, int32_t *buf, int64_t cap, int64_t *len);

/* Candidate (order, restriction set, analytic cost) triples in the order the
 * reference model scores them (reference src/schedule_IEP.cpp:67-177).  Pass
 * orders = NULL to query the count.  orders: cap*n ints; restricts: cap*
 * GI_MAX_PREFIX*2 ints; n_restricts, costs, divisors: cap entries (divisor 0
 * marks a restriction set that does not count every subgraph equally). */
int gi_plan_candidates(int n, const char *adj, int32_t v_cnt, int64_t e_cnt, int64_t tri_cnt, int enable_iep,
                       int32_t *orders, int32_t *restricts, int32_t *n_restricts, double *costs,
                       int32_t *divisors, int64_t cap, int64_t *count);

/* --------------------------------------------------------------- counting */

typedef struct gi_stats {
    double kernel_ms;        /* device time of the counting kernel(s), CUDA events */
    uint64_t raw_sum;        /* sum before the division by redundancy (mod 2^64) */
    uint64_t tasks;          /* first-level edge tasks that passed the depth-1 filters */
    uint64_t alg_bytes;      /* algorithmic bytes, filled when count_bytes != 0 */
    int32_t count_bytes;     /* in: 1 = run the instrumented kernel that also sums alg_bytes */
    double budget_ms;        /* in: > 0 = stop claiming work after this much device time and
                                return GI_ETIMEOUT (checked between tasks, never a wait) */
    int32_t grid_blocks;     /* out: persistent blocks launched */
    int32_t block_threads;   /* out */
    int32_t kernel_launches; /* out: kernels of this library launched by the call */
    int32_t allow_partial;   /* in (gi_count_shard only): with budget_ms > 0, return GI_OK and a
                                partial raw_sum when the budget runs out.  Work items are then
                                visited in a fixed pseudo-random order, no new item starts after
                                budget_ms and items still running at 3 * budget_ms are dropped,
                                so the completed items are a random sample of the shard */
    int64_t chunks_done;     /* out: work chunks (GI_TASK_CHUNK subtasks each) counted */
    int64_t chunks_total;    /* out: work chunks in the shard */
    double prep_ms;          /* out: device time of the work-split pre-pass (once per count,
                                not included in kernel_ms) */
    int64_t sample_chunks;   /* in (gi_count_shard only): > 0 = count only the first
                                sample_chunks chunks of the shard in the same fixed pseudo-random
                                order, all of them to completion: a uniform sample whose chunks,
                                and hence raw_sum, are the same on every call */
    int64_t edge_step;       /* in (gi_count_shard only): > 1 = count only the first-level tasks of
                                the directed edges e with e % edge_step == edge_offset, each whole:
                                the raw sum the reference's per-edge task (reference
                                src/graph.cpp:392-427) gives summed over exactly those edges.
                                Subsets of offsets 0 .. edge_step-1 add up to the whole count */
    int64_t edge_offset;     /* in: 0 <= edge_offset < edge_step */
} gi_stats;

/* Replaces gpu_pattern_matching<<<...>>> + the D2H of dev_sum + the
 * division by redundancy (reference gpu/gpu_graph.cu:22-51,
 * gpu/src/gpu_pattern_matching.cuh:14-104).  Blocks until the count is on
 * the host.  stats may be NULL. */
int gi_count(const gi_graph *g, const gi_plan *p, gi_stream stream, uint64_t *out_count, gi_stats *stats);

#define GI_TASK_CHUNK 32 /* consecutive first-level edges per claimed work item */

/* Partial count over shard `shard` of `num_shards`.  First-level tasks (the
 * directed edges) are grouped in chunks of GI_TASK_CHUNK consecutive edges;
 * chunk c belongs to shard c % num_shards — the reference's static
 * multi-device interleave (reference gpu/src/
 * gpu_pattern_matching_static_task.cuh:63, driven per device by
 * gpu/gpu_graph_static_task.cu).  *raw_sum receives the shard's sum modulo
 * 2^64, not divided: the shards' sums add up (mod 2^64) to the whole
 * graph's raw sum, which the caller divides by gi_plan_desc.count_divisor
 * after reducing across devices.  stats->alg_bytes excludes the per-start-
 * vertex depth-0 aliases that gi_count adds. */
int gi_count_shard(const gi_graph *g, const gi_plan *p, int32_t shard, int32_t num_shards, gi_stream stream,
                   uint64_t *raw_sum, gi_stats *stats);

/* -------------------------------------------------------------- autotuner */

/* Kernel variant of a plan: changes the counting kernel's speed, never its
 * counts.  The reference has one configuration, fixed at compile time
 * (reference gpu/function/pattern_matching.cuh:7-9, gpu/gpu_graph.cu:33). */
typedef struct gi_variant {
    int32_t leaf_flat;   /* 1: leaf probes spread evenly over a warp's lanes; 0: a candidate per lane */
    int32_t lane_budget; /* leaf_flat 0: candidates costlier than this run on the whole warp (0 = keep) */
    int32_t occupancy;   /* resident blocks per SM the kernel is built for: 1, 16, or 0 = by pattern size */
    int32_t split;       /* depth-2 candidates per work item (0 = 256 when depth 2 is the leaf, else 32) */
    int32_t leaf_handoff; /* leaf loop ranges of at least twice this go to idle warps (0 = 64) */
    int32_t mid_handoff; /* intermediate loop ranges of at least twice this go to idle warps (0 = 4) */
    int32_t edge_triangles; /* 1: count from per-edge triangle counts of the degree-oriented DAG; only
                               for plans ending at depth 2 in an IEP tail over N(v0), N(v1) and
                               N(v0) ∩ N(v1) (the diamond, books), else ignored */
} gi_variant;
int gi_plan_get_variant(const gi_plan *p, gi_variant *out);
int gi_plan_set_variant(gi_plan *p, const gi_variant *v);

typedef struct gi_tune_options {
    int64_t sample_edges; /* first-level edges in the timed sample (0 = 16384) */
    double max_ms;        /* a variant slower than this on the sample is dropped (0 = 250) */
    int32_t reps;         /* timed runs per variant, the fastest kept (0 = 2) */
    int32_t use_cache;    /* 1: reuse a choice cached for the same class of plan and graph */
    int32_t quick;        /* 1: a short search (the leaf modes and the edge-triangle path at the
                             default occupancy, the other occupancy, the split; one run each),
                             for callers that tune many classes at once */
    int32_t lookup_only;  /* 1: only apply a cached choice; time nothing (cached = 0 when none) */
} gi_tune_options;

typedef struct gi_tune_info {
    gi_variant chosen;
    int32_t cached;       /* 1: taken from the cache, nothing timed */
    int32_t candidates;   /* variants timed */
    double best_ms;       /* the chosen variant's time on the sample */
    double default_ms;    /* the plan's own variant's time on the sample */
    int64_t sample_edges; /* first-level edges timed */
} gi_tune_info;

/* Times every variant (leaf spread or per lane with lane budgets 256 and
 * 2048, each at occupancy 1 and 16) on an edge subset of g (each task
 * whole; every variant must give the same raw sum, else GI_ECUDA; the
 * subset is first resized until the plan's own variant takes between a
 * fiftieth of max_ms and max_ms, starting from sample_edges edges), sets
 * the fastest in p and caches it for the class of (p, g): pattern size, IEP
 * depth, depth-2 split, first-level restriction, log4 of the edge count and
 * of the largest degree.  gi_batch_create applies cached choices to its
 * jobs.  opt and info may be NULL.  The call changes p's variant (never its
 * counts): do not run it while another thread counts with p. */
int gi_autotune(const gi_graph *g, gi_plan *p, gi_stream stream, const gi_tune_options *opt, gi_tune_info *info);
int gi_autotune_clear(void);

/* No counterpart in the reference.  The count of gi_count for callers that
 * must not allocate device memory when they ask for it: code whose GPU
 * memory is owned by another framework's pool, a serving loop that cannot
 * afford cudaMalloc's latency and implicit synchronisation, a plug-in host
 * that forbids allocations inside a request.  The caller passes the CSR it
 * already holds on the current device (d_vertex[v_cnt+1] int64 offsets,
 * d_edge[e_cnt] int32 sorted adjacency, as for gi_graph_create) and a device
 * buffer d_result of two uint64: [0] the count, [1] the raw sum modulo 2^64.
 * All working memory comes from one fixed device array of
 * GI_NOALLOC_SCRATCH_BYTES that every GPU loading this code holds until the
 * process exits; the call allocates nothing (no cudaMalloc, no cudaFree, no
 * allocating library routine).  It launches as many warps as that array
 * holds and returns GI_EOVERFLOW when even one block of four warps would
 * need more (4 x materialised sets x second-largest degree x 4 bytes).  The
 * first call on a device looks up the array's device address, so make that
 * first call before any stream capture.  Calls share the array: two calls
 * that overlap on the GPU (other streams, other threads) race and give wrong
 * results.  Synchronous like gi_count; the CSR is checked on the device and
 * a malformed one gives GI_EINVAL. */
#define GI_NOALLOC_SCRATCH_BYTES (64u << 20)
int gi_count_noalloc(const int64_t *d_vertex, const int32_t *d_edge, int32_t v_cnt, int64_t e_cnt,
                     const gi_plan *p, gi_stream stream, uint64_t *d_result);

/* Replaces gpu_clique (reference gpu/gpu_clique.cu:573-639) when
 * orientation = 0: k-cliques on the id-oriented DAG (keep u < v,
 * reference src/graph.cpp:710-735); and gpu_kclique (reference
 * gpu/gpu_kclique.cu:517-546) when orientation = 1: degree orientation
 * (reference src/graph.cpp:821-859).  3 <= k <= 7. */
int gi_clique_count(const gi_graph *g, int k, int orientation, gi_stream stream, uint64_t *out_count,
                    gi_stats *stats);

/* No reference counterpart (the reference enumerates, gpu/gpu_kclique.cu).
 * The number of k-cliques for every k in [1, kmax] at once, counts[k]
 * (counts needs kmax + 1 entries; counts[0] = 0), by clique-tree pivoting
 * (Jain and Seshadhri, WSDM 2020) on the degree-oriented DAG's per-vertex
 * bitmaps, which gi_clique_count(..., 1) builds and keeps: one warp per root
 * vertex, cost growing with the pivot tree rather than with the number of
 * cliques.  1 <= kmax <= 7.  GI_ENOTSUP when an out-degree exceeds the
 * bitmap limit (4096), GI_ENOMEM when the bitmaps do not fit. */
int gi_clique_counts_pivot(const gi_graph *g, int kmax, gi_stream stream, uint64_t *counts, gi_stats *stats);

/* Replaces gpu_mc (reference gpu/gpu_mc.cu:62-119): edge-induced counts of
 * every connected k-vertex pattern in the reference MotifGenerator order
 * (reference src/motif_generator.cpp:5-43).  out_counts needs room for
 * gi_motif_num(k) entries; adj_out (optional) receives k*k chars per motif. */
int gi_motif_num(int k);
int gi_motif_patterns(int k, char *adj_out, int cap);
int gi_motif_count(const gi_graph *g, int k, gi_stream stream, uint64_t *out_counts, int cap, gi_stats *stats);

/* -------------------------------------------------------- batched counts */

/* No single reference counterpart: the reference launches one kernel per
 * (pattern, graph) (gpu/gpu_graph.cu:22-51; gpu/gpu_mc.cu:93-112 loops over
 * patterns).  A batch fixes n_jobs (graph, plan) pairs, job i =
 * (graphs[i], plans[i]), all graphs on one device; the handles must outlive
 * the batch.  gi_batch_run counts every job in one persistent launch (the
 * first run captures it in a CUDA graph, later runs replay it) and writes
 * counts[i] (gpu_graph semantics, as gi_count) and, optionally, job_ms[i]:
 * device time from the launch's first warp to the end of job i's last work
 * item.  Runs of one batch must not overlap. */
typedef struct gi_batch gi_batch;
int gi_batch_create(gi_graph *const *graphs, const gi_plan *const *plans, int n_jobs, gi_batch **out);
int gi_batch_run(gi_batch *b, gi_stream stream, uint64_t *counts, double *job_ms, gi_stats *stats);
int gi_batch_destroy(gi_batch *b);

/* ------------------------------------------- learned schedule cost model */

/* No reference counterpart: the reference picks a schedule with its analytic
 * model only (src/schedule_IEP.cpp:307-382).  A small MLP trained on
 * engine-measured device times (graphindor_b200/schedule_cost/train.py)
 * re-ranks the best valid candidate schedules (order + restriction set) of a
 * pattern for a graph described by GI_GRAPH_FEATURES floats. */
#define GI_GRAPH_FEATURES 19
/* Loads the model file written by train.py (process-wide; replaces any
 * loaded model). */
int gi_cost_model_load(const char *path);
/* The graph features of a graph handle, or of host CSR offsets. */
int gi_graph_features(const gi_graph *g, float *out, int cap);
int gi_graph_features_host(const int64_t *vertex, int32_t v_cnt, int64_t tri_cnt, float *out, int cap);
/* The model re-ranks the GI_LEARNED_CANDIDATES valid candidates of lowest
 * analytic cost (ties: enumeration order), the region of the candidate space
 * its training timings cover; the analytic model stays the first filter. */
#define GI_LEARNED_CANDIDATES 16
/* Of those, the one with the smallest predicted time (ties: enumeration
 * order), as gi_plan_create_explicit builds it (exact counts).  predicted_ms
 * (optional) receives the model's prediction. */
int gi_plan_create_learned(int n, const char *adj, int32_t v_cnt, int64_t e_cnt, int64_t tri_cnt,
                           const float *graph_features, int enable_iep, gi_plan **out, double *predicted_ms);
/* Training kernels of that model (3-layer MLP, fp32, ReLU, mean squared
 * error, Adam).  params: W1 [hidden x in], b1, W2 [hidden x hidden], b2, w3,
 * b3, the model file's order.  gi_mlp_grad: the loss gradient over all rows
 * (rows x in inputs X, targets y) and the loss; gi_mlp_train: `epochs`
 * passes of minibatches of `batch` rows in a seeded shuffle, weight decay wd
 * on W1, W2 and w3, params updated in place, loss = the final loss over all
 * rows. */
int gi_mlp_grad(const float *X, const float *y, int rows, int in, int hidden, const float *params, float *grad_out,
                float *loss_out);
/* The model's output (log10 predicted ms) for each of `rows` normalised
 * feature rows, on the GPU. */
int gi_mlp_predict(const float *X, int rows, int in, int hidden, const float *params, float *y_out);
int gi_mlp_train(const float *X, const float *y, int rows, int in, int hidden, int epochs, int batch, float lr,
                 float wd, uint64_t seed, float *params_inout, float *loss_out);

/* --------------------------------------------------- labeled graphs + FSM */

/* Replaces DataLoader::load_labeled_data (reference src/dataloader.cpp:
 * 381-625).  The input is the reference's .adj content: v_cnt vertices,
 * each with an original label value and a neighbour list (both directions
 * of every edge listed; self-loops are skipped as the reference skips
 * them; duplicates are kept).  Labels are renamed 0..l_cnt-1 by descending
 * maximum degree (first-seen order, then the reference's unstable sort for
 * ties), vertices are renumbered by (label, -degree, id), and every
 * neighbour list is bucketed by neighbour label.  `order` lists the vertices
 * in the order their lines appeared (NULL = ascending id); it fixes the
 * first-seen label order.  GI_EINVAL for an id out of range or a neighbour
 * list that is not symmetric.  The structure is copied to the current device. */
int gi_labeled_graph_create(int32_t v_cnt, const int64_t *vertex, const int32_t *edge, const uint32_t *labels,
                            const int32_t *order, gi_labeled_graph **out);
/* The same structure as gi_labeled_graph_create, built on the current device
 * (GPU ingest; reference src/dataloader.cpp:440-620 does it on the host):
 * degrees, the symmetry check, the renumbering by (label, -degree, id), the
 * renamed and sorted neighbour lists and the label buckets are computed by
 * kernels and device sorts; only the first-seen label pass and the sort of
 * at most 255 (label, maximum degree) pairs run on the host.  The bucketed
 * lists stay on the device (gi_labeled_graph_export downloads them).
 * Additionally GI_EOVERFLOW for 2^31 or more neighbour entries. */
int gi_labeled_graph_create_device(int32_t v_cnt, const int64_t *vertex, const int32_t *edge, const uint32_t *labels,
                                   const int32_t *order, gi_stream stream, gi_labeled_graph **out);
/* Parses a .adj text file: first token v_cnt, then one line per vertex
 * "id label nbr nbr ...". */
int gi_labeled_graph_load_adj(const char *path, gi_labeled_graph **out);
int gi_labeled_graph_destroy(gi_labeled_graph *g);

typedef struct gi_labeled_graph_info {
    int32_t v_cnt;
    int64_t e_cnt; /* directed entries */
    int32_t l_cnt;
    int32_t device;
} gi_labeled_graph_info;
int gi_labeled_graph_get_info(const gi_labeled_graph *g, gi_labeled_graph_info *out);
/* Host copies of the renumbered structure: new_id[v_cnt] (original id -> new
 * id), v_label[v_cnt], label_value[l_cnt] (original value of each new
 * label), label_start[l_cnt+1], bucket[v_cnt*l_cnt+1] (start of the bucket
 * of (v, l) in edge), edge[e_cnt].  Any pointer may be NULL. */
int gi_labeled_graph_export(const gi_labeled_graph *g, int32_t *new_id, int32_t *v_label, uint32_t *label_value,
                            uint32_t *label_start, uint32_t *bucket, uint32_t *edge);

#define GI_FSM_MAX_PATTERNS 64
/* One unlabeled pattern of an FSM run, as planned and as counted. */
typedef struct gi_fsm_pattern {
    int32_t n;                   /* vertices */
    int32_t edges;
    char adj[GI_MAX_PATTERN * GI_MAX_PATTERN]; /* '0'/'1', in schedule order */
    int32_t n_restricts;
    int32_t restricts[21][2];    /* (d, r): label at d <= label at r */
    int32_t n_automorphisms;
    int64_t jobs;                /* labeled patterns whose sub-patterns are all frequent */
    int64_t frequent;            /* of those, with MNI support >= min_support */
    double kernel_ms;
} gi_fsm_pattern;

typedef struct gi_fsm_stats {
    double kernel_ms;            /* device time of the support kernels */
    double total_ms;             /* host wall time of the whole call */
    int64_t jobs;
    int64_t candidates;          /* (labeled pattern, vertex, candidate) checks run */
    int32_t kernel_launches;
    int32_t n_patterns;          /* entries written to `patterns` */
    gi_fsm_pattern *patterns;    /* in: optional array of GI_FSM_MAX_PATTERNS */
} gi_fsm_stats;

/* Replaces gpu_fsm's fsm_init (reference gpu/gpu_fsm.cu:779-925) and
 * LabeledGraph::fsm (reference src/labeled_graph.cpp:540-606): the number of
 * frequent labeled patterns with exactly max_edge edges.  Every connected
 * pattern with at most max_edge edges is planned with the analytic model on
 * (v_cnt, e_cnt, tri_cnt) — the reference passes a fixed triangle count per
 * dataset (gpu_fsm: YouTube 103017122, fsm_test: Patents 7515023).  Labeled
 * patterns are enumerated under the plan's restrictions with Apriori
 * pruning; a labeled pattern is frequent when its MNI support (minimum over
 * pattern vertices of the number of distinct graph vertices that vertex
 * maps to) reaches min_support >= 1.  0 <= max_edge <= 6. */
int gi_fsm(gi_labeled_graph *g, int max_edge, int64_t min_support, int64_t tri_cnt, gi_stream stream,
           int64_t *out_fsm_cnt, gi_fsm_stats *stats);
/* Plans only (no device work): fills `patterns` as gi_fsm would, with jobs
 * and frequent left at 0. */
int gi_fsm_plan(int max_edge, int32_t v_cnt, int64_t e_cnt, int64_t tri_cnt, gi_fsm_pattern *patterns, int cap,
                int *count);

#ifdef __cplusplus
}
#endif

#endif /* GRAPHINDOR_B200_GI_H */
