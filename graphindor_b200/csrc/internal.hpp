// Shared definitions behind the C ABI (include/gi.h).
#pragma once

#include <cstdint>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/gi.h"
#include "planner.hpp"

namespace gi {

// Records a failure message for gi_last_error() and returns the status.
int fail(int status, const std::string &msg);

// Connected k-vertex patterns (row-major k*k 0/1 matrices) in the order of
// the reference MotifGenerator; k >= 2.  With max_edges, only those with at
// most that many edges (the same patterns, in the same order, as filtering
// the full list).
std::vector<std::vector<int>> motif_list(int k, int max_edges = 1 << 30);

// Makes `device` current for a scope and restores the caller's device on
// every exit path.
class DeviceGuard {
  public:
    explicit DeviceGuard(int device);
    ~DeviceGuard();
    DeviceGuard(const DeviceGuard &) = delete;
    DeviceGuard &operator=(const DeviceGuard &) = delete;

  private:
    int prev_ = -1, device_ = -1;
};

// CUDA events (timing) destroyed with the scope.
class ScopedEvents {
  public:
    explicit ScopedEvents(int n);
    ~ScopedEvents();
    ScopedEvents(const ScopedEvents &) = delete;
    ScopedEvents &operator=(const ScopedEvents &) = delete;
    void *operator[](int i) const { return ev_[i]; }  // a cudaEvent_t

  private:
    void *ev_[4] = {nullptr, nullptr, nullptr, nullptr};
    int n_ = 0;
};

// Per-prefix build mode used by the counting kernels.
enum PrefixMode : int32_t {
    kAlias = 0,        // father == -1: the set is N(v) itself, no copy
    kMaterialize = 1,  // S_father ∩ N(v) written to the warp's scratch slot
    kSizeOnly = 2,     // only |S_father ∩ N(v)| is ever read
};

// The plan as the device reads it: flat, fixed-size, passed by value as a
// kernel parameter.  Built once per gi_plan from the Schedule_IEP arrays.
struct DevPlan {
    int32_t n;                  // pattern size
    int32_t iep_k;              // in_exclusion_optimize_num (0 = no IEP tail)
    int32_t total_prefix;
    int32_t n_slots;            // materialised prefixes = scratch slots per warp
    int32_t first_restricted;   // restrict_last[1] != -1: tasks need v1 < v0
    int32_t vertex_induced;
    int32_t stop;               // depth closed in form: n - iep_k with IEP, else n - 1
    int32_t leaf_depth;         // stop - 1 when its candidates run one per lane, else -1
    int32_t lane_budget;        // leaf candidates costlier than this for one lane go to the warp
    int32_t leaf_flat;          // 1: leaf probes spread evenly over the warp's lanes (leaf_level_flat)
    int32_t flat_first;         // 1: the DFS ends at depth 2 and a chunk's edges are counted as one flat leaf
    int32_t flat_first_ok;      // the plan allows flat_first (set with leaf_flat)
    int32_t occupancy;          // resident blocks per SM the kernel is built for: 0 by pattern size, 1 or 16
    int32_t split;              // depth-2 candidates per subtask (0: 256 when depth 2 is the leaf, else 32)
    int32_t leaf_handoff;       // leaf ranges of at least twice this are donated (0: 64)
    int32_t mid_handoff;        // intermediate ranges of at least twice this are donated (0: 4)
    int32_t tri_ok;             // the plan can be counted from edge-triangle counts (tri_edge.cu)
    int32_t tri_edge;           // 1: count it that way (a variant; needs tri_ok)
    int32_t loop2_kind;         // bound of the depth-2 loop set: 0 d(v0), 1 d(v1), 2 min, -1 none
    int32_t pdepth[GI_MAX_PREFIX];  // last member (position) of each prefix
    int32_t father[GI_MAX_PREFIX];
    int32_t next[GI_MAX_PREFIX];
    int32_t break_size[GI_MAX_PREFIX];
    int32_t mode[GI_MAX_PREFIX];
    int32_t slot[GI_MAX_PREFIX];
    int32_t last[GI_MAX_PATTERN + 1];
    int32_t loop_set[GI_MAX_PATTERN + 1];
    int32_t restrict_last[GI_MAX_PATTERN + 1];
    int32_t restrict_next[GI_MAX_PREFIX];
    int32_t restrict_index[GI_MAX_PREFIX];
    int32_t adj[GI_MAX_PATTERN * GI_MAX_PATTERN];
    int32_t iep_nsets;
    int32_t iep_nterms;
    int32_t iep_set[GI_MAX_IEP_SETS];
    int32_t iep_set_flag[GI_MAX_IEP_SETS];
    int32_t iep_set_coef[GI_MAX_IEP_SETS];
    int32_t iep_coef[GI_MAX_IEP_TERMS];
    int32_t iep_flag[GI_MAX_IEP_TERMS];
    int32_t iep_pos[GI_MAX_IEP_TERMS];
};

// The even-spread leaf (leaf_level_flat) numbers the probes of 32 candidates
// with 32-bit ints: it is used only on graphs whose largest degree is below
// this.
constexpr int64_t kFlatLeafMaxDegree = int64_t(1) << 26;

// The plan as a kernel receives it for a graph of the given largest degree.
inline DevPlan plan_for_graph(const DevPlan &P, int64_t max_degree) {
    DevPlan d = P;
    if (max_degree >= kFlatLeafMaxDegree) d.leaf_flat = d.flat_first = 0;
    return d;
}

// Kernel variants (autotune.cpp): set a variant's fields in a plan, and the
// plan with the cached tuned variant of its class on graph g (false when
// none is cached).
void variant_apply(DevPlan &P, const gi_variant &v);
bool tuned_plan(const gi_graph *g, const DevPlan &P, DevPlan &out);

}  // namespace gi

struct gi_plan {
    std::unique_ptr<gi::Schedule_IEP> sched;
    gi::DevPlan dev;
    int multiplicity = 0;
    bool iep_tables_rebuilt = false;
};

// Implemented in device code (graph.cu / count.cu).
struct gi_graph {
    int device = 0;
    int32_t v_cnt = 0;
    int64_t e_cnt = 0;
    int64_t tri_cnt = 0;
    int32_t max_degree = 0;
    int32_t max_isect = 0;
    int64_t *d_vertex = nullptr;
    int32_t *d_edge = nullptr;
    uint32_t *d_edge_from = nullptr;
    // Scratch for the counting kernels, grown on demand; counts on one graph
    // handle are serialised by `mu`.
    std::mutex mu;
    void *d_scratch = nullptr;
    size_t scratch_bytes = 0;
    unsigned long long *d_counters = nullptr;  // [0] sum, [1] task cursor, [2] bytes, [3] tasks, ...
    // Per-edge subtask offsets (exclusive scan) for splitting the depth-2
    // loop, and the cub scan workspace; grown on demand.
    int64_t *d_offsets = nullptr;
    void *d_scan_tmp = nullptr;
    size_t scan_tmp_bytes = 0;
    // Features of the learned schedule cost model (schedule_cost.cpp):
    // log10 v_cnt, edges and triangles, then the share of vertices per
    // power-of-two degree bin.
    float graph_features[3 + 16] = {};
    // Work-donation queue of the counting kernel (kept between counts, its
    // ready flags tagged with a per-launch epoch so it never needs clearing).
    void *d_handoff = nullptr;
    uint32_t handoff_epoch = 0;
    // Lazily built derived graphs (clique orientations).
    gi_graph *oriented[2] = {nullptr, nullptr};
    // Per-vertex adjacency bitmaps of a degree-oriented DAG (kclique.cu),
    // built by the first k-clique count and kept: row i of vertex u has bit j
    // when out-neighbour j of u is an out-neighbour of out-neighbour i.
    uint32_t *d_bitmap = nullptr;
    int64_t *d_bitmap_off = nullptr;  // v_cnt + 1 word offsets
    int64_t bitmap_words = 0;
    // Roots of the clique-tree pivoting search, largest out-degree first
    // (kclique.cu), built with the bitmaps' first pivoting count and kept.
    int32_t *d_roots = nullptr;
    // Adjacency bitmaps of the hubs (every vertex of degree >= hub_min_degree;
    // graph.cu): n_hubs rows of hub_words 32-bit words, and hub_row[v] = the
    // row of hub v (-1 for other vertices).  Read by the counting DFS.
    uint32_t *d_hub_bits = nullptr;
    int32_t *d_hub_row = nullptr;
    int32_t n_hubs = 0;
    int32_t hub_min_degree = 0x7fffffff;
    int64_t hub_words = 0;
    // Open-addressing hash sets of the adjacency lists of every vertex of
    // degree >= hash_min_degree (graph.cu): vertex v's table is
    // d_hash[d_hash_off[v] .. d_hash_off[v+1]), a power of two at least twice
    // its degree, empty slots 0xffffffff.  Read by the counting DFS.
    uint32_t *d_hash = nullptr;
    int64_t *d_hash_off = nullptr;
    int32_t hash_min_degree = 0x7fffffff;
    int64_t hash_slots = 0;
    // Per-arc triangle counts of the degree-oriented DAG (tri_edge.cu),
    // recomputed by every edge-triangle count; the buffer is kept.
    void *d_tri_arc = nullptr;
    int64_t tri_arc_cap = 0;
};
