// Labeled graphs and frequent subgraph mining (FSM): the structures shared
// by the host driver (fsm_host.cpp) and the support kernel (fsm.cu).
#pragma once

#include <cstdint>
#include <mutex>
#include <vector>

#include "../../include/gi.h"

// A labeled graph after the reference loader's renaming (reference
// src/dataloader.cpp:381-625): labels 0..l_cnt-1 by descending maximum
// degree, vertices sorted by (label, -degree, id), and each neighbour list
// sorted by (neighbour label, neighbour id) so that the neighbours of v with
// label l are edge[bucket[v*l_cnt+l] .. bucket[v*l_cnt+l+1]).
struct gi_labeled_graph {
    int device = 0;
    int32_t v_cnt = 0;
    int64_t e_cnt = 0;
    int32_t l_cnt = 0;
    std::vector<int32_t> new_id;           // original id -> new id
    std::vector<int32_t> v_label;          // by new id
    std::vector<uint32_t> label_value;     // original value of each new label
    std::vector<int64_t> label_frequency;  // vertices per label
    std::vector<uint32_t> label_start;     // l_cnt + 1
    std::vector<uint32_t> bucket;          // v_cnt * l_cnt + 1
    std::vector<uint32_t> edge;            // e_cnt
    uint32_t *d_edge = nullptr;
    uint32_t *d_bucket = nullptr;
    uint32_t *d_label_start = nullptr;
    // Built on the device (labeled_ingest.cu): edge and bucket exist only
    // there until an export downloads them.
    bool device_built = false;
    std::mutex mu;  // serialises the FSM runs on one handle
};

namespace gi {

// One unlabeled pattern as the support kernel reads it.  For every pattern
// vertex r the kernel can root an existence search at r: order[r][t] is the
// pattern vertex matched at step t (order[r][0] = r), and bit t' of
// parents[r][t] is set when steps t' < t and t are adjacent.
struct FsmDevPattern {
    int32_t n = 0;
    int32_t l_cnt = 0;
    int64_t min_support = 0;
    uint8_t order[GI_MAX_PATTERN][GI_MAX_PATTERN] = {};
    uint8_t parents[GI_MAX_PATTERN][GI_MAX_PATTERN] = {};
    uint8_t adj_mask[GI_MAX_PATTERN] = {};  // pattern neighbours of each vertex, as a bit mask
};

struct FsmRunStats {
    double kernel_ms = 0.0;
    int64_t candidates = 0;
    int launches = 0;
};

// Host copies of the lists and buckets of a graph built on the device
// (labeled_ingest.cu); nothing to do for a host-built graph.
int labeled_graph_download(const gi_labeled_graph *g);

// Copies the bucketed structure to the graph's device (fsm.cu).
int fsm_upload(gi_labeled_graph *g);
void fsm_free(gi_labeled_graph *g);

// Decides, for each of n_jobs labeled patterns (labels[j*n + i] = label of
// pattern vertex i), whether its MNI support reaches P.min_support; writes
// frequent[j] = 0/1.  One launch of the support kernel (fsm.cu).
int fsm_support(gi_labeled_graph *g, const FsmDevPattern &P, const std::vector<uint8_t> &labels, int64_t n_jobs,
                void *stream, std::vector<uint8_t> &frequent, FsmRunStats &st);

}  // namespace gi
