// Test and baseline infrastructure: times the reference's own CPU counting
// code on a bounded sample of a workload.  Built only by oracle/Makefile
// against the reference sources (output in oracle/_ref/, never shipped).
//
// The reference's pm_test counts a whole graph (hours at the workload's
// size).  This driver enters the reference's DFS through its per-edge task,
// Graph::pattern_matching_edge_task (reference src/graph.cpp:392-427: depth 0
// and 1 built from one directed edge, then pattern_matching_aggressive_func),
// on every stride-th directed edge, with the plan the reference's own
// Schedule_IEP(pattern, valid, 1, 1, iep, v_cnt, e_cnt, tri_cnt) makes from
// the .g header (reference gpu/gpu_graph.cu:102).  Summed over all edges
// these tasks give the whole raw count.
//
//   ref_edge_sample <graph.g> <iep 0|1> <target_seconds> <threads> <n> <adj> [<n> <adj> ...]
//
// Per pattern the stride starts at 2^22 and is divided by 4 until one sample
// takes at least target/4 seconds (or the stride is 1); no edge is begun once
// 2 * target seconds have passed.  One line per pattern:
//   <adj> raw <raw sum mod 2^64> done <edges counted> stride <s> seconds <t> redundancy <r>
// The time covers the counting only (the graph is loaded before).
#include "dataloader.h"
#include "graph.h"
#include "pattern.h"
#include "schedule_IEP.h"
#include "vertex_set.h"

#include <omp.h>

#include <atomic>
#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>

namespace {

double now_s() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// One timed sample: edges 0, stride, 2 * stride, ... with no edge begun once
// max_seconds have passed.  Returns the raw sum; *done = edges counted.
unsigned long long sample(Graph *g, const Schedule_IEP &s, long long stride, double max_seconds, int threads,
                          long long *done, double *seconds) {
    const long long n_items = (static_cast<long long>(g->e_cnt) + stride - 1) / stride;
    std::atomic<bool> stop(false);
    unsigned long long raw = 0;
    long long counted = 0;
    const double t0 = now_s();
#pragma omp parallel num_threads(threads) reduction(+ : raw, counted)
    {
        int *ans_buffer = new int[s.in_exclusion_optimize_vertex_id.size() + 1];
        VertexSet *sets = new VertexSet[s.get_total_prefix_num() + 10];
        VertexSet partial, tmp;
        partial.init();
        tmp.init();
#pragma omp for schedule(dynamic, 1)
        for (long long k = 0; k < n_items; ++k) {
            if (stop.load(std::memory_order_relaxed)) continue;
            if (now_s() - t0 > max_seconds) {
                stop.store(true, std::memory_order_relaxed);
                continue;
            }
            raw += static_cast<unsigned long long>(
                g->pattern_matching_edge_task(s, static_cast<int>(k * stride), sets, partial, tmp, ans_buffer));
            ++counted;
        }
        delete[] sets;
        delete[] ans_buffer;
    }
    *seconds = now_s() - t0;
    *done = counted;
    return raw;
}

}  // namespace

int main(int argc, char **argv) {
    if (argc < 7 || (argc - 5) % 2 != 0) {
        std::fprintf(stderr, "usage: %s graph.g iep target_seconds threads n adj [n adj ...]\n", argv[0]);
        return 2;
    }
    const bool iep = std::atoi(argv[2]) != 0;
    const double target = std::atof(argv[3]);
    const int threads = std::max(1, std::atoi(argv[4]));
    DataLoader loader;
    Graph *g = nullptr;
    if (!loader.fast_load(g, argv[1])) {
        std::fprintf(stderr, "cannot load %s\n", argv[1]);
        return 1;
    }
    // Source of every directed edge (the reference's GPU path fills the same
    // array, gpu/function/pattern_matching.cuh:27-31).
    g->edge_from = new int[g->e_cnt];
    for (int v = 0; v < g->v_cnt; ++v)
        for (long long e = g->vertex[v]; e < g->vertex[v + 1]; ++e) g->edge_from[e] = v;
    for (int a = 5; a + 1 < argc; a += 2) {
        const int n = std::atoi(argv[a]);
        const char *adj = argv[a + 1];
        if (n < 3 || n > 7 || static_cast<int>(std::strlen(adj)) < n * n) {
            std::fprintf(stderr, "bad pattern %s\n", adj);
            return 2;
        }
        Pattern p(n, adj);
        bool valid = true;
        Schedule_IEP s(p, valid, 1, 1, iep, g->v_cnt, g->e_cnt, g->tri_cnt);
        if (!valid) {
            std::fprintf(stderr, "invalid pattern %s\n", adj);
            return 1;
        }
        long long stride = 1ll << 22, done = 0;
        double seconds = 0.0;
        unsigned long long raw = 0;
        while (true) {
            raw = sample(g, s, stride, 2.0 * target, threads, &done, &seconds);
            if (seconds >= target / 4.0 || stride == 1) break;
            stride /= 4;
        }
        std::printf("%s raw %llu done %lld stride %lld seconds %.6f redundancy %lld\n", adj, raw, done, stride,
                    seconds, static_cast<long long>(s.get_in_exclusion_optimize_redundancy()));
        std::fflush(stdout);
    }
    delete g;
    return 0;
}
