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
// Per pattern the stride starts at e_cnt rounded down to a power of 4 and is
// divided by 4 until one sample takes at least target/4 seconds (or the
// stride is 1); no edge is begun once 2 * target seconds have passed.  One
// line per pattern:
//   <adj> raw <raw sum mod 2^64> done <edges counted> stride <s> seconds <t> redundancy <r>
//
//   ref_edge_sample --edges <step> <offset> <parts> <graph.g> <iep> <threads> <n> <adj> [...]
//
// A fixed edge subset, counted whole: the directed edges e with
// e % step == offset (the engine's gi_stats.edge_step / edge_offset), in
// `parts` timed parts; part i holds the subset's edges offset + (i + j *
// parts) * step.  One line per pattern and part:
//   <adj> part <i> raw <raw sum mod 2^64> done <edges> seconds <t> redundancy <r>
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

// One timed sample: edges first, first + stride, first + 2 * stride, ...
// with no edge begun once max_seconds have passed (max_seconds <= 0: no
// limit).  Returns the raw sum; *done = edges counted.
unsigned long long sample(Graph *g, const Schedule_IEP &s, long long first, long long stride, double max_seconds,
                          int threads, long long *done, double *seconds) {
    const long long e_cnt = static_cast<long long>(g->e_cnt);
    const long long n_items = first < e_cnt ? (e_cnt - first + stride - 1) / stride : 0;
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
            if (max_seconds > 0 && now_s() - t0 > max_seconds) {
                stop.store(true, std::memory_order_relaxed);
                continue;
            }
            raw += static_cast<unsigned long long>(g->pattern_matching_edge_task(
                s, static_cast<int>(first + k * stride), sets, partial, tmp, ans_buffer));
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
    // Either "graph.g iep target threads patterns..." (adaptive stride) or
    // "--edges step offset parts graph.g iep threads patterns..." (fixed subset).
    long long fixed_step = 0, fixed_offset = 0, fixed_parts = 0;
    int a = 1;
    if (argc > 1 && std::strcmp(argv[1], "--edges") == 0) {
        if (argc < 5) return 2;
        fixed_step = std::atoll(argv[2]);
        fixed_offset = std::atoll(argv[3]);
        fixed_parts = std::atoll(argv[4]);
        if (fixed_step < 1 || fixed_offset < 0 || fixed_offset >= fixed_step || fixed_parts < 1) {
            std::fprintf(stderr, "bad --edges step offset parts\n");
            return 2;
        }
        a = 5;
    }
    const int fixed_args = fixed_step > 0 ? 3 : 4;  // graph, iep, [target,] threads
    const int first_pattern = a + fixed_args;
    if (argc < first_pattern + 2 || (argc - first_pattern) % 2 != 0) {
        std::fprintf(stderr,
                     "usage: %s graph.g iep target_seconds threads n adj [n adj ...]\n"
                     "       %s --edges step offset parts graph.g iep threads n adj [n adj ...]\n",
                     argv[0], argv[0]);
        return 2;
    }
    const char *path = argv[a];
    const bool iep = std::atoi(argv[a + 1]) != 0;
    const double target = fixed_step > 0 ? 0.0 : std::atof(argv[a + 2]);
    const int threads = std::max(1, std::atoi(argv[first_pattern - 1]));
    DataLoader loader;
    Graph *g = nullptr;
    if (!loader.fast_load(g, path)) {
        std::fprintf(stderr, "cannot load %s\n", path);
        return 1;
    }
    // Source of every directed edge (the reference's GPU path fills the same
    // array, gpu/function/pattern_matching.cuh:27-31).
    g->edge_from = new int[g->e_cnt];
    for (int v = 0; v < g->v_cnt; ++v)
        for (long long e = g->vertex[v]; e < g->vertex[v + 1]; ++e) g->edge_from[e] = v;
    for (int k = first_pattern; k + 1 < argc; k += 2) {
        const int n = std::atoi(argv[k]);
        const char *adj = argv[k + 1];
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
        const long long redundancy = static_cast<long long>(s.get_in_exclusion_optimize_redundancy());
        long long done = 0;
        double seconds = 0.0;
        unsigned long long raw = 0;
        if (fixed_step > 0) {
            for (long long part = 0; part < fixed_parts; ++part) {
                raw = sample(g, s, fixed_offset + part * fixed_step, fixed_step * fixed_parts, 0.0, threads, &done,
                             &seconds);
                std::printf("%s part %lld raw %llu done %lld seconds %.6f redundancy %lld\n", adj, part, raw, done,
                            seconds, redundancy);
                std::fflush(stdout);
            }
            continue;
        }
        long long stride = 1;
        while (stride * 4 <= static_cast<long long>(g->e_cnt)) stride *= 4;
        while (true) {
            raw = sample(g, s, 0, stride, 2.0 * target, threads, &done, &seconds);
            if (seconds >= target / 4.0 || stride == 1) break;
            stride /= 4;
        }
        std::printf("%s raw %llu done %lld stride %lld seconds %.6f redundancy %lld\n", adj, raw, done, stride,
                    seconds, redundancy);
        std::fflush(stdout);
    }
    delete g;
    return 0;
}
