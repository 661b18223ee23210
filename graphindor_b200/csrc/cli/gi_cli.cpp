// Command-line front ends with the reference's argv and stdout lines, so the
// reference's orchestration (reproduce/utils.py parses "Counting time cost")
// keeps working.  Each tool is this file compiled with -DGI_TOOL=<n>:
//   1 gpu_graph   <graph.g> <pattern_size> <pattern_adj> [enable_iep]  (reference gpu/gpu_graph.cu:53-114)
//   2 gpu_clique  <graph.g> <clique_size>                             (reference gpu/gpu_clique.cu:573-639)
//   3 gpu_kclique <graph.g> <clique_size>                             (reference gpu/gpu_kclique.cu:517-546)
//   4 gpu_mc      <graph.g> <motif_size>                              (reference gpu/gpu_mc.cu:62-119)
//   5 gpu_fsm     <graph.adj> <max_edge> <min_support>                (reference gpu/gpu_fsm.cu:926-950)
// Each prints the same result line as the reference tool ("Pattern count:",
// "count", "Answer:", one "Pattern count:" per motif, "fsm cnt =") and
// "Counting time cost: X s".  Failures go to stderr with the status text; no tool calls
// exit() from inside the library.
#include <sys/time.h>

#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "gi.h"

#ifndef GI_TOOL
#define GI_TOOL 1
#endif

namespace {

double now_s() {
    timeval tv;
    gettimeofday(&tv, nullptr);
    return tv.tv_sec + tv.tv_usec * 1e-6;
}

int report(int status, const char *what) {
    std::fprintf(stderr, "%s: %s (%s)\n", what, gi_status_string(status), gi_last_error());
    return 1;
}

// Edges (i, j), i < j, as the reference's Pattern::print does.
void print_pattern(int n, const char *adj) {
    for (int i = 0; i < n; ++i)
        for (int j = i + 1; j < n; ++j)
            if (adj[i * n + j] == '1' || adj[j * n + i] == '1') std::printf("(%d,%d) ", i, j);
    std::printf("\n");
}

gi_graph *load(const char *path) {
    gi_graph *g = nullptr;
    const double t0 = now_s();
    const int st = gi_graph_load_g(path, &g);
    if (st != GI_OK) {
        report(st, "data load failure");
        return nullptr;
    }
    std::fprintf(stderr, "Load data success! time: %g seconds\n", now_s() - t0);
    return g;
}

// Plans and counts one pattern; prints "Pattern count:"; returns seconds.
double count_one(gi_graph *g, int n, const char *adj, int iep, bool &ok) {
    gi_graph_info info;
    gi_graph_get_info(g, &info);
    gi_plan *p = nullptr;
    int st = gi_plan_create(n, adj, info.v_cnt, info.e_cnt, info.tri_cnt, 1, iep, &p);
    if (st != GI_OK) {
        ok = false;
        report(st, "pattern is invalid!");
        return 0;
    }
    // The kernel variant for this class of (plan, graph), timed on a sample
    // before the count (like planning, outside the counting time);
    // GI_TUNE=0 keeps the default variant.
    const char *tune = std::getenv("GI_TUNE");
    if (!tune || std::atoi(tune) != 0) {
        const double tt = now_s();
        gi_tune_info ti;
        if (gi_autotune(g, p, nullptr, nullptr, &ti) == GI_OK)
            std::fprintf(stderr, "Tuning time: %g seconds (leaf_flat %d, occupancy %d, split %d, edge_triangles %d)\n",
                         now_s() - tt, ti.chosen.leaf_flat, ti.chosen.occupancy, ti.chosen.split,
                         ti.chosen.edge_triangles);
    }
    const double t0 = now_s();
    uint64_t count = 0;
    st = gi_count(g, p, nullptr, &count, nullptr);
    const double dt = now_s() - t0;
    gi_plan_destroy(p);
    if (st != GI_OK) {
        ok = false;
        report(st, "count failed");
        return 0;
    }
    std::printf("Pattern count: %llu\n", static_cast<unsigned long long>(count));
    return dt;
}

}  // namespace

int main(int argc, char **argv) {
#if GI_TOOL == 1
    if (argc < 4) {
        std::fprintf(stderr, "Usage: %s graph_file pattern_size pattern_string <1/0 for enable iep or not>\n", argv[0]);
        return 1;
    }
    int iep = 1;
    if (argc >= 5) {
        iep = std::atoi(argv[4]);
        if (iep != 0 && iep != 1) {
            std::fprintf(stderr, "Usage: %s graph_file pattern_size pattern_string <1/0 for enable iep or not>\n",
                         argv[0]);
            return 1;
        }
    }
    gi_graph *g = load(argv[1]);
    if (!g) return 1;
    const int n = std::atoi(argv[2]);
    if (static_cast<int>(std::string(argv[3]).size()) < n * n) return report(GI_EINVAL, "pattern string too short");
    std::printf("pattern = ");
    print_pattern(n, argv[3]);
    bool ok = true;
    const double dt = count_one(g, n, argv[3], iep, ok);
    if (ok) std::printf("Counting time cost: %ld.%06ld s.\n", static_cast<long>(dt), static_cast<long>((dt - static_cast<long>(dt)) * 1e6));
    gi_graph_destroy(g);
    return ok ? 0 : 1;
#elif GI_TOOL == 2 || GI_TOOL == 3
    if (argc != 3) {
        std::printf("usage: %s graph_file clique_size\n", argv[0]);
        return 0;
    }
    gi_graph *g = load(argv[1]);
    if (!g) return 1;
    const int k = std::atoi(argv[2]);
    gi_graph_info info;
    gi_graph_get_info(g, &info);
    const double t0 = now_s();
    uint64_t count = 0;
    int st = GI_OK;
    if (k == 1) {
        count = static_cast<uint64_t>(info.v_cnt);
    } else if (k == 2) {
        count = static_cast<uint64_t>(info.e_cnt / 2);
    } else {
        st = gi_clique_count(g, k, GI_TOOL == 2 ? 0 : 1, nullptr, &count, nullptr);
    }
    const double dt = now_s() - t0;
    gi_graph_destroy(g);
    if (st != GI_OK) return report(st, "clique count failed");
    if (GI_TOOL == 2)
        std::printf("count %llu\n", static_cast<unsigned long long>(count));
    else
        std::printf("Answer: %llu\n", static_cast<unsigned long long>(count));
    std::printf("Counting time cost: %.6lf s.\n", dt);
    return 0;
#elif GI_TOOL == 5
    if (argc < 4) {
        std::fprintf(stderr, "Usage: %s graph.adj max_edge min_support\n", argv[0]);
        return 1;
    }
    gi_labeled_graph *g = nullptr;
    const double t_load = now_s();
    int st = gi_labeled_graph_load_adj(argv[1], &g);
    if (st != GI_OK) return report(st, "data load failure");
    std::fprintf(stderr, "Load data success! time: %g seconds\n", now_s() - t_load);
    const int max_edge = std::atoi(argv[2]);
    const long long min_support = std::atoll(argv[3]);
    // gpu_fsm plans with the YouTube triangle count (reference gpu/gpu_fsm.cu:939).
    const double t0 = now_s();
    int64_t cnt = 0;
    st = gi_fsm(g, max_edge, min_support, 103017122LL, nullptr, &cnt, nullptr);
    const double dt = now_s() - t0;
    gi_labeled_graph_destroy(g);
    if (st != GI_OK) return report(st, "fsm failed");
    std::printf("Counting time cost: %ld.%06ld s.\n", static_cast<long>(dt),
                static_cast<long>((dt - static_cast<long>(dt)) * 1e6));
    std::printf("fsm cnt = %lld\n", static_cast<long long>(cnt));
    return 0;
#else
    if (argc < 3) {
        std::fprintf(stderr, "Usage: %s graph_file pattern_size\n", argv[0]);
        return 1;
    }
    gi_graph *g = load(argv[1]);
    if (!g) return 1;
    const int k = std::atoi(argv[2]);
    std::printf("motif_size: %d\n", k);
    const int m = gi_motif_num(k);
    if (m < 0) return report(GI_EINVAL, "motif size must be between 3 and 7");
    std::printf("Motifs number = %d\n", m);
    std::vector<char> adj(static_cast<size_t>(m) * k * k + 1);
    gi_motif_patterns(k, adj.data(), m);
    double total = 0;
    bool ok = true;
    for (int i = 0; i < m && ok; ++i) {
        std::string a(adj.data() + static_cast<size_t>(i) * k * k, static_cast<size_t>(k) * k);
        std::printf("pattern = ");
        print_pattern(k, a.c_str());
        total += count_one(g, k, a.c_str(), 1, ok);
    }
    gi_graph_destroy(g);
    if (!ok) return 1;
    std::printf("Counting time cost: %.6lf s\n", total);
    return 0;
#endif
}
