// Test infrastructure: prints every field of the reference's Schedule_IEP as
// one JSON object per input line, so the engine's planner can be compared
// field by field with the reference planner.  Built only by oracle/Makefile
// against the reference sources (output in oracle/_ref/, never shipped).
//
// stdin, one job per line:
//   full    <n> <adj-string> <v_cnt> <e_cnt> <tri_cnt> <enable_iep>
//       -> Schedule_IEP(Pattern(n, adj), valid, 1, 1, iep, v, e, tri)
//          (reference include/schedule_IEP.h:15-18, as gpu/gpu_graph.cu:102)
//   induced <n> <adj-string>
//       -> Schedule_IEP(adj_mat, n)  (reference src/schedule_IEP.cpp:249)
#include "pattern.h"
#include "schedule_IEP.h"
#include "motif_generator.h"

#include <cstdio>
#include <cstring>
#include <iostream>
#include <sstream>
#include <string>
#include <vector>

static void arr(const char *name, const int *p, int n) {
    printf("\"%s\":[", name);
    for (int i = 0; i < n; ++i) printf("%s%d", i ? "," : "", p[i]);
    printf("],");
}

template <class V> static void vec(const char *name, const V &v) {
    printf("\"%s\":[", name);
    for (size_t i = 0; i < v.size(); ++i) printf("%s%d", i ? "," : "", (int)v[i]);
    printf("],");
}

static void dump(const Schedule_IEP &s) {
    const int n = s.get_size();
    const int maxp = n * (n - 1) / 2 + 1;
    printf("{");
    printf("\"size\":%d,", n);
    arr("adj_mat", s.get_adj_mat_ptr(), n * n);
    printf("\"total_prefix_num\":%d,\"basic_prefix_num\":%d,", s.get_total_prefix_num(),
           s.get_basic_prefix_num());
    arr("father_prefix_id", s.get_father_prefix_id_ptr(), s.get_total_prefix_num());
    arr("last", s.get_last_ptr(), n);
    arr("next", s.get_next_ptr(), s.get_total_prefix_num());
    arr("loop_set_prefix_id", s.get_loop_set_prefix_id_ptr(), n);
    arr("break_size", s.get_break_size_ptr(), s.get_total_prefix_num());
    std::vector<int> only(s.get_total_prefix_num());
    for (int i = 0; i < s.get_total_prefix_num(); ++i) only[i] = s.get_prefix_only_need_size(i);
    vec("only_need_size", only);
    printf("\"total_restrict_num\":%d,", s.get_total_restrict_num());
    arr("restrict_last", s.get_restrict_last_ptr(), n);
    arr("restrict_next", s.get_restrict_next_ptr(), s.get_total_restrict_num());
    arr("restrict_index", s.get_restrict_index_ptr(), s.get_total_restrict_num());
    printf("\"restrict_pair\":[");
    for (size_t i = 0; i < s.restrict_pair.size(); ++i)
        printf("%s[%d,%d]", i ? "," : "", s.restrict_pair[i].first, s.restrict_pair[i].second);
    printf("],");
    printf("\"in_exclusion_optimize_num\":%d,", s.get_in_exclusion_optimize_num());
    vec("iep_vertex_id", s.in_exclusion_optimize_vertex_id);
    vec("iep_vertex_flag", s.in_exclusion_optimize_vertex_flag);
    vec("iep_vertex_coef", s.in_exclusion_optimize_vertex_coef);
    vec("iep_coef", s.in_exclusion_optimize_coef);
    vec("iep_flag", s.in_exclusion_optimize_flag);
    vec("iep_ans_pos", s.in_exclusion_optimize_ans_pos);
    printf("\"is_vertex_induced\":%d,", (int)s.is_vertex_induced);
    printf("\"redundancy\":%lld,\"maxp\":%d}\n", s.get_in_exclusion_optimize_redundancy(), maxp);
    (void)maxp;
}

int main() {
    std::string line;
    while (std::getline(std::cin, line)) {
        if (line.empty() || line[0] == '#') continue;
        std::istringstream in(line);
        std::string mode, adj;
        int n = 0;
        in >> mode >> n >> adj;
        try {
            if (mode == "full") {
                long long v = 0, e = 0, tri = 0;
                int iep = 1;
                in >> v >> e >> tri >> iep;
                Pattern p(n, adj.c_str());
                bool valid = false;
                Schedule_IEP s(p, valid, 1, 1, iep != 0, (int)v, (int64_t)e, tri);
                dump(s);
            } else if (mode == "induced") {
                std::vector<int> m(n * n, 0);
                for (int i = 0; i < n; ++i)
                    for (int j = 0; j < n; ++j)
                        if (adj[i * n + j] == '1') m[i * n + j] = m[j * n + i] = 1;
                Schedule_IEP s(m.data(), n);
                dump(s);
            } else if (mode == "motifs") {
                // motifs <k> -: the MotifGenerator list (reference
                // src/motif_generator.cpp:33-43) as n*n adjacency strings.
                MotifGenerator mg(n);
                std::vector<Pattern> list = mg.generate();
                printf("{\"motifs\":[");
                for (size_t m = 0; m < list.size(); ++m) {
                    printf("%s\"", m ? "," : "");
                    for (int i = 0; i < n * n; ++i) printf("%d", list[m].get_adj_mat_ptr()[i] ? 1 : 0);
                    printf("\"");
                }
                printf("]}\n");
            } else {
                printf("{\"error\":\"bad mode\"}\n");
            }
        } catch (const std::exception &ex) {
            printf("{\"error\":\"%s\"}\n", ex.what());
        }
        fflush(stdout);
    }
    return 0;
}
