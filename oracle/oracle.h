/*
 * ORACLE — test infrastructure only.
 *
 * A plain-C restatement of the reference's CPU counting path, used by tests/,
 * the smoke check and bench.py's CPU-baseline leg to check and time the CUDA
 * engine.  Nothing in the engine links, loads or calls it.
 *
 * Parity is pinned by tests against (a) the reference's own binaries built
 * from its sources by oracle/Makefile (counts on seeded graphs, committed
 * under tests/golden/) and (b) the reference's published triangle count for
 * Wiki-Vote and the survey-measured Wiki-Vote pattern counts.
 */
#ifndef GI_ORACLE_H
#define GI_ORACLE_H

#include <stdint.h>

#include "../include/gi.h"

#ifdef __cplusplus
extern "C" {
#endif

/* Count of the plan on the graph with the reference CPU path's semantics
 * (reference src/graph.cpp:305-355 pattern_matching, :429-566
 * pattern_matching_aggressive_func, src/vertex_set.cpp:203-277).  Start
 * vertices v0 in [v_begin, v_end) only (the whole graph: 0, v_cnt), run over
 * `threads` OpenMP threads (0 = all).  *raw_sum receives the sum before the
 * division by redundancy, modulo 2^64.  If alg_bytes is non-NULL it receives
 * the algorithmic bytes of the traversal (see oracle.c).  Returns 0, or -1
 * on bad input. */
int oracle_count(const gi_plan_desc *plan, const int64_t *vertex, const int32_t *edge, int32_t v_cnt,
                 int32_t v_begin, int32_t v_end, int threads, uint64_t *raw_sum, uint64_t *alg_bytes);

/* The same over the start vertices v_begin, v_begin + stride, ... < v_end:
 * an unbiased sample when vertex ids are randomly assigned (a contiguous id
 * range is not: restrictions anchor each subgraph at one end of its id
 * order).  Used for the timed CPU baseline. */
int oracle_count_strided(const gi_plan_desc *plan, const int64_t *vertex, const int32_t *edge, int32_t v_cnt,
                         int32_t v_begin, int32_t v_end, int32_t stride, int threads, uint64_t *raw_sum,
                         uint64_t *alg_bytes);

/* As oracle_count_strided, but no start vertex is begun once max_seconds
 * have passed; *processed receives how many start vertices were counted
 * (the sample is then those vertices). */
int oracle_count_timed(const gi_plan_desc *plan, const int64_t *vertex, const int32_t *edge, int32_t v_cnt,
                       int32_t stride, int threads, double max_seconds, uint64_t *raw_sum, int64_t *processed);

/* The same count over the directed edges e = offset, offset + stride,
 * offset + 2*stride, ... (0 <= offset < stride): the reference's depth-1
 * loop entered per sampled edge (reference src/graph.cpp:392-427; summed
 * over all offsets it is the whole count).  No edge is begun once
 * max_seconds have passed (0 = no limit); *processed receives how many were
 * counted.  The sampling unit of the timed CPU baseline and the edge subset
 * of the engine's gi_stats.edge_step / edge_offset. */
int oracle_count_edges_timed(const gi_plan_desc *plan, const int64_t *vertex, const int32_t *edge, int32_t v_cnt,
                             int64_t stride, int64_t offset, int threads, double max_seconds, uint64_t *raw_sum,
                             int64_t *processed);

/* Independent brute force: number of subgraphs of the graph isomorphic to
 * the n-vertex pattern adj (n*n '0'/'1'), edge-induced (induced = 0) or
 * vertex-induced (induced = 1), as #injective maps / #automorphisms.  For
 * small graphs only. */
uint64_t oracle_brute_count(int n, const char *adj, int induced, const int64_t *vertex, const int32_t *edge,
                            int32_t v_cnt);

/* Number of k-cliques (undirected), by brute force over increasing vertex
 * tuples.  For small graphs only. */
uint64_t oracle_clique_count(int k, const int64_t *vertex, const int32_t *edge, int32_t v_cnt);

/* Number of k-cliques for every k in [1, kmax] at once (out[k], modulo 2^64;
 * out needs kmax + 1 entries) by clique-tree pivoting (Jain and Seshadhri,
 * "The Power of Pivoting for Exact Clique Counting", WSDM 2020): vertices in
 * (degree, id) order; for each v the candidates are its later neighbours; a
 * node with candidates S picks the pivot u of S with the most neighbours in S
 * and has one child S ∩ N(u) in which u is optional, and one child per other
 * w ∈ S \ N(u), S ∩ N(w) minus the earlier such w, in which w is required.
 * A leaf with h required and q optional vertices holds C(q, k - h)
 * k-cliques.  A node three or fewer vertices short of kmax is counted in
 * closed form from its candidates' number, induced edges and induced
 * triangles (no descent), so the search never goes below h = kmax - 3.
 * Each root's candidates
 * and their induced adjacency are bit rows of ceil(|N+(v)| / 64) words.  An
 * independent check of the engine's k-clique counts for large k, where
 * enumeration is too slow.  Returns 0, or -1 on bad input or no memory. */
int oracle_clique_counts_pivot(int kmax, const int64_t *vertex, const int32_t *edge, int32_t v_cnt, int threads,
                               uint64_t *out);

/* Exact triangle count (each triangle once) by merging sorted lists,
 * reference src/graph.cpp:1006-1043 (motif_counting_3). */
uint64_t oracle_triangles(const int64_t *vertex, const int32_t *edge, int32_t v_cnt, int threads);

/* MNI support of labeled patterns by the reference's CPU enumeration
 * (reference src/labeled_graph.cpp:120-353, get_support_pattern_matching and
 * get_support_pattern_matching_aggressive_func, with the loop sets of
 * Schedule_IEP::update_loop_invariant_for_fsm, src/schedule_IEP.cpp:393-418):
 * for every start vertex of label[0], every embedding below it is
 * enumerated (in the schedule's vertex order; the loop set of depth d is the
 * intersection of the label-d buckets of its earlier neighbours, minus the
 * vertices already matched), the vertices of each complete embedding go into
 * per-position sets, and the scan stops once the smallest set holds
 * min_support vertices.  Graph: the bucketed structure of the reference
 * loader (bucket[v*l_cnt+l] .. bucket[v*l_cnt+l+1] in edge are v's
 * neighbours with label l; label_start[l] .. label_start[l+1] the vertices
 * with label l).  Pattern: n vertices, adj n*n 0/1 ints in schedule order.
 * labels[j*n + i] is job j's label of position i.  support[j] receives the
 * support at the point the scan stopped, frequent[j] = support >= min_support
 * and at least one embedding found.  Returns 0, or -1 on bad input. */
int oracle_fsm_support(int32_t v_cnt, int32_t l_cnt, const uint32_t *bucket, const uint32_t *edge,
                       const uint32_t *label_start, int n, const int *adj, int64_t n_jobs, const uint8_t *labels,
                       int64_t min_support, int threads, int64_t *support, uint8_t *frequent);

#ifdef __cplusplus
}
#endif

#endif
