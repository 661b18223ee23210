/*
 * graphindor_b200 — seeded synthetic graph generators (host only).
 *
 * No counterpart in the reference, which reads SNAP files; these stand in
 * for its datasets with seeded graphs of the same shapes.  Every generator is
 * deterministic for a given seed, independent of the number of host threads:
 * sample i draws its random bits from splitmix64 of (seed, i).  Output is a
 * simple undirected graph in the reference's CSR layout (both directions,
 * sorted, no self-loops, no duplicates) after a seeded random relabelling.
 */
#ifndef GRAPHINDOR_B200_GI_GEN_H
#define GRAPHINDOR_B200_GI_GEN_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct gi_host_csr {
    int32_t v_cnt;
    int64_t e_cnt;        /* directed entries */
    int64_t *vertex;      /* v_cnt + 1 */
    int32_t *edge;        /* e_cnt */
    int32_t max_degree;
    int32_t max_intersection_size;
} gi_host_csr;

/* R-MAT: edge_factor * 2^scale sampled pairs, quadrant probabilities a, b, c
 * and d = 1 - a - b - c at every level. */
int gi_gen_rmat(int scale, double edge_factor, double a, double b, double c, uint64_t seed, gi_host_csr **out);
/* Chung-Lu: n vertices with weights (i + i0)^(-1/(gamma-1)); m sampled pairs
 * with both endpoints drawn proportionally to weight; i0 is chosen so that
 * the heaviest vertex's expected degree is max_degree. */
int gi_gen_chung_lu(int32_t n, int64_t m, double gamma, double max_degree, uint64_t seed, gi_host_csr **out);
/* Erdős–Rényi G(n, m): m uniformly sampled pairs. */
int gi_gen_er(int32_t n, int64_t m, uint64_t seed, gi_host_csr **out);
/* Restricts a graph to the vertices with id < keep (used to carve a
 * 100k-vertex graph out of an R-MAT). */
int gi_csr_restrict(const gi_host_csr *in, int32_t keep, gi_host_csr **out);
void gi_host_csr_free(gi_host_csr *g);

#ifdef __cplusplus
}
#endif

#endif
