/*
 * ORACLE — test infrastructure only (see oracle.h).  Plain C11 + OpenMP.
 *
 * oracle_count restates the reference CPU path:
 *   Graph::pattern_matching             reference src/graph.cpp:305-355
 *   Graph::pattern_matching_aggressive_func           src/graph.cpp:429-566
 *   Graph::remove_anti_edge_vertices                  src/graph.cpp:195-232
 *   VertexSet::build_vertex_set / intersection        src/vertex_set.cpp:83-91,203-215
 *   VertexSet::unordered_subtraction_size             src/vertex_set.cpp:264-277
 * on the plan arrays of a gi_plan_desc (the Schedule_IEP fields).
 *
 * Algorithmic bytes (counted when asked), per the engine's measurement
 * definition, on this traversal:
 *   materialised S_f ∩ N(v):      4 * (|S_f| + d(v) + |result|)
 *   size-only S_f ∩ N(v):         4 * (|S_f| + d(v))
 *   alias of N(v) (no father):    16
 *   last-level count:             4 * size_after_restrict
 *   IEP tail:                     4 * |S| for every set whose size alone is not enough
 * where "size-only" marks a prefix with no child, not walked as a loop set
 * before the IEP tail or the last position, and not needed by the IEP tail
 * as members.
 */
#include "oracle.h"

#include <omp.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
    const gi_plan_desc *P;
    const int64_t *vertex;
    const int32_t *edge;
    int32_t v_cnt;
    int n, k;
    int32_t *buf[GI_MAX_PREFIX];
    int32_t *diff[GI_MAX_PATTERN + 1];
    const int32_t *ptr[GI_MAX_PREFIX];
    int32_t size[GI_MAX_PREFIX];
    int size_only[GI_MAX_PREFIX];
    int32_t emb[GI_MAX_PATTERN + 1];
    int depth_emb;
    int ans[GI_MAX_IEP_SETS];
    uint64_t sum;
    uint64_t bytes;
    int want_bytes;
} dfs_t;

static int lower_bound_i32(const int32_t *a, int n, int32_t x) {
    int lo = 0, hi = n;
    while (lo < hi) {
        int mid = (lo + hi) >> 1;
        if (a[mid] < x) lo = mid + 1;
        else hi = mid;
    }
    return lo;
}

static int contains_i32(const int32_t *a, int n, int32_t x) {
    int i = lower_bound_i32(a, n, x);
    return i < n && a[i] == x;
}

/* |set0[0, size0) - emb[0, d)| — reference src/vertex_set.cpp:264-277 */
static int subtraction_size(const int32_t *set0, int size0, const int32_t *emb, int d) {
    int ret = size0;
    for (int j = 0; j < d; ++j)
        if (contains_i32(set0, size0, emb[j])) --ret;
    return ret;
}

static int merge_intersect(const int32_t *a, int na, const int32_t *b, int nb, int32_t *out) {
    int i = 0, j = 0, c = 0;
    while (i < na && j < nb) {
        if (a[i] < b[j]) ++i;
        else if (a[i] > b[j]) ++j;
        else {
            out[c++] = a[i];
            ++i;
            ++j;
        }
    }
    return c;
}

/* reference src/vertex_set.cpp:203-215: father -1 aliases N(v), otherwise
 * S_father ∩ N(v). */
static void build_vertex_set(dfs_t *s, int p, int32_t v) {
    const int64_t l = s->vertex[v], r = s->vertex[v + 1];
    const int32_t *nb = s->edge + l;
    const int deg = (int)(r - l);
    const int f = s->P->father_prefix_id[p];
    if (f == -1) {
        s->ptr[p] = nb;
        s->size[p] = deg;
        if (s->want_bytes) s->bytes += 16;
    } else {
        const int fn = s->size[f];
        const int c = merge_intersect(s->ptr[f], fn, nb, deg, s->buf[p]);
        s->ptr[p] = s->buf[p];
        s->size[p] = c;
        if (s->want_bytes) s->bytes += 4ull * (uint64_t)(fn + deg + (s->size_only[p] ? 0 : c));
    }
}

/* reference src/graph.cpp:195-232 */
static int remove_anti_edge(dfs_t *s, const int32_t *in, int n_in, int32_t *out, int vp) {
    int c = 0;
    const int n = s->n;
    for (int i = 0; i < n_in; ++i) {
        int keep = 1;
        for (int u = 0; u < vp && keep; ++u) {
            if (s->P->adj_mat[u * n + vp]) continue;
            const int32_t v = s->emb[u];
            const int64_t l = s->vertex[v], r = s->vertex[v + 1];
            if (contains_i32(s->edge + l, (int)(r - l), in[i])) keep = 0;
        }
        if (keep) out[c++] = in[i];
    }
    return c;
}

static int has_data(const dfs_t *s, int d, int32_t v) {
    for (int i = 0; i < d; ++i)
        if (s->emb[i] == v) return 1;
    return 0;
}

/* reference src/graph.cpp:429-566 */
static void aggressive(dfs_t *s, int depth) {
    const gi_plan_desc *P = s->P;
    const int n = s->n, k = s->k;
    const int ls = P->loop_set_prefix_id[depth];
    const int32_t *vset = s->ptr[ls];
    int loop_size = s->size[ls];
    if (loop_size <= 0) return;
    if (P->is_vertex_induced) {
        loop_size = remove_anti_edge(s, vset, loop_size, s->diff[depth], depth);
        vset = s->diff[depth];
    }
    if (depth == n - k) {
        /* IEP tail, reference src/graph.cpp:456-493 */
        for (int i = 0; i < P->iep_vertex_id_size; ++i) {
            const int p = P->iep_vertex_id[i];
            if (P->iep_vertex_flag[i]) {
                s->ans[i] = s->size[p] - P->iep_vertex_coef[i];
            } else {
                s->ans[i] = subtraction_size(s->ptr[p], s->size[p], s->emb, depth);
                if (s->want_bytes) s->bytes += 4ull * (uint64_t)s->size[p];
            }
        }
        int last_pos = -1;
        uint64_t val = 0;
        for (int pos = 0; pos < P->iep_term_count; ++pos) {
            const int64_t a = s->ans[P->iep_ans_pos[pos]];
            if (pos == last_pos + 1) val = (uint64_t)a;
            else if (val != 0) val = val * (uint64_t)a;
            if (P->iep_flag[pos]) {
                last_pos = pos;
                s->sum += val * (uint64_t)(int64_t)P->iep_coef[pos];
            }
        }
        return;
    }
    if (depth == n - 1) {
        int size_after = loop_size;
        if (P->total_restrict_num > 0) {
            int32_t min_vertex = s->v_cnt;
            for (int i = P->restrict_last[depth]; i != -1; i = P->restrict_next[i])
                if (min_vertex > s->emb[P->restrict_index[i]]) min_vertex = s->emb[P->restrict_index[i]];
            size_after = lower_bound_i32(vset, loop_size, min_vertex);
        }
        if (s->want_bytes) s->bytes += 4ull * (uint64_t)size_after;
        if (size_after > 0) s->sum += (uint64_t)(int64_t)subtraction_size(vset, size_after, s->emb, depth);
        return;
    }
    int32_t min_vertex = s->v_cnt;
    for (int i = P->restrict_last[depth]; i != -1; i = P->restrict_next[i])
        if (min_vertex > s->emb[P->restrict_index[i]]) min_vertex = s->emb[P->restrict_index[i]];
    for (int i = 0; i < loop_size; ++i) {
        const int32_t v = vset[i];
        if (min_vertex <= v) break;
        if (has_data(s, depth, v)) continue;
        int zero = 0;
        for (int p = P->last[depth]; p != -1; p = P->next[p]) {
            build_vertex_set(s, p, v);
            if (s->size[p] == P->break_size[p]) {
                zero = 1;
                break;
            }
        }
        if (zero) continue;
        s->emb[depth] = v;
        aggressive(s, depth + 1);
    }
}

static void classify(const gi_plan_desc *P, int *size_only) {
    const int tp = P->total_prefix_num, n = P->size, k = P->in_exclusion_optimize_num;
    int need[GI_MAX_PREFIX] = {0};
    for (int p = 0; p < tp; ++p)
        if (P->father_prefix_id[p] >= 0) need[P->father_prefix_id[p]] = 1;
    const int end = k > 0 ? n - k : n;
    for (int d = 1; d < end; ++d)
        if (P->loop_set_prefix_id[d] >= 0) need[P->loop_set_prefix_id[d]] = 1;
    for (int i = 0; i < P->iep_vertex_id_size && k > 0; ++i)
        if (!P->iep_vertex_flag[i]) need[P->iep_vertex_id[i]] = 1;
    for (int p = 0; p < tp; ++p) size_only[p] = P->father_prefix_id[p] >= 0 && !need[p];
}

int oracle_count(const gi_plan_desc *P, const int64_t *vertex, const int32_t *edge, int32_t v_cnt,
                 int32_t v_begin, int32_t v_end, int threads, uint64_t *raw_sum, uint64_t *alg_bytes) {
    return oracle_count_strided(P, vertex, edge, v_cnt, v_begin, v_end, 1, threads, raw_sum, alg_bytes);
}

static int count_core(const gi_plan_desc *P, const int64_t *vertex, const int32_t *edge, int32_t v_cnt,
                      int32_t v_begin, int32_t v_end, int32_t stride, int threads, double max_seconds,
                      uint64_t *raw_sum, uint64_t *alg_bytes, int64_t *processed);

int oracle_count_strided(const gi_plan_desc *P, const int64_t *vertex, const int32_t *edge, int32_t v_cnt,
                         int32_t v_begin, int32_t v_end, int32_t stride, int threads, uint64_t *raw_sum,
                         uint64_t *alg_bytes) {
    return count_core(P, vertex, edge, v_cnt, v_begin, v_end, stride, threads, 0.0, raw_sum, alg_bytes, NULL);
}

int oracle_count_timed(const gi_plan_desc *P, const int64_t *vertex, const int32_t *edge, int32_t v_cnt,
                       int32_t stride, int threads, double max_seconds, uint64_t *raw_sum, int64_t *processed) {
    return count_core(P, vertex, edge, v_cnt, 0, v_cnt, stride, threads, max_seconds, raw_sum, NULL, processed);
}

static int count_core(const gi_plan_desc *P, const int64_t *vertex, const int32_t *edge, int32_t v_cnt,
                      int32_t v_begin, int32_t v_end, int32_t stride, int threads, double max_seconds,
                      uint64_t *raw_sum, uint64_t *alg_bytes, int64_t *processed) {
    if (!P || !vertex || !raw_sum || P->size < 3 || P->size > GI_MAX_PATTERN || v_cnt < 1 || stride < 1) return -1;
    const double deadline = max_seconds > 0 ? omp_get_wtime() + max_seconds : 0.0;
    int64_t done = 0;
    if (v_begin < 0) v_begin = 0;
    if (v_end > v_cnt) v_end = v_cnt;
    const int64_t n_start = v_end > v_begin ? ((int64_t)v_end - v_begin + stride - 1) / stride : 0;
    int max_deg = 1;
    for (int32_t v = 0; v < v_cnt; ++v) {
        const int d = (int)(vertex[v + 1] - vertex[v]);
        if (d > max_deg) max_deg = d;
    }
    uint64_t total = 0, total_bytes = 0;
    int size_only[GI_MAX_PREFIX];
    classify(P, size_only);
    if (threads <= 0) threads = omp_get_max_threads();
#pragma omp parallel num_threads(threads) reduction(+ : total, total_bytes, done)
    {
        dfs_t s;
        memset(&s, 0, sizeof(s));
        s.P = P;
        s.vertex = vertex;
        s.edge = edge;
        s.v_cnt = v_cnt;
        s.n = P->size;
        s.k = P->in_exclusion_optimize_num;
        s.want_bytes = alg_bytes != NULL;
        memcpy(s.size_only, size_only, sizeof(size_only));
        for (int p = 0; p < P->total_prefix_num; ++p) s.buf[p] = (int32_t *)malloc(sizeof(int32_t) * (size_t)max_deg);
        for (int d = 0; d <= GI_MAX_PATTERN; ++d) s.diff[d] = (int32_t *)malloc(sizeof(int32_t) * (size_t)max_deg);
#pragma omp for schedule(dynamic, 16) nowait
        for (int64_t it = 0; it < n_start; ++it) {
            if (deadline > 0 && omp_get_wtime() > deadline) continue;
            const int32_t v = (int32_t)(v_begin + it * stride);
            for (int p = P->last[0]; p != -1; p = P->next[p]) build_vertex_set(&s, p, v);
            s.emb[0] = v;
            aggressive(&s, 1);
            ++done;
        }
        total += s.sum;
        total_bytes += s.bytes;
        for (int p = 0; p < P->total_prefix_num; ++p) free(s.buf[p]);
        for (int d = 0; d <= GI_MAX_PATTERN; ++d) free(s.diff[d]);
    }
    *raw_sum = total;
    if (alg_bytes) *alg_bytes = total_bytes;
    if (processed) *processed = done;
    return 0;
}

/* One iteration of the depth-1 loop of the reference CPU path (reference
 * src/graph.cpp:537-565 at depth 1) for the candidate v1 of start vertex v0:
 * restriction bound, injectivity, vertex-induced filter, the depth-1 prefix
 * builds with the break-size prune, then the DFS from depth 2.  Summed over
 * every directed edge (v0, v1) this is the whole count. */
static void edge_task(dfs_t *s, int32_t v0, int32_t v1) {
    const gi_plan_desc *P = s->P;
    for (int p = P->last[0]; p != -1; p = P->next[p]) build_vertex_set(s, p, v0);
    s->emb[0] = v0;
    int32_t min_vertex = s->v_cnt;
    for (int i = P->restrict_last[1]; i != -1; i = P->restrict_next[i])
        if (min_vertex > s->emb[P->restrict_index[i]]) min_vertex = s->emb[P->restrict_index[i]];
    if (min_vertex <= v1 || v1 == v0) return;
    if (P->is_vertex_induced) {
        int32_t out;
        if (remove_anti_edge(s, &v1, 1, &out, 1) == 0) return;
    }
    for (int p = P->last[1]; p != -1; p = P->next[p]) {
        build_vertex_set(s, p, v1);
        if (s->size[p] == P->break_size[p]) return;
    }
    s->emb[1] = v1;
    aggressive(s, 2);
}

int oracle_count_edges_timed(const gi_plan_desc *P, const int64_t *vertex, const int32_t *edge, int32_t v_cnt,
                             int64_t stride, int64_t offset, int threads, double max_seconds, uint64_t *raw_sum,
                             int64_t *processed) {
    if (!P || !vertex || !raw_sum || P->size < 3 || P->size > GI_MAX_PATTERN || v_cnt < 1 || stride < 1 ||
        offset < 0 || offset >= stride)
        return -1;
    const int64_t e_cnt = vertex[v_cnt];
    const int64_t n_edges = offset < e_cnt ? (e_cnt - offset + stride - 1) / stride : 0;
    const double deadline = max_seconds > 0 ? omp_get_wtime() + max_seconds : 0.0;
    int max_deg = 1;
    for (int32_t v = 0; v < v_cnt; ++v) {
        const int d = (int)(vertex[v + 1] - vertex[v]);
        if (d > max_deg) max_deg = d;
    }
    uint64_t total = 0;
    int64_t done = 0;
    if (threads <= 0) threads = omp_get_max_threads();
#pragma omp parallel num_threads(threads) reduction(+ : total, done)
    {
        dfs_t s;
        memset(&s, 0, sizeof(s));
        s.P = P;
        s.vertex = vertex;
        s.edge = edge;
        s.v_cnt = v_cnt;
        s.n = P->size;
        s.k = P->in_exclusion_optimize_num;
        for (int p = 0; p < P->total_prefix_num; ++p) s.buf[p] = (int32_t *)malloc(sizeof(int32_t) * (size_t)max_deg);
        for (int d = 0; d <= GI_MAX_PATTERN; ++d) s.diff[d] = (int32_t *)malloc(sizeof(int32_t) * (size_t)max_deg);
#pragma omp for schedule(dynamic, 64) nowait
        for (int64_t it = 0; it < n_edges; ++it) {
            if (deadline > 0 && omp_get_wtime() > deadline) continue;
            const int64_t e = offset + it * stride;
            /* source vertex: the last v with vertex[v] <= e */
            int32_t lo = 0, hi = v_cnt;
            while (hi - lo > 1) {
                const int32_t mid = lo + (hi - lo) / 2;
                if (vertex[mid] <= e) lo = mid;
                else hi = mid;
            }
            edge_task(&s, lo, edge[e]);
            ++done;
        }
        total += s.sum;
        for (int p = 0; p < P->total_prefix_num; ++p) free(s.buf[p]);
        for (int d = 0; d <= GI_MAX_PATTERN; ++d) free(s.diff[d]);
    }
    *raw_sum = total;
    if (processed) *processed = done;
    return 0;
}

/* ------------------------------------------------------------ brute force */

static int adjacent(const int64_t *vertex, const int32_t *edge, int32_t a, int32_t b) {
    return contains_i32(edge + vertex[a], (int)(vertex[a + 1] - vertex[a]), b);
}

typedef struct {
    int n, induced;
    int adj[GI_MAX_PATTERN * GI_MAX_PATTERN];
    int order[GI_MAX_PATTERN];   /* pattern vertices in BFS order */
    int anchor[GI_MAX_PATTERN];  /* an earlier BFS neighbour, -1 for the root */
    const int64_t *vertex;
    const int32_t *edge;
    int32_t v_cnt;
    int32_t map[GI_MAX_PATTERN];
    uint64_t count;
} brute_t;

static void brute_rec(brute_t *b, int i) {
    if (i == b->n) {
        ++b->count;
        return;
    }
    const int pv = b->order[i];
    const int32_t *cand;
    int nc;
    int32_t all_dummy = 0;
    if (b->anchor[i] < 0) {
        cand = NULL;
        nc = b->v_cnt;
    } else {
        const int32_t a = b->map[b->anchor[i]];
        cand = b->edge + b->vertex[a];
        nc = (int)(b->vertex[a + 1] - b->vertex[a]);
    }
    (void)all_dummy;
    for (int c = 0; c < nc; ++c) {
        const int32_t x = cand ? cand[c] : c;
        int ok = 1;
        for (int j = 0; j < i && ok; ++j) {
            const int qv = b->order[j];
            const int32_t y = b->map[qv];
            if (y == x) ok = 0;
            else if (b->adj[pv * b->n + qv]) ok = adjacent(b->vertex, b->edge, x, y);
            else if (b->induced) ok = !adjacent(b->vertex, b->edge, x, y);
        }
        if (!ok) continue;
        b->map[pv] = x;
        brute_rec(b, i + 1);
    }
}

static uint64_t automorphisms(int n, const int *adj) {
    int p[GI_MAX_PATTERN], c[GI_MAX_PATTERN] = {0};
    for (int i = 0; i < n; ++i) p[i] = i;
    uint64_t count = 0;
    /* Heap's algorithm over all n! permutations. */
    int i = 0;
    for (;;) {
        int ok = 1;
        for (int a = 0; a < n && ok; ++a)
            for (int b = 0; b < n; ++b)
                if (adj[a * n + b] != adj[p[a] * n + p[b]]) {
                    ok = 0;
                    break;
                }
        count += (uint64_t)ok;
        while (i < n && c[i] >= i) c[i++] = 0;
        if (i >= n) break;
        if (i % 2 == 0) {
            int t = p[0]; p[0] = p[i]; p[i] = t;
        } else {
            int t = p[c[i]]; p[c[i]] = p[i]; p[i] = t;
        }
        ++c[i];
        i = 0;
    }
    return count;
}

uint64_t oracle_brute_count(int n, const char *adj, int induced, const int64_t *vertex, const int32_t *edge,
                            int32_t v_cnt) {
    brute_t b;
    memset(&b, 0, sizeof(b));
    b.n = n;
    b.induced = induced;
    b.vertex = vertex;
    b.edge = edge;
    b.v_cnt = v_cnt;
    for (int i = 0; i < n * n; ++i) b.adj[i] = adj[i] == '1';
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j)
            if (b.adj[i * n + j]) b.adj[j * n + i] = 1;
    int seen[GI_MAX_PATTERN] = {0};
    int cnt = 0;
    b.order[cnt] = 0;
    b.anchor[cnt++] = -1;
    seen[0] = 1;
    for (int h = 0; h < cnt; ++h)
        for (int j = 0; j < n; ++j)
            if (b.adj[b.order[h] * n + j] && !seen[j]) {
                seen[j] = 1;
                b.anchor[cnt] = b.order[h];
                b.order[cnt++] = j;
            }
    if (cnt != n) return 0; /* disconnected patterns are rejected by the engine */
    brute_rec(&b, 0);
    return b.count / automorphisms(n, b.adj);
}

static uint64_t clique_rec(const int64_t *vertex, const int32_t *edge, int32_t *pick, int depth, int k,
                           int32_t v_cnt) {
    if (depth == k) return 1;
    uint64_t c = 0;
    const int32_t last = pick[depth - 1];
    for (int64_t e = vertex[last]; e < vertex[last + 1]; ++e) {
        const int32_t x = edge[e];
        if (x <= last) continue;
        int ok = 1;
        for (int j = 0; j < depth - 1 && ok; ++j) ok = adjacent(vertex, edge, x, pick[j]);
        if (!ok) continue;
        pick[depth] = x;
        c += clique_rec(vertex, edge, pick, depth + 1, k, v_cnt);
    }
    return c;
}

uint64_t oracle_clique_count(int k, const int64_t *vertex, const int32_t *edge, int32_t v_cnt) {
    uint64_t total = 0;
    int32_t pick[GI_MAX_PATTERN + 1];
    if (k < 1 || k > GI_MAX_PATTERN) return 0;
    for (int32_t v = 0; v < v_cnt; ++v) {
        pick[0] = v;
        total += clique_rec(vertex, edge, pick, 1, k, v_cnt);
    }
    return total;
}

uint64_t oracle_triangles(const int64_t *vertex, const int32_t *edge, int32_t v_cnt, int threads) {
    uint64_t total = 0;
    if (threads <= 0) threads = omp_get_max_threads();
#pragma omp parallel for num_threads(threads) schedule(dynamic, 64) reduction(+ : total)
    for (int32_t v = 0; v < v_cnt; ++v) {
        for (int64_t e = vertex[v]; e < vertex[v + 1]; ++e) {
            const int32_t u = edge[e];
            if (u >= v) break;
            /* w < u < v, w in N(u) ∩ N(v) */
            int64_t i = vertex[v], j = vertex[u];
            const int64_t ie = vertex[v + 1], je = vertex[u + 1];
            while (i < ie && j < je) {
                const int32_t a = edge[i], b = edge[j];
                if (a >= u || b >= u) break;
                if (a < b) ++i;
                else if (a > b) ++j;
                else {
                    ++total;
                    ++i;
                    ++j;
                }
            }
        }
    }
    return total;
}

/* ------------------------------------------------------------------ FSM */

typedef struct {
    int32_t v_cnt, l_cnt;
    const uint32_t *bucket, *edge;
    int n;
    const int *adj;
    const uint8_t *lab;
    uint32_t *cand[GI_MAX_PATTERN]; /* loop set of each depth */
    int64_t ncand[GI_MAX_PATTERN];
    uint32_t *tmp;
    int32_t m[GI_MAX_PATTERN];      /* matched vertices (the subtraction set) */
    uint64_t *bits[GI_MAX_PATTERN]; /* per-position image sets */
    int64_t count[GI_MAX_PATTERN];
} fsm_t;

static void fsm_insert(fsm_t *s, int d, uint32_t v) {
    uint64_t *w = &s->bits[d][v >> 6];
    const uint64_t b = (uint64_t)1 << (v & 63);
    if (!(*w & b)) {
        *w |= b;
        ++s->count[d];
    }
}

/* Loop set of depth d: the intersection of the label-d buckets of the
 * earlier pattern neighbours of d (the chain of prefixes the reference
 * builds for d).  Returns its size. */
static int64_t fsm_loop_set(fsm_t *s, int d) {
    int first = 1;
    int64_t size = 0;
    for (int j = 0; j < d; ++j) {
        if (!s->adj[d * s->n + j]) continue;
        const int64_t b = (int64_t)s->m[j] * s->l_cnt + s->lab[d];
        const uint32_t *src = s->edge + s->bucket[b];
        const int64_t len = (int64_t)s->bucket[b + 1] - s->bucket[b];
        if (first) {
            memcpy(s->cand[d], src, (size_t)len * sizeof(uint32_t));
            size = len;
            first = 0;
        } else {
            int64_t i = 0, k = 0, o = 0;
            while (i < size && k < len) {
                if (s->cand[d][i] < src[k]) ++i;
                else if (s->cand[d][i] > src[k]) ++k;
                else {
                    s->tmp[o++] = s->cand[d][i];
                    ++i;
                    ++k;
                }
            }
            memcpy(s->cand[d], s->tmp, (size_t)o * sizeof(uint32_t));
            size = o;
        }
        if (size == 0) break;
    }
    s->ncand[d] = size;
    return size;
}

static int fsm_used(const fsm_t *s, int d, uint32_t v) {
    for (int j = 0; j < d; ++j)
        if ((uint32_t)s->m[j] == v) return 1;
    return 0;
}

/* Whether some embedding extends m[0..d-1]; inserts the vertices of every
 * such embedding.  The reference skips a vertex as soon as one of the prefix
 * sets it builds for a later depth is empty; here the later depth finds an
 * empty loop set instead, with the same outcome. */
static int fsm_rec(fsm_t *s, int d) {
    if (d >= GI_MAX_PATTERN || fsm_loop_set(s, d) == 0) return 0;
    int match = 0;
    if (d == s->n - 1) {
        for (int64_t i = 0; i < s->ncand[d]; ++i) {
            const uint32_t v = s->cand[d][i];
            if (fsm_used(s, d, v)) continue;
            match = 1;
            fsm_insert(s, d, v);
        }
        return match;
    }
    /* cand[d] is overwritten by deeper calls only at deeper depths */
    for (int64_t i = 0; i < s->ncand[d]; ++i) {
        const uint32_t v = s->cand[d][i];
        if (fsm_used(s, d, v)) continue;
        s->m[d] = (int32_t)v;
        if (fsm_rec(s, d + 1)) {
            match = 1;
            fsm_insert(s, d, v);
        }
    }
    return match;
}

int oracle_fsm_support(int32_t v_cnt, int32_t l_cnt, const uint32_t *bucket, const uint32_t *edge,
                       const uint32_t *label_start, int n, const int *adj, int64_t n_jobs, const uint8_t *labels,
                       int64_t min_support, int threads, int64_t *support, uint8_t *frequent) {
    if (n < 2 || n > GI_MAX_PATTERN || v_cnt < 1 || l_cnt < 1) return -1;
    uint32_t max_deg = 0;
    for (int32_t v = 0; v < v_cnt; ++v) {
        const uint32_t d = bucket[(int64_t)(v + 1) * l_cnt] - bucket[(int64_t)v * l_cnt];
        if (d > max_deg) max_deg = d;
    }
    if (threads <= 0) threads = omp_get_max_threads();
    const size_t words = ((size_t)v_cnt + 63) / 64;
#pragma omp parallel num_threads(threads)
    {
        fsm_t s;
        memset(&s, 0, sizeof(s));
        s.v_cnt = v_cnt;
        s.l_cnt = l_cnt;
        s.bucket = bucket;
        s.edge = edge;
        s.n = n;
        s.adj = adj;
        for (int d = 0; d < n; ++d) {
            s.cand[d] = (uint32_t *)malloc(((size_t)max_deg + 1) * sizeof(uint32_t));
            s.bits[d] = (uint64_t *)malloc(words * sizeof(uint64_t));
        }
        s.tmp = (uint32_t *)malloc(((size_t)max_deg + 1) * sizeof(uint32_t));
#pragma omp for schedule(dynamic, 1)
        for (int64_t j = 0; j < n_jobs; ++j) {
            s.lab = labels + j * n;
            for (int d = 0; d < n; ++d) {
                memset(s.bits[d], 0, words * sizeof(uint64_t));
                s.count[d] = 0;
            }
            int64_t sup = v_cnt;
            int any = 0;
            const uint32_t end = label_start[s.lab[0] + 1];
            for (uint32_t v = label_start[s.lab[0]]; v < end; ++v) {
                s.m[0] = (int32_t)v;
                if (!fsm_rec(&s, 1)) continue;
                any = 1;
                fsm_insert(&s, 0, v);
                sup = v_cnt;
                for (int d = 0; d < n; ++d)
                    if (s.count[d] < sup) sup = s.count[d];
                if (sup >= min_support) break;
            }
            sup = v_cnt;
            for (int d = 0; d < n; ++d)
                if (s.count[d] < sup) sup = s.count[d];
            support[j] = sup;
            frequent[j] = (uint8_t)(any && sup >= min_support);
        }
        for (int d = 0; d < n; ++d) {
            free(s.cand[d]);
            free(s.bits[d]);
        }
        free(s.tmp);
    }
    return 0;
}

/* ------------------------------------------------- clique-tree pivoting */

/* One root's search: the candidates are the root's later neighbours, numbered
 * 0..n-1 in id order; adj[i] is row i of their induced adjacency as a bit
 * row of W words.  Candidate sets are bit rows too, one per recursion depth
 * (cand), with a spare row per depth for the non-neighbour children (rest). */
typedef struct {
    int kmax;
    int64_t W;
    uint64_t *adj;
    uint64_t *cand;
    uint64_t *rest;
    const uint64_t *binom; /* binom[q * (kmax + 1) + j] = C(q, j) modulo 2^64 */
    uint64_t acc[GI_MAX_PATTERN + 1];
} pivot_t;

static int64_t row_popcount_and(const uint64_t *a, const uint64_t *b, int64_t W) {
    int64_t c = 0;
    for (int64_t i = 0; i < W; ++i) c += __builtin_popcountll(a[i] & b[i]);
    return c;
}

/* Node with candidate row cand[depth], h required and q optional vertices. */
static void pivot_rec(pivot_t *t, int64_t depth, int h, int64_t q) {
    const int64_t W = t->W;
    const uint64_t *S = t->cand + depth * W;
    const int K1 = t->kmax + 1;
    if (h >= t->kmax - 3) {
        /* The subtree of this node counts every clique R ∪ P' ∪ C once, R the
         * h required vertices, P' a subset of the q optional ones and C a
         * clique of G[S].  With at most three vertices left to add up to
         * kmax, the k-clique count is sum_j C(q, j) cl(k - h - j), where
         * cl(0) = 1, cl(1) = |S|, cl(2) = the edges and cl(3) = the
         * triangles of G[S]; no descent needed. */
        uint64_t cl[4] = {1, 0, 0, 0};
        for (int64_t w = 0; w < W; ++w) cl[1] += (uint64_t)__builtin_popcountll(S[w]);
        if (h <= t->kmax - 2) {
            uint64_t *R = t->rest + depth * W; /* free: this node has no children */
            uint64_t twice = 0, tri = 0;
            for (int64_t w = 0; w < W; ++w)
                for (uint64_t b = S[w]; b; b &= b - 1) {
                    const int64_t x = w * 64 + __builtin_ctzll(b);
                    const uint64_t *ax = t->adj + x * W;
                    twice += (uint64_t)row_popcount_and(S, ax, W);
                    if (h > t->kmax - 3) continue;
                    /* triangles x < y < z: R = S ∩ N(x) above x, then
                     * |R ∩ N(y)| above y for each y in R */
                    for (int64_t i = 0; i < W; ++i) R[i] = i < w ? 0 : S[i] & ax[i];
                    R[w] &= x % 64 == 63 ? 0 : ~((2ull << (x % 64)) - 1);
                    for (int64_t wy = w; wy < W; ++wy)
                        for (uint64_t by = R[wy]; by; by &= by - 1) {
                            const int64_t y = wy * 64 + __builtin_ctzll(by);
                            const uint64_t *ay = t->adj + y * W;
                            uint64_t c = (uint64_t)__builtin_popcountll(
                                R[wy] & ay[wy] & (y % 64 == 63 ? 0 : ~((2ull << (y % 64)) - 1)));
                            for (int64_t i = wy + 1; i < W; ++i) c += (uint64_t)__builtin_popcountll(R[i] & ay[i]);
                            tri += c;
                        }
                }
            cl[2] = twice / 2;
            cl[3] = tri;
        }
        for (int k = h; k <= t->kmax; ++k)
            for (int j = 0; j <= k - h && j <= q; ++j) t->acc[k] += t->binom[q * K1 + j] * cl[k - h - j];
        return;
    }
    int64_t u = -1, best = -1;
    for (int64_t w = 0; w < W; ++w)
        for (uint64_t b = S[w]; b; b &= b - 1) {
            const int64_t x = w * 64 + __builtin_ctzll(b);
            const int64_t c = row_popcount_and(S, t->adj + x * W, W);
            if (c > best) {
                best = c;
                u = x;
            }
        }
    if (u < 0) { /* leaf */
        for (int k = h; k <= t->kmax && k - h <= q; ++k) t->acc[k] += t->binom[q * K1 + (k - h)];
        return;
    }
    uint64_t *next = t->cand + (depth + 1) * W;
    const uint64_t *au = t->adj + u * W;
    for (int64_t w = 0; w < W; ++w) next[w] = S[w] & au[w];
    pivot_rec(t, depth + 1, h, q + 1);
    /* Each non-neighbour w of u other than u is required in its child, whose
     * candidates are S ∩ N(w) minus the earlier such w. */
    uint64_t *cur = t->rest + depth * W;
    for (int64_t w = 0; w < W; ++w) cur[w] = S[w];
    for (int64_t w = 0; w < W; ++w) {
        uint64_t b = S[w] & ~au[w];
        if (w == u / 64) b &= ~(1ull << (u % 64));
        for (; b; b &= b - 1) {
            const int64_t x = w * 64 + __builtin_ctzll(b);
            const uint64_t *ax = t->adj + x * W;
            for (int64_t i = 0; i < W; ++i) next[i] = cur[i] & ax[i];
            pivot_rec(t, depth + 1, h + 1, q);
            cur[w] &= ~(1ull << (x % 64));
        }
    }
}

int oracle_clique_counts_pivot(int kmax, const int64_t *vertex, const int32_t *edge, int32_t v_cnt, int threads,
                               uint64_t *out) {
    if (kmax < 1 || kmax > GI_MAX_PATTERN || v_cnt < 1) return -1;
    /* Later neighbours in (degree, id) order, each list in id order. */
    int64_t *off = (int64_t *)malloc(sizeof(int64_t) * ((size_t)v_cnt + 1));
    if (!off) return -1;
    off[0] = 0;
    int64_t dmax = 0;
    for (int32_t v = 0; v < v_cnt; ++v) {
        const int64_t dv = vertex[v + 1] - vertex[v];
        int64_t later = 0;
        for (int64_t e = vertex[v]; e < vertex[v + 1]; ++e) {
            const int64_t dw = vertex[edge[e] + 1] - vertex[edge[e]];
            later += dw > dv || (dw == dv && edge[e] > v);
        }
        off[v + 1] = off[v] + later;
        if (later > dmax) dmax = later;
    }
    int32_t *out_nb = (int32_t *)malloc(sizeof(int32_t) * ((size_t)off[v_cnt] + 1));
    /* Every vertex chosen along a path of the recursion is adjacent to all the
     * later candidates, so the depth (and q) is at most dmax + 1. */
    const int64_t qmax = dmax + 2;
    uint64_t *binom = (uint64_t *)malloc(sizeof(uint64_t) * (size_t)(qmax + 1) * (size_t)(kmax + 1));
    if (!out_nb || !binom) {
        free(off);
        free(out_nb);
        free(binom);
        return -1;
    }
    for (int32_t v = 0; v < v_cnt; ++v) {
        const int64_t dv = vertex[v + 1] - vertex[v];
        int64_t o = off[v];
        for (int64_t e = vertex[v]; e < vertex[v + 1]; ++e) {
            const int32_t w = edge[e];
            const int64_t dw = vertex[w + 1] - vertex[w];
            if (dw > dv || (dw == dv && w > v)) out_nb[o++] = w;
        }
    }
    for (int64_t a = 0; a <= qmax; ++a)
        for (int b = 0; b <= kmax; ++b)
            binom[a * (kmax + 1) + b] =
                b == 0 ? 1 : (a == 0 ? 0 : binom[(a - 1) * (kmax + 1) + b - 1] + binom[(a - 1) * (kmax + 1) + b]);
    for (int k = 0; k <= kmax; ++k) out[k] = 0;
    if (threads <= 0) threads = omp_get_max_threads();
    int fail = 0;
    const int64_t Wmax = (dmax + 63) / 64 > 0 ? (dmax + 63) / 64 : 1;
#pragma omp parallel num_threads(threads)
    {
        pivot_t t;
        memset(&t, 0, sizeof(t));
        t.kmax = kmax;
        t.binom = binom;
        const int64_t levels = dmax + 3;
        t.adj = (uint64_t *)malloc(sizeof(uint64_t) * (size_t)(dmax > 0 ? dmax : 1) * (size_t)Wmax);
        t.cand = (uint64_t *)malloc(sizeof(uint64_t) * (size_t)levels * (size_t)Wmax);
        t.rest = (uint64_t *)malloc(sizeof(uint64_t) * (size_t)levels * (size_t)Wmax);
        int32_t *pos = (int32_t *)calloc((size_t)v_cnt, sizeof(int32_t)); /* local index + 1, or 0 */
        if (!t.adj || !t.cand || !t.rest || !pos) {
#pragma omp atomic write
            fail = 1;
        } else {
#pragma omp for schedule(dynamic, 64)
            for (int32_t v = 0; v < v_cnt; ++v) {
                const int32_t *L = out_nb + off[v];
                const int64_t n = off[v + 1] - off[v];
                const int64_t W = t.W = n > 64 ? (n + 63) / 64 : 1; /* row width of this root */
                for (int64_t i = 0; i < n; ++i) pos[L[i]] = (int32_t)(i + 1);
                memset(t.adj, 0, sizeof(uint64_t) * (size_t)n * (size_t)W);
                /* Both ends of an edge inside L: the later one is in the
                 * earlier one's out-list. */
                for (int64_t i = 0; i < n; ++i)
                    for (int64_t e = off[L[i]]; e < off[L[i] + 1]; ++e) {
                        const int32_t p = pos[out_nb[e]];
                        if (!p) continue;
                        const int64_t j = p - 1;
                        t.adj[i * W + j / 64] |= 1ull << (j % 64);
                        t.adj[j * W + i / 64] |= 1ull << (i % 64);
                    }
                memset(t.cand, 0, sizeof(uint64_t) * (size_t)W);
                for (int64_t i = 0; i < n; ++i) t.cand[i / 64] |= 1ull << (i % 64);
                pivot_rec(&t, 0, 1, 0);
                for (int64_t i = 0; i < n; ++i) pos[L[i]] = 0;
            }
        }
#pragma omp critical
        for (int k = 0; k <= kmax; ++k) out[k] += t.acc[k];
        free(t.adj);
        free(t.cand);
        free(t.rest);
        free(pos);
    }
    free(off);
    free(out_nb);
    free(binom);
    return fail ? -1 : 0;
}
