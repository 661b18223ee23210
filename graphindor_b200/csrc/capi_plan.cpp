// C ABI: status strings, plans and motif enumeration (host only).
#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <new>
#include <set>
#include <stdexcept>

#include "internal.hpp"

namespace gi {

namespace {
thread_local std::string g_last_error;
}

int fail(int status, const std::string &msg) {
    g_last_error = msg;
    return status;
}

// Decide how the kernels build each prefix and flatten the plan.  A prefix
// is materialised when a later set is intersected with it, when the DFS
// iterates over it, or when the IEP tail needs its members; otherwise only
// its size is ever read.  The IEP tables are the entries the reference reads
// (the leading entries of its never-cleared vectors).
static int build_dev_plan(const Schedule_IEP &s, DevPlan &d) {
    std::memset(&d, 0, sizeof(d));
    const int n = s.get_size();
    const int tp = s.get_total_prefix_num();
    if (tp > GI_MAX_PREFIX) return fail(GI_EINVAL, "plan has too many prefixes");
    if (s.get_total_restrict_num() > GI_MAX_PREFIX) return fail(GI_EINVAL, "plan has too many restrictions");
    d.n = n;
    d.iep_k = s.get_in_exclusion_optimize_num();
    d.total_prefix = tp;
    d.vertex_induced = s.is_vertex_induced ? 1 : 0;
    d.first_restricted = s.get_restrict_last(1) != -1 ? 1 : 0;
    for (int i = 0; i < GI_MAX_PATTERN + 1; ++i) {
        d.last[i] = i < n ? s.get_last(i) : -1;
        d.loop_set[i] = i < n ? s.get_loop_set_prefix_id(i) : -1;
        d.restrict_last[i] = i < n ? s.get_restrict_last(i) : -1;
    }
    for (int i = 0; i < n * n; ++i) d.adj[i] = s.get_adj_mat_ptr()[i];
    for (int i = 0; i < GI_MAX_PREFIX; ++i) {
        d.father[i] = i < tp ? s.get_father_prefix_id(i) : -1;
        d.next[i] = i < tp ? s.get_next(i) : -1;
        d.break_size[i] = i < tp ? s.get_break_size(i) : -1;
        d.restrict_next[i] = i < s.get_total_restrict_num() ? s.get_restrict_next(i) : -1;
        d.restrict_index[i] = i < s.get_total_restrict_num() ? s.get_restrict_index(i) : -1;
        d.slot[i] = -1;
    }
    const int nsets = static_cast<int>(s.in_exclusion_optimize_vertex_id.size());
    const int nterms = static_cast<int>(s.in_exclusion_optimize_coef.size());
    if (d.iep_k > 0) {
        if (nsets > GI_MAX_IEP_SETS || nterms > GI_MAX_IEP_TERMS)
            return fail(GI_EINVAL, "IEP tables exceed the engine's limits");
        d.iep_nsets = nsets;
        d.iep_nterms = nterms;
        for (int i = 0; i < nsets; ++i) {
            d.iep_set[i] = s.in_exclusion_optimize_vertex_id[i];
            d.iep_set_flag[i] = s.in_exclusion_optimize_vertex_flag[i];
            d.iep_set_coef[i] = s.in_exclusion_optimize_vertex_coef[i];
        }
        for (int t = 0; t < nterms; ++t) {
            d.iep_coef[t] = s.in_exclusion_optimize_coef[t];
            d.iep_flag[t] = s.in_exclusion_optimize_flag[t];
            d.iep_pos[t] = s.in_exclusion_optimize_ans_pos[t];
            if (d.iep_pos[t] < 0 || d.iep_pos[t] >= nsets)
                return fail(GI_EINVAL, "plan's IEP table points past its set list");
        }
    }
    // Which prefixes need their members.
    std::vector<int> need(tp, 0);
    for (int p = 0; p < tp; ++p)
        if (d.father[p] >= 0) need[d.father[p]] = 1;
    const int iter_end = d.iep_k > 0 ? n - d.iep_k : n;  // depths whose loop sets are walked or counted
    for (int dep = 1; dep < iter_end; ++dep)
        if (d.loop_set[dep] >= 0) need[d.loop_set[dep]] = 1;
    for (int i = 0; i < d.iep_nsets; ++i)
        if (!d.iep_set_flag[i]) need[d.iep_set[i]] = 1;
    int slots = 0;
    for (int p = 0; p < tp; ++p) {
        if (d.father[p] == -1) {
            d.mode[p] = kAlias;
        } else if (need[p]) {
            d.mode[p] = kMaterialize;
            d.slot[p] = slots++;
        } else {
            d.mode[p] = kSizeOnly;
        }
    }
    d.n_slots = slots;

    // Lane-parallel leaf level: the candidates at depth stop - 1 are
    // evaluated one per lane (sizes and counts only, no materialisation).
    // Needs stop - 1 >= 2 and, for vertex-induced plans, no non-edge in the
    // pattern (the per-candidate anti-edge filter stays warp-cooperative).
    d.stop = d.iep_k > 0 ? n - d.iep_k : n - 1;
    bool anti_edge = false;
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j)
            if (i != j && !d.adj[i * n + j]) anti_edge = true;
    d.leaf_depth = (d.stop - 1 >= 2 && !(d.vertex_induced && anti_edge)) ? d.stop - 1 : -1;
    // Lane-versus-warp split of leaf candidates, measured on the B200 (R-MAT
    // scales 14-17): plans with an IEP tail evaluate several intersections per
    // candidate and run best when only cheap candidates stay on one lane
    // (house 11 %, prism 5 %, 6-cycle + chord 4 % faster at 256 than at 2048);
    // plans without one (cliques) prefer the lanes (5-clique 36 % faster at 2048).
    d.lane_budget = d.iep_k > 0 ? 256 : 2048;
    // Leaf probes spread over the lanes (one element test per lane and step)
    // instead of one candidate per lane; GI_LEAF_FLAT=0/1 overrides.
    d.leaf_flat = 0;
    if (const char *e = std::getenv("GI_LEAF_FLAT")) d.leaf_flat = std::atoi(e) != 0;
    // A DFS that ends at depth 2 (triangle- and diamond-like plans): the
    // first-level edges of a chunk are themselves the flat leaf's candidates.
    d.flat_first_ok = d.stop == 2 && !(d.vertex_induced && anti_edge);
    d.flat_first = d.leaf_flat && d.flat_first_ok;
    d.occupancy = 0;
    for (int p = 0; p < GI_MAX_PREFIX; ++p) d.pdepth[p] = p < tp ? s.get_prefix_data(p).back() : -1;
    // Edge-triangle counting (tri_edge.cu) serves plans whose DFS ends at
    // depth 2 in an IEP tail and whose sets before it are N(v0), N(v1) and
    // N(v0) ∩ N(v1) only.
    d.tri_ok = d.iep_k > 0 && d.stop == 2 && !d.vertex_induced;
    for (int p = 0; p < tp && d.tri_ok; ++p) {
        const int f = d.father[p];
        if (d.pdepth[p] == 0 && f != -1) d.tri_ok = 0;
        if (d.pdepth[p] == 1 && f != -1 && (d.pdepth[f] != 0 || d.father[f] != -1)) d.tri_ok = 0;
    }
    d.tri_edge = 0;
    // Splitting of the depth-2 loop: its set's members are a subset of {0, 1}.
    d.loop2_kind = -1;
    if (d.stop > 2 && d.loop_set[2] >= 0) {
        const auto &data = s.get_prefix_data(d.loop_set[2]);
        if (data.size() == 1) d.loop2_kind = data[0];
        else d.loop2_kind = 2;
    }
    return GI_OK;
}

static bool parse_adj(int n, const char *adj) {
    if (!adj) return false;
    for (int i = 0; i < n * n; ++i)
        if (adj[i] == '\0') return false;
    return true;
}

static int finish_plan(std::unique_ptr<Schedule_IEP> s, gi_plan **out) {
    auto *p = new (std::nothrow) gi_plan;
    if (!p) return fail(GI_ENOMEM, "out of host memory");
    p->sched = std::move(s);
    int st = build_dev_plan(*p->sched, p->dev);
    if (st != GI_OK) {
        delete p;
        return st;
    }
    p->multiplicity = p->sched->get_multiplicity();
    *out = p;
    return GI_OK;
}

}  // namespace gi

using namespace gi;

extern "C" {

const char *gi_status_string(int status) {
    switch (status) {
        case GI_OK: return "ok";
        case GI_EINVAL: return "invalid argument";
        case GI_ENOMEM: return "out of memory";
        case GI_ECUDA: return "CUDA error";
        case GI_ETIMEOUT: return "device work budget exhausted";
        case GI_EOVERFLOW: return "size overflow";
        case GI_EIO: return "I/O error";
        case GI_ENOTSUP: return "not supported";
        case GI_EDISCONNECTED: return "pattern is not connected";
        default: return "unknown status";
    }
}

const char *gi_last_error(void) { return g_last_error.c_str(); }

int gi_version(void) { return 1; }

int gi_plan_create(int n, const char *adj, int32_t v_cnt, int64_t e_cnt, int64_t tri_cnt, int model,
                   int enable_iep, gi_plan **out) {
    if (!out) return fail(GI_EINVAL, "out is NULL");
    *out = nullptr;
    if (n < 3 || n > GI_MAX_PATTERN) return fail(GI_EINVAL, "pattern size must be between 3 and 7");
    if (!parse_adj(n, adj)) return fail(GI_EINVAL, "adjacency string shorter than n*n");
    if (model < 0 || model > 2) return fail(GI_EINVAL, "model must be 0, 1 or 2");
    if (model >= 1 && (v_cnt <= 0 || e_cnt <= 0)) return fail(GI_EINVAL, "the analytic model needs v_cnt, e_cnt > 0");
    try {
        Pattern pat(n, adj);
        if (!pat.check_connected()) return fail(GI_EDISCONNECTED, "pattern is not connected");
        if (model == 2) {
            Schedule_IEP::Candidate c;
            if (!Schedule_IEP::choose_validated(pat, enable_iep != 0, v_cnt, e_cnt, tri_cnt, c))
                return fail(GI_EINVAL, "no candidate schedule has a valid restriction set");
            auto s = std::make_unique<Schedule_IEP>(pat, c.order, c.restricts, enable_iep != 0);
            return finish_plan(std::move(s), out);
        }
        bool valid = false;
        auto s = std::make_unique<Schedule_IEP>(pat, valid, model, 1, enable_iep != 0, v_cnt, e_cnt, tri_cnt);
        if (s->iep_tables_out_of_range()) {
            // The reference would read its IEP answer buffer out of bounds
            // for this plan (an undefined count).  Keep its order and
            // restrictions and rebuild the IEP tables cleanly.
            auto clean = std::make_unique<Schedule_IEP>(pat, s->get_order(), s->get_chosen_restricts(),
                                                        enable_iep != 0, /*exact=*/false);
            const int st = finish_plan(std::move(clean), out);
            if (st == GI_OK) (*out)->iep_tables_rebuilt = true;
            return st;
        }
        return finish_plan(std::move(s), out);
    } catch (const std::runtime_error &e) {
        return fail(GI_EDISCONNECTED, e.what());
    } catch (const std::bad_alloc &) {
        return fail(GI_ENOMEM, "out of host memory");
    } catch (const std::exception &e) {
        return fail(GI_EINVAL, e.what());
    }
}

int gi_plan_create_explicit(int n, const char *adj, const int32_t *order, const int32_t *restricts,
                            int n_restricts, int enable_iep, gi_plan **out) {
    if (!out) return fail(GI_EINVAL, "out is NULL");
    *out = nullptr;
    if (n < 3 || n > GI_MAX_PATTERN) return fail(GI_EINVAL, "pattern size must be between 3 and 7");
    if (!parse_adj(n, adj) || !order) return fail(GI_EINVAL, "missing adjacency string or order");
    if (n_restricts < 0 || n_restricts > GI_MAX_PREFIX || (n_restricts > 0 && !restricts))
        return fail(GI_EINVAL, "bad restriction list");
    try {
        Pattern pat(n, adj);
        std::vector<int> ord(order, order + n);
        std::vector<std::pair<int, int>> r;
        for (int i = 0; i < n_restricts; ++i) r.emplace_back(restricts[2 * i], restricts[2 * i + 1]);
        auto s = std::make_unique<Schedule_IEP>(pat, ord, r, enable_iep != 0);
        return finish_plan(std::move(s), out);
    } catch (const std::runtime_error &e) {
        return fail(GI_EDISCONNECTED, e.what());
    } catch (const std::exception &e) {
        return fail(GI_EINVAL, e.what());
    }
}

int gi_plan_create_induced(int n, const char *adj, gi_plan **out) {
    if (!out) return fail(GI_EINVAL, "out is NULL");
    *out = nullptr;
    if (n < 3 || n > GI_MAX_PATTERN) return fail(GI_EINVAL, "pattern size must be between 3 and 7");
    if (!parse_adj(n, adj)) return fail(GI_EINVAL, "adjacency string shorter than n*n");
    try {
        Pattern pat(n, adj);
        auto s = std::make_unique<Schedule_IEP>(pat.get_adj_mat_ptr(), n);
        return finish_plan(std::move(s), out);
    } catch (const std::runtime_error &e) {
        return fail(GI_EDISCONNECTED, e.what());
    } catch (const std::exception &e) {
        return fail(GI_EINVAL, e.what());
    }
}

int gi_plan_destroy(gi_plan *p) {
    delete p;
    return GI_OK;
}

int gi_plan_export(const gi_plan *p, gi_plan_desc *o) {
    if (!p || !o) return fail(GI_EINVAL, "NULL argument");
    const Schedule_IEP &s = *p->sched;
    std::memset(o, 0, sizeof(*o));
    const int n = s.get_size();
    const int tp = s.get_total_prefix_num();
    o->size = n;
    for (int i = 0; i < n * n; ++i) o->adj_mat[i] = s.get_adj_mat_ptr()[i];
    for (int i = 0; i < n; ++i) {
        o->order[i] = s.get_order()[i];
        o->last[i] = s.get_last(i);
        o->loop_set_prefix_id[i] = s.get_loop_set_prefix_id(i);
        o->restrict_last[i] = s.get_restrict_last(i);
    }
    o->total_prefix_num = tp;
    o->basic_prefix_num = s.get_basic_prefix_num();
    for (int i = 0; i < tp; ++i) {
        o->father_prefix_id[i] = s.get_father_prefix_id(i);
        o->next[i] = s.get_next(i);
        o->break_size[i] = s.get_break_size(i);
        o->only_need_size[i] = s.get_prefix_only_need_size(i);
        const auto &data = s.get_prefix_data(i);
        o->prefix_len[i] = static_cast<int32_t>(data.size());
        for (size_t j = 0; j < data.size() && j < GI_MAX_PATTERN; ++j) o->prefix_data[i][j] = data[j];
    }
    o->total_restrict_num = s.get_total_restrict_num();
    for (int i = 0; i < o->total_restrict_num; ++i) {
        o->restrict_next[i] = s.get_restrict_next(i);
        o->restrict_index[i] = s.get_restrict_index(i);
    }
    o->n_restrict_pairs = static_cast<int32_t>(std::min<size_t>(s.restrict_pair.size(), GI_MAX_PREFIX));
    for (int i = 0; i < o->n_restrict_pairs; ++i) {
        o->restrict_pairs[i][0] = s.restrict_pair[i].first;
        o->restrict_pairs[i][1] = s.restrict_pair[i].second;
    }
    o->in_exclusion_optimize_num = s.get_in_exclusion_optimize_num();
    const DevPlan &d = p->dev;
    o->iep_vertex_id_size = static_cast<int32_t>(s.in_exclusion_optimize_vertex_id.size());
    for (int i = 0; i < o->iep_vertex_id_size && i < GI_MAX_IEP_SETS; ++i) {
        o->iep_vertex_id[i] = s.in_exclusion_optimize_vertex_id[i];
        o->iep_vertex_flag[i] = s.in_exclusion_optimize_vertex_flag[i];
        o->iep_vertex_coef[i] = s.in_exclusion_optimize_vertex_coef[i];
    }
    o->iep_term_count = static_cast<int32_t>(s.in_exclusion_optimize_coef.size());
    for (int t = 0; t < o->iep_term_count && t < GI_MAX_IEP_TERMS; ++t) {
        o->iep_coef[t] = s.in_exclusion_optimize_coef[t];
        o->iep_flag[t] = s.in_exclusion_optimize_flag[t];
        o->iep_ans_pos[t] = s.in_exclusion_optimize_ans_pos[t];
    }
    (void)d;
    o->iep_vertex_flag_raw_len = static_cast<int64_t>(s.in_exclusion_optimize_vertex_flag.size());
    o->iep_ans_pos_raw_len = static_cast<int64_t>(s.in_exclusion_optimize_ans_pos.size());
    o->is_vertex_induced = s.is_vertex_induced ? 1 : 0;
    o->redundancy = s.get_in_exclusion_optimize_redundancy();
    o->k_val = s.get_k_val();
    o->multiplicity = p->multiplicity;
    o->model_cost = s.get_model_cost();
    o->iep_tables_rebuilt = p->iep_tables_rebuilt ? 1 : 0;
    o->count_divisor = s.get_count_divisor();
    if (s.is_vertex_induced) {
        o->exact = -1;
    } else {
        std::vector<std::pair<int, int>> applied;
        for (const auto &pr : s.restrict_pair)
            if (pr.second < n - s.get_in_exclusion_optimize_num()) applied.push_back(pr);
        o->exact = restriction_multiplicity(s.get_adj_mat_ptr(), n, applied) == s.get_count_divisor() ? 1 : 0;
    }
    return GI_OK;
}

int gi_plan_export_raw(const gi_plan *p, int which, int32_t *buf, int64_t cap, int64_t *len) {
    if (!p || !len) return fail(GI_EINVAL, "NULL argument");
    const Schedule_IEP &s = *p->sched;
    const std::vector<int> *v = nullptr;
    if (which == 0) v = &s.in_exclusion_optimize_vertex_flag;
    else if (which == 1) v = &s.in_exclusion_optimize_vertex_coef;
    else if (which == 2) v = &s.in_exclusion_optimize_ans_pos;
    else return fail(GI_EINVAL, "which must be 0, 1 or 2");
    *len = static_cast<int64_t>(v->size());
    if (buf)
        for (int64_t i = 0; i < cap && i < *len; ++i) buf[i] = (*v)[i];
    return GI_OK;
}

int gi_plan_candidates(int n, const char *adj, int32_t v_cnt, int64_t e_cnt, int64_t tri_cnt, int enable_iep,
                       int32_t *orders, int32_t *restricts, int32_t *n_restricts, double *costs,
                       int32_t *divisors, int64_t cap,
                       int64_t *count) {
    if (!count) return fail(GI_EINVAL, "count is NULL");
    if (n < 3 || n > GI_MAX_PATTERN || !parse_adj(n, adj)) return fail(GI_EINVAL, "bad pattern");
    try {
        Pattern pat(n, adj);
        if (!pat.check_connected()) return fail(GI_EDISCONNECTED, "pattern is not connected");
        auto c = Schedule_IEP::enumerate_candidates(pat, enable_iep != 0, v_cnt, e_cnt, tri_cnt);
        *count = static_cast<int64_t>(c.size());
        if (!orders) return GI_OK;
        for (int64_t i = 0; i < cap && i < *count; ++i) {
            for (int j = 0; j < n; ++j) orders[i * n + j] = c[i].order[j];
            const int nr = static_cast<int>(std::min<size_t>(c[i].restricts.size(), GI_MAX_PREFIX));
            if (n_restricts) n_restricts[i] = nr;
            if (restricts)
                for (int j = 0; j < nr; ++j) {
                    restricts[(i * GI_MAX_PREFIX + j) * 2] = c[i].restricts[j].first;
                    restricts[(i * GI_MAX_PREFIX + j) * 2 + 1] = c[i].restricts[j].second;
                }
            if (costs) costs[i] = c[i].model_cost;
            if (divisors) divisors[i] = c[i].divisor;
        }
        return GI_OK;
    } catch (const std::exception &e) {
        return fail(GI_EINVAL, e.what());
    }
}

// Connected k-vertex patterns in the order of the reference MotifGenerator
// (reference src/motif_generator.cpp:5-43): edges (i,j), i<j, taken in
// row-major order with "use the edge" explored before "skip it"; a pattern is
// emitted when it is connected and no relabelling of it was emitted before.
}  // extern "C"

std::vector<std::vector<int>> gi::motif_list(int k, int max_edges) {
    std::vector<std::vector<int>> out;
    std::set<std::set<int>> seen;
    std::vector<std::pair<int, int>> edges;
    for (int i = 0; i < k; ++i)
        for (int j = i + 1; j < k; ++j) edges.emplace_back(i, j);
    std::vector<std::vector<int>> perms;
    {
        std::vector<int> p(k);
        for (int i = 0; i < k; ++i) p[i] = i;
        do perms.push_back(p);
        while (std::next_permutation(p.begin(), p.end()));
    }
    std::vector<int> adj(k * k, 0);
    std::set<int> edge_set;
    std::function<void(size_t)> rec = [&](size_t e) {
        if (e == edges.size()) {
            if (seen.count(edge_set)) return;
            Pattern p(k);
            for (int i = 0; i < k * k; ++i)
                if (adj[i]) p.add_ordered_edge(i / k, i % k);
            if (!p.check_connected()) return;
            out.push_back(adj);
            for (const auto &v : perms) {
                std::set<int> es;
                for (int i = 0; i < k; ++i)
                    for (int j = i + 1; j < k; ++j)
                        if (adj[i * k + j]) es.insert(v[i] < v[j] ? v[i] * k + v[j] : v[j] * k + v[i]);
                seen.insert(es);
            }
            return;
        }
        const int i = edges[e].first, j = edges[e].second;
        // Patterns over max_edges edges are never emitted; they are not
        // isomorphic to any kept pattern, so dropping them leaves the kept
        // patterns, their labellings and their order unchanged.
        if (static_cast<int>(edge_set.size()) < max_edges) {
            edge_set.insert(i * k + j);
            adj[i * k + j] = adj[j * k + i] = 1;
            rec(e + 1);
            adj[i * k + j] = adj[j * k + i] = 0;
            edge_set.erase(i * k + j);
        }
        rec(e + 1);
    };
    rec(0);
    return out;
}

extern "C" {

int gi_motif_num(int k) {
    if (k < 3 || k > GI_MAX_PATTERN) return -1;
    return static_cast<int>(motif_list(k).size());
}

int gi_motif_patterns(int k, char *adj_out, int cap) {
    if (k < 3 || k > GI_MAX_PATTERN) return fail(GI_EINVAL, "motif size must be between 3 and 7");
    auto list = motif_list(k);
    if (!adj_out) return GI_OK;
    for (int m = 0; m < cap && m < static_cast<int>(list.size()); ++m)
        for (int i = 0; i < k * k; ++i) adj_out[m * k * k + i] = list[m][i] ? '1' : '0';
    return GI_OK;
}

}  // extern "C"
