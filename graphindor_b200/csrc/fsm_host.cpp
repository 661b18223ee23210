// Labeled graphs and the frequent subgraph mining driver (host side).
//
// The driver follows LabeledGraph::fsm / gpu_fsm's fsm_init (reference
// src/labeled_graph.cpp:435-606, gpu/gpu_fsm.cu:779-925):
//   1. every connected pattern with at most max_edge edges, sorted by edge
//      count (reference src/labeled_graph.cpp:180-196), each planned with the
//      analytic model (reference :438-452);
//   2. for each pattern, in that order, the labeled patterns whose labels
//      satisfy the plan's restrictions (label at d <= label at r, reference
//      :393-433) and whose sub-patterns are all frequent: the induced prefix
//      of every depth, and every sub-pattern that drops one edge and keeps
//      the last vertex connected (reference :96-178);
//   3. the MNI support of those labeled patterns on the GPU (fsm.cu), and the
//      frequent ones marked in the frequent table under every automorphism
//      (reference gpu/gpu_fsm.cu:497-511);
//   4. the result is the number of frequent labeled patterns with exactly
//      max_edge edges (reference src/labeled_graph.cpp:580-581).
#include <sys/time.h>

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <numeric>
#include <sstream>
#include <string>
#include <unordered_map>

#include "fsm.hpp"
#include "internal.hpp"

namespace gi {
namespace {

double wall_ms() {
    timeval tv;
    gettimeofday(&tv, nullptr);
    return tv.tv_sec * 1e3 + tv.tv_usec * 1e-3;
}

// Renames labels and vertices and buckets the neighbour lists, as the
// reference loader does (reference src/dataloader.cpp:440-620).
int build_labeled(int32_t v_cnt, const int64_t *vertex, const int32_t *edge, const uint32_t *labels,
                  const int32_t *order, gi_labeled_graph **out) {
    if (!out) return fail(GI_EINVAL, "out is NULL");
    *out = nullptr;
    if (v_cnt < 1 || !vertex || !labels) return fail(GI_EINVAL, "empty labeled graph");
    if (vertex[0] != 0) return fail(GI_EINVAL, "vertex[0] must be 0");
    for (int32_t v = 0; v < v_cnt; ++v)
        if (vertex[v + 1] < vertex[v]) return fail(GI_EINVAL, "vertex offsets decrease");
    const int64_t entries = vertex[v_cnt];
    if (entries > 0 && !edge) return fail(GI_EINVAL, "edge is NULL");
    for (int64_t i = 0; i < entries; ++i)
        if (edge[i] < 0 || edge[i] >= v_cnt) return fail(GI_EINVAL, "neighbour id out of range");
    std::vector<int32_t> seq(v_cnt);
    if (order) {
        std::vector<char> seen(v_cnt, 0);
        for (int32_t i = 0; i < v_cnt; ++i) {
            if (order[i] < 0 || order[i] >= v_cnt || seen[order[i]]) return fail(GI_EINVAL, "order is not a permutation");
            seen[order[i]] = 1;
            seq[i] = order[i];
        }
    } else {
        std::iota(seq.begin(), seq.end(), 0);
    }
    // Degree = listed neighbours without self-loops (duplicates count).
    std::vector<int64_t> degree(v_cnt, 0);
    for (int32_t v = 0; v < v_cnt; ++v)
        for (int64_t i = vertex[v]; i < vertex[v + 1]; ++i) degree[v] += edge[i] != v;
    const int64_t e_cnt = std::accumulate(degree.begin(), degree.end(), int64_t(0));
    if (e_cnt >= (int64_t(1) << 32)) return fail(GI_EOVERFLOW, "more than 2^32 - 1 neighbour entries");
    // Symmetry: u in N(v) iff v in N(u).
    {
        std::vector<int32_t> sorted(edge, edge + entries);
        for (int32_t v = 0; v < v_cnt; ++v) std::sort(sorted.begin() + vertex[v], sorted.begin() + vertex[v + 1]);
        for (int32_t v = 0; v < v_cnt; ++v)
            for (int64_t i = vertex[v]; i < vertex[v + 1]; ++i) {
                const int32_t u = sorted[i];
                if (u == v) continue;
                if (!std::binary_search(sorted.begin() + vertex[u], sorted.begin() + vertex[u + 1], v))
                    return fail(GI_EINVAL, "neighbour lists are not symmetric");
            }
    }
    // Labels in first-seen order, then renamed by descending maximum degree.
    std::unordered_map<uint32_t, int32_t> first;
    std::vector<uint32_t> first_value;
    std::vector<int32_t> tmp_label(v_cnt);
    for (int32_t v : seq) {
        auto it = first.find(labels[v]);
        if (it == first.end()) {
            it = first.emplace(labels[v], static_cast<int32_t>(first_value.size())).first;
            first_value.push_back(labels[v]);
        }
        tmp_label[v] = it->second;
    }
    const int32_t l_cnt = static_cast<int32_t>(first_value.size());
    if (l_cnt > 255) return fail(GI_ENOTSUP, "more than 255 labels");
    if (static_cast<int64_t>(v_cnt) * l_cnt >= (int64_t(1) << 31))
        return fail(GI_EOVERFLOW, "v_cnt * l_cnt does not fit the bucket index");
    std::vector<int64_t> max_deg(l_cnt, 0);
    for (int32_t v = 0; v < v_cnt; ++v) max_deg[tmp_label[v]] = std::max(max_deg[tmp_label[v]], degree[v]);
    // The reference sorts (label, max degree) pairs with std::sort, which is
    // not stable: the same call on the same sequence resolves ties the same
    // way (reference src/dataloader.cpp:528-536).
    std::vector<std::pair<int, double>> by_deg;
    by_deg.reserve(l_cnt);
    for (int32_t l = 0; l < l_cnt; ++l) by_deg.emplace_back(l, static_cast<double>(max_deg[l]));
    std::sort(by_deg.begin(), by_deg.end(),
              [](const std::pair<int, double> &a, const std::pair<int, double> &b) { return a.second > b.second; });
    std::vector<int32_t> rename(l_cnt);
    for (int32_t i = 0; i < l_cnt; ++i) rename[by_deg[i].first] = i;

    auto *g = new (std::nothrow) gi_labeled_graph;
    if (!g) return fail(GI_ENOMEM, "host allocation");
    g->v_cnt = v_cnt;
    g->e_cnt = e_cnt;
    g->l_cnt = l_cnt;
    g->label_value.resize(l_cnt);
    for (int32_t l = 0; l < l_cnt; ++l) g->label_value[rename[l]] = first_value[l];
    std::vector<int32_t> lab(v_cnt);
    for (int32_t v = 0; v < v_cnt; ++v) lab[v] = rename[tmp_label[v]];
    // New ids by (label, -degree, id) (reference src/dataloader.cpp:542-553).
    std::vector<int32_t> rank(v_cnt);
    std::iota(rank.begin(), rank.end(), 0);
    std::sort(rank.begin(), rank.end(), [&](int32_t a, int32_t b) {
        if (lab[a] != lab[b]) return lab[a] < lab[b];
        if (degree[a] != degree[b]) return degree[a] > degree[b];
        return a < b;
    });
    g->new_id.resize(v_cnt);
    g->v_label.resize(v_cnt);
    for (int32_t i = 0; i < v_cnt; ++i) {
        g->new_id[rank[i]] = i;
        g->v_label[i] = lab[rank[i]];
    }
    g->label_frequency.assign(l_cnt, 0);
    for (int32_t v = 0; v < v_cnt; ++v) ++g->label_frequency[lab[v]];
    g->label_start.assign(l_cnt + 1, 0);
    for (int32_t l = 0; l < l_cnt; ++l) g->label_start[l + 1] = g->label_start[l] + static_cast<uint32_t>(g->label_frequency[l]);
    // Neighbour lists in new ids, sorted by (label, id); bucket[v*L+l] is the
    // first entry of v with label >= l (reference src/dataloader.cpp:576-616).
    g->edge.resize(e_cnt);
    g->bucket.assign(static_cast<size_t>(v_cnt) * l_cnt + 1, 0);
    int64_t pos = 0;
    std::vector<uint32_t> list;
    for (int32_t u = 0; u < v_cnt; ++u) {
        const int32_t x = rank[u];
        list.clear();
        for (int64_t i = vertex[x]; i < vertex[x + 1]; ++i)
            if (edge[i] != x) list.push_back(static_cast<uint32_t>(g->new_id[edge[i]]));
        std::sort(list.begin(), list.end(), [&](uint32_t a, uint32_t b) {
            const int32_t la = g->v_label[a], lb = g->v_label[b];
            return la != lb ? la < lb : a < b;
        });
        size_t k = 0;
        for (int32_t l = 0; l < l_cnt; ++l) {
            while (k < list.size() && g->v_label[list[k]] < l) ++k;
            g->bucket[static_cast<size_t>(u) * l_cnt + l] = static_cast<uint32_t>(pos + k);
        }
        std::copy(list.begin(), list.end(), g->edge.begin() + pos);
        pos += static_cast<int64_t>(list.size());
    }
    g->bucket[static_cast<size_t>(v_cnt) * l_cnt] = static_cast<uint32_t>(e_cnt);
    *out = g;  // copied to the device by the first gi_fsm
    return GI_OK;
}

// ----------------------------------------------------------------- patterns

int edge_count(const std::vector<int> &adj, int n) {
    int c = 0;
    for (int i = 0; i < n; ++i)
        for (int j = i + 1; j < n; ++j) c += adj[i * n + j] != 0;
    return c;
}

struct Check {
    int s0;                // earlier pattern
    std::vector<int> map;  // vertex k of s0 -> vertex of this pattern
};

struct FsmPattern {
    int n = 1;
    int edges = 0;
    std::vector<int> adj{0};                    // schedule order
    std::vector<std::vector<int>> restrict_of;  // per depth d: r with label[d] <= label[r]
    std::vector<std::vector<int>> auts;
    std::vector<std::vector<Check>> checks;     // per depth
    uint64_t base = 0;                          // first entry in the frequent table
};

// Finds an earlier pattern isomorphic to `sub` (m vertices, e edges) and an
// isomorphism onto it.  Sub-patterns always have fewer edges than the
// pattern they come from, so they precede it in the edge-sorted list.
bool find_iso(const std::vector<FsmPattern> &pats, size_t before, const std::vector<int> &sub, int m, int e,
              Check &out) {
    std::vector<int> perm(m);
    for (size_t s = 0; s < before; ++s) {
        const FsmPattern &p = pats[s];
        if (p.n != m || p.edges != e) continue;
        std::iota(perm.begin(), perm.end(), 0);
        do {
            bool ok = true;
            for (int a = 0; a < m && ok; ++a)
                for (int b = a + 1; b < m; ++b)
                    if ((p.adj[a * m + b] != 0) != (sub[perm[a] * m + perm[b]] != 0)) {
                        ok = false;
                        break;
                    }
            if (ok) {
                out.s0 = static_cast<int>(s);
                out.map = perm;
                return true;
            }
        } while (std::next_permutation(perm.begin(), perm.end()));
    }
    return false;
}

// The sub-pattern checks of pattern `idx` (reference
// src/labeled_graph.cpp:96-178): depth d < n-1 checks the induced prefix of
// vertices 0..d; depth n-1 checks every one-edge-smaller sub-pattern that
// keeps the last vertex, the edge count dropping by exactly one.
void build_checks(std::vector<FsmPattern> &pats, size_t idx) {
    FsmPattern &s = pats[idx];
    const int n = s.n;
    s.checks.assign(n, {});
    for (int d = 0; d + 1 < n; ++d) {
        const int m = d + 1;
        std::vector<int> sub(m * m);
        for (int a = 0; a < m; ++a)
            for (int b = 0; b < m; ++b) sub[a * m + b] = s.adj[a * n + b];
        Check c;
        if (find_iso(pats, idx, sub, m, edge_count(sub, m), c)) s.checks[d].push_back(c);
    }
    std::vector<int> tmp = s.adj;
    for (int i = 0; i < n; ++i)
        for (int j = i + 1; j < n; ++j) {
            if (!s.adj[i * n + j]) continue;
            tmp[i * n + j] = tmp[j * n + i] = 0;
            std::vector<int> comp{n - 1};
            std::vector<char> seen(n, 0);
            seen[n - 1] = 1;
            for (size_t h = 0; h < comp.size(); ++h)
                for (int w = 0; w < n; ++w)
                    if (tmp[comp[h] * n + w] && !seen[w]) {
                        seen[w] = 1;
                        comp.push_back(w);
                    }
            const int m = static_cast<int>(comp.size());
            std::vector<int> sub(m * m);
            for (int a = 0; a < m; ++a)
                for (int b = 0; b < m; ++b) sub[a * m + b] = tmp[comp[a] * n + comp[b]];
            tmp[i * n + j] = tmp[j * n + i] = 1;
            const int e = edge_count(sub, m);
            if (e != s.edges - 1) continue;
            Check c;
            if (find_iso(pats, idx, sub, m, e, c)) {
                for (int &k : c.map) k = comp[k];
                s.checks[n - 1].push_back(c);
            }
        }
}

// The patterns of an FSM run with their plans, checks and table offsets.
int plan_patterns(int max_edge, int32_t v_cnt, int64_t e_cnt, int64_t tri_cnt, int32_t l_cnt,
                  std::vector<FsmPattern> &pats) {
    pats.clear();
    pats.emplace_back();  // the single vertex
    std::vector<std::pair<int, std::vector<int>>> found;  // (n, adj)
    for (int k = 2; k <= max_edge + 1; ++k)
        for (auto &adj : motif_list(k, max_edge))
            if (edge_count(adj, k) <= max_edge) found.emplace_back(k, adj);
    std::stable_sort(found.begin(), found.end(), [](const auto &a, const auto &b) {
        return edge_count(a.second, a.first) < edge_count(b.second, b.first);
    });
    if (found.size() + 1 > GI_FSM_MAX_PATTERNS) return fail(GI_ENOTSUP, "too many patterns for max_edge");
    for (auto &f : found) {
        const int n = f.first;
        std::string s(n * n, '0');
        for (int i = 0; i < n * n; ++i) s[i] = f.second[i] ? '1' : '0';
        Pattern p(n, s.c_str());
        bool valid = false;
        // Model 1, restrictions type 1, IEP on: the reference's FSM schedules
        // (reference src/labeled_graph.cpp:446).
        Schedule_IEP sched(p, valid, 1, 1, true, v_cnt, e_cnt, tri_cnt);
        FsmPattern fp;
        fp.n = n;
        fp.edges = edge_count(f.second, n);
        fp.adj.assign(sched.get_adj_mat_ptr(), sched.get_adj_mat_ptr() + n * n);
        fp.restrict_of.assign(n, {});
        for (int d = 0; d < n; ++d)
            for (int r = sched.get_restrict_last(d); r != -1; r = sched.get_restrict_next(r))
                fp.restrict_of[d].push_back(sched.get_restrict_index(r));
        std::vector<int> perm(n);
        std::iota(perm.begin(), perm.end(), 0);
        do {
            bool ok = true;
            for (int a = 0; a < n && ok; ++a)
                for (int b = 0; b < n; ++b)
                    if (fp.adj[a * n + b] != fp.adj[perm[a] * n + perm[b]]) {
                        ok = false;
                        break;
                    }
            if (ok) fp.auts.push_back(perm);
        } while (std::next_permutation(perm.begin(), perm.end()));
        pats.push_back(std::move(fp));
        build_checks(pats, pats.size() - 1);
    }
    uint64_t base = 0;
    for (auto &fp : pats) {
        fp.base = base;
        uint64_t span = 1;
        for (int i = 0; i < fp.n; ++i) span *= static_cast<uint64_t>(std::max(l_cnt, 1));
        base += span;
        if (base > (uint64_t(1) << 36)) return fail(GI_ENOTSUP, "label space too large for max_edge");
    }
    return GI_OK;
}

struct FreqTable {
    std::vector<uint64_t> words;
    void init(uint64_t bits) { words.assign((bits + 63) / 64, 0); }
    bool test(uint64_t i) const { return (words[i >> 6] >> (i & 63)) & 1; }
    void set(uint64_t i) { words[i >> 6] |= uint64_t(1) << (i & 63); }
};

uint64_t table_index(const FsmPattern &p, const Check *c, const uint8_t *lab, int32_t l_cnt, const int *perm) {
    uint64_t idx = p.base, pw = 1;
    for (int k = 0; k < p.n; ++k) {
        const int src = c ? c->map[k] : perm[k];
        idx += lab[src] * pw;
        pw *= static_cast<uint64_t>(l_cnt);
    }
    return idx;
}

// Labeled patterns of pattern `s` under its restrictions whose sub-patterns
// are all frequent, in the reference's depth-first label order.
void enumerate_jobs(const std::vector<FsmPattern> &pats, const FsmPattern &s, const FreqTable &freq, int32_t l_cnt,
                    std::vector<uint8_t> &jobs) {
    uint8_t lab[GI_MAX_PATTERN] = {};
    const int n = s.n;
    auto rec = [&](auto &&self, int d) -> void {
        if (d == n) {
            jobs.insert(jobs.end(), lab, lab + n);
            return;
        }
        int top = l_cnt - 1;
        for (int r : s.restrict_of[d])
            if (r < d) top = std::min<int>(top, lab[r]);
        for (int l = 0; l <= top; ++l) {
            lab[d] = static_cast<uint8_t>(l);
            bool ok = true;
            for (const Check &c : s.checks[d])
                if (!freq.test(table_index(pats[c.s0], &c, lab, l_cnt, nullptr))) {
                    ok = false;
                    break;
                }
            if (ok) self(self, d + 1);
        }
    };
    rec(rec, 0);
}

// Rooted matching orders for the support kernel: from each root, repeatedly
// the unvisited vertex with the most visited neighbours (lowest id on ties).
FsmDevPattern device_pattern(const FsmPattern &s, int32_t l_cnt, int64_t min_support) {
    FsmDevPattern P;
    const int n = s.n;
    P.n = n;
    P.l_cnt = l_cnt;
    P.min_support = min_support;
    for (int a = 0; a < n; ++a)
        for (int b = 0; b < n; ++b)
            if (s.adj[a * n + b]) P.adj_mask[a] |= static_cast<uint8_t>(1u << b);
    for (int r = 0; r < n; ++r) {
        std::vector<char> in(n, 0);
        in[r] = 1;
        P.order[r][0] = static_cast<uint8_t>(r);
        for (int t = 1; t < n; ++t) {
            int best = -1, best_links = -1;
            for (int q = 0; q < n; ++q) {
                if (in[q]) continue;
                int links = 0;
                for (int u = 0; u < t; ++u) links += s.adj[q * n + P.order[r][u]] != 0;
                if (links > best_links) {
                    best = q;
                    best_links = links;
                }
            }
            in[best] = 1;
            P.order[r][t] = static_cast<uint8_t>(best);
            for (int u = 0; u < t; ++u)
                if (s.adj[best * n + P.order[r][u]]) P.parents[r][t] |= static_cast<uint8_t>(1u << u);
        }
    }
    return P;
}

void describe(const FsmPattern &fp, gi_fsm_pattern &o) {
    std::memset(&o, 0, sizeof(o));
    o.n = fp.n;
    o.edges = fp.edges;
    for (int i = 0; i < GI_MAX_PATTERN * GI_MAX_PATTERN; ++i) o.adj[i] = '0';
    for (int i = 0; i < fp.n * fp.n; ++i) o.adj[i] = fp.adj[i] ? '1' : '0';
    for (int d = 0; d < fp.n; ++d)
        for (int r : fp.restrict_of[d])
            if (o.n_restricts < 21) {
                o.restricts[o.n_restricts][0] = d;
                o.restricts[o.n_restricts][1] = r;
                ++o.n_restricts;
            }
    o.n_automorphisms = static_cast<int32_t>(fp.auts.size());
}

}  // namespace
}  // namespace gi

using namespace gi;

extern "C" {

int gi_labeled_graph_create(int32_t v_cnt, const int64_t *vertex, const int32_t *edge, const uint32_t *labels,
                            const int32_t *order, gi_labeled_graph **out) {
    try {
        return build_labeled(v_cnt, vertex, edge, labels, order, out);
    } catch (const std::bad_alloc &) {
        return fail(GI_ENOMEM, "host allocation");
    }
}

int gi_labeled_graph_load_adj(const char *path, gi_labeled_graph **out) {
    if (!path || !out) return fail(GI_EINVAL, "NULL argument");
    std::ifstream in(path);
    if (!in) return fail(GI_EIO, std::string("cannot open ") + path);
    try {
        int64_t v_cnt = -1;
        if (!(in >> v_cnt) || v_cnt < 1 || v_cnt > INT32_MAX) return fail(GI_EIO, "bad vertex count");
        std::string line;
        std::getline(in, line);
        std::vector<uint32_t> labels(v_cnt, 0);
        std::vector<int32_t> order;
        std::vector<std::vector<int32_t>> nbr(v_cnt);
        std::vector<char> seen(v_cnt, 0);
        order.reserve(v_cnt);
        while (std::getline(in, line)) {
            std::istringstream ls(line);
            int64_t x;
            uint64_t y;
            if (!(ls >> x)) continue;  // blank line
            if (!(ls >> y)) return fail(GI_EIO, "vertex line without a label");
            if (x < 0 || x >= v_cnt) return fail(GI_EINVAL, "vertex id out of range");
            if (seen[x]) return fail(GI_EINVAL, "vertex listed twice");
            seen[x] = 1;
            order.push_back(static_cast<int32_t>(x));
            labels[x] = static_cast<uint32_t>(y);
            int64_t w;
            while (ls >> w) {
                if (w < 0 || w >= v_cnt) return fail(GI_EINVAL, "neighbour id out of range");
                nbr[x].push_back(static_cast<int32_t>(w));
            }
        }
        if (static_cast<int64_t>(order.size()) != v_cnt) return fail(GI_EIO, "vertex number error");
        std::vector<int64_t> vertex(v_cnt + 1, 0);
        for (int64_t v = 0; v < v_cnt; ++v) vertex[v + 1] = vertex[v] + static_cast<int64_t>(nbr[v].size());
        std::vector<int32_t> edge(vertex[v_cnt]);
        for (int64_t v = 0; v < v_cnt; ++v) std::copy(nbr[v].begin(), nbr[v].end(), edge.begin() + vertex[v]);
        return build_labeled(static_cast<int32_t>(v_cnt), vertex.data(), edge.data(), labels.data(), order.data(),
                             out);
    } catch (const std::bad_alloc &) {
        return fail(GI_ENOMEM, "host allocation");
    }
}

int gi_labeled_graph_destroy(gi_labeled_graph *g) {
    if (!g) return GI_OK;
    fsm_free(g);
    delete g;
    return GI_OK;
}

int gi_labeled_graph_get_info(const gi_labeled_graph *g, gi_labeled_graph_info *out) {
    if (!g || !out) return fail(GI_EINVAL, "NULL argument");
    out->v_cnt = g->v_cnt;
    out->e_cnt = g->e_cnt;
    out->l_cnt = g->l_cnt;
    out->device = g->device;
    return GI_OK;
}

int gi_labeled_graph_export(const gi_labeled_graph *g, int32_t *new_id, int32_t *v_label, uint32_t *label_value,
                            uint32_t *label_start, uint32_t *bucket, uint32_t *edge) {
    if (!g) return fail(GI_EINVAL, "NULL graph");
    if (bucket || edge) {
        const int st = labeled_graph_download(g);
        if (st != GI_OK) return st;
    }
    if (new_id) std::copy(g->new_id.begin(), g->new_id.end(), new_id);
    if (v_label) std::copy(g->v_label.begin(), g->v_label.end(), v_label);
    if (label_value) std::copy(g->label_value.begin(), g->label_value.end(), label_value);
    if (label_start) std::copy(g->label_start.begin(), g->label_start.end(), label_start);
    if (bucket) std::copy(g->bucket.begin(), g->bucket.end(), bucket);
    if (edge) std::copy(g->edge.begin(), g->edge.end(), edge);
    return GI_OK;
}

int gi_fsm_plan(int max_edge, int32_t v_cnt, int64_t e_cnt, int64_t tri_cnt, gi_fsm_pattern *patterns, int cap,
                int *count) {
    if (max_edge < 0 || max_edge > GI_MAX_PATTERN - 1) return fail(GI_EINVAL, "max_edge must be in [0, 6]");
    try {
        std::vector<FsmPattern> pats;
        const int st = plan_patterns(max_edge, v_cnt, e_cnt, tri_cnt, 1, pats);
        if (st != GI_OK) return st;
        if (count) *count = static_cast<int>(pats.size()) - 1;
        for (size_t i = 1; i < pats.size() && patterns && static_cast<int>(i) - 1 < cap; ++i)
            describe(pats[i], patterns[i - 1]);
        return GI_OK;
    } catch (const std::exception &e) {
        return fail(GI_EINVAL, e.what());
    }
}

int gi_fsm(gi_labeled_graph *g, int max_edge, int64_t min_support, int64_t tri_cnt, gi_stream stream,
           int64_t *out_fsm_cnt, gi_fsm_stats *stats) {
    if (!g || !out_fsm_cnt) return fail(GI_EINVAL, "NULL argument");
    if (max_edge < 0 || max_edge > GI_MAX_PATTERN - 1) return fail(GI_EINVAL, "max_edge must be in [0, 6]");
    if (min_support < 1) return fail(GI_EINVAL, "min_support must be at least 1");
    std::lock_guard<std::mutex> lock(g->mu);
    const double t0 = wall_ms();
    if (!g->d_edge) {
        const int st = fsm_upload(g);
        if (st != GI_OK) {
            fsm_free(g);
            return st;
        }
    }
    try {
        std::vector<FsmPattern> pats;
        int st = plan_patterns(max_edge, g->v_cnt, g->e_cnt, tri_cnt, g->l_cnt, pats);
        if (st != GI_OK) return st;
        FreqTable freq;
        freq.init(pats.back().base + [&] {
            uint64_t span = 1;
            for (int i = 0; i < pats.back().n; ++i) span *= static_cast<uint64_t>(g->l_cnt);
            return span;
        }());
        int64_t fsm_cnt = 0;
        // Single vertices: frequent when the label occurs min_support times
        // (reference gpu/gpu_fsm.cu:791-797).
        for (int32_t l = 0; l < g->l_cnt; ++l)
            if (g->label_frequency[l] >= min_support) {
                freq.set(pats[0].base + static_cast<uint64_t>(l));
                if (max_edge == 0) ++fsm_cnt;
            }
        FsmRunStats rs;
        int64_t all_jobs = 0;
        int written = 0;
        for (size_t i = 1; i < pats.size(); ++i) {
            const FsmPattern &s = pats[i];
            std::vector<uint8_t> jobs;
            enumerate_jobs(pats, s, freq, g->l_cnt, jobs);
            const int64_t n_jobs = static_cast<int64_t>(jobs.size()) / s.n;
            std::vector<uint8_t> frequent;
            const double k0 = rs.kernel_ms;
            if (n_jobs > 0) {
                st = fsm_support(g, device_pattern(s, g->l_cnt, min_support), jobs, n_jobs, stream, frequent, rs);
                if (st != GI_OK) return st;
            }
            int64_t hits = 0;
            for (int64_t j = 0; j < n_jobs; ++j) {
                if (!frequent[j]) continue;
                ++hits;
                const uint8_t *lab = jobs.data() + j * s.n;
                for (const auto &aut : s.auts) freq.set(table_index(s, nullptr, lab, g->l_cnt, aut.data()));
            }
            if (s.edges == max_edge) fsm_cnt += hits;
            all_jobs += n_jobs;
            if (stats && stats->patterns && written < GI_FSM_MAX_PATTERNS) {
                gi_fsm_pattern &o = stats->patterns[written++];
                describe(s, o);
                o.jobs = n_jobs;
                o.frequent = hits;
                o.kernel_ms = rs.kernel_ms - k0;
            }
        }
        *out_fsm_cnt = fsm_cnt;
        if (stats) {
            stats->kernel_ms = rs.kernel_ms;
            stats->total_ms = wall_ms() - t0;
            stats->jobs = all_jobs;
            stats->candidates = rs.candidates;
            stats->kernel_launches = rs.launches;
            stats->n_patterns = written;
        }
        return GI_OK;
    } catch (const std::bad_alloc &) {
        return fail(GI_ENOMEM, "host allocation");
    } catch (const std::exception &e) {
        return fail(GI_EINVAL, e.what());
    }
}

}  // extern "C"
