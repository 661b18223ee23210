// Host-side planner: Pattern and Schedule_IEP (see planner.hpp).
//
// Every step below follows the reference planner (reference
// src/schedule_IEP.cpp, src/pattern.cpp) so that the plan it emits is the
// same plan, field for field.  Floating-point expressions of the analytic
// model keep the reference's evaluation order; this file must be compiled
// without FMA contraction (-ffp-contract=off) so that ties between candidate
// orders break the same way.
#include "planner.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <numeric>
#include <tuple>
#include <unordered_map>

namespace gi {

// ---------------------------------------------------------------- Pattern

Pattern::Pattern(int n, bool clique) : n_(n), adj_(static_cast<size_t>(n) * n, 0) {
    if (clique)
        for (int i = 0; i < n; ++i)
            for (int j = 0; j < i; ++j) add_edge(i, j);
}

Pattern::Pattern(int n, const char *adj_string) : n_(n), adj_(static_cast<size_t>(n) * n, 0) {
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j)
            if (adj_string[i * n + j] == '1') add_edge(i, j);
}

void Pattern::add_edge(int x, int y) { adj_[x * n_ + y] = adj_[y * n_ + x] = 1; }
void Pattern::del_edge(int x, int y) { adj_[x * n_ + y] = adj_[y * n_ + x] = 0; }

int Pattern::edge_count() const {
    int c = 0;
    for (int i = 0; i < n_; ++i)
        for (int j = i + 1; j < n_; ++j) c += adj_[i * n_ + j] != 0;
    return c;
}

bool Pattern::check_connected() const {
    std::vector<char> seen(n_, 0);
    std::vector<int> queue{0};
    seen[0] = 1;
    for (size_t h = 0; h < queue.size(); ++h)
        for (int i = 0; i < n_; ++i)
            if (adj_[queue[h] * n_ + i] && !seen[i]) {
                seen[i] = 1;
                queue.push_back(i);
            }
    return static_cast<int>(queue.size()) == n_;
}

// Kahn's algorithm over the directed entries adj(x,y) > 0.
bool Pattern::is_dag() const {
    std::vector<int> indeg(n_, 0), queue;
    for (int i = 0; i < n_; ++i)
        for (int j = 0; j < n_; ++j)
            if (adj_[i * n_ + j] > 0) ++indeg[j];
    for (int i = 0; i < n_; ++i)
        if (!indeg[i]) queue.push_back(i);
    for (size_t h = 0; h < queue.size(); ++h)
        for (int j = 0; j < n_; ++j)
            if (adj_[queue[h] * n_ + j] > 0 && --indeg[j] == 0) queue.push_back(j);
    return static_cast<int>(queue.size()) == n_;
}

// ----------------------------------------------------------- small helpers

namespace {

// All permutations of 0..n-1 in lexicographic order (the order of the
// reference's get_full_permutation DFS), built once per n.
const std::vector<std::vector<int>> &all_permutations(int n) {
    static const std::vector<std::vector<std::vector<int>>> table = [] {
        std::vector<std::vector<std::vector<int>>> t(kMaxPatternSize + 1);
        for (int m = 0; m <= kMaxPatternSize; ++m) {
            std::vector<int> p(m);
            std::iota(p.begin(), p.end(), 0);
            do t[m].push_back(p);
            while (std::next_permutation(p.begin(), p.end()));
        }
        return t;
    }();
    return table.at(n);
}

// Cycle decomposition of a permutation, cycles listed from their smallest
// unvisited start (reference src/schedule_IEP.cpp:1016-1040).
std::vector<std::vector<int>> cycles_of(const std::vector<int> &perm) {
    const int n = static_cast<int>(perm.size());
    std::vector<char> used(n, 0);
    std::vector<std::vector<int>> res;
    for (int i = 0; i < n; ++i) {
        if (used[i]) continue;
        std::vector<int> c{i};
        used[i] = 1;
        for (int x = perm[i]; !used[x]; x = perm[x]) {
            used[x] = 1;
            c.push_back(x);
        }
        res.push_back(c);
    }
    return res;
}

uint64_t adj_key(const int *adj, int n) {
    uint64_t k = static_cast<uint64_t>(n);
    for (int i = 0; i < n; ++i)
        for (int j = i + 1; j < n; ++j) k = (k << 1) | (adj[i * n + j] ? 1u : 0u);
    return k;
}

using Pairs = std::vector<std::pair<int, int>>;

// A restriction list of up to 20 pairs over positions < 8, packed 6 bits a
// pair (a * 8 + b + 1, never 0) into two words, with a tag word: a hash key
// for the planner's memo tables.
struct PackedKey {
    uint64_t tag, w0, w1;
    bool operator==(const PackedKey &o) const { return tag == o.tag && w0 == o.w0 && w1 == o.w1; }
};
struct PackedKeyHash {
    size_t operator()(const PackedKey &k) const {
        uint64_t h = k.tag * 0x9E3779B97F4A7C15ull;
        h ^= k.w0 + 0x9E3779B97F4A7C15ull + (h << 6) + (h >> 2);
        h ^= k.w1 + 0x9E3779B97F4A7C15ull + (h << 6) + (h >> 2);
        return static_cast<size_t>(h);
    }
};
bool pack_pairs(uint64_t tag, const Pairs &r, PackedKey &out) {
    if (r.size() > 20) return false;
    out = {tag, 0, 0};
    for (size_t i = 0; i < r.size(); ++i) {
        const auto &p = r[i];
        if (p.first < 0 || p.first >= 8 || p.second < 0 || p.second >= 8) return false;
        const uint64_t v = static_cast<uint64_t>(p.first * 8 + p.second + 1);
        (i < 10 ? out.w0 : out.w1) |= v << (6 * (i % 10));
    }
    return true;
}

// Depth-first search of restriction sets (reference
// src/schedule_IEP.cpp:785-840).
void restriction_dfs(const Pattern &base_dag, std::vector<std::vector<int>> iso,
                     std::vector<std::vector<std::vector<int>>> groups, const Pairs &pairs,
                     std::vector<Pairs> &out) {
    for (size_t i = 0; i < iso.size();) {
        Pattern test(base_dag);
        for (const auto &p : pairs) test.add_ordered_edge(iso[i][p.first], iso[i][p.second]);
        if (!test.is_dag()) {
            groups.erase(groups.begin() + i);
            iso.erase(iso.begin() + i);
        } else {
            ++i;
        }
    }
    if (iso.size() == 1) {
        out.push_back(pairs);
        return;
    }
    for (size_t i = 0; i < groups.size();) {
        int two = 0;
        for (const auto &cyc : groups[i]) {
            if (cyc.size() != 2) continue;
            ++two;
            auto next_groups = groups;
            auto next_iso = iso;
            Pairs next_pairs = pairs;
            Pattern next_dag = base_dag;
            next_groups.erase(next_groups.begin() + i);
            next_iso.erase(next_iso.begin() + i);
            next_pairs.emplace_back(cyc[0], cyc[1]);
            next_dag.add_ordered_edge(cyc[0], cyc[1]);
            restriction_dfs(next_dag, next_iso, next_groups, next_pairs, out);
        }
        if (two >= 1) break;
        ++i;
    }
}

// Fraction of the n! vertex labelings that satisfy each prefix of a sorted
// restriction list, turned into conditional selectivities (reference
// src/schedule_IEP.cpp:330-346).  Memoised per thread.
const std::vector<double> &restriction_selectivity(const Pairs &sorted, int n) {
    thread_local std::unordered_map<PackedKey, std::vector<double>, PackedKeyHash> cache;
    thread_local std::map<std::pair<int, Pairs>, std::vector<double>> long_cache;  // lists that do not pack
    PackedKey key;
    const bool packed = pack_pairs(static_cast<uint64_t>(n), sorted, key);
    if (packed) {
        auto it = cache.find(key);
        if (it != cache.end()) return it->second;
    } else {
        auto it = long_cache.find(std::make_pair(n, sorted));
        if (it != long_cache.end()) return it->second;
    }
    const int rs = static_cast<int>(sorted.size());
    std::vector<double> sum(rs, 0.0);
    std::vector<int> tmp(n);
    std::iota(tmp.begin(), tmp.end(), 0);
    do {
        for (int i = 0; i < rs; ++i) {
            if (tmp[sorted[i].first] > tmp[sorted[i].second])
                sum[i] += 1;
            else
                break;
        }
    } while (std::next_permutation(tmp.begin(), tmp.end()));
    double total = 1;
    for (int i = 2; i <= n; ++i) total *= i;
    for (int i = 0; i < rs; ++i) sum[i] = sum[i] / total;
    for (int i = rs - 1; i > 0; --i) sum[i] /= sum[i - 1];
    if (packed) return cache.emplace(key, std::move(sum)).first->second;
    return long_cache.emplace(std::make_pair(n, sorted), std::move(sum)).first->second;
}

// Drops pairs implied by two others, as add_restrict does (reference
// src/schedule_IEP.cpp:650-668).
Pairs filter_implied(Pairs r) {
    for (size_t i = 0; i < r.size();) {
        bool tag = true;
        for (size_t j = 0; j < r.size() && tag; ++j) {
            if (i != j && r[j].first == r[i].first)
                for (size_t k = 0; k < r.size(); ++k)
                    if (i != k && j != k && r[k].second == r[i].second && r[j].second == r[k].first) {
                        tag = false;
                        break;
                    }
        }
        if (!tag)
            r.erase(r.begin() + i);
        else
            ++i;
    }
    return r;
}

}  // namespace

// An embedding f and its automorphic images f∘σ cover one subgraph.  A
// restriction set R (pairs (a, b): value at b < value at a) counts that
// subgraph #{σ in Aut : the ranking of f∘σ satisfies R} times, which depends
// only on the ranking π of f's values.  Returns that number when it is the
// same for every ranking π (then count = raw / it), or 0 when it varies (R
// over- or under-counts some subgraphs).  Memoised per thread.
int restriction_multiplicity(const int *adj, int n, const std::vector<std::pair<int, int>> &R) {
    thread_local std::unordered_map<PackedKey, int, PackedKeyHash> cache;
    PackedKey key;
    const bool packed = pack_pairs(adj_key(adj, n), R, key);
    if (packed) {
        auto it = cache.find(key);
        if (it != cache.end()) return it->second;
    }
    // Automorphisms by backtracking: position i takes an unused vertex of the
    // same degree whose adjacency to the earlier positions matches.
    std::vector<std::vector<int>> aut;
    {
        int deg[kMaxPatternSize] = {};
        for (int i = 0; i < n; ++i)
            for (int j = 0; j < n; ++j) deg[i] += adj[i * n + j] != 0;
        std::vector<int> p(n);
        bool used[kMaxPatternSize] = {};
        auto extend = [&](auto &&self, int i) -> void {
            if (i == n) {
                aut.push_back(p);
                return;
            }
            for (int x = 0; x < n; ++x) {
                if (used[x] || deg[x] != deg[i]) continue;
                bool ok = true;
                for (int j = 0; j < i && ok; ++j) ok = (adj[j * n + i] != 0) == (adj[p[j] * n + x] != 0);
                if (!ok) continue;
                p[i] = x;
                used[x] = true;
                self(self, i + 1);
                used[x] = false;
            }
        };
        extend(extend, 0);
    }
    int common = -1;
    if (R.empty()) {
        common = static_cast<int>(aut.size());  // every ranking satisfies no restriction
    } else if (aut.size() == 1) {
        common = 0;  // some ranking breaks a restriction: count 0 for it
    }
    if (common == -1) {
        // c(pi) = automorphisms s whose ranking pi∘s satisfies R; it must be
        // the same, and nonzero, for every ranking pi.
        int first = -1;
        for (const auto &pi : all_permutations(n)) {
            int c = 0;
            for (const auto &s : aut) {
                bool sat = true;
                for (const auto &r : R)
                    if (!(pi[s[r.second]] < pi[s[r.first]])) { sat = false; break; }
                c += sat;
            }
            if (first == -1) first = c;
            if (c != first || c == 0) {
                first = 0;
                break;
            }
        }
        common = first < 0 ? 0 : first;
    }
    if (packed) cache.emplace(key, common);
    return common;
}

// ---------------------------------------------------------- Schedule_IEP

// Pattern-only state of the model constructor, shared by every plan of the
// same pattern (any graph).  Bounded: the whole cache is dropped when it
// holds more than kModelCacheEntries patterns.
struct Schedule_IEP::ModelKey {
    int n;
    uint64_t adj;
    bool use_iep;
    bool vertex_induced;
    bool operator<(const ModelKey &o) const {
        return std::tie(n, adj, use_iep, vertex_induced) < std::tie(o.n, o.adj, o.use_iep, o.vertex_induced);
    }
};

struct Schedule_IEP::ModelState {
    std::vector<std::vector<int>> candidates;  // orders of maximal IEP depth, in enumeration order
    std::vector<std::vector<Pairs>> sets;      // restriction sets per order
    std::vector<int> iep_num;                  // IEP depth per order
    std::vector<int> rep;                      // first order with the same ordered adjacency (same scores)
    std::unique_ptr<const Schedule_IEP> replayed;  // state after the replay of every order
    mutable std::mutex mu;
    mutable std::map<std::pair<int, int>, long long> redundancy;  // by chosen (order, set); set -1 = none
};

namespace {
constexpr size_t kModelCacheEntries = 4096;
std::mutex g_model_mu;
std::map<Schedule_IEP::ModelKey, std::shared_ptr<const Schedule_IEP::ModelState>> g_model_cache;
}  // namespace

std::shared_ptr<const Schedule_IEP::ModelState> Schedule_IEP::model_cache_find(const ModelKey &k) {
    std::lock_guard<std::mutex> lock(g_model_mu);
    auto it = g_model_cache.find(k);
    return it == g_model_cache.end() ? nullptr : it->second;
}

std::shared_ptr<const Schedule_IEP::ModelState> Schedule_IEP::model_cache_insert(const ModelKey &k,
                                                                                std::shared_ptr<ModelState> s) {
    std::lock_guard<std::mutex> lock(g_model_mu);
    if (g_model_cache.size() >= kModelCacheEntries) g_model_cache.clear();
    return g_model_cache.emplace(k, std::move(s)).first->second;
}


void Schedule_IEP::alloc(int n) {
    size = n;
    const int maxp = n * (n - 1) / 2 + 1;
    adj_mat.assign(static_cast<size_t>(n) * n, 0);
    father_prefix_id.assign(maxp, -1);
    last.assign(n, -1);
    next.assign(maxp, -1);
    break_size.assign(maxp, -1);
    loop_set_prefix_id.assign(n, -1);
    prefix.assign(maxp, Prefix());
    restrict_last.assign(n, -1);
    restrict_next.assign(maxp, -1);
    restrict_index.assign(maxp, -1);
    order_.resize(n);
    std::iota(order_.begin(), order_.end(), 0);
}

Schedule_IEP::Schedule_IEP(const Pattern &pattern, bool &is_pattern_valid, int performance_modeling_type,
                           int restricts_type, bool use_in_exclusion_optimize, int v_cnt, int64_t e_cnt,
                           long long tri_cnt, bool vertex_induced) {
    const int n = pattern.get_size();
    if (n < 2 || n > kMaxPatternSize)
        throw std::invalid_argument("pattern size must be between 3 and 7");
    if (performance_modeling_type < 0 || performance_modeling_type > 1)
        throw std::invalid_argument("only performance_modeling_type 0 and 1 are supported");
    if (restricts_type < 0 || restricts_type > 1)
        throw std::invalid_argument("only restricts_type 0 and 1 are supported");
    if (performance_modeling_type == 1 && restricts_type != 1)
        throw std::invalid_argument("the analytic model needs restricts_type 1");
    is_vertex_induced = vertex_induced;
    if (vertex_induced) {
        use_in_exclusion_optimize = false;
        in_exclusion_optimize_redundancy = 1;
    }
    if (performance_modeling_type == 1 && tri_cnt == -1)
        throw std::logic_error("Fatal: Can not use performance modeling if not have triangle number of this dataset.\n");
    is_pattern_valid = true;
    alloc(n);
    std::copy(pattern.get_adj_mat_ptr(), pattern.get_adj_mat_ptr() + n * n, adj_mat.begin());
    if (!pattern.check_connected()) {
        is_pattern_valid = false;
        throw std::runtime_error("pattern is not connected");
    }

    Pairs best_pairs;
    std::shared_ptr<const ModelState> st;  // model path: the pattern's cached state
    std::pair<int, int> best_ck(-1, -1);   // model path: chosen (order, restriction set) index
    if (performance_modeling_type != 0) {
        const int *src = pattern.get_adj_mat_ptr();
        // Everything the model loop does apart from scoring depends on the
        // pattern alone: the candidate orders, their restriction sets and
        // IEP depths, and the state the sequential replay leaves behind (the
        // never-cleared IEP vectors and prefix flags).  It is computed once
        // per pattern and reused for every graph; only the scores are
        // recomputed from (v_cnt, e_cnt, tri_cnt).
        const ModelKey key{n, adj_key(src, n), use_in_exclusion_optimize, vertex_induced};
        st = model_cache_find(key);
        if (st) {
            *this = *st->replayed;
        } else {
            auto ns = std::make_shared<ModelState>();
            auto candidates = all_permutations(n);
            // reference src/schedule_IEP.cpp:2019-2042: every position after
            // the first must touch an earlier one.
            candidates.erase(std::remove_if(candidates.begin(), candidates.end(),
                                            [&](const std::vector<int> &v) { return get_vec_optimize_num(v) < 0; }),
                             candidates.end());
            int max_val = 0;
            for (const auto &v : candidates) max_val = std::max(max_val, get_vec_optimize_num(v));
            k_val = max_val;
            candidates.erase(std::remove_if(candidates.begin(), candidates.end(),
                                            [&](const std::vector<int> &v) {
                                                return get_vec_optimize_num(v) != max_val;
                                            }),
                             candidates.end());
            ns->sets.resize(candidates.size());
            ns->iep_num.resize(candidates.size());
            // Restriction sets per order, on per-thread copies in parallel.
#pragma omp parallel
            {
                Schedule_IEP w;
                w.alloc(n);
#pragma omp for schedule(dynamic, 1)
                for (size_t c = 0; c < candidates.size(); ++c) {
                    w.copy_adj_mat_from(candidates[c], src);
                    w.setup_optimization_info(use_in_exclusion_optimize);
                    w.restricts_generate(ns->sets[c]);
                    ns->iep_num[c] = w.in_exclusion_optimize_num;
                }
            }
            // The replay, in the reference's order (setup_optimization_info
            // appends to vectors the reference never clears).
            for (const auto &vec : candidates) {
                copy_adj_mat_from(vec, src);
                setup_optimization_info(use_in_exclusion_optimize);
            }
            // Orders that give the same ordered adjacency have the same
            // restriction sets, IEP depth and scores.
            {
                std::map<uint64_t, int> first;
                Schedule_IEP w;
                w.alloc(n);
                ns->rep.resize(candidates.size());
                for (size_t c = 0; c < candidates.size(); ++c) {
                    w.copy_adj_mat_from(candidates[c], src);
                    ns->rep[c] = first.emplace(adj_key(w.adj_mat.data(), n), static_cast<int>(c)).first->second;
                }
            }
            ns->candidates = std::move(candidates);
            ns->replayed.reset(new Schedule_IEP(*this));
            st = model_cache_insert(key, std::move(ns));
        }
        // Scores, in parallel; the minimum is taken in the reference's order
        // (the first of equal scores wins).
        const auto &cands = st->candidates;
        std::vector<std::vector<double>> costs(cands.size());
#pragma omp parallel
        {
            Schedule_IEP w;
            w.alloc(n);
#pragma omp for schedule(dynamic, 8)
            for (size_t c = 0; c < cands.size(); ++c) {
                if (st->rep[c] != static_cast<int>(c)) continue;
                w.copy_adj_mat_from(cands[c], src);
                w.in_exclusion_optimize_num = st->iep_num[c];
                if (st->sets[c].empty()) {
                    costs[c].push_back(w.new_estimate_schedule_restrict(Pairs(), v_cnt, e_cnt, tri_cnt));
                } else {
                    for (const auto &pairs : st->sets[c])
                        costs[c].push_back(w.new_estimate_schedule_restrict(pairs, v_cnt, e_cnt, tri_cnt));
                }
            }
        }
        std::vector<int> best_order(n, 0);
        double min_val = 1e18;
        bool have_best = false;
        for (size_t c = 0; c < cands.size(); ++c) {
            const auto &sets = st->sets[c];
            const std::vector<double> &cost = costs[st->rep[c]];
            if (sets.empty()) {
                if (!have_best || cost[0] < min_val) {
                    have_best = true;
                    min_val = cost[0];
                    best_order = cands[c];
                    best_pairs.clear();
                    best_ck = {static_cast<int>(c), -1};
                }
            }
            for (size_t k = 0; k < sets.size(); ++k) {
                if (!have_best || cost[k] < min_val) {
                    have_best = true;
                    min_val = cost[k];
                    best_order = cands[c];
                    best_pairs = sets[k];
                    best_ck = {static_cast<int>(c), static_cast<int>(k)};
                }
            }
        }
        copy_adj_mat_from(best_order, src);
        order_ = best_order;
        model_cost_ = min_val;
    } else if (restricts_type != 0) {
        std::vector<Pairs> restricts_vector;
        restricts_generate(restricts_vector);
        bool have_best = false;
        double min_val = 0;
        for (const auto &pairs : restricts_vector) {
            double val = new_estimate_schedule_restrict(pairs, v_cnt, e_cnt, tri_cnt);
            if (!have_best || val < min_val) {
                have_best = true;
                min_val = val;
                best_pairs = pairs;
            }
        }
        model_cost_ = min_val;
    }

    if (!check_connectivity()) {
        is_pattern_valid = false;
        throw std::runtime_error("pattern is not connected");
    }
    setup_optimization_info(use_in_exclusion_optimize);
    chosen_pairs_ = best_pairs;
    if (restricts_type != 0) add_restrict(best_pairs);
    if (!st) {
        set_in_exclusion_optimize_redundancy();
        return;
    }
    // The redundancy depends on the pattern's replayed state and the chosen
    // (order, restriction set) only.
    {
        std::lock_guard<std::mutex> lock(st->mu);
        auto it = st->redundancy.find(best_ck);
        if (it != st->redundancy.end()) {
            in_exclusion_optimize_redundancy = it->second;
            return;
        }
    }
    set_in_exclusion_optimize_redundancy();
    std::lock_guard<std::mutex> lock(st->mu);
    st->redundancy.emplace(best_ck, in_exclusion_optimize_redundancy);
}

Schedule_IEP::Schedule_IEP(const Pattern &pattern, const std::vector<int> &order, const Pairs &restricts,
                           bool use_in_exclusion_optimize, bool exact) {
    const int n = pattern.get_size();
    if (n < 2 || n > kMaxPatternSize)
        throw std::invalid_argument("pattern size must be between 3 and 7");
    if (static_cast<int>(order.size()) != n)
        throw std::invalid_argument("order must list every pattern vertex once");
    std::vector<int> seen(n, 0);
    for (int v : order) {
        if (v < 0 || v >= n || seen[v]++) throw std::invalid_argument("order must be a permutation");
    }
    for (const auto &p : restricts)
        if (p.first < 0 || p.first >= n || p.second < 0 || p.second >= n || p.first == p.second)
            throw std::invalid_argument("restriction out of range");
    alloc(n);
    copy_adj_mat_from(order, pattern.get_adj_mat_ptr());
    order_ = order;
    if (!check_connectivity()) throw std::runtime_error("pattern is not connected");
    setup_optimization_info(use_in_exclusion_optimize);
    add_restrict(restricts);
    set_in_exclusion_optimize_redundancy();
    if (!exact) return;  // keep the reference's redundancy as the divisor
    // Explicit schedules are counted exactly: the divisor is the number of
    // automorphic images of each subgraph that pass the restrictions the DFS
    // applies (those below the IEP tail), and it must not depend on the
    // subgraph.
    std::vector<std::pair<int, int>> applied;
    for (const auto &p : restrict_pair)
        if (p.second < size - in_exclusion_optimize_num) applied.push_back(p);
    count_divisor_ = restriction_multiplicity(adj_mat.data(), size, applied);
    if (count_divisor_ == 0)
        throw std::invalid_argument("restriction set does not count every subgraph the same number of times");
}

Schedule_IEP::Schedule_IEP(const int *adj, int n) {
    if (n < 2 || n > kMaxPatternSize + 1)
        throw std::invalid_argument("pattern size must be between 2 and 8");
    alloc(n);
    std::copy(adj, adj + n * n, adj_mat.begin());
    is_vertex_induced = true;
    if (!check_connectivity()) throw std::runtime_error("pattern is not connected");
    build_loop_invariant(0);
    set_in_exclusion_optimize_redundancy();
}

// reference src/schedule_IEP.cpp:384-391: position rank[vec[i]] = i.
void Schedule_IEP::copy_adj_mat_from(const std::vector<int> &vec, const int *src) {
    std::vector<int> rank(size);
    for (int i = 0; i < size; ++i) rank[vec[i]] = i;
    for (int i = 0; i < size; ++i)
        for (int j = 0; j < size; ++j) adj_mat[rank[i] * size + rank[j]] = src[i * size + j];
}

bool Schedule_IEP::check_connectivity() const {
    for (int i = 1; i < size; ++i) {
        bool ok = false;
        for (int j = 0; j < i && !ok; ++j) ok = adj_mat[i * size + j] != 0;
        if (!ok) return false;
    }
    return true;
}

int Schedule_IEP::get_max_degree() const {
    int mx = 0;
    for (int i = 0; i < size; ++i) {
        int c = 0;
        for (int j = 0; j < size; ++j) c += adj_mat[i * size + j];
        mx = std::max(mx, c);
    }
    return mx;
}

// reference src/schedule_IEP.cpp:420-449.  The three IEP vertex vectors and
// the Prefix flags are deliberately not reset.
void Schedule_IEP::setup_optimization_info(bool use_iep) {
    const int maxp = size * (size - 1) / 2;
    std::fill(father_prefix_id.begin(), father_prefix_id.begin() + maxp, -1);
    std::fill(last.begin(), last.end(), -1);
    std::fill(next.begin(), next.begin() + maxp, -1);
    std::fill(break_size.begin(), break_size.begin() + maxp, -1);
    std::fill(restrict_last.begin(), restrict_last.end(), -1);
    std::fill(restrict_next.begin(), restrict_next.begin() + maxp, -1);
    total_prefix_num = 0;
    total_restrict_num = 0;
    if (use_iep) {
        std::vector<int> ident(size);
        std::iota(ident.begin(), ident.end(), 0);
        in_exclusion_optimize_num = get_vec_optimize_num(ident);
        if (in_exclusion_optimize_num <= 1)
            in_exclusion_optimize_num = 0;
        else
            init_in_exclusion_optimize();
    } else {
        in_exclusion_optimize_num = 0;
    }
    build_loop_invariant(in_exclusion_optimize_num);
}

// reference src/schedule_IEP.cpp:1762-1789: how many trailing positions are
// pairwise non-adjacent (the IEP tail length), or -1 for an invalid order.
int Schedule_IEP::get_vec_optimize_num(const std::vector<int> &vec) const {
    for (int i = 1; i < size; ++i) {
        bool have_edge = false;
        for (int j = 0; j < i && !have_edge; ++j) have_edge = adj_mat[vec[i] * size + vec[j]] != 0;
        if (!have_edge) return -1;
    }
    for (int k = 2; k <= size - 2; ++k) {
        for (int i = size - k + 1; i < size; ++i)
            if (adj_mat[vec[size - k] * size + vec[i]]) return k - 1;
    }
    return size - 2;
}

// reference src/schedule_IEP.cpp:480-627
void Schedule_IEP::build_loop_invariant(int iep_num) {
    std::vector<int> tmp(size);
    loop_set_prefix_id[0] = -1;
    for (int i = 1; i < size; ++i) {
        int ds = 0;
        for (int j = 0; j < i; ++j)
            if (adj_mat[i * size + j]) tmp[ds++] = j;
        loop_set_prefix_id[i] = find_father_prefix(ds, tmp.data());
    }
    basic_prefix_num = total_prefix_num;

    // break_size[p]: earlier positions (below the prefix's last member) that
    // are adjacent to every member; a set of exactly that size holds only
    // already-embedded vertices.
    for (int p = 0; p < basic_prefix_num; ++p) {
        const auto &d = prefix[p].data;
        int cnt = 0;
        for (int node = 0; node < d.back(); ++node) {
            bool in_data = false, not_connect = false;
            for (int x : d) {
                if (node == x) { in_data = true; break; }
                if (!adj_mat[node * size + x]) { not_connect = true; break; }
            }
            if (!in_data && !not_connect) ++cnt;
        }
        break_size[p] = cnt;
    }

    if (iep_num > 0) {
        in_exclusion_optimize_vertex_id.clear();
        in_exclusion_optimize_coef.clear();
        in_exclusion_optimize_flag.clear();
        const int base = size - iep_num;
        for (size_t rank = 0; rank < in_exclusion_optimize_group.size(); ++rank) {
            const auto &cur = in_exclusion_optimize_group[rank];
            const int val = in_exclusion_optimize_val[rank];
            for (size_t b = 0; b < cur.size(); ++b) {
                int ds = 0;
                for (int node = 0; node < base; ++node)
                    for (int m : cur[b])
                        if (adj_mat[node * size + m + base]) { tmp[ds++] = node; break; }
                const int my_id = find_father_prefix(ds, tmp.data());
                int equal = -1;
                for (size_t i = 0; i < in_exclusion_optimize_vertex_id.size(); ++i)
                    if (in_exclusion_optimize_vertex_id[i] == my_id) { equal = static_cast<int>(i); break; }
                if (equal == -1) {
                    in_exclusion_optimize_vertex_id.push_back(my_id);
                    equal = static_cast<int>(in_exclusion_optimize_vertex_id.size()) - 1;
                    int in_set = 0, full_connect = 0;
                    for (int i = 0; i < base; ++i) {
                        int cnt = 0;
                        bool hit = false;
                        for (int j = 0; j < ds; ++j) {
                            if (tmp[j] == i) { hit = true; break; }
                            if (adj_mat[i * size + tmp[j]]) ++cnt;
                        }
                        if (hit) ++in_set;
                        else if (cnt == ds) ++full_connect;
                    }
                    in_exclusion_optimize_vertex_flag.push_back(in_set + full_connect == base ? 1 : 0);
                    in_exclusion_optimize_vertex_coef.push_back(full_connect);
                }
                in_exclusion_optimize_ans_pos.push_back(equal);
                const bool block_last = b + 1 == cur.size();
                in_exclusion_optimize_coef.push_back(block_last ? val : 0);
                in_exclusion_optimize_flag.push_back(block_last ? 1 : 0);
            }
        }
        for (size_t i = 0; i < in_exclusion_optimize_vertex_flag.size(); ++i) {
            if (in_exclusion_optimize_vertex_flag[i] && i < in_exclusion_optimize_vertex_id.size()) {
                const int p = in_exclusion_optimize_vertex_id[i];
                if (!prefix[p].has_child) prefix[p].only_need_size = true;
            }
        }
    }

    // The per-depth lists were built newest-first; reverse them so prefixes
    // are visited in creation order (reference src/schedule_IEP.cpp:607-623).
    for (int i = 0; i < size; ++i) {
        if (last[i] == -1) continue;
        std::vector<int> buf;
        for (int id = last[i]; id != -1; id = next[id]) buf.push_back(id);
        last[i] = buf.back();
        for (int id = static_cast<int>(buf.size()) - 1; id > 0; --id) next[buf[id]] = buf[id - 1];
        next[buf[0]] = -1;
    }
}

// reference src/schedule_IEP.cpp:629-648
int Schedule_IEP::find_father_prefix(int ds, const int *data) {
    if (ds == 0) return -1;
    const int num = data[ds - 1];
    for (int p = last[num]; p != -1; p = next[p])
        if (static_cast<int>(prefix[p].data.size()) == ds && std::equal(data, data + ds, prefix[p].data.begin()))
            return p;
    const int father = find_father_prefix(ds - 1, data);
    if (father >= 0) prefix[father].has_child = true;
    father_prefix_id[total_prefix_num] = father;
    next[total_prefix_num] = last[num];
    last[num] = total_prefix_num;
    prefix[total_prefix_num].data.assign(data, data + ds);
    return total_prefix_num++;
}

// reference src/schedule_IEP.cpp:650-684.  A pair is dropped when two others
// already imply it transitively.
void Schedule_IEP::add_restrict(const Pairs &restricts) {
    restrict_pair = restricts;
    for (size_t i = 0; i < restrict_pair.size();) {
        bool tag = true;
        for (size_t j = 0; j < restrict_pair.size() && tag; ++j) {
            if (i != j && restrict_pair[j].first == restrict_pair[i].first)
                for (size_t k = 0; k < restrict_pair.size(); ++k)
                    if (i != k && j != k && restrict_pair[k].second == restrict_pair[i].second &&
                        restrict_pair[j].second == restrict_pair[k].first) {
                        tag = false;
                        break;
                    }
        }
        if (!tag)
            restrict_pair.erase(restrict_pair.begin() + i);
        else
            ++i;
    }
    const int maxp = size * (size - 1) / 2;
    std::fill(restrict_last.begin(), restrict_last.end(), -1);
    std::fill(restrict_next.begin(), restrict_next.begin() + maxp, -1);
    total_restrict_num = 0;
    for (const auto &p : restrict_pair) {
        restrict_index[total_restrict_num] = p.first;
        restrict_next[total_restrict_num] = restrict_last[p.second];
        restrict_last[p.second] = total_restrict_num;
        ++total_restrict_num;
    }
}

// The permutations v with adj(i, j) => adj(v[i], v[j]) (the automorphisms),
// in lexicographic order like a scan of all n! permutations: positions are
// filled in turn with the smallest unused vertex of the same degree whose
// edges to the earlier positions are kept.
std::vector<std::vector<int>> Schedule_IEP::get_isomorphism_vec() const {
    std::vector<std::vector<int>> out;
    const int n = size;
    int deg[kMaxPatternSize] = {};
    for (int i = 0; i < n; ++i)
        for (int j = 0; j < n; ++j) deg[i] += adj_mat[i * n + j] != 0;
    std::vector<int> v(n, -1);
    bool used[kMaxPatternSize] = {};
    int cand[kMaxPatternSize + 1];  // next vertex to try at each position
    int i = 0;
    cand[0] = 0;
    while (i >= 0) {
        if (i == n) {
            out.push_back(v);
            --i;
            used[v[i]] = false;
            continue;
        }
        int x = cand[i];
        for (; x < n; ++x) {
            if (used[x] || deg[x] != deg[i]) continue;
            bool ok = true;
            for (int j = 0; j < i && ok; ++j)
                if (adj_mat[j * n + i] && !adj_mat[v[j] * n + x]) ok = false;
            if (ok) break;
        }
        if (x == n) {  // position i exhausted: back to i - 1
            --i;
            if (i >= 0) used[v[i]] = false;
            continue;
        }
        v[i] = x;
        used[x] = true;
        cand[i] = x + 1;
        ++i;
        if (i < n) cand[i] = 0;
    }
    return out;
}

int Schedule_IEP::get_multiplicity() const { return static_cast<int>(get_isomorphism_vec().size()); }

// reference src/schedule_IEP.cpp:732-783
void Schedule_IEP::aggressive_optimize_get_all_pairs(std::vector<Pairs> &out) const {
    auto iso = get_isomorphism_vec();
    std::vector<std::vector<std::vector<int>>> groups;
    for (const auto &v : iso) groups.push_back(cycles_of(v));
    out.clear();
    Pairs pairs;
    // Automorphisms that are a single transposition give a forced pair.
    for (size_t i = 0; i < groups.size();) {
        int two = 0;
        std::pair<int, int> found;
        for (const auto &c : groups[i]) {
            if (c.size() == 2) {
                ++two;
                found = {c[0], c[1]};
            } else if (c.size() != 1) {
                two = -1;
                break;
            }
        }
        if (two == 1) {
            groups.erase(groups.begin() + i);
            iso.erase(iso.begin() + i);
            pairs.push_back(found);
        } else {
            ++i;
        }
    }
    Pattern base_dag(size);
    for (const auto &p : pairs) base_dag.add_ordered_edge(p.first, p.second);
    restriction_dfs(base_dag, iso, groups, pairs, out);
}

// reference src/schedule_IEP.cpp:1737-1760: keep the restriction sets whose
// count on K_{n+1} equals the unrestricted count divided by the number of
// automorphisms.  The check runs on a vertex-induced scratch plan, as in the
// reference.  Results are memoised per thread by adjacency matrix.
void Schedule_IEP::restricts_generate(std::vector<Pairs> &out) const {
    thread_local std::map<uint64_t, std::vector<Pairs>> cache;
    const uint64_t key = adj_key(adj_mat.data(), size);
    auto it = cache.find(key);
    if (it != cache.end()) {
        out = it->second;
        return;
    }
    Schedule_IEP plain(adj_mat.data(), size);
    plain.aggressive_optimize_get_all_pairs(out);
    const long long ans = plain.count_on_complete_graph(size + 1) / plain.get_multiplicity();
    for (size_t i = 0; i < out.size();) {
        Schedule_IEP cur(plain.get_adj_mat_ptr(), size);
        cur.add_restrict(out[i]);
        if (cur.count_on_complete_graph(size + 1) != ans)
            out.erase(out.begin() + i);
        else
            ++i;
    }
    cache.emplace(key, out);
}

// reference src/schedule_IEP.cpp:307-382
double Schedule_IEP::new_estimate_schedule_restrict(const Pairs &pairs, int v_cnt, int64_t e_cnt,
                                                    long long tri_cnt) const {
    const int max_degree = get_max_degree();
    const int len = std::max(max_degree, 2);
    std::vector<double> p_size(len, 0.0), pp_size(len, 0.0);
    const double p0 = e_cnt * 1.0 / v_cnt / v_cnt;
    const double p1 = tri_cnt * 1.0 * v_cnt / e_cnt / e_cnt;
    p_size[0] = v_cnt;
    for (int i = 1; i < max_degree; ++i) p_size[i] = p_size[i - 1] * p0;
    pp_size[0] = 1;
    for (int i = 1; i < max_degree; ++i) pp_size[i] = pp_size[i - 1] * p1;

    Pairs restricts = pairs;
    std::sort(restricts.begin(), restricts.end());
    const std::vector<double> &sum = restriction_selectivity(restricts, size);

    std::vector<std::vector<int>> invariant_size(size);
    double val = 1;
    for (int i = size - in_exclusion_optimize_num - 1; i >= 0; --i) {
        int cnt_forward = 0;
        for (int j = 0; j < i; ++j)
            if (adj_mat[j * size + i]) ++cnt_forward;
        int c = cnt_forward;
        for (int j = i - 1; j >= 0; --j)
            if (adj_mat[j * size + i]) invariant_size[j].push_back(c--);
        // The reference is built with GCC's default FMA contraction on an
        // FMA-capable -march, which fuses this update into one fma; the
        // fusion is written out so ties between orders break the same way.
        for (int s : invariant_size[i])
            if (s > 1) val = std::fma(p_size[1] * pp_size[s - 2], std::log2(p_size[1]), val);
        for (size_t j = 0; j < restricts.size(); ++j)
            if (restricts[j].second == i) val *= sum[j];
        if (i)
            val *= p_size[1] * pp_size[cnt_forward - 1];
        else
            val *= p_size[0];
    }
    return val;
}

// reference src/schedule_IEP.cpp:1400-1451: (#even, #odd) connected spanning
// edge subsets of K_n for n = 1..k, then every set partition of the k tail
// positions with its signed coefficient.
void Schedule_IEP::init_in_exclusion_optimize() {
    const int k = in_exclusion_optimize_num;
    std::vector<int> iep_val(2 * k, 0);
    for (int n = 1; n <= k; ++n) {
        if (n == 1) {
            iep_val[0] = 1;
            continue;
        }
        std::vector<std::pair<int, int>> edges;
        for (int i = 0; i < n; ++i)
            for (int j = 0; j < i; ++j) edges.emplace_back(i, j);
        const int m = static_cast<int>(edges.size());
        std::vector<int> parent(n);
        for (int s = 0; s < (1 << m); ++s) {
            std::iota(parent.begin(), parent.end(), 0);
            int comps = n, bits = 0;
            auto find = [&](int x) {
                while (parent[x] != x) x = parent[x] = parent[parent[x]];
                return x;
            };
            for (int i = 0; i < m; ++i)
                if (s & (1 << i)) {
                    ++bits;
                    int a = find(edges[i].first), b = find(edges[i].second);
                    if (a != b) {
                        parent[a] = b;
                        --comps;
                    }
                }
            if (comps == 1) ++iep_val[2 * n - 2 + (bits & 1)];
        }
    }
    in_exclusion_optimize_group.clear();
    in_exclusion_optimize_val.clear();
    std::vector<int> id(k);
    get_in_exclusion_optimize_group(0, id.data(), 0, iep_val.data());
}

// reference src/schedule_IEP.cpp:1453-1496 (restricted-growth enumeration)
void Schedule_IEP::get_in_exclusion_optimize_group(int depth, int *id, int id_cnt, const int *iep_val) {
    const int k = in_exclusion_optimize_num;
    if (depth == k) {
        std::vector<int> sz(id_cnt, 0);
        for (int i = 0; i < k; ++i) sz[id[i]]++;
        int v0 = iep_val[sz[0] * 2 - 2], v1 = iep_val[sz[0] * 2 - 1];
        for (int i = 1; i < id_cnt; ++i) {
            const int t0 = v0, t1 = v1;
            v0 = t0 * iep_val[sz[i] * 2 - 2] + t1 * iep_val[sz[i] * 2 - 1];
            v1 = t0 * iep_val[sz[i] * 2 - 1] + t1 * iep_val[sz[i] * 2 - 2];
        }
        std::vector<std::vector<int>> group(id_cnt);
        for (int i = 0; i < id_cnt; ++i)
            for (int j = 0; j < k; ++j)
                if (id[j] == i) group[i].push_back(j);
        in_exclusion_optimize_group.push_back(group);
        in_exclusion_optimize_val.push_back(v0 - v1);
        return;
    }
    id[depth] = id_cnt;
    get_in_exclusion_optimize_group(depth + 1, id, id_cnt + 1, iep_val);
    for (int i = 0; i < id_cnt; ++i) {
        id[depth] = i;
        get_in_exclusion_optimize_group(depth + 1, id, id_cnt, iep_val);
    }
}

// reference src/schedule_IEP.cpp:2050-2068: redundancy = IEP count / plain
// count, both on the complete graph K_n.
void Schedule_IEP::set_in_exclusion_optimize_redundancy() {
    const int tmp = in_exclusion_optimize_num;
    if (tmp <= 1) {
        in_exclusion_optimize_redundancy = 1;
        return;
    }
    in_exclusion_optimize_redundancy = 1;
    const long long ans = count_on_complete_graph(size);
    in_exclusion_optimize_num = 0;
    const long long true_ans = count_on_complete_graph(size);
    in_exclusion_optimize_num = tmp;
    in_exclusion_optimize_redundancy = true_ans ? ans / true_ans : 1;
}

// ------------------------------------------------- complete-graph counting
//
// The reference CPU DFS (src/graph.cpp:305-355, 429-566; set semantics from
// src/vertex_set.cpp) specialised to K_kn, whose adjacency list of v is every
// other vertex in increasing order.  Planning only ever runs it on graphs of
// at most eight vertices.
namespace {

struct CompleteDfs {
    const Schedule_IEP &s;
    int kn;
    std::vector<std::vector<int>> sets;  // per prefix
    std::vector<int> emb;
    std::vector<int> ans_buf;
    long long ans = 0;

    CompleteDfs(const Schedule_IEP &sched, int n) : s(sched), kn(n) {
        sets.resize(std::max(1, s.get_total_prefix_num()));
        ans_buf.resize(s.in_exclusion_optimize_vertex_id.size() + 1);
    }
    bool has(int v) const { return std::find(emb.begin(), emb.end(), v) != emb.end(); }
    int subtract_size(const std::vector<int> &set0, int size0) const {
        int ret = size0;
        for (int x : emb)
            if (std::binary_search(set0.begin(), set0.begin() + size0, x)) --ret;
        return ret;
    }
    // S_p = S_father ∩ N(v); in K_kn, N(v) is every vertex but v, so the
    // intersection is the father's set without v (all vertices but v for a
    // prefix without father).
    void build(int p, int v) {
        const int f = s.get_father_prefix_id(p);
        std::vector<int> &out = sets[p];
        out.clear();
        if (f == -1) {
            for (int u = 0; u < kn; ++u)
                if (u != v) out.push_back(u);
        } else {
            for (int u : sets[f])
                if (u != v) out.push_back(u);
        }
    }
    void run() {
        for (int v = 0; v < kn; ++v) {
            for (int p = s.get_last(0); p != -1; p = s.get_next(p)) build(p, v);
            emb.push_back(v);
            dfs(1);
            emb.pop_back();
        }
    }
    void dfs(int depth) {
        const int n = s.get_size();
        const int k = s.get_in_exclusion_optimize_num();
        std::vector<int> vset = sets[s.get_loop_set_prefix_id(depth)];
        if (vset.empty()) return;
        if (s.is_vertex_induced) {
            // Drop candidates adjacent to an earlier vertex the pattern does
            // not connect to this position; in K_kn that is every candidate
            // other than that earlier vertex itself.
            std::vector<int> kept;
            for (int x : vset) {
                bool keep = true;
                for (int u = 0; u < depth && keep; ++u)
                    if (!s.get_adj_mat_ptr()[u * n + depth] && x != emb[u]) keep = false;
                if (keep) kept.push_back(x);
            }
            vset.swap(kept);
        }
        if (depth == n - k) {
            const auto &vid = s.in_exclusion_optimize_vertex_id;
            for (size_t i = 0; i < vid.size(); ++i) {
                const auto &set = sets[vid[i]];
                ans_buf[i] = s.in_exclusion_optimize_vertex_flag[i]
                                 ? static_cast<int>(set.size()) - s.in_exclusion_optimize_vertex_coef[i]
                                 : subtract_size(set, static_cast<int>(set.size()));
            }
            long long val = 0;
            int last_pos = -1;
            for (size_t pos = 0; pos < s.in_exclusion_optimize_coef.size(); ++pos) {
                // Out-of-range entries are the reference's uninitialised
                // reads; such plans are rebuilt with clean tables, so any
                // value works here.
                const int ap = s.in_exclusion_optimize_ans_pos[pos];
                const int a = ap >= 0 && ap < static_cast<int>(vid.size()) ? ans_buf[ap] : 0;
                if (static_cast<int>(pos) == last_pos + 1)
                    val = a;
                else if (val != 0)
                    val = val * a;
                if (s.in_exclusion_optimize_flag[pos]) {
                    last_pos = static_cast<int>(pos);
                    ans += val * s.in_exclusion_optimize_coef[pos];
                }
            }
            return;
        }
        if (depth == n - 1) {
            if (s.get_total_restrict_num() > 0) {
                int min_vertex = kn;
                for (int i = s.get_restrict_last(depth); i != -1; i = s.get_restrict_next(i))
                    min_vertex = std::min(min_vertex, emb[s.get_restrict_index(i)]);
                const int after = static_cast<int>(std::lower_bound(vset.begin(), vset.end(), min_vertex) - vset.begin());
                if (after > 0) ans += subtract_size(vset, after);
            } else {
                ans += subtract_size(vset, static_cast<int>(vset.size()));
            }
            return;
        }
        int min_vertex = kn;
        for (int i = s.get_restrict_last(depth); i != -1; i = s.get_restrict_next(i))
            min_vertex = std::min(min_vertex, emb[s.get_restrict_index(i)]);
        for (int v : vset) {
            if (min_vertex <= v) break;
            if (has(v)) continue;
            bool zero = false;
            for (int p = s.get_last(depth); p != -1; p = s.get_next(p)) {
                build(p, v);
                if (static_cast<int>(sets[p].size()) == s.get_break_size(p)) { zero = true; break; }
            }
            if (zero) continue;
            emb.push_back(v);
            dfs(depth + 1);
            emb.pop_back();
        }
    }
};

}  // namespace

bool Schedule_IEP::iep_tables_out_of_range() const {
    if (in_exclusion_optimize_num <= 0) return false;
    const int nsets = static_cast<int>(in_exclusion_optimize_vertex_id.size());
    for (size_t t = 0; t < in_exclusion_optimize_coef.size(); ++t)
        if (in_exclusion_optimize_ans_pos[t] < 0 || in_exclusion_optimize_ans_pos[t] >= nsets) return true;
    return false;
}

long long Schedule_IEP::count_on_complete_graph(int kn) const {
    if (is_vertex_induced) {
        // Every vertex of K_kn is adjacent to every other, so the
        // vertex-induced filter keeps, at a position with a non-adjacent
        // earlier position u, only the vertex already matched to u: the
        // count of a pattern that is not complete is 0.
        for (int i = 0; i < size; ++i)
            for (int j = i + 1; j < size; ++j)
                if (!adj_mat[i * size + j]) return 0;
    }
    CompleteDfs d(*this, kn);
    d.run();
    return d.ans / in_exclusion_optimize_redundancy;
}

std::vector<Schedule_IEP::Candidate> Schedule_IEP::enumerate_candidates(const Pattern &pattern, bool use_iep,
                                                                       int v_cnt, int64_t e_cnt,
                                                                       long long tri_cnt) {
    std::vector<Candidate> out;
    const int n = pattern.get_size();
    if (n < 2 || n > kMaxPatternSize || !pattern.check_connected()) return out;
    const int *src = pattern.get_adj_mat_ptr();
    // The candidates without their scores depend on the pattern alone and
    // are kept per pattern (bounded like the model constructor's state);
    // score_of[i] is the first candidate with candidate i's ordered
    // adjacency and restriction set, whose score it shares.
    struct EnumState {
        std::vector<Candidate> cands;
        std::vector<int> score_of;
    };
    static std::mutex mu;
    static std::map<std::pair<uint64_t, bool>, std::shared_ptr<const EnumState>> cache;
    const auto key = std::make_pair(adj_key(src, n), use_iep);
    std::shared_ptr<const EnumState> st;
    {
        std::lock_guard<std::mutex> lock(mu);
        auto it = cache.find(key);
        if (it != cache.end()) st = it->second;
    }
    if (!st) {
        Schedule_IEP s;
        s.alloc(n);
        std::copy(src, src + n * n, s.adj_mat.begin());
        auto candidates = all_permutations(n);
        candidates.erase(std::remove_if(candidates.begin(), candidates.end(),
                                        [&](const std::vector<int> &v) { return s.get_vec_optimize_num(v) < 0; }),
                         candidates.end());
        int max_val = 0;
        for (const auto &v : candidates) max_val = std::max(max_val, s.get_vec_optimize_num(v));
        candidates.erase(std::remove_if(candidates.begin(), candidates.end(),
                                        [&](const std::vector<int> &v) {
                                            return s.get_vec_optimize_num(v) != max_val;
                                        }),
                         candidates.end());
        // Orders are independent: evaluated in parallel on per-thread copies,
        // concatenated in order.
        std::vector<std::vector<Candidate>> per(candidates.size());
        std::vector<uint64_t> okey(candidates.size());
#pragma omp parallel
        {
            Schedule_IEP w;
            w.alloc(n);
#pragma omp for schedule(dynamic, 1)
            for (size_t c = 0; c < candidates.size(); ++c) {
                const auto &vec = candidates[c];
                w.copy_adj_mat_from(vec, src);
                okey[c] = adj_key(w.adj_mat.data(), n);
                w.setup_optimization_info(use_iep);
                std::vector<Pairs> rv;
                w.restricts_generate(rv);
                if (rv.empty()) rv.push_back(Pairs());
                for (const auto &pairs : rv) {
                    std::vector<std::pair<int, int>> applied;
                    for (const auto &p : filter_implied(pairs))
                        if (p.second < n - w.in_exclusion_optimize_num) applied.push_back(p);
                    const int div = restriction_multiplicity(w.adj_mat.data(), n, applied);
                    per[c].push_back({vec, pairs, 0.0, div, w.in_exclusion_optimize_num});
                }
            }
        }
        auto ns = std::make_shared<EnumState>();
        std::map<std::pair<uint64_t, size_t>, int> first;
        for (size_t c = 0; c < per.size(); ++c)
            for (size_t k = 0; k < per[c].size(); ++k) {
                const int i = static_cast<int>(ns->cands.size());
                ns->score_of.push_back(first.emplace(std::make_pair(okey[c], k), i).first->second);
                ns->cands.push_back(std::move(per[c][k]));
            }
        std::lock_guard<std::mutex> lock(mu);
        if (cache.size() >= 4096) cache.clear();
        st = cache.emplace(key, std::move(ns)).first->second;
    }
    out = st->cands;
    const int total = static_cast<int>(out.size());
#pragma omp parallel
    {
        Schedule_IEP w;
        w.alloc(n);
#pragma omp for schedule(dynamic, 8)
        for (int i = 0; i < total; ++i) {
            if (st->score_of[i] != i) continue;
            w.copy_adj_mat_from(out[i].order, src);
            w.in_exclusion_optimize_num = out[i].iep_k;
            out[i].model_cost = w.new_estimate_schedule_restrict(out[i].restricts, v_cnt, e_cnt, tri_cnt);
        }
    }
    for (int i = 0; i < total; ++i) out[i].model_cost = out[st->score_of[i]].model_cost;
    return out;
}

}  // namespace gi

namespace gi {

bool Schedule_IEP::choose_validated(const Pattern &pattern, bool use_iep, int v_cnt, int64_t e_cnt,
                                    long long tri_cnt, Candidate &best) {
    bool have = false;
    for (auto &c : enumerate_candidates(pattern, use_iep, v_cnt, e_cnt, tri_cnt)) {
        if (c.divisor <= 0) continue;
        if (!have || c.model_cost < best.model_cost) {
            best = c;
            have = true;
        }
    }
    return have;
}

}  // namespace gi
