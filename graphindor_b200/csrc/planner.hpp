// Host-side planner: Pattern and Schedule_IEP.
//
// These mirror the reference's host classes (reference include/pattern.h,
// include/schedule_IEP.h) closely enough that a caller of the reference finds
// the same names, arguments and errors.  The planning algorithm is restated
// step for step because the engine's results must be bit-identical to the
// reference's: the vertex order, the restriction set, the prefix DAG, the
// inclusion-exclusion (IEP) tables and the redundancy divisor all feed the
// count, and the reference reads some IEP tables from state left over by
// earlier candidate orders (see Schedule_IEP::setup_optimization_info).
#pragma once

#include <cstdint>
#include <memory>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

namespace gi {

constexpr int kMaxPatternSize = 7;  // reference gpu/function/pattern_matching.cuh:7

// Number of automorphic images of any subgraph that satisfy restriction set
// R on the pattern adj (n*n), or 0 if that number depends on the subgraph.
int restriction_multiplicity(const int *adj, int n, const std::vector<std::pair<int, int>> &R);

// Undirected pattern graph on n vertices stored as an n*n 0/1 matrix.
// Follows reference src/pattern.cpp.
class Pattern {
public:
    explicit Pattern(int n, bool clique = false);
    // n*n characters; any '1' at (i,j) adds the undirected edge {i,j}
    // (reference src/pattern.cpp:22-31).
    Pattern(int n, const char *adj_string);
    void add_edge(int x, int y);
    void del_edge(int x, int y);
    void add_ordered_edge(int x, int y) { adj_[x * n_ + y] = 1; }
    int get_size() const { return n_; }
    const int *get_adj_mat_ptr() const { return adj_.data(); }
    bool check_connected() const;  // reference src/pattern.cpp:227-252
    bool is_dag() const;           // reference src/pattern.cpp:296-325
    int edge_count() const;

private:
    int n_;
    std::vector<int> adj_;
};

// One node of the prefix DAG: the sorted list of earlier pattern vertices
// whose neighbourhoods are intersected (reference include/prefix.h).
struct Prefix {
    std::vector<int> data;
    bool has_child = false;
    bool only_need_size = false;
};

// The plan for one pattern.  Field names follow the reference
// (include/schedule_IEP.h:30-110).
class Schedule_IEP {
public:
    // reference src/schedule_IEP.cpp:12-247.  performance_modeling_type 0 = keep
    // the given order, 1 = the reference's analytic model; restricts_type 0 = no
    // symmetry breaking, 1 = the reference's restriction generator.  Throws
    // std::invalid_argument for sizes outside [3, 7] and std::runtime_error
    // ("pattern is not connected") like the reference.
    Schedule_IEP(const Pattern &pattern, bool &is_pattern_valid, int performance_modeling_type,
                 int restricts_type, bool use_in_exclusion_optimize, int v_cnt, int64_t e_cnt,
                 long long tri_cnt = 0, bool vertex_induced = false);
    // Same, with an explicit vertex order (order[i] = pattern vertex placed at
    // position i) and restriction set, for timing candidate schedules.
    // Restrictions are (first, second) pairs over positions: the vertex at
    // position `second` must have a smaller id than the one at `first`.
    Schedule_IEP(const Pattern &pattern, const std::vector<int> &order,
                 const std::vector<std::pair<int, int>> &restricts, bool use_in_exclusion_optimize,
                 bool exact = true);
    // Vertex-induced plan with the pattern's own order and no restrictions
    // (reference src/schedule_IEP.cpp:249-290).
    Schedule_IEP(const int *adj_mat, int size);

    int get_size() const { return size; }
    int get_total_prefix_num() const { return total_prefix_num; }
    int get_basic_prefix_num() const { return basic_prefix_num; }
    int get_father_prefix_id(int p) const { return father_prefix_id[p]; }
    int get_loop_set_prefix_id(int d) const { return loop_set_prefix_id[d]; }
    int get_last(int d) const { return last[d]; }
    int get_next(int p) const { return next[p]; }
    int get_break_size(int p) const { return break_size[p]; }
    bool get_prefix_only_need_size(int p) const { return prefix[p].only_need_size; }
    const std::vector<int> &get_prefix_data(int p) const { return prefix[p].data; }
    int get_in_exclusion_optimize_num() const { return in_exclusion_optimize_num; }
    int get_total_restrict_num() const { return total_restrict_num; }
    int get_restrict_last(int d) const { return restrict_last[d]; }
    int get_restrict_next(int i) const { return restrict_next[i]; }
    int get_restrict_index(int i) const { return restrict_index[i]; }
    long long get_in_exclusion_optimize_redundancy() const { return in_exclusion_optimize_redundancy; }
    const int *get_adj_mat_ptr() const { return adj_mat.data(); }
    int get_k_val() const { return k_val; }
    // Position -> original pattern vertex of the chosen order.
    const std::vector<int> &get_order() const { return order_; }
    int get_multiplicity() const;  // number of automorphisms
    double get_model_cost() const { return model_cost_; }
    // The restriction set the model picked, before add_restrict drops pairs
    // implied by others.
    const std::vector<std::pair<int, int>> &get_chosen_restricts() const { return chosen_pairs_; }
    // True when the never-cleared IEP vectors, read from index 0 as the
    // reference reads them, point past the final IEP set list.  The
    // reference's count is then undefined (it reads uninitialised memory).
    bool iep_tables_out_of_range() const;

    void add_restrict(const std::vector<std::pair<int, int>> &restricts);
    // reference src/schedule_IEP.cpp:732-783
    void aggressive_optimize_get_all_pairs(std::vector<std::vector<std::pair<int, int>>> &out) const;
    // reference src/schedule_IEP.cpp:307-382: the analytic cost of the current
    // order under a restriction set.
    double new_estimate_schedule_restrict(const std::vector<std::pair<int, int>> &pairs, int v_cnt,
                                          int64_t e_cnt, long long tri_cnt) const;
    // All (order, restriction set) candidates the reference model scores, in
    // the reference's enumeration order.  Used by the learned cost model.
    struct Candidate {
        std::vector<int> order;
        std::vector<std::pair<int, int>> restricts;
        double model_cost;
        int divisor;  // exact count divisor, 0 when the restriction set is not valid
        int iep_k = 0;  // in_exclusion_optimize_num of the order
    };
    // The lowest-cost candidate whose restriction set is valid (ties: first
    // in enumeration order).  Returns false if there is none.
    static bool choose_validated(const Pattern &pattern, bool use_iep, int v_cnt, int64_t e_cnt, long long tri_cnt,
                                 Candidate &out);
    // What the count of this plan is divided by: the reference's redundancy
    // for plans made the reference's way, the exact multiplicity for
    // explicit plans.
    long long get_count_divisor() const { return count_divisor_ > 0 ? count_divisor_ : in_exclusion_optimize_redundancy; }
    static std::vector<Candidate> enumerate_candidates(const Pattern &pattern, bool use_iep, int v_cnt,
                                                       int64_t e_cnt, long long tri_cnt);

    // Public state, as in the reference.
    std::vector<std::pair<int, int>> restrict_pair;
    // These three vectors are appended to by every setup_optimization_info()
    // call and never cleared, exactly as in the reference; readers index them
    // from 0, so entries from the first candidate order win.
    std::vector<int> in_exclusion_optimize_vertex_id;
    std::vector<int> in_exclusion_optimize_vertex_flag;
    std::vector<int> in_exclusion_optimize_vertex_coef;
    std::vector<int> in_exclusion_optimize_coef;
    std::vector<int> in_exclusion_optimize_flag;
    std::vector<int> in_exclusion_optimize_ans_pos;
    std::vector<int> break_size;
    bool is_vertex_induced = false;

    // Count of the current plan on the complete graph K_kn, with the
    // reference CPU path's semantics (reference src/graph.cpp:305-355,429-566).
    // Planning uses it on K_n and K_{n+1} only.
    long long count_on_complete_graph(int kn) const;

    // Internal helpers (public for the restriction generator's scratch plans).
    void setup_optimization_info(bool use_in_exclusion_optimize);
    void set_in_exclusion_optimize_num(int k) { in_exclusion_optimize_num = k; }

private:
    Schedule_IEP() = default;
    // Not copyable from outside, as in the reference (schedule_IEP.h:27-28);
    // the model constructor copies the state it caches per pattern.
    Schedule_IEP(const Schedule_IEP &) = default;
    Schedule_IEP &operator=(const Schedule_IEP &) = default;
    void alloc(int n);
    bool check_connectivity() const;
    int get_max_degree() const;
    void copy_adj_mat_from(const std::vector<int> &vec, const int *src);
    void build_loop_invariant(int iep_num);
    int find_father_prefix(int data_size, const int *data);
    void init_in_exclusion_optimize();
    void get_in_exclusion_optimize_group(int depth, int *id, int id_cnt, const int *iep_val);
    int get_vec_optimize_num(const std::vector<int> &vec) const;
    void restricts_generate(std::vector<std::vector<std::pair<int, int>>> &out) const;
    void set_in_exclusion_optimize_redundancy();
    std::vector<std::vector<int>> get_isomorphism_vec() const;

public:
    struct ModelKey;
    struct ModelState;

private:
    static std::shared_ptr<const ModelState> model_cache_find(const ModelKey &k);
    static std::shared_ptr<const ModelState> model_cache_insert(const ModelKey &k, std::shared_ptr<ModelState> s);

    int size = 0;
    std::vector<int> adj_mat;
    std::vector<int> father_prefix_id, last, next, loop_set_prefix_id;
    std::vector<Prefix> prefix;
    std::vector<int> restrict_last, restrict_next, restrict_index;
    int total_prefix_num = 0, basic_prefix_num = 0, total_restrict_num = 0;
    int in_exclusion_optimize_num = 0;
    int k_val = 0;
    long long in_exclusion_optimize_redundancy = 1;
    std::vector<std::vector<std::vector<int>>> in_exclusion_optimize_group;
    std::vector<int> in_exclusion_optimize_val;
    std::vector<int> order_;
    double model_cost_ = 0.0;
    std::vector<std::pair<int, int>> chosen_pairs_;
    long long count_divisor_ = 0;  // 0: use the redundancy
};

}  // namespace gi
