// Autotuner of the counting kernel's variants.
//
// The reference has one kernel configuration, fixed at compile time
// (gpu/function/pattern_matching.cuh:7-9: 4 warps per block, a
// binary-search intersection; gpu/gpu_graph.cu:33: 1024 blocks).  Here a
// plan carries a kernel variant that changes speed, never counts:
//   * the leaf level: probes spread evenly over the lanes (leaf_flat), or one
//     candidate per lane with candidates costlier than lane_budget handed to
//     the whole warp;
//   * the occupancy the kernel is compiled for: 1 (registers unconstrained,
//     4 blocks of 128 threads per SM) or 16 blocks per SM (32 registers,
//     some spilling, four times the resident warps).
// gi_autotune times every variant on a sample of the graph's first-level
// edges (an edge subset, each task counted whole, so every variant counts
// the same work and must return the same raw sum) and keeps the fastest in
// the plan.  Choices are cached per class of (plan, graph): pattern size, IEP
// depth, depth-2 split, first-level restriction, and the graph's edge count
// and largest degree in powers of two.  Batches (batch.cu) apply the cached
// choice of each job's class to their copy of its plan.
#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

#include "internal.hpp"

namespace gi {
namespace {

using TuneKey = std::tuple<int, int, int, int, int, int>;

std::mutex g_tune_mu;
std::map<TuneKey, gi_variant> g_tune_cache;

int log2_bucket(int64_t x) {
    int b = 0;
    while (x > 1) {
        x >>= 1;
        ++b;
    }
    return b;
}

TuneKey key_of(const gi_graph *g, const DevPlan &P) {
    return TuneKey{P.n, P.iep_k, P.loop2_kind >= 0 ? 1 : 0, P.first_restricted, log2_bucket(g->e_cnt) / 2,
                   log2_bucket(g->max_degree) / 2};
}

}  // namespace

void variant_apply(DevPlan &P, const gi_variant &v) {
    P.leaf_flat = v.leaf_flat ? 1 : 0;
    P.flat_first = P.leaf_flat && P.flat_first_ok;
    if (v.lane_budget > 0) P.lane_budget = v.lane_budget;
    P.occupancy = v.occupancy;
    P.split = v.split;
    P.leaf_handoff = v.leaf_handoff;
    P.mid_handoff = v.mid_handoff;
    P.tri_edge = v.edge_triangles && P.tri_ok ? 1 : 0;
}

gi_variant variant_of(const DevPlan &P) {
    gi_variant v{};
    v.leaf_flat = P.leaf_flat;
    v.lane_budget = P.lane_budget;
    v.occupancy = P.occupancy;
    v.split = P.split;
    v.leaf_handoff = P.leaf_handoff;
    v.mid_handoff = P.mid_handoff;
    v.edge_triangles = P.tri_edge;
    return v;
}

// The plan with the tuned variant of its class on graph g, when one is cached.
bool tuned_plan(const gi_graph *g, const DevPlan &P, DevPlan &out) {
    std::lock_guard<std::mutex> lock(g_tune_mu);
    const auto it = g_tune_cache.find(key_of(g, P));
    if (it == g_tune_cache.end()) return false;
    out = P;
    variant_apply(out, it->second);
    return true;
}

}  // namespace gi

using namespace gi;

extern "C" {

int gi_plan_get_variant(const gi_plan *p, gi_variant *out) {
    if (!p || !out) return fail(GI_EINVAL, "NULL argument");
    *out = variant_of(p->dev);
    return GI_OK;
}

int gi_plan_set_variant(gi_plan *p, const gi_variant *v) {
    if (!p || !v) return fail(GI_EINVAL, "NULL argument");
    if (v->occupancy != 0 && v->occupancy != 1 && v->occupancy != 16)
        return fail(GI_EINVAL, "occupancy must be 0, 1 or 16");
    if (v->lane_budget < 0) return fail(GI_EINVAL, "lane_budget must be >= 0");
    if (v->split < 0 || v->split > (1 << 20) || v->leaf_handoff < 0 || v->mid_handoff < 0)
        return fail(GI_EINVAL, "split, leaf_handoff and mid_handoff must be >= 0 (split at most 2^20)");
    variant_apply(p->dev, *v);
    return GI_OK;
}

int gi_autotune(const gi_graph *g, gi_plan *p, gi_stream stream, const gi_tune_options *opt, gi_tune_info *info) {
    if (!g || !p) return fail(GI_EINVAL, "NULL argument");
    gi_tune_options o{};
    o.sample_edges = 16384;
    o.max_ms = 250.0;
    o.reps = 2;
    o.use_cache = 1;
    if (opt) {
        if (opt->sample_edges > 0) o.sample_edges = opt->sample_edges;
        if (opt->max_ms > 0) o.max_ms = opt->max_ms;
        if (opt->reps > 0) o.reps = opt->reps;
        o.use_cache = opt->use_cache;
        o.quick = opt->quick;
        o.lookup_only = opt->lookup_only;
        if (o.quick) o.reps = 1;
    }
    gi_tune_info res{};
    const TuneKey key = key_of(g, p->dev);
    if (o.use_cache) {
        std::lock_guard<std::mutex> lock(g_tune_mu);
        const auto it = g_tune_cache.find(key);
        if (it != g_tune_cache.end()) {
            variant_apply(p->dev, it->second);
            res.chosen = it->second;
            res.cached = 1;
            if (info) *info = res;
            return GI_OK;
        }
    }
    if (o.lookup_only) {  // nothing cached: the plan keeps its variant
        res.chosen = variant_of(p->dev);
        if (info) *info = res;
        return GI_OK;
    }
    const DevPlan original = p->dev;
    // Calibrate the sample with the plan's own variant: fewer edges while it
    // runs past max_ms, more while it takes under a fiftieth of it.
    int64_t step = std::max<int64_t>(1, g->e_cnt / std::max<int64_t>(1, o.sample_edges));
    for (int round = 0; round < (o.quick ? 4 : 12); ++round) {
        gi_stats s{};
        s.edge_step = step;
        s.budget_ms = o.max_ms;
        uint64_t raw = 0;
        const int rc = gi_count_shard(g, p, 0, 1, stream, &raw, &s);
        if (rc == GI_ETIMEOUT) {
            if (step >= g->e_cnt) break;  // a single edge is already too slow
            step = std::min<int64_t>(std::max<int64_t>(g->e_cnt, 1), step * 8);
            continue;
        }
        if (rc != GI_OK) return rc;
        if (s.kernel_ms + s.prep_ms < o.max_ms / 50 && step > 1) {
            step = std::max<int64_t>(1, step / 4);
            continue;
        }
        break;
    }
    // Times variant v on the sample (the fastest of o.reps runs; INFINITY
    // when it runs past max_ms) and checks its raw sum against the others.
    bool have_sum = false;
    uint64_t sum = 0;
    auto time_variant = [&](const gi_variant &v, double &t) -> int {
        p->dev = original;
        variant_apply(p->dev, v);
        t = INFINITY;
        for (int r = 0; r < o.reps; ++r) {
            gi_stats s{};
            s.edge_step = step;
            s.edge_offset = 0;
            s.budget_ms = o.max_ms;
            uint64_t raw = 0;
            const int rc = gi_count_shard(g, p, 0, 1, stream, &raw, &s);
            if (rc == GI_ETIMEOUT) break;  // slower than max_ms: not a candidate
            if (rc != GI_OK) return rc;
            if (have_sum && raw != sum) return fail(GI_ECUDA, "kernel variants counted the same sample differently");
            sum = raw;
            have_sum = true;
            t = std::min(t, s.kernel_ms + s.prep_ms);
        }
        ++res.candidates;
        return GI_OK;
    };
    double best = INFINITY;
    gi_variant chosen = variant_of(original);
    int st = GI_OK;
    // Stage 1: the leaf level and the occupancy.
    const int budgets[2] = {256, 2048};
    const int default_occ = original.occupancy ? original.occupancy : (original.n >= 6 ? 16 : 1);
    std::vector<gi_variant> cands;
    if (o.quick) {
        cands.push_back(gi_variant{0, original.lane_budget, default_occ, 0, 0, 0, 0});
        cands.push_back(gi_variant{1, original.lane_budget, default_occ, 0, 0, 0, 0});
        cands.push_back(gi_variant{1, original.lane_budget, default_occ == 1 ? 16 : 1, 0, 0, 0, 0});
    } else {
        for (int occ : {1, 16}) {
            cands.push_back(gi_variant{1, original.lane_budget, occ, 0, 0, 0, 0});
            for (int b : budgets) cands.push_back(gi_variant{0, b, occ, 0, 0, 0, 0});
        }
    }
    if (original.tri_ok) cands.push_back(gi_variant{0, original.lane_budget, 0, 0, 0, 0, 1});
    for (const gi_variant &v : cands) {
        double t;
        if ((st = time_variant(v, t)) != GI_OK) break;
        if (v.leaf_flat == original.leaf_flat && v.lane_budget == original.lane_budget && v.occupancy == default_occ)
            res.default_ms = t;
        if (t < best) {
            best = t;
            chosen = v;
        }
    }
    // Stage 2: the work split of the depth-2 loop (a quarter and four times
    // the default), then stage 3: the leaf donation threshold.
    if (st == GI_OK && original.loop2_kind >= 0) {
        const int d = original.leaf_depth == 2 ? 256 : 32;
        for (int sp : {d / 4, d * 4}) {
            gi_variant v = chosen;
            v.split = sp;
            double t;
            if ((st = time_variant(v, t)) != GI_OK) break;
            if (t < best) {
                best = t;
                chosen = v;
            }
        }
    }
    if (st == GI_OK && original.leaf_depth >= 2 && !o.quick) {
        for (int lh : {16, 256}) {
            gi_variant v = chosen;
            v.leaf_handoff = lh;
            double t;
            if ((st = time_variant(v, t)) != GI_OK) break;
            if (t < best) {
                best = t;
                chosen = v;
            }
        }
    }
    p->dev = original;
    if (st != GI_OK) return st;
    variant_apply(p->dev, chosen);
    res.chosen = chosen;
    res.best_ms = std::isfinite(best) ? best : -1.0;
    res.sample_edges = (g->e_cnt + step - 1) / step;
    {
        std::lock_guard<std::mutex> lock(g_tune_mu);
        g_tune_cache[key] = chosen;
    }
    if (info) *info = res;
    return GI_OK;
}

int gi_autotune_clear(void) {
    std::lock_guard<std::mutex> lock(g_tune_mu);
    g_tune_cache.clear();
    return GI_OK;
}

}  // extern "C"
