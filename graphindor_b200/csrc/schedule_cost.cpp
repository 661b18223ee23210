// Learned schedule cost model: re-ranks the analytic model's best valid
// candidate schedules of a pattern (vertex order + restriction set,
// reference src/schedule_IEP.cpp:67-189 enumerates them; the analytic model
// is src/schedule_IEP.cpp:307-382) by the device time a small MLP predicts
// for them on a graph.  The MLP (3 layers, hidden 128,
// fp32) is trained offline on engine-measured times
// (graphindor_b200/schedule_cost/train.py); the feature layout here must
// match graphindor_b200/schedule_cost/features.py.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>
#include <vector>

#include "internal.hpp"

namespace gi {

namespace {

constexpr int kMaxN = 7;
constexpr int kPairs = kMaxN * (kMaxN - 1) / 2;  // 21 position pairs
constexpr int kDegBins = 16;
constexpr int kGraphDim = 3 + kDegBins;
constexpr int kPlanDim = 2 * kPairs + 6;
constexpr int kDim = kPlanDim + kGraphDim;

struct Mlp {
    int in = 0, hidden = 0;
    std::vector<float> mu, sd, W1, b1, W2, b2, w3;
    float b3 = 0.f;
};

std::mutex g_model_mu;
Mlp g_model;  // in == 0: none loaded

int pair_index(int i, int j) {  // i < j, row-major over the upper triangle
    int k = 0;
    for (int a = 0; a < kMaxN; ++a)
        for (int b = a + 1; b < kMaxN; ++b) {
            if (a == i && b == j) return k;
            ++k;
        }
    return -1;
}

void plan_features(int n, const int *adj, const std::vector<int> &order, const std::vector<std::pair<int, int>> &rs,
                   double model_cost, int iep_k, float *f) {
    std::memset(f, 0, sizeof(float) * kPlanDim);
    int edges = 0;
    for (int i = 0; i < n; ++i)
        for (int j = i + 1; j < n; ++j)
            if (adj[order[i] * n + order[j]]) {
                f[pair_index(i, j)] = 1.f;
                ++edges;
            }
    for (const auto &r : rs) {
        const int i = std::min(r.first, r.second), j = std::max(r.first, r.second);
        f[kPairs + pair_index(i, j)] = 1.f;
    }
    const double lc = std::log10(std::max(model_cost, 1.0));
    float *t = f + 2 * kPairs;
    t[0] = static_cast<float>(n / 7.0);
    t[1] = static_cast<float>(edges / 21.0);
    t[2] = static_cast<float>(rs.size() / 21.0);
    t[3] = static_cast<float>(iep_k / 5.0);
    t[4] = static_cast<float>(lc / 10.0);
    t[5] = static_cast<float>((lc / 10.0) * (lc / 10.0));
}

float forward(const Mlp &m, const float *x) {
    std::vector<float> z(m.in), h1(m.hidden), h2(m.hidden);
    for (int i = 0; i < m.in; ++i) z[i] = (x[i] - m.mu[i]) / m.sd[i];
    for (int o = 0; o < m.hidden; ++o) {
        float a = m.b1[o];
        const float *w = &m.W1[static_cast<size_t>(o) * m.in];
        for (int i = 0; i < m.in; ++i) a += w[i] * z[i];
        h1[o] = a > 0.f ? a : 0.f;
    }
    for (int o = 0; o < m.hidden; ++o) {
        float a = m.b2[o];
        const float *w = &m.W2[static_cast<size_t>(o) * m.hidden];
        for (int i = 0; i < m.hidden; ++i) a += w[i] * h1[i];
        h2[o] = a > 0.f ? a : 0.f;
    }
    float y = m.b3;
    for (int i = 0; i < m.hidden; ++i) y += m.w3[i] * h2[i];
    return y;
}

}  // namespace

// log10 of v_cnt, undirected edges and triangles, then the share of vertices
// per power-of-two degree bin [2^b, 2^(b+1)) (bin 0 also holds degree 0).
void cost_model_graph_features(const int64_t *vertex, int32_t v_cnt, int64_t tri_cnt, float *out) {
    double bins[kDegBins] = {};
    for (int32_t v = 0; v < v_cnt; ++v) {
        const int64_t d = vertex[v + 1] - vertex[v];
        int b = 0;
        while (b + 1 < kDegBins && (int64_t(1) << (b + 1)) <= d) ++b;
        bins[b] += 1.0;
    }
    const double e = static_cast<double>(vertex[v_cnt]) / 2.0;
    out[0] = static_cast<float>(std::log10(std::max<double>(v_cnt, 1)));
    out[1] = static_cast<float>(std::log10(std::max<double>(std::floor(e), 1)));
    out[2] = static_cast<float>(std::log10(std::max<double>(static_cast<double>(tri_cnt), 1)));
    for (int b = 0; b < kDegBins; ++b) out[3 + b] = static_cast<float>(bins[b] / std::max<double>(v_cnt, 1));
}

}  // namespace gi

using namespace gi;

extern "C" {

int gi_cost_model_load(const char *path) {
    if (!path) return fail(GI_EINVAL, "NULL path");
    FILE *f = std::fopen(path, "rb");
    if (!f) return fail(GI_EIO, std::string("cannot open ") + path);
    Mlp m;
    char magic[8];
    int32_t dims[2];
    bool ok = std::fread(magic, 1, 8, f) == 8 && std::memcmp(magic, "GIMLP1\0\0", 8) == 0 &&
              std::fread(dims, 4, 2, f) == 2 && dims[0] == kDim && dims[1] > 0 && dims[1] <= 4096;
    if (ok) {
        m.in = dims[0];
        m.hidden = dims[1];
        auto rd = [&](std::vector<float> &v, size_t n) {
            v.resize(n);
            return std::fread(v.data(), 4, n, f) == n;
        };
        std::vector<float> b3(1);
        ok = rd(m.mu, m.in) && rd(m.sd, m.in) && rd(m.W1, static_cast<size_t>(m.hidden) * m.in) &&
             rd(m.b1, m.hidden) && rd(m.W2, static_cast<size_t>(m.hidden) * m.hidden) && rd(m.b2, m.hidden) &&
             rd(m.w3, m.hidden) && rd(b3, 1);
        m.b3 = b3[0];
    }
    std::fclose(f);
    if (!ok) return fail(GI_EIO, "not a schedule cost model file of this build");
    std::lock_guard<std::mutex> lock(g_model_mu);
    g_model = std::move(m);
    return GI_OK;
}

int gi_graph_features_host(const int64_t *vertex, int32_t v_cnt, int64_t tri_cnt, float *out, int cap) {
    if (!vertex || !out || v_cnt < 1) return fail(GI_EINVAL, "bad arguments");
    if (cap < kGraphDim) return fail(GI_EINVAL, "feature buffer too small");
    cost_model_graph_features(vertex, v_cnt, tri_cnt, out);
    return GI_OK;
}

int gi_graph_features(const gi_graph *g, float *out, int cap) {
    if (!g || !out) return fail(GI_EINVAL, "NULL argument");
    if (cap < kGraphDim) return fail(GI_EINVAL, "feature buffer too small");
    std::memcpy(out, g->graph_features, sizeof(float) * kGraphDim);
    return GI_OK;
}

int gi_plan_create_learned(int n, const char *adj, int32_t v_cnt, int64_t e_cnt, int64_t tri_cnt,
                           const float *graph_features, int enable_iep, gi_plan **out, double *predicted_ms) {
    if (!out || !adj || !graph_features) return fail(GI_EINVAL, "NULL argument");
    *out = nullptr;
    if (n < 3 || n > GI_MAX_PATTERN) return fail(GI_EINVAL, "pattern size must be between 3 and 7");
    for (int i = 0; i < n * n; ++i)
        if (adj[i] == '\0') return fail(GI_EINVAL, "adjacency string shorter than n*n");
    Mlp m;
    {
        std::lock_guard<std::mutex> lock(g_model_mu);
        if (g_model.in == 0) return fail(GI_EINVAL, "no schedule cost model loaded (gi_cost_model_load)");
        m = g_model;
    }
    try {
        Pattern pat(n, adj);
        if (!pat.check_connected()) return fail(GI_EDISCONNECTED, "pattern is not connected");
        const auto cands = Schedule_IEP::enumerate_candidates(pat, enable_iep != 0, v_cnt, e_cnt, tri_cnt);
        // The valid candidates of lowest analytic cost, back in enumeration
        // order; the first of equal predictions wins.
        std::vector<int> top;
        for (size_t i = 0; i < cands.size(); ++i)
            if (cands[i].divisor > 0) top.push_back(static_cast<int>(i));
        std::stable_sort(top.begin(), top.end(),
                         [&](int a, int b) { return cands[a].model_cost < cands[b].model_cost; });
        if (top.size() > static_cast<size_t>(GI_LEARNED_CANDIDATES)) top.resize(GI_LEARNED_CANDIDATES);
        std::sort(top.begin(), top.end());
        std::vector<float> x(kDim);
        std::memcpy(x.data() + kPlanDim, graph_features, sizeof(float) * kGraphDim);
        int best = -1;
        float best_y = 0.f;
        for (int i : top) {
            const auto &c = cands[static_cast<size_t>(i)];
            plan_features(n, pat.get_adj_mat_ptr(), c.order, c.restricts, c.model_cost, c.iep_k, x.data());
            const float y = forward(m, x.data());
            if (best < 0 || y < best_y) {
                best = i;
                best_y = y;
            }
        }
        if (best < 0) return fail(GI_EINVAL, "pattern has no valid candidate schedule");
        const auto &c = cands[best];
        std::vector<int32_t> rs;
        for (const auto &r : c.restricts) {
            rs.push_back(r.first);
            rs.push_back(r.second);
        }
        if (predicted_ms) *predicted_ms = std::pow(10.0, static_cast<double>(best_y));
        return gi_plan_create_explicit(n, adj, c.order.data(), rs.empty() ? nullptr : rs.data(),
                                       static_cast<int>(c.restricts.size()), enable_iep, out);
    } catch (const std::exception &e) {
        return fail(GI_EINVAL, e.what());
    }
}

}  // extern "C"
