// Seeded synthetic graph generators (include/gi_gen.h).
#include <parallel/algorithm>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <new>
#include <vector>

#include "../../include/gi_gen.h"
#include "internal.hpp"

namespace {

inline uint64_t splitmix64(uint64_t x) {
    x += 0x9e3779b97f4a7c15ull;
    x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ull;
    x = (x ^ (x >> 27)) * 0x94d049bb133111ebull;
    return x ^ (x >> 31);
}

// Counter-based stream: value j of sample i under seed.
inline uint64_t rnd(uint64_t seed, uint64_t i, uint64_t j) {
    return splitmix64(splitmix64(seed ^ 0x5851f42d4c957f2dull) ^ splitmix64(i * 0x9e3779b97f4a7c15ull + j));
}

inline double unit(uint64_t x) { return static_cast<double>(x >> 11) * (1.0 / 9007199254740992.0); }

// Seeded permutation of 0..n-1 (Fisher-Yates; sequential, deterministic).
std::vector<int32_t> permutation(int32_t n, uint64_t seed) {
    std::vector<int32_t> p(n);
    for (int32_t i = 0; i < n; ++i) p[i] = i;
    for (int32_t i = n - 1; i > 0; --i) {
        const int32_t j = static_cast<int32_t>(rnd(seed, 0x7065726dull, static_cast<uint64_t>(i)) % (static_cast<uint64_t>(i) + 1));
        std::swap(p[i], p[j]);
    }
    return p;
}

// Symmetrise, drop self-loops, sort, deduplicate, build the CSR.
int finish(std::vector<uint64_t> &keys, int32_t n, gi_host_csr **out) {
    __gnu_parallel::sort(keys.begin(), keys.end());
    keys.erase(std::unique(keys.begin(), keys.end()), keys.end());
    auto *g = new (std::nothrow) gi_host_csr;
    if (!g) return gi::fail(GI_ENOMEM, "out of host memory");
    std::memset(g, 0, sizeof(*g));
    g->v_cnt = n;
    g->e_cnt = static_cast<int64_t>(keys.size());
    g->vertex = new (std::nothrow) int64_t[static_cast<size_t>(n) + 1];
    g->edge = new (std::nothrow) int32_t[keys.empty() ? 1 : keys.size()];
    if (!g->vertex || !g->edge) {
        gi_host_csr_free(g);
        return gi::fail(GI_ENOMEM, "out of host memory");
    }
    std::vector<int64_t> deg(static_cast<size_t>(n) + 1, 0);
    for (uint64_t k : keys) ++deg[static_cast<size_t>(k >> 32)];
    g->vertex[0] = 0;
    for (int32_t v = 0; v < n; ++v) g->vertex[v + 1] = g->vertex[v] + deg[v];
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < g->e_cnt; ++i) g->edge[i] = static_cast<int32_t>(keys[i] & 0xffffffffull);
    int64_t a = 0, b = 0;
    for (int32_t v = 0; v < n; ++v) {
        if (deg[v] > a) {
            b = a;
            a = deg[v];
        } else if (deg[v] > b) {
            b = deg[v];
        }
    }
    g->max_degree = static_cast<int32_t>(a);
    g->max_intersection_size = static_cast<int32_t>(b);
    *out = g;
    return GI_OK;
}

// Turns sampled pairs (already relabelled) into both directed keys.
void push_pair(std::vector<uint64_t> &keys, size_t slot, uint32_t u, uint32_t v) {
    keys[2 * slot] = (static_cast<uint64_t>(u) << 32) | v;
    keys[2 * slot + 1] = (static_cast<uint64_t>(v) << 32) | u;
}

void drop_self_loops(std::vector<uint64_t> &keys) {
    keys.erase(std::remove_if(keys.begin(), keys.end(), [](uint64_t k) { return (k >> 32) == (k & 0xffffffffull); }),
               keys.end());
}

}  // namespace

extern "C" {

int gi_gen_rmat(int scale, double edge_factor, double a, double b, double c, uint64_t seed, gi_host_csr **out) {
    if (!out || scale < 1 || scale > 30 || edge_factor <= 0 || a < 0 || b < 0 || c < 0 || a + b + c > 1)
        return gi::fail(GI_EINVAL, "bad R-MAT parameters");
    const int32_t n = int32_t(1) << scale;
    const int64_t m = static_cast<int64_t>(std::llround(edge_factor * n));
    std::vector<uint64_t> keys;
    try {
        keys.resize(static_cast<size_t>(2 * m));
    } catch (const std::bad_alloc &) {
        return gi::fail(GI_ENOMEM, "out of host memory");
    }
    const auto perm = permutation(n, seed);
    const double ab = a + b, abc = a + b + c;
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < m; ++i) {
        uint32_t u = 0, v = 0;
        for (int lvl = 0; lvl < scale; ++lvl) {
            const double r = unit(rnd(seed, static_cast<uint64_t>(i), static_cast<uint64_t>(lvl)));
            const uint32_t bit = 1u << (scale - 1 - lvl);
            if (r < a) {
            } else if (r < ab) {
                v |= bit;
            } else if (r < abc) {
                u |= bit;
            } else {
                u |= bit;
                v |= bit;
            }
        }
        push_pair(keys, static_cast<size_t>(i), static_cast<uint32_t>(perm[u]), static_cast<uint32_t>(perm[v]));
    }
    drop_self_loops(keys);
    return finish(keys, n, out);
}

int gi_gen_chung_lu(int32_t n, int64_t m, double gamma, double max_degree, uint64_t seed, gi_host_csr **out) {
    if (!out || n < 2 || m < 1 || gamma <= 1.0 || max_degree <= 0) return gi::fail(GI_EINVAL, "bad Chung-Lu parameters");
    const double alpha = 1.0 / (gamma - 1.0);
    // Pick i0 by bisection so that 2m * w_0 / W equals max_degree.
    auto top_degree = [&](double i0) {
        double W = 0;
        for (int32_t i = 0; i < n; ++i) W += std::pow(i + i0, -alpha);
        return 2.0 * static_cast<double>(m) * std::pow(i0, -alpha) / W;
    };
    double lo = 1e-3, hi = static_cast<double>(n);
    for (int it = 0; it < 80; ++it) {
        const double mid = std::sqrt(lo * hi);
        if (top_degree(mid) > max_degree) lo = mid;
        else hi = mid;
    }
    const double i0 = std::sqrt(lo * hi);
    std::vector<double> cdf(n);
    double acc = 0;
    for (int32_t i = 0; i < n; ++i) {
        acc += std::pow(i + i0, -alpha);
        cdf[i] = acc;
    }
    for (auto &x : cdf) x /= acc;
    std::vector<uint64_t> keys;
    try {
        keys.resize(static_cast<size_t>(2 * m));
    } catch (const std::bad_alloc &) {
        return gi::fail(GI_ENOMEM, "out of host memory");
    }
    const auto perm = permutation(n, seed);
    auto draw = [&](uint64_t r) {
        const double x = unit(r);
        int32_t i = static_cast<int32_t>(std::upper_bound(cdf.begin(), cdf.end(), x) - cdf.begin());
        return std::min(i, n - 1);
    };
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < m; ++i) {
        const int32_t u = draw(rnd(seed, static_cast<uint64_t>(i), 0));
        const int32_t v = draw(rnd(seed, static_cast<uint64_t>(i), 1));
        push_pair(keys, static_cast<size_t>(i), static_cast<uint32_t>(perm[u]), static_cast<uint32_t>(perm[v]));
    }
    drop_self_loops(keys);
    return finish(keys, n, out);
}

int gi_gen_er(int32_t n, int64_t m, uint64_t seed, gi_host_csr **out) {
    if (!out || n < 2 || m < 1) return gi::fail(GI_EINVAL, "bad G(n, m) parameters");
    std::vector<uint64_t> keys;
    try {
        keys.resize(static_cast<size_t>(2 * m));
    } catch (const std::bad_alloc &) {
        return gi::fail(GI_ENOMEM, "out of host memory");
    }
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < m; ++i) {
        const uint32_t u = static_cast<uint32_t>(rnd(seed, static_cast<uint64_t>(i), 0) % static_cast<uint64_t>(n));
        const uint32_t v = static_cast<uint32_t>(rnd(seed, static_cast<uint64_t>(i), 1) % static_cast<uint64_t>(n));
        push_pair(keys, static_cast<size_t>(i), u, v);
    }
    drop_self_loops(keys);
    return finish(keys, n, out);
}

int gi_csr_restrict(const gi_host_csr *in, int32_t keep, gi_host_csr **out) {
    if (!in || !out || keep < 2 || keep > in->v_cnt) return gi::fail(GI_EINVAL, "bad restriction size");
    std::vector<uint64_t> keys;
    for (int32_t v = 0; v < keep; ++v)
        for (int64_t e = in->vertex[v]; e < in->vertex[v + 1]; ++e)
            if (in->edge[e] < keep) keys.push_back((static_cast<uint64_t>(v) << 32) | static_cast<uint32_t>(in->edge[e]));
    return finish(keys, keep, out);
}

void gi_host_csr_free(gi_host_csr *g) {
    if (!g) return;
    delete[] g->vertex;
    delete[] g->edge;
    delete g;
}

}  // extern "C"
