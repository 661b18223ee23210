// Clique-tree pivoting (Jain and Seshadhri, "The Power of Pivoting for Exact
// Clique Counting", WSDM 2020) over the k-clique bitmaps of the
// degree-oriented DAG: the counts of every clique size up to kmax at once.
//
// The root of a search is a vertex v with its out-neighbours N+(v) as
// candidates (every clique is found once, from its lowest vertex in the DAG
// order).  The root's bitmap (kclique.cu) holds the induced DAG on N+(v):
// row i has bit j when N+(v)[j] is an out-neighbour of N+(v)[i].  The search
// needs the undirected induced graph, so it first ORs each row with the
// matching column (A = D | D^T).  A node of the search has candidate set S,
// h required and q optional vertices.  It picks the pivot u of S with the
// most neighbours in S and has one child S ∩ N(u) in which u is optional,
// and one child per other w ∈ S \ N(u), on S ∩ N(w) minus the earlier such
// w, in which w is required.  A leaf (S empty) holds C(q, k - h) k-cliques.
// A node at most three vertices short of kmax is closed without descent:
// its k-clique count is sum_j C(q, j) cl(k - h - j), with cl(0) = 1, cl(1) =
// |S|, cl(2) = the edges and cl(3) = the triangles of G[S].
//
// The same code serves a warp (one root per warp, lanes over rows, words
// and candidates, all control flow warp-uniform) and, through a one-lane
// policy, a host build that the tests check against the host oracle.  The
// recursion is an explicit stack in the worker's scratch; every step either
// pops a node or pushes a child whose candidate set is strictly smaller, so
// the search ends.
#pragma once

#include <cstddef>
#include <cstdint>

#if defined(__CUDACC__)
#define GI_PIVOT_FN __device__ __forceinline__
#define GI_PIVOT_HD __host__ __device__ __forceinline__
#else
#define GI_PIVOT_FN inline
#define GI_PIVOT_HD inline
#endif

namespace gi {
namespace pivot {

constexpr int kMaxK = 7;  // counts for cliques of up to kMaxK vertices
constexpr int kBinomCols = kMaxK + 1;

// One node of the explicit stack.
struct Frame {
    int32_t h;      // required vertices (the root is one)
    int32_t q;      // optional vertices
    int32_t u;      // the pivot once chosen
    int32_t phase;  // 0: new node; 1: pivot child done, non-neighbour children next
};

// A worker's scratch, in 32-bit words: the root's symmetric rows (dmax rows
// of wmax words), the candidate and remaining sets per stack level, and the
// frames.  Rows of a root with out-degree d use a stride of ceil(d / 32).
struct Layout {
    int64_t dmax = 0, wmax = 1, levels = 0;
    GI_PIVOT_HD int64_t a_words() const { return dmax * wmax; }
    GI_PIVOT_HD int64_t set_words() const { return levels * wmax; }
    GI_PIVOT_HD int64_t words() const { return a_words() + 2 * set_words() + 4 * levels; }
};

GI_PIVOT_FN int popc32(uint32_t x) {
#if defined(__CUDA_ARCH__)
    return __popc(x);
#else
    return __builtin_popcount(x);
#endif
}

GI_PIVOT_FN int low_bit(uint32_t x) {  // x != 0
#if defined(__CUDA_ARCH__)
    return __ffs(x) - 1;
#else
    return __builtin_ctz(x);
#endif
}

// Bits above position b of its word (b in [0, 32)).
GI_PIVOT_FN uint32_t above(int b) { return b == 31 ? 0u : ~((2u << b) - 1u); }

// Counts below one root.  D: the root's directed rows (nullptr when it has
// fewer than two out-neighbours), d: its out-degree, kmax <= kMaxK, binom:
// C(q, j) modulo 2^64 for q < L.levels + 1 and j < kBinomCols.  acc[k] gets
// the root's k-cliques (warp-uniform).  Returns false when the search needs
// more than L.levels stack levels (nothing is then added).
template <class Wp>
GI_PIVOT_FN bool count_root(const Wp &wp, const uint32_t *D, int d, int kmax, const uint64_t *binom,
                            const Layout &L, uint32_t *scratch, uint64_t *acc) {
    const int W = d > 32 ? (d + 31) / 32 : 1;
    uint32_t *A = scratch;
    uint32_t *cand = A + L.a_words();
    uint32_t *rest = cand + L.set_words();
    Frame *frames = reinterpret_cast<Frame *>(rest + L.set_words());
    const int lane = wp.lane(), width = wp.width();
    uint64_t part[kMaxK + 1];
    for (int k = 0; k <= kMaxK; ++k) part[k] = 0;

    // A = D | D^T, one row per lane.
    for (int i = lane; i < d; i += width)
        for (int w = 0; w < W; ++w) {
            uint32_t word = D ? D[static_cast<int64_t>(i) * W + w] : 0u;
            if (D)
                for (int b = 0; b < 32 && 32 * w + b < d; ++b)
                    if ((D[static_cast<int64_t>(32 * w + b) * W + (i >> 5)] >> (i & 31)) & 1u) word |= 1u << b;
            A[static_cast<int64_t>(i) * W + w] = word;
        }
    // Level 0: every out-neighbour.
    for (int w = lane; w < W; w += width) {
        const int bits = d - 32 * w;
        cand[w] = bits >= 32 ? 0xffffffffu : (bits > 0 ? (1u << bits) - 1u : 0u);
    }
    if (lane == 0) frames[0] = Frame{1, 0, -1, 0};
    wp.sync();

    int level = 0;
    while (level >= 0) {
        const Frame F = frames[level];
        const uint32_t *S = cand + static_cast<int64_t>(level) * W;
        uint32_t *R = rest + static_cast<int64_t>(level) * W;
        if (F.phase == 0) {
            if (F.h >= kmax - 3) {
                // Closed form: |S|, edges and triangles of G[S].
                uint64_t c1 = 0, twice = 0, tri = 0;
                for (int w = lane; w < W; w += width) c1 += popc32(S[w]);
                if (F.h <= kmax - 2)
                    for (int x = lane; x < d; x += width) {
                        if (!((S[x >> 5] >> (x & 31)) & 1u)) continue;
                        const uint32_t *ax = A + static_cast<int64_t>(x) * W;
                        for (int w = 0; w < W; ++w) twice += popc32(S[w] & ax[w]);
                        if (F.h > kmax - 3) continue;
                        // triangles x < y < z
                        for (int wy = x >> 5; wy < W; ++wy) {
                            uint32_t by = S[wy] & ax[wy];
                            if (wy == (x >> 5)) by &= above(x & 31);
                            for (; by; by &= by - 1) {
                                const int y = 32 * wy + low_bit(by);
                                const uint32_t *ay = A + static_cast<int64_t>(y) * W;
                                uint64_t c = popc32(S[wy] & ax[wy] & ay[wy] & above(y & 31));
                                for (int w = wy + 1; w < W; ++w) c += popc32(S[w] & ax[w] & ay[w]);
                                tri += c;
                            }
                        }
                    }
                const uint64_t cl[4] = {1, wp.sum(c1), wp.sum(twice) / 2, wp.sum(tri)};
                for (int k = F.h; k <= kmax; ++k)
                    for (int j = 0; j <= k - F.h && j <= F.q; ++j)
                        part[k] += binom[static_cast<int64_t>(F.q) * kBinomCols + j] * cl[k - F.h - j];
                --level;
                continue;
            }
            // Pivot: the candidate with the most neighbours in S (ties: the
            // smallest index).
            int64_t best = -1;
            int32_t u = 0x7fffffff;
            for (int x = lane; x < d; x += width) {
                if (!((S[x >> 5] >> (x & 31)) & 1u)) continue;
                const uint32_t *ax = A + static_cast<int64_t>(x) * W;
                int64_t c = 0;
                for (int w = 0; w < W; ++w) c += popc32(S[w] & ax[w]);
                if (c > best) {
                    best = c;
                    u = x;
                }
            }
            wp.argmax(best, u);
            if (best < 0) {  // leaf
                for (int k = F.h; k <= kmax && k - F.h <= F.q; ++k)
                    part[k] += binom[static_cast<int64_t>(F.q) * kBinomCols + (k - F.h)];
                --level;
                continue;
            }
            if (level + 1 >= L.levels) return false;
            const uint32_t *au = A + static_cast<int64_t>(u) * W;
            uint32_t *next = cand + static_cast<int64_t>(level + 1) * W;
            for (int w = lane; w < W; w += width) {
                R[w] = S[w];
                next[w] = S[w] & au[w];
            }
            if (lane == 0) {
                frames[level] = Frame{F.h, F.q, u, 1};
                frames[level + 1] = Frame{F.h, F.q + 1, -1, 0};
            }
            wp.sync();
            ++level;
            continue;
        }
        // Next non-neighbour x of the pivot still in R (the earlier ones
        // are gone from R).
        const uint32_t *au = A + static_cast<int64_t>(F.u) * W;
        int x = -1;
        for (int base = 0; base < W && x < 0; base += width) {
            const int w = base + lane;
            uint32_t m = 0;
            if (w < W) {
                m = R[w] & ~au[w];
                if (w == (F.u >> 5)) m &= ~(1u << (F.u & 31));
            }
            const unsigned hit = wp.ballot(m != 0);
            if (hit) {
                const int src = low_bit(hit);
                x = 32 * (base + src) + low_bit(wp.shfl(m, src));
            }
        }
        if (x < 0) {
            --level;
            continue;
        }
        if (level + 1 >= L.levels) return false;
        const uint32_t *ax = A + static_cast<int64_t>(x) * W;
        uint32_t *next = cand + static_cast<int64_t>(level + 1) * W;
        for (int w = lane; w < W; w += width) next[w] = R[w] & ax[w];
        wp.sync();
        if (lane == 0) {
            R[x >> 5] &= ~(1u << (x & 31));
            frames[level + 1] = Frame{F.h + 1, F.q, -1, 0};
        }
        wp.sync();
        ++level;
    }
    for (int k = 0; k <= kMaxK; ++k) acc[k] += part[k];
    return true;
}

// One lane: the host build of the search.
struct HostLane {
    int lane() const { return 0; }
    int width() const { return 1; }
    void sync() const {}
    unsigned ballot(bool p) const { return p ? 1u : 0u; }
    uint32_t shfl(uint32_t v, int) const { return v; }
    uint64_t sum(uint64_t v) const { return v; }
    void argmax(int64_t &, int32_t &) const {}
};

#if defined(__CUDACC__)
// A whole warp; every lane calls every member (warp-uniform call sites).
struct WarpLanes {
    int l;
    __device__ int lane() const { return l; }
    __device__ int width() const { return 32; }
    __device__ void sync() const { __syncwarp(); }
    __device__ unsigned ballot(bool p) const { return __ballot_sync(0xffffffffu, p); }
    __device__ uint32_t shfl(uint32_t v, int src) const { return __shfl_sync(0xffffffffu, v, src); }
    __device__ uint64_t sum(uint64_t v) const {
        for (int o = 16; o; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
        return v;
    }
    // The largest value over the lanes, the smallest key among equal values.
    __device__ void argmax(int64_t &val, int32_t &key) const {
        for (int o = 16; o; o >>= 1) {
            const int64_t ov = __shfl_xor_sync(0xffffffffu, val, o);
            const int32_t ok = __shfl_xor_sync(0xffffffffu, key, o);
            if (ov > val || (ov == val && ok < key)) {
                val = ov;
                key = ok;
            }
        }
    }
};
#endif

}  // namespace pivot
}  // namespace gi
