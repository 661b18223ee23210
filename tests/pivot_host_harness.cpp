// Test harness, built by tests/test_pivot_host.py: the host (one-lane) build
// of the clique-tree pivoting search in graphindor_b200/csrc/pivot.cuh, the
// same code the GPU kernel runs a warp at a time, over bitmaps laid out as
// the k-clique bitmap kernels lay them out.
#include "../graphindor_b200/csrc/pivot.cuh"

#include <algorithm>
#include <vector>

using gi::pivot::HostLane;
using gi::pivot::Layout;

// dvertex / off: the DAG's offsets and each vertex's bitmap word offset
// (v_cnt + 1 entries); bitmap rows as in kclique.cu.  counts gets kmax + 1
// entries.  Returns 0, or -1 when the search needs more than `levels`.
extern "C" int pivot_host_counts(const int64_t *dvertex, int32_t v_cnt, const int64_t *off, const uint32_t *bitmap,
                                 int kmax, int levels, uint64_t *counts) {
    Layout L;
    for (int32_t v = 0; v < v_cnt; ++v) L.dmax = std::max<int64_t>(L.dmax, dvertex[v + 1] - dvertex[v]);
    L.dmax = std::max<int64_t>(L.dmax, 1);
    L.wmax = (L.dmax + 31) / 32;
    L.levels = levels;
    const int cols = gi::pivot::kBinomCols;
    std::vector<uint64_t> binom(static_cast<size_t>(levels + 1) * cols, 0);
    for (int q = 0; q <= levels; ++q)
        for (int j = 0; j < cols; ++j)
            binom[q * cols + j] = j == 0 ? 1 : (q == 0 ? 0 : binom[(q - 1) * cols + j - 1] + binom[(q - 1) * cols + j]);
    std::vector<uint32_t> scratch(static_cast<size_t>(L.words()));
    uint64_t acc[gi::pivot::kMaxK + 1] = {};
    for (int32_t v = 0; v < v_cnt; ++v) {
        const int d = static_cast<int>(dvertex[v + 1] - dvertex[v]);
        const uint32_t *D = d >= 2 ? bitmap + off[v] : nullptr;
        if (!gi::pivot::count_root(HostLane{}, D, d, kmax, binom.data(), L, scratch.data(), acc)) return -1;
    }
    counts[0] = 0;
    for (int k = 1; k <= kmax; ++k) counts[k] = acc[k];
    return 0;
}
