"""The bench's timed edge subsets are the ones whose raw sums the reference
pinned (tests/golden/configs.json, section c2_sample): the same graph
parameters, the same step per pattern, the same pattern strings.  A change
of bench.py's subsets without regenerated fixtures fails here, on CPU."""
from __future__ import annotations

import json
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def test_bench_subsets_match_the_pinned_fixtures():
    sys.path.insert(0, str(ROOT))
    import bench
    c = json.loads((ROOT / "tests" / "golden" / "configs.json").read_text())["c2_sample"]
    assert c["params"] == {"scale": bench.SCALE, "edge_factor": bench.EDGE_FACTOR, "seed": bench.SEED}
    assert set(c["subsets"]) == {name for name, _, _ in bench.PATTERNS}
    for name, _, _ in bench.PATTERNS:
        rows = c["subsets"][name]
        assert [(r["step"], r["offset"]) for r in rows] == [(bench.SAMPLE_EDGE_STEP[name], 0)], name
    from test_gpu_configs import WORKLOAD
    assert {name: (n, adj) for name, n, adj in bench.PATTERNS} == WORKLOAD


def test_config3_fixtures_present():
    c = json.loads((ROOT / "tests" / "golden" / "configs.json").read_text())
    assert {int(k) for k in c["c3_cliques"]["cliques"]} == {3, 4, 5, 6}
    assert [(r["max_edge"], r["min_support"], r["fsm_cnt"]) for r in c["c3_fsm"]["runs"]] == [(3, 1000, 1167),
                                                                                             (3, 3000, 46)]
