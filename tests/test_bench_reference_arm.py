"""bench.py's reference arm runs on host cores only: its JSON line at a small
scale, the same edge subsets as the GPU arm (their raw sums add up over the
arm's parts to the oracle's count of the subset), and the silent exit of a
non-zero rank under torchrun."""
from __future__ import annotations

import json
import os
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def _run(extra_env=None, *args):
    env = dict(os.environ, **(extra_env or {}))
    return subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--scale", "13", "--steps",
                           "3", "--warmup", "1", "--step-scale", "64", *args], capture_output=True, text=True,
                          env=env, timeout=600)


def test_reference_arm_prints_its_line(native, oracle):
    import bench
    import graphindor_b200 as gi
    from conftest import plan_desc
    r = _run()
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["value"] > 0 and line["unit"] == "embeddings/s"
    # The reference's own code when its sources were compiled here, else the port.
    built = os.access(ROOT / "oracle" / "_ref" / "ref_edge_sample", os.X_OK)
    assert line["cpu_baseline"]["kind"] == ("reference" if built else "port")
    assert line["cpu_baseline"]["cores"] >= 1
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["d2h_bytes_per_step"] == 0
    # Over its three parts the arm counted exactly each pattern's subset.
    g = bench.make_graph(13)
    tri = oracle.triangles(g.vertex, g.edge)
    for name, n, adj in bench.PATTERNS[:5]:
        step = line["config"]["edge_step"][name]
        d = plan_desc(gi.Schedule_IEP(gi.Pattern(n, adj), g.v_cnt, g.e_cnt, tri))
        want, done = oracle.count_edges_timed(d, g.vertex, g.edge, step)
        got = line["config"]["per_pattern"][name]
        assert got["raw_sum"] == want and got["edges"] == done, name


def test_reference_arm_other_ranks_exit_quietly(native):
    r = _run({"WORLD_SIZE": "2", "RANK": "1", "LOCAL_RANK": "1"})
    assert r.returncode == 0 and r.stdout.strip() == ""
