"""bench.py's reference arm runs on host cores only: its JSON line at a small
scale, and the silent exit of a non-zero rank under torchrun."""
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
                           "1", "--warmup", "1", "--cpu-target-s", "0.2", *args], capture_output=True, text=True,
                          env=env, timeout=300)


def test_reference_arm_prints_its_line(native, oracle):
    r = _run()
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference" and line["value"] > 0 and line["unit"] == "embeddings/s"
    # The reference's own code when its sources were compiled here, else the port.
    built = os.access(ROOT / "oracle" / "_ref" / "ref_edge_sample", os.X_OK)
    assert line["cpu_baseline"]["kind"] == ("reference" if built else "port")
    assert line["cpu_baseline"]["cores"] >= 1
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["d2h_bytes_per_step"] == 0


def test_reference_arm_other_ranks_exit_quietly(native):
    r = _run({"WORLD_SIZE": "2", "RANK": "1", "LOCAL_RANK": "1"})
    assert r.returncode == 0 and r.stdout.strip() == ""
