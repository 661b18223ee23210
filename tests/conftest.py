"""Shared fixtures.  GPU tests carry @pytest.mark.gpu; everything else runs
on a CPU-only host."""
from __future__ import annotations

import json
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
GOLDEN = ROOT / "tests" / "golden"
for p in (str(ROOT), str(ROOT / "oracle")):
    if p not in sys.path:
        sys.path.insert(0, p)


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (runs on the B200 box)")


@pytest.fixture(scope="session")
def native():
    """The engine library, built in-tree if it is missing."""
    from graphindor_b200 import _native, build
    if not _native.LIB_PATH.exists():
        build.build()
    return _native.lib()


@pytest.fixture(scope="session")
def oracle():
    import oracle_py
    oracle_py.build()
    return oracle_py


@pytest.fixture(scope="session")
def golden_counts():
    with open(GOLDEN / "counts.json") as f:
        return json.load(f)


@pytest.fixture(scope="session")
def golden_graphs(golden_counts, native):
    """The seeded graphs behind counts.json, regenerated and checked against
    their recorded sha1."""
    import hashlib
    from graphindor_b200 import gen
    out = {}
    for name, meta in golden_counts["graphs"].items():
        p = meta["params"]
        if meta["kind"] == "rmat":
            g = gen.rmat(p["scale"], p["edge_factor"], p["seed"])
        elif meta["kind"] == "er":
            g = gen.erdos_renyi(p["n"], p["m"], p["seed"])
        else:
            g = gen.chung_lu(p["n"], p["m"], p["gamma"], p["max_degree"], p["seed"])
        h = hashlib.sha1()
        h.update(g.vertex.tobytes())
        h.update(g.edge.tobytes())
        assert h.hexdigest() == meta["sha1"], f"generator drift for {name}"
        out[name] = g
    return out


def plan_desc(schedule):
    """The C struct of a plan, as the oracle consumes it."""
    import ctypes as C
    from graphindor_b200 import _native as N
    d = N.PlanDesc()
    N.check(N.lib().gi_plan_export(schedule.handle, C.byref(d)), "gi_plan_export")
    return d


@pytest.fixture(scope="session")
def golden_fsm():
    with open(GOLDEN / "fsm.json") as f:
        return json.load(f)


@pytest.fixture(scope="session")
def fsm_graphs(golden_fsm, native, tmp_path_factory):
    """The seeded labeled graphs behind fsm.json: name -> (CSR, labels, path of
    the regenerated .adj file), each checked against its recorded sha1."""
    import hashlib
    from graphindor_b200 import gen
    d = tmp_path_factory.mktemp("fsm")
    out = {}
    for name, meta in golden_fsm["graphs"].items():
        g, labels = gen.labeled_rmat(**meta["params"])
        path = d / f"{name}.adj"
        gen.write_adj(str(path), g, labels)
        assert hashlib.sha1(path.read_bytes()).hexdigest() == meta["adj_sha1"], f"generator drift for {name}"
        out[name] = (g, labels, path)
    return out
