"""Regenerates the golden fixtures in this directory from the reference itself.

Run in a checkout that has the reference sources ($GI_REFERENCE, else a
"reference" directory beside this repository)
after ``make -C oracle ref`` has built the reference CPU binaries into
oracle/_ref/:

    python tests/golden/make_golden.py [--ref <reference checkout>]

Writes
  plans.jsonl   every Schedule_IEP field of the reference planner for each job
                (reference src/schedule_IEP.cpp), long never-cleared vectors
                stored as (length, sha1, first 256 entries);
  counts.json   reference pm_test / clique_test / motif_counting_test counts on
                seeded synthetic graphs, with each graph's generator parameters
                and a sha1 of its CSR arrays so tests can regenerate it;
  fsm.json      reference fsm_test results on seeded labeled graphs (generator
                parameters, sha1 of the .adj text) and the reference planner's
                FSM schedules for each graph.

The tests never read the reference; they only read these files.
"""
from __future__ import annotations

import argparse
import hashlib
import json
import os
import re
import subprocess
import sys
import tempfile
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))

import graphindor_b200 as gi  # noqa: E402
from graphindor_b200 import gen  # noqa: E402

HERE = Path(__file__).resolve().parent
REF_BIN = ROOT / "oracle" / "_ref"

# The reference's own test patterns (reference test/gpu_pattern_matching_test.cu:19-26,
# reproduce/pattern_matching.py:6-11).
REF_TEST_PATTERNS = [
    (5, "0111010011100011100001100"),
    (6, "011011101110110101011000110000101000"),
    (6, "011111101000110111101010101101101010"),
    (6, "011110101101110000110000100001010010"),
    (7, "0111111101111111011101110100111100011100001100000"),
    (7, "0111111101111111011001110100111100011000001100000"),
]
# The six patterns of the R-MAT scale-22 workload.
WORKLOAD_PATTERNS = [
    (4, "0111101111001100"),                        # diamond
    (4, "0110100110010110"),                        # 4-cycle
    (5, "0101110101010101010011000"),               # house
    (5, "0111110111110111110111110"),               # 5-clique
    (6, "011100101010110001100011010101001110"),    # prism
    (6, "010101101000010100101010000101100010"),    # 6-cycle + chord (0,3)
]
GRAPHS = {
    "rmat_s9_ef8": ("rmat", dict(scale=9, edge_factor=8.0, seed=11)),
    "rmat_s10_ef12": ("rmat", dict(scale=10, edge_factor=12.0, seed=12)),
    "er_n600_m4000": ("er", dict(n=600, m=4000, seed=13)),
    "cl_n2000_m12000": ("chung_lu", dict(n=2000, m=12000, gamma=2.2, max_degree=200.0, seed=14)),
}


def make_graph(kind: str, params: dict) -> gen.CSR:
    if kind == "rmat":
        return gen.rmat(params["scale"], params["edge_factor"], params["seed"])
    if kind == "er":
        return gen.erdos_renyi(params["n"], params["m"], params["seed"])
    if kind == "chung_lu":
        return gen.chung_lu(params["n"], params["m"], params["gamma"], params["max_degree"], params["seed"])
    raise ValueError(kind)


def csr_sha1(g: gen.CSR) -> str:
    h = hashlib.sha1()
    h.update(g.vertex.tobytes())
    h.update(g.edge.tobytes())
    return h.hexdigest()


def compact(vec: list) -> dict:
    return {"len": len(vec), "sha1": hashlib.sha1(json.dumps(vec).encode()).hexdigest(), "head": vec[:256]}


def plan_jobs(ref_root: Path):
    motifs = {}
    out = subprocess.run([str(REF_BIN / "ref_plan_dump")], input="".join(f"motifs {k} -\n" for k in range(3, 8)),
                         capture_output=True, text=True, check=True).stdout.splitlines()
    for k, line in zip(range(3, 8), out):
        motifs[k] = json.loads(line)["motifs"]
    stats = [(7115, 201524, 608389), (4194304, 86000000, 123456789), (1000, 5000, 0)]
    jobs = []
    for k in range(3, 7):
        for adj in motifs[k]:
            for v, e, t in stats:
                for iep in (1, 0):
                    jobs.append(f"full {k} {adj} {v} {e} {t} {iep}")
            jobs.append(f"induced {k} {adj}")
    import random
    for adj in random.Random(5).sample(motifs[7], 24):
        jobs.append(f"full 7 {adj} 4194304 86000000 123456789 1")
    for n, adj in REF_TEST_PATTERNS + WORKLOAD_PATTERNS:
        for v, e, t in stats[:2]:
            jobs.append(f"full {n} {adj} {v} {e} {t} 1")
    return jobs, motifs


def write_plans(jobs):
    res = subprocess.run([str(REF_BIN / "ref_plan_dump")], input="\n".join(jobs) + "\n", capture_output=True,
                         text=True, check=True).stdout.splitlines()
    with open(HERE / "plans.jsonl", "w") as f:
        for job, line in zip(jobs, res):
            d = json.loads(line)
            for key in ("iep_vertex_flag", "iep_vertex_coef", "iep_ans_pos"):
                if key in d:
                    d[key] = compact(d[key])
            d.pop("maxp", None)
            f.write(json.dumps({"job": job, "ref": d}) + "\n")


def run_ref(binary: str, *args, timeout=600) -> str:
    return subprocess.run([str(REF_BIN / binary), *map(str, args)], capture_output=True, text=True, check=True,
                          timeout=timeout).stdout


def write_counts(motifs):
    out = {"graphs": {}, "patterns": {}, "cliques": {}, "motifs": {}}
    pats = [(k, a) for k in (3, 4, 5) for a in motifs[k]] + WORKLOAD_PATTERNS + REF_TEST_PATTERNS
    with tempfile.TemporaryDirectory() as td:
        for name, (kind, params) in GRAPHS.items():
            g = make_graph(kind, params)
            path = Path(td) / f"{name}.g"
            gi.write_g(str(path), g.vertex, g.edge, g.max_intersection_size, 0)
            out["graphs"][name] = {"kind": kind, "params": params, "v_cnt": g.v_cnt, "e_cnt": g.e_cnt,
                                   "sha1": csr_sha1(g)}
            rows = {}
            for n, adj in pats:
                t = time.time()
                txt = run_ref("pm_test", path, n, adj)
                m = re.search(r"Ans: (-?\d+)", txt)
                rows[adj] = int(m.group(1))
                print(name, adj, rows[adj], f"{time.time() - t:.2f}s", flush=True)
            out["patterns"][name] = rows
            cl = {}
            for k in (3, 4, 5, 6):
                txt = run_ref("clique_test", path, k)
                cl[str(k)] = int(re.search(r"ans: (-?\d+)", txt).group(1))
            out["cliques"][name] = cl
            mo = {}
            txt = run_ref("motif_counting_test", path, 3)
            m = re.search(r"triangle: (\d+) wedge: (\d+)", txt)
            mo["3"] = [int(m.group(1)), int(m.group(2))]
            txt = run_ref("motif_counting_test", path, 4)
            mo["4"] = [int(x) for x in re.findall(r"^ans: (-?\d+)", txt, re.M)]
            out["motifs"][name] = mo
    with open(HERE / "counts.json", "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)


# Labeled graphs for FSM: (scale, edge_factor, seed, keep, n_labels, zipf_s,
# label_seed) of graphindor_b200.gen.labeled_rmat, and the (max_edge,
# min_support) runs of the reference fsm_test on each.
FSM_GRAPHS = {
    "lrmat_s10_l5": (dict(scale=10, edge_factor=8.0, seed=5, keep=900, n_labels=5, zipf_s=1.1, label_seed=7),
                     [(me, ms) for me in (1, 2, 3) for ms in (5, 20, 60)] + [(4, 40)]),
    "lrmat_s11_l12": (dict(scale=11, edge_factor=10.0, seed=21, keep=1800, n_labels=12, zipf_s=1.1, label_seed=8),
                      [(me, ms) for me in (2, 3) for ms in (10, 40)]),
    "lrmat_s12_l29": (dict(scale=12, edge_factor=12.0, seed=31, keep=3500, n_labels=29, zipf_s=1.1, label_seed=9),
                      [(me, ms) for me in (2, 3) for ms in (15, 50)]),
    "lrmat_s12_l3": (dict(scale=12, edge_factor=6.0, seed=41, keep=4096, n_labels=3, zipf_s=0.3, label_seed=10),
                     [(3, 200), (3, 800)]),
}
FSM_TRI_CNT = 7515023  # fsm_test plans with the Patents constant (reference src/fsm_test.cpp:27)


def adj_sha1(path: Path) -> str:
    return hashlib.sha1(path.read_bytes()).hexdigest()


def fsm_plans(motifs_by_k, max_edge, v_cnt, e_cnt):
    """The reference's FSM plans: Schedule_IEP(p, valid, 1, 1, 1, v, e, tri)
    of every connected pattern with at most max_edge edges (reference
    src/labeled_graph.cpp:180-196, :438-452), as (schedule-order adjacency,
    label restrictions (d, r))."""
    pats = []
    for k in range(2, max_edge + 2):
        for adj in motifs_by_k[k]:
            e = sum(adj[i * k + j] == "1" for i in range(k) for j in range(i + 1, k))
            if e <= max_edge:
                pats.append((e, k, adj))
    pats.sort(key=lambda t: t[0])  # stable
    jobs = [f"full {k} {adj} {v_cnt} {e_cnt} {FSM_TRI_CNT} 1" for _, k, adj in pats]
    res = subprocess.run([str(REF_BIN / "ref_plan_dump")], input="\n".join(jobs) + "\n", capture_output=True,
                         text=True, check=True).stdout.splitlines()
    out = []
    for (e, k, _), line in zip(pats, res):
        d = json.loads(line)
        restricts = []
        for depth in range(k):
            r = d["restrict_last"][depth]
            while r != -1:
                restricts.append([depth, d["restrict_index"][r]])
                r = d["restrict_next"][r]
        out.append({"n": k, "edges": e, "adj": "".join(str(x) for x in d["adj_mat"]), "restricts": restricts})
    return out


def write_fsm():
    motifs_by_k = {}
    lines = subprocess.run([str(REF_BIN / "ref_plan_dump")], input="".join(f"motifs {k} -\n" for k in range(2, 6)),
                           capture_output=True, text=True, check=True).stdout.splitlines()
    for k, line in zip(range(2, 6), lines):
        motifs_by_k[k] = json.loads(line)["motifs"]
    out = {"tri_cnt": FSM_TRI_CNT, "graphs": {}}
    with tempfile.TemporaryDirectory() as td:
        for name, (params, runs) in FSM_GRAPHS.items():
            g, labels = gen.labeled_rmat(**params)
            path = Path(td) / f"{name}.adj"
            gen.write_adj(str(path), g, labels)
            e_cnt = int(g.e_cnt)
            max_me = max(me for me, _ in runs)
            rows = []
            for me, ms in runs:
                t = time.time()
                txt = run_ref("fsm_test", path, me, ms)
                cnt = int(re.findall(r"fsm_cnt = (-?\d+)", txt)[-1])
                rows.append({"max_edge": me, "min_support": ms, "fsm_cnt": cnt})
                print(name, me, ms, cnt, f"{time.time() - t:.2f}s", flush=True)
            out["graphs"][name] = {"params": params, "v_cnt": g.v_cnt, "e_cnt": e_cnt, "adj_sha1": adj_sha1(path),
                                   "runs": rows, "plans": fsm_plans(motifs_by_k, max_me, g.v_cnt, e_cnt)}
    with open(HERE / "fsm.json", "w") as f:
        json.dump(out, f, indent=1, sort_keys=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--ref", default=os.environ.get("GI_REFERENCE", str(ROOT.parent / "reference")))
    ap.add_argument("--skip-plans", action="store_true")
    ap.add_argument("--only-fsm", action="store_true")
    a = ap.parse_args()
    if a.only_fsm:
        write_fsm()
        return
    jobs, motifs = plan_jobs(Path(a.ref))
    if not a.skip_plans:
        write_plans(jobs)
    write_counts(motifs)
    write_fsm()


if __name__ == "__main__":
    main()
