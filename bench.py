"""Benchmark: pattern counting with IEP on an R-MAT scale-22 graph, six patterns.

Workload: a seeded R-MAT graph, scale 22 (4.19M vertices), edge factor 10.6
(about 43M undirected edges once symmetrised, deduplicated and stripped of
self-loops), a/b/c = 0.57/0.19/0.19, random relabelling; the six patterns
diamond, 4-cycle, house, 5-clique, prism and 6-cycle with chord (0,3), each
planned as the reference's gpu_graph plans them (analytic model, the
reference's restriction generator, IEP on).

The whole six-pattern job runs for days on any machine, so the bench
measures a fixed random sample of it.  First-level work is cut into chunks of
GI_TASK_CHUNK subtasks; for pattern p a step counts the first M_p chunks of a
fixed pseudo-random order over all of them (gi_stats.sample_chunks), each to
completion, with M_p = SAMPLE_CHUNKS[p].  The sample, and so its count, is the
same on every run; only the time varies.  Under torchrun rank r samples shard r of
world (weak scaling: every rank counts its own M_p chunks).

value = whole-job throughput estimated from the samples:
          sum_p (embeddings counted for p) / f_p  over  sum_p (device time for p) / f_p
        with f_p = M_p / chunks_p and the graph resident in HBM (device time
        from CUDA events).
e2e   = the same whole job through the public API from pinned host buffers:
        graph upload (H2D) + planning + counts + result reads (D2H).
cpu_baseline / --impl reference: the reference's CPU path on all host cores
        over every s_p-th directed edge (an unbiased slice: ids are random),
        extrapolated the same way.  It is the reference's own code where its
        sources were compiled into oracle/_ref (ref_edge_sample: its per-edge
        task, Graph::pattern_matching_edge_task, with its own plans from the
        .g header; kind "reference"), else the oracle, a C restatement of
        reference src/graph.cpp:305-566 (kind "port").
"""
from __future__ import annotations

import argparse
import atexit
import ctypes as C
import json
import os
import shutil
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

SCALE, EDGE_FACTOR, SEED = 22, 10.6, 2
PATTERNS = [
    ("diamond", 4, "0111101111001100"),
    ("4-cycle", 4, "0110100110010110"),
    ("house", 5, "0101110101010101010011000"),
    ("5-clique", 5, "0111110111110111110111110"),
    ("prism", 6, "011100101010110001100011010101001110"),
    ("6-cycle+chord", 6, "010101101000010100101010000101100010"),
]
# Chunks of each pattern's fixed sample (0 = all of them).  Sized on a B200 at
# scale 22 so that each sample takes about 0.5 - 7 s: the prism and 6-cycle +
# chord jobs are so heavy-tailed (5.8e6 and ~1e8 device-seconds whole) that 64
# and 16 chunks already take seconds; their estimates are the roughest.
SAMPLE_CHUNKS = {"diamond": 0, "4-cycle": 65536, "house": 16384, "5-clique": 16384, "prism": 64,
                 "6-cycle+chord": 16}
CPU_TARGET_S = 3.0           # host time of one pattern's CPU slice
MEASURED = ROOT / "MEASURED_PEAKS.json"
METRIC = "pattern-match embeddings/s, whole six-pattern job (R-MAT s22, IEP), 1 B200"


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--scale", type=int, default=SCALE)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--sample-scale", type=float, default=1.0, help="multiplies every sample size")
    ap.add_argument("--workload", choices=["patterns", "batch"], default="patterns",
                    help="batch: many small (pattern, graph) jobs in one launch vs one launch per job")
    ap.add_argument("--cpu-target-s", type=float, default=CPU_TARGET_S)
    return ap.parse_args()


def make_graph(scale: int):
    from graphindor_b200 import gen
    return gen.rmat(scale, EDGE_FACTOR, SEED)


_PINNED = []  # keeps the pinned host buffers alive


def pinned(a: np.ndarray) -> np.ndarray:
    import torch
    t = torch.empty(a.shape, dtype={np.int64: torch.int64, np.int32: torch.int32}[a.dtype.type], pin_memory=True)
    _PINNED.append(t)
    out = t.numpy()
    out[...] = a
    return out


class Clocks:
    """nvidia-smi samples (200 ms) taken during the timed region."""

    def __init__(self, gpu_index: int):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--id={gpu_index}", f"--query-gpu={q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def stop(self) -> dict:
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.p.terminate()
        self.p.wait()
        self.f.seek(0)
        rows = [[x.strip() for x in r.split(",")] for r in self.f.read().splitlines() if r.strip()]
        os.unlink(self.f.name)
        num = lambda s: s.replace(".", "", 1).isdigit()  # noqa: E731
        sm = [float(r[1]) for r in rows if len(r) >= 9 and num(r[1])]
        mx = [float(r[2]) for r in rows if len(r) >= 9 and num(r[2])]
        reasons = set()
        for r in rows:
            if len(r) < 9:
                continue
            for name, val in zip(["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"], r[5:9]):
                if val == "Active":
                    reasons.add(name)
        busy = [x for x in sm if x > 500] or sm
        return {"sm_mhz": statistics.median(busy) if busy else None, "sm_max_mhz": max(mx) if mx else None,
                "samples": len(rows), "reasons": sorted(reasons)}


def run_ours(args, world, rank, local):
    import torch

    import graphindor_b200 as gi
    from graphindor_b200 import _native as N

    torch.cuda.set_device(local)
    L = gi.lib()
    g = make_graph(args.scale)
    vertex_h, edge_h = pinned(g.vertex), pinned(g.edge)
    stream = torch.cuda.Stream()
    sp = C.c_void_p(stream.cuda_stream)
    dg = gi.Graph.from_csr(vertex_h, edge_h, stream=stream.cuda_stream)
    tri = gi.clique_count(dg, 3, 1, stream=stream.cuda_stream).count  # the .g header's triangle count
    del dg
    dg = gi.Graph.from_csr(vertex_h, edge_h, tri_cnt=tri, stream=stream.cuda_stream)
    plans = {name: gi.Schedule_IEP(gi.Pattern(n, adj), dg.v_cnt, dg.e_cnt, tri) for name, n, adj in PATTERNS}
    divisors = {name: plans[name].export()["count_divisor"] for name, _, _ in PATTERNS}

    # Chunks per pattern (shard `rank` of `world`), then the fixed sample sizes.
    sample = {}
    for name, _, _ in PATTERNS:
        st = N.Stats()
        st.sample_chunks = 1
        raw = C.c_uint64()
        N.check(L.gi_count_shard(dg.handle, plans[name].handle, rank, world, sp, C.byref(raw), C.byref(st)),
                "gi_count_shard")
        want = SAMPLE_CHUNKS[name]
        m = st.chunks_total if want == 0 else max(1, int(round(want * args.sample_scale)))
        sample[name] = (min(m, st.chunks_total), st.chunks_total)

    def one_step(graph, plan_map, step, acc, count_bytes=False):
        for name, _, _ in PATTERNS:
            st = N.Stats()
            st.count_bytes = 1 if count_bytes else 0
            st.sample_chunks = sample[name][0]
            raw = C.c_uint64()
            N.check(L.gi_count_shard(graph.handle, plan_map[name].handle, rank, world, sp, C.byref(raw),
                                     C.byref(st)), "gi_count_shard")
            f = st.chunks_done / max(1, st.chunks_total * world)  # fraction of the whole job
            a = acc.setdefault(name, {"emb": 0.0, "ms": 0.0, "launches": 0, "bytes_per_chunk": 0.0, "chunks": 0,
                                      "job_emb": 0.0, "job_ms": 0.0, "prep_ms": 0.0})
            a["emb"] += raw.value / divisors[name]
            a["ms"] += st.kernel_ms
            a["prep_ms"] += st.prep_ms
            a["launches"] += st.kernel_launches
            a["chunks"] += st.chunks_done
            if count_bytes and st.chunks_done:
                a["bytes_per_chunk"] = st.alg_bytes / st.chunks_done
            if f > 0:
                a["job_emb"] += raw.value / divisors[name] / f
                a["job_ms"] += st.prep_ms + st.kernel_ms / f

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            torch.distributed.barrier()

    steps = range(args.warmup, args.warmup + args.steps)
    for s in range(args.warmup):
        one_step(dg, plans, s, {})
    instr = {}
    one_step(dg, plans, 0, instr, count_bytes=True)  # algorithmic bytes of the (fixed) sample, untimed

    clocks = Clocks(torch.cuda.current_device())
    barrier()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    acc = {}
    for s in steps:
        one_step(dg, plans, s, acc)
    ev1.record(stream)
    barrier()
    clk = clocks.stop()
    dev_ms = ev0.elapsed_time(ev1)

    # End to end through the public API, every step: upload from pinned host
    # memory, planning, the shard counts, the result reads.
    del dg
    barrier()
    e2e = {"upload_ms": 0.0, "plan_ms": 0.0}
    e2e_acc = {}
    for s in steps:
        e0, e1, e2, e3 = (torch.cuda.Event(enable_timing=True) for _ in range(4))
        e0.record(stream)
        g2 = gi.Graph.from_csr(vertex_h, edge_h, tri_cnt=tri, stream=stream.cuda_stream)
        e1.record(stream)
        p2 = {name: gi.Schedule_IEP(gi.Pattern(n, adj), g2.v_cnt, g2.e_cnt, tri) for name, n, adj in PATTERNS}
        e2.record(stream)
        one_step(g2, p2, s, e2e_acc)
        e3.record(stream)
        e3.synchronize()
        e2e["upload_ms"] += e0.elapsed_time(e1)
        e2e["plan_ms"] += e1.elapsed_time(e2)
        del g2, p2
    barrier()

    # Whole-job estimates, averaged over the steps and summed over ranks
    # (each rank samples its own shards; the job's time is the ranks' max).
    names = [n for n, _, _ in PATTERNS]
    k = len(names)
    vec = [acc[n]["job_emb"] for n in names] + [acc[n]["job_ms"] for n in names] + \
          [e2e_acc[n]["job_ms"] for n in names] + [acc[n]["ms"] for n in names] + \
          [instr[n]["bytes_per_chunk"] * acc[n]["chunks"] for n in names] + [float(acc[n]["launches"]) for n in names] + \
          [dev_ms, e2e["upload_ms"], e2e["plan_ms"]]
    t = torch.tensor(vec, dtype=torch.float64, device="cuda")
    if world > 1:
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.SUM)
        t /= world
    v = t.tolist()
    job_emb_p = dict(zip(names, v[0:k]))
    job_ms_p = dict(zip(names, v[k:2 * k]))
    e2e_job_ms_p = dict(zip(names, v[2 * k:3 * k]))
    ms_p = dict(zip(names, v[3 * k:4 * k]))
    bytes_p = dict(zip(names, v[4 * k:5 * k]))
    launch_p = dict(zip(names, v[5 * k:6 * k]))
    dev_ms, up_ms, plan_ms = v[6 * k:6 * k + 3]
    job_emb = sum(job_emb_p.values()) / args.steps
    job_ms = sum(job_ms_p.values()) / args.steps
    job_e2e_ms = (up_ms + plan_ms + sum(e2e_job_ms_p.values())) / args.steps

    peaks = json.loads(MEASURED.read_text()) if MEASURED.exists() else {}
    hbm = float(peaks.get("hbm_gbs", 6650.0))
    total_bytes = sum(bytes_p.values())
    count_ms = sum(ms_p.values())
    achieved = total_bytes / (count_ms / 1e3) / 1e9 if count_ms else 0.0
    line = {
        "metric": METRIC,
        "value": job_emb * world / (job_ms / 1e3),
        "unit": "embeddings/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": dev_ms / args.steps,
        "higher_is_better": True,
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "u32 ids / u64 counts",
        "data": "synthetic (seeded R-MAT, no dataset)",
        "config": {
            "workload": f"R-MAT scale {args.scale}, edge factor {EDGE_FACTOR}, seed {SEED}: {g.v_cnt} vertices, "
                        f"{g.e_cnt // 2} undirected edges; six patterns with IEP, reference plans; whole-job "
                        f"throughput estimated from a fixed seeded random sample of each pattern's work chunks "
                        f"(the same sample every step and run)",
            "sample_chunks": {n: {"sampled": sample[n][0], "of": sample[n][1]} for n in names},
            "patterns": {n: adj for n, _, adj in PATTERNS},
            "per_pattern_job_s_estimate": {n: job_ms_p[n] / 1e3 / args.steps for n in names},
            "per_pattern_embeddings_estimate": {n: job_emb_p[n] / args.steps for n in names},
            "l2": "inputs larger than L2 (CSR %.2f GB vs 126 MB)" % ((g.vertex.nbytes + g.edge.nbytes) / 1e9),
            "parallelism": f"dp{world}: shards interleaved across ranks",
        },
        "e2e": {"value": job_emb * world / (job_e2e_ms / 1e3), "unit": "embeddings/s",
                "h2d_bytes_per_step": int(g.vertex.nbytes + g.edge.nbytes),
                "d2h_bytes_per_step": int(2 * 64 * len(PATTERNS)),
                "upload_ms_per_step": up_ms / args.steps, "plan_ms_per_step": plan_ms / args.steps},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                     "frac": achieved / hbm if hbm else None, "traffic": None, "kernel": "dfs_count_kernel",
                     "peak_source": "MEASURED_PEAKS.json hbm_gbs (of measured)" if MEASURED.exists() else "fallback",
                     "note": "achieved = algorithmic bytes of the counting launches (merge-intersection "
                             "accounting, counted by the instrumented kernel) / their CUDA-event time"},
        "gpu_launches": int(round(sum(launch_p.values()) * world)),
        "clocks": clk,
    }
    return line, g, plans, divisors, tri


def plan_descs(plans):
    import graphindor_b200 as gi
    from graphindor_b200 import _native as N
    out = {}
    for name, s in plans.items():
        d = N.PlanDesc()
        N.check(gi.lib().gi_plan_export(s.handle, C.byref(d)), "gi_plan_export")
        out[name] = d
    return out


REF_SAMPLER = ROOT / "oracle" / "_ref" / "ref_edge_sample"
_g_files: dict = {}


def _g_file(g, tri: int) -> str:
    """The graph as a .g file (written once per graph, removed at exit)."""
    import graphindor_b200 as gi
    key = (id(g), tri)
    if key not in _g_files:
        d = tempfile.mkdtemp(prefix="gi_bench_")
        atexit.register(shutil.rmtree, d, True)
        path = os.path.join(d, "graph.g")
        gi.write_g(path, g.vertex, g.edge, int(g.max_intersection_size), int(tri))
        _g_files[key] = path
    return _g_files[key]


def ref_cpu_job(g, tri, threads, target_s):
    """The reference's own CPU code (oracle/_ref/ref_edge_sample) on every
    s_p-th directed edge per pattern, s_p the power of 4 whose slice takes
    about target_s; returns (whole-job embeddings/s, sample text), or None
    when the reference was not compiled here."""
    if not os.access(REF_SAMPLER, os.X_OK):
        return None
    args = [str(REF_SAMPLER), _g_file(g, tri), "1", repr(float(target_s)), str(threads)]
    for _, n, adj in PATTERNS:
        args += [str(n), adj]
    out = subprocess.run(args, capture_output=True, text=True, check=True).stdout
    rows = {f[0]: f for f in (line.split() for line in out.splitlines() if " raw " in line)}
    job_emb = job_s = 0.0
    parts = []
    for name, _, adj in PATTERNS:
        f = rows[adj]
        raw, done, stride, dt, red = int(f[2]), int(f[4]), int(f[6]), float(f[8]), int(f[10])
        scale = g.e_cnt / max(1, done)
        job_emb += raw / red * scale
        job_s += dt * scale
        parts.append(f"{name}: {done} edges (every {stride}th), {dt:.2f}s")
    return (job_emb / job_s if job_s else 0.0), "; ".join(parts)


def cpu_baseline_job(g, tri, descs, divisors, threads, target_s):
    """(embeddings/s, sample text, kind): the reference's own code when it
    was compiled here, else the oracle port."""
    r = ref_cpu_job(g, tri, threads, target_s)
    if r is not None:
        return r[0], r[1], "reference"
    v, sample = cpu_job(g, descs, divisors, threads, target_s)
    return v, sample, "port"


def cpu_job(g, descs, divisors, threads, target_s):
    """The reference CPU path (oracle) on every s_p-th directed edge per
    pattern, s_p the power of 4 whose slice takes about target_s; returns
    (whole-job embeddings/s, sample text)."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle_py
    job_emb = job_s = 0.0
    parts = []
    m = g.e_cnt
    for name, _, _ in PATTERNS:
        stride = 1 << 22
        while True:
            t0 = time.perf_counter()
            # Every stride-th directed edge (the reference's depth-1 loop
            # entered per edge); no edge is begun after 2 * target_s and the
            # extrapolation uses those counted.
            raw, done = oracle_py.count_edges_timed(descs[name], g.vertex, g.edge, stride, 2.0 * target_s, threads)
            dt = time.perf_counter() - t0
            if dt >= target_s / 4.0 or stride == 1:
                break
            stride //= 4
        scale = m / max(1, done)
        job_emb += raw / divisors[name] * scale
        job_s += dt * scale
        parts.append(f"{name}: {done} edges (every {stride}th), {dt:.2f}s")
    return job_emb / job_s if job_s else 0.0, "; ".join(parts)


def run_reference(args, world):
    """Reference arm: the reference's CPU path on all host cores."""
    sys.path.insert(0, str(ROOT / "oracle"))
    import oracle_py

    import graphindor_b200 as gi
    g = make_graph(args.scale)
    tri = int(oracle_py.triangles(g.vertex, g.edge))
    plans = {name: gi.Schedule_IEP(gi.Pattern(n, adj), g.v_cnt, g.e_cnt, tri) for name, n, adj in PATTERNS}
    descs = plan_descs(plans)
    divisors = {n: descs[n].count_divisor for n in descs}
    threads = os.cpu_count() or 1
    values, sample, kind = [], "", "port"
    t0 = time.perf_counter()
    for s in range(args.warmup + args.steps):
        v, sample, kind = cpu_baseline_job(g, tri, descs, divisors, threads, args.cpu_target_s / max(1, args.steps))
        if s >= args.warmup:
            values.append(v)
    wall = time.perf_counter() - t0
    value = statistics.median(values) if values else 0.0
    return {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "embeddings/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": wall * 1e3 / (args.warmup + args.steps),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32 ids / u64 counts",
        "data": "synthetic (seeded R-MAT, no dataset)",
        "config": {"workload": f"R-MAT scale {args.scale}, edge factor {EDGE_FACTOR}, seed {SEED}; six patterns with "
                               "IEP, reference plans; whole-job throughput of the reference CPU path extrapolated "
                               "from strided first-level edge slices"},
        "cpu_baseline": {"value": value, "unit": "embeddings/s", "cores": threads, "kind": kind, "sample": sample},
        "e2e": {"value": value, "unit": "embeddings/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def run_batch(args):
    """Batched serving: 64 seeded random connected patterns of 4-6 vertices
    (edge density 0.4-1.0) against 8 seeded R-MAT graphs of scales 10-12
    (edge factor 8-16), all 512 jobs in one persistent launch replayed from a
    CUDA graph, against one gi_count launch per job; counts must agree.  Also
    end to end with planning: learned plans in one batch against analytic
    plans with one launch per job."""
    import random

    import torch

    import graphindor_b200 as gi
    from graphindor_b200 import gen
    from graphindor_b200.schedule_cost.collect import random_connected
    rng = random.Random(5)
    graphs = []
    for i in range(8):
        g = gen.rmat(rng.randint(10, 12), rng.uniform(8, 16), 100 + i)
        dg = gi.Graph.from_csr(g.vertex, g.edge)
        tri = gi.clique_count(dg, 3, 1).count  # the triangle count the analytic model plans with
        graphs.append(gi.Graph.from_csr(g.vertex, g.edge, tri_cnt=tri))
    pats = []
    for _ in range(64):
        n = rng.randint(4, 6)
        pats.append((n, random_connected(n, rng.uniform(0.4, 1.0), rng)))
    # End to end first, while no plan of these patterns is kept yet: the
    # engine's path (learned selection, one batched launch from a CUDA graph)
    # against the reference's way (analytic plans, one launch per job), each
    # planning every job; graphs are resident for both.
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    ljobs = [(g, gi.Schedule_IEP.learned(gi.Pattern(n, adj), g)) for g in graphs for n, adj in pats]
    lcounts, _, _ = gi.Batch(ljobs).run()
    e2e_learned_batched = time.perf_counter() - t0
    t0 = time.perf_counter()
    jobs, pcounts = [], []
    for g in graphs:
        for n, adj in pats:
            s = gi.Schedule_IEP(gi.Pattern(n, adj), g.v_cnt, g.e_cnt, g.tri_cnt)
            jobs.append((g, s))
            pcounts.append(gi.pattern_matching(g, s).count)
    e2e_analytic_single = time.perf_counter() - t0
    assert lcounts == pcounts
    batch = gi.Batch(jobs)
    for _ in range(max(1, args.warmup)):
        counts, _, _ = batch.run()
    times, lat = [], []
    for _ in range(args.steps):
        c2, ms, kms = batch.run()
        assert c2 == counts
        times.append(kms)
        lat = ms
    # One launch per job, timed on the device per job.
    single, single_counts = [], []
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    for g, s in jobs:
        gi.pattern_matching(g, s)  # warm
    torch.cuda.synchronize()
    t_all0 = time.perf_counter()
    for g, s in jobs:
        ev0.record()
        r = gi.pattern_matching(g, s)
        ev1.record()
        ev1.synchronize()
        single.append(ev0.elapsed_time(ev1))
        single_counts.append(r.count)
    t_all = time.perf_counter() - t_all0
    assert single_counts == counts
    batch_ms = statistics.median(times)
    lat_sorted = sorted(lat)
    pct = lambda xs, q: xs[min(len(xs) - 1, int(q * len(xs)))]  # noqa: E731
    return {"metric": "batched pattern-count jobs/s, 1 B200", "value": len(jobs) / (batch_ms / 1e3),
            "unit": "jobs/s", "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": batch_ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u32 ids / u64 counts",
            "data": "synthetic (seeded R-MAT graphs, seeded random patterns)",
            "config": {"workload": f"{len(pats)} random connected patterns of 4-6 vertices x {len(graphs)} R-MAT "
                                   f"graphs (scales 10-12) = {len(jobs)} jobs, one launch from a CUDA graph",
                       "job_latency_ms_p50": pct(lat_sorted, 0.5), "job_latency_ms_p99": pct(lat_sorted, 0.99),
                       "one_launch_per_job": {"jobs_per_s_device": len(jobs) / (sum(single) / 1e3),
                                              "jobs_per_s_wall": len(jobs) / t_all,
                                              "job_ms_p50": pct(sorted(single), 0.5),
                                              "job_ms_p99": pct(sorted(single), 0.99)},
                       "end_to_end_s": {"learned_plans_one_batch": e2e_learned_batched,
                                        "analytic_plans_one_launch_per_job": e2e_analytic_single,
                                        "speedup": e2e_analytic_single / max(e2e_learned_batched, 1e-9)}}}


def main():
    args = parse_args()
    if args.workload == "batch":
        print(json.dumps(run_batch(args)), flush=True)
        return
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        if rank == 0:
            print(json.dumps(run_reference(args, world)), flush=True)
        return
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=900))
    line, g, plans, divisors, tri = run_ours(args, world, rank, local)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        v, sample, kind = cpu_baseline_job(g, tri, plan_descs(plans), divisors, os.cpu_count() or 1,
                                           args.cpu_target_s)
        line["cpu_baseline"] = {"value": v, "unit": "embeddings/s", "cores": os.cpu_count() or 1, "kind": kind,
                                "sample": sample}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
