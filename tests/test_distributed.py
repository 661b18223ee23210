"""The multi-rank path on CPU: world-size-2 gloo process groups run the
exchanges of graphindor_b200.distributed with the oracle standing in for each
rank's GPU work (vertex-strided shards of one count; the jobs of a batch),
and check the results against single-process counts; the modulo-2^64
reduction; the job assignment; and a rank that fails before the exchange."""
from __future__ import annotations

import datetime
import os
import socket
import sys
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _init(rank, world, port, timeout_s=30):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=timeout_s))


def _count_worker(rank, world, port, q):
    sys.path[:0] = [str(ROOT), str(ROOT / "oracle"), str(ROOT / "tests")]
    try:
        import torch.distributed as dist
        import graphindor_b200 as gi
        from graphindor_b200 import distributed as gd, gen
        import oracle_py
        from conftest import plan_desc
        _init(rank, world, port)
        g = gen.rmat(10, 12.0, 12)
        out = {}
        for n, adj in [(4, "0110100110010110"), (5, "0101110101010101010011000"), (4, "0111101111001100")]:
            s = gi.Schedule_IEP(gi.Pattern(n, adj), g.v_cnt, g.e_cnt, 0)
            desc = plan_desc(s)

            def shard(r, w):
                return oracle_py.count_strided(desc, g.vertex, g.edge, w, v_begin=r)
            out[adj] = gd.count(None, s, shard_fn=shard)
        wrap = gd.allreduce_u64([(1 << 64) - 1 - rank, (1 << 63) + rank, 5])
        dist.destroy_process_group()
        q.put((rank, out, wrap))
    except Exception as e:  # reported to the parent
        q.put((rank, "error", repr(e)))


def _batch_worker(rank, world, port, q):
    sys.path[:0] = [str(ROOT), str(ROOT / "oracle"), str(ROOT / "tests")]
    try:
        import torch.distributed as dist
        import graphindor_b200 as gi
        from graphindor_b200 import distributed as gd, gen
        import oracle_py
        from conftest import plan_desc
        _init(rank, world, port)
        jobs = _batch_jobs(gi, gen)
        ran = []

        def runner(local):
            ran.extend(id(j) for j in local)
            return [oracle_py.count(plan_desc(s), g.vertex, g.edge)[0] // plan_desc(s).count_divisor
                    for g, s in local]
        counts = gd.batch_counts(jobs, runner=runner)
        mine = sorted(i for i, j in enumerate(jobs) if id(j) in ran)
        dist.destroy_process_group()
        q.put((rank, counts, mine))
    except Exception as e:  # reported to the parent
        q.put((rank, "error", repr(e)))


def _batch_jobs(gi, gen):
    graphs = [gen.rmat(9, 8.0, 21), gen.rmat(10, 6.0, 22), gen.erdos_renyi(600, 5000, 23)]
    pats = [(3, "011101110"), (4, "0110100110010110"), (4, "0111101111001100"), (5, "0101110101010101010011000")]
    return [(g, gi.Schedule_IEP(gi.Pattern(n, a), g.v_cnt, g.e_cnt, 0)) for g in graphs for n, a in pats]


def test_batch_jobs_spread_over_two_ranks(oracle, native):
    """Each rank counts only the jobs assigned to it, the two sets cover all
    jobs once, and both ranks end with every job's count."""
    import graphindor_b200 as gi
    from graphindor_b200 import gen
    from conftest import plan_desc
    res = _run(_batch_worker)
    jobs = _batch_jobs(gi, gen)
    want = [oracle.count(plan_desc(s), g.vertex, g.edge)[0] // plan_desc(s).count_divisor for g, s in jobs]
    for rank, counts, mine in res:
        assert counts != "error", mine
        assert counts == want
    assert sorted(res[0][2] + res[1][2]) == list(range(len(jobs)))
    assert res[0][2] and res[1][2]


def test_job_assignment_is_balanced_and_deterministic():
    from graphindor_b200.distributed import assign_jobs
    costs = [9.0, 1.0, 8.0, 2.0, 7.0, 3.0, 6.0, 4.0, 5.0, 0.0]
    owner = assign_jobs(costs, 3)
    assert owner == assign_jobs(list(costs), 3)
    load = [sum(c for c, o in zip(costs, owner) if o == r) for r in range(3)]
    assert max(load) - min(load) <= max(costs)
    assert assign_jobs(costs, 1) == [0] * len(costs)
    assert assign_jobs([], 4) == []
    with pytest.raises(ValueError):
        assign_jobs(costs, 0)


def _fail_worker(rank, world, port, q):
    sys.path[:0] = [str(ROOT)]
    try:
        from graphindor_b200 import distributed as gd
        _init(rank, world, port, timeout_s=5)
        if rank == 1:
            raise RuntimeError("rank 1 fails before the exchange")
        gd.allreduce_u64([1])
        q.put((rank, "no error"))
    except Exception as e:
        q.put((rank, type(e).__name__))


def _run(target, world=2, timeout=240):
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=target, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    res = [q.get(timeout=timeout) for _ in range(world)]
    for p in procs:
        p.join(timeout=60)
        if p.is_alive():
            p.kill()
    return sorted(res, key=lambda r: r[0])


def test_two_ranks_add_up_to_the_whole_count(oracle, native):
    import graphindor_b200 as gi
    from graphindor_b200 import gen
    from conftest import plan_desc
    res = _run(_count_worker)
    g = gen.rmat(10, 12.0, 12)
    for rank, out, wrap in res:
        assert out != "error", wrap
        for adj, got in out.items():
            n = int(round(len(adj) ** 0.5))
            s = gi.Schedule_IEP(gi.Pattern(n, adj), g.v_cnt, g.e_cnt, 0)
            d = plan_desc(s)
            raw, _ = oracle.count(d, g.vertex, g.edge)
            assert got == raw // d.count_divisor, adj
        # (2^64 - 1) + (2^64 - 2), (2^63) + (2^63 + 1), 5 + 5, all modulo 2^64
        assert wrap == [(1 << 64) - 3, 1, 10]


def test_a_rank_that_fails_before_the_exchange_ends_the_others_with_an_error():
    res = _run(_fail_worker, timeout=120)
    assert res[1][1] == "RuntimeError"
    assert res[0][1] != "no error"
