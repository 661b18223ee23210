"""Counts across the ranks of a torch.distributed process group, one GPU per
rank (reference gpu/gpu_graph_static_task.cu, gpu/gpu_graph_mpi.cu).

``count``: every rank holds a replica of the graph on its own GPU and counts
its shard of the first-level work with ``gi_count_shard`` (chunk c belongs to shard
c mod world, the reference's static interleave,
gpu/src/gpu_pattern_matching_static_task.cuh:63).  The only exchange is one
all-reduce of the raw sums, added modulo 2^64 as the reference's GPU sum is;
the total is divided by the plan's count divisor once, as a single-GPU count
divides its whole sum (reference gpu/gpu_graph.cu:42-44).

``batch_counts``: many (graph, pattern) jobs are spread over the ranks by
their analytic cost; each rank counts its own jobs in one batched launch and
one all-reduce of the per-job counts gives every rank all of them.
"""
from __future__ import annotations

import ctypes as C
from typing import Callable, Optional, Sequence

from . import _native as N
from ._native import check, lib

MASK64 = (1 << 64) - 1


def shard_raw_sum(graph, schedule, rank: int, world: int, stream: int = 0) -> int:
    """Raw sum (before the division, modulo 2^64) of this rank's shard."""
    raw = C.c_uint64()
    check(lib().gi_count_shard(graph.handle, schedule.handle, rank, world, C.c_void_p(stream) if stream else None,
                               C.byref(raw), None), "gi_count_shard")
    return raw.value


def allreduce_u64(values: Sequence[int], group=None) -> list[int]:
    """Element-wise sum modulo 2^64 over the group's ranks.  Each value
    travels as two 32-bit halves in int64 lanes so that no backend ever adds
    past the int64 range (exact for up to 2^31 ranks)."""
    import torch
    import torch.distributed as dist

    backend = dist.get_backend(group)
    device = torch.device("cuda", torch.cuda.current_device()) if backend == "nccl" else torch.device("cpu")
    halves = []
    for v in values:
        v &= MASK64
        halves += [v & 0xFFFFFFFF, v >> 32]
    t = torch.tensor(halves, dtype=torch.int64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.SUM, group=group)
    h = t.tolist()
    return [((h[2 * i + 1] << 32) + h[2 * i]) & MASK64 for i in range(len(values))]


def count(graph, schedule, group=None, *, stream: int = 0,
          shard_fn: Optional[Callable[[int, int], int]] = None) -> int:
    """The whole count of the schedule's pattern, every rank returning it.
    ``shard_fn(rank, world) -> raw sum`` replaces the GPU shard count (a CPU
    stand-in lets the exchange run on hosts without GPUs)."""
    import torch.distributed as dist

    rank, world = dist.get_rank(group), dist.get_world_size(group)
    raw = shard_fn(rank, world) if shard_fn else shard_raw_sum(graph, schedule, rank, world, stream)
    total = allreduce_u64([raw], group)[0]
    return total // divisor(schedule)


def divisor(schedule) -> int:
    """The plan's count divisor (redundancy, or the exact multiplicity)."""
    d = N.PlanDesc()
    check(lib().gi_plan_export(schedule.handle, C.byref(d)), "gi_plan_export")
    return int(d.count_divisor)


def assign_jobs(costs: Sequence[float], world: int) -> list[int]:
    """Owner rank of each job: longest first onto the least-loaded rank
    (ties to the lower job index and the lower rank), so every rank computes
    the same assignment from the same costs."""
    if world < 1:
        raise ValueError("world must be >= 1")
    order = sorted(range(len(costs)), key=lambda j: (-float(costs[j]), j))
    load = [0.0] * world
    owner = [0] * len(costs)
    for j in order:
        r = min(range(world), key=lambda x: (load[x], x))
        owner[j] = r
        load[r] += max(float(costs[j]), 0.0)
    return owner


def batch_counts(jobs: Sequence, group=None, *, costs: Optional[Sequence[float]] = None,
                 runner: Optional[Callable[[list], Sequence[int]]] = None) -> list[int]:
    """Counts of many (graph, schedule) jobs spread over the group's ranks,
    one GPU each.  Every rank passes the same job list (its own graph
    handles, on its own GPU), runs the jobs ``assign_jobs`` gives it as one
    batch (``graphindor_b200.Batch``), and one all-reduce of the counts (0
    where another rank owns the job) hands every rank all of them.  ``costs``
    orders the assignment (default: each schedule's analytic model cost);
    ``runner(local_jobs) -> counts`` replaces the batch (a CPU stand-in lets
    the exchange run on hosts without GPUs)."""
    import torch.distributed as dist

    rank, world = dist.get_rank(group), dist.get_world_size(group)
    if costs is None:
        costs = [s.export()["model_cost"] for _, s in jobs]
    if len(costs) != len(jobs):
        raise ValueError("one cost per job")
    owner = assign_jobs(costs, world)
    mine = [j for j in range(len(jobs)) if owner[j] == rank]
    local: Sequence[int] = []
    if mine:
        local_jobs = [jobs[j] for j in mine]
        if runner is not None:
            local = runner(local_jobs)
        else:
            from . import Batch
            local = Batch(local_jobs).run()[0]
        if len(local) != len(mine):
            raise RuntimeError("the runner returned the wrong number of counts")
    values = [0] * len(jobs)
    for j, c in zip(mine, local):
        values[j] = int(c)
    return allreduce_u64(values, group)
