"""Multi-GPU execution of a batch: one process per GPU, instances sharded.

The instances of a batch are independent domains (the reference advances
one, src/main.cpp:718-1164), so a batch spread over several GPUs needs no
exchange on the data path: rank r builds one handle over its own shard of
the instances and steps it.  Collectives appear only around the timed
region -- a barrier before and after, and the maximum of the ranks' device
times -- and when results are gathered on one rank.

``shard`` balances node counts greedily (largest instance first onto the
least loaded rank); ``job_time_ms`` is the max over ranks of each rank's
CUDA-event time; ``gather_by_instance`` collects per-instance results in
instance order.  All three work on any torch.distributed backend (NCCL on
the GPUs, gloo in the CPU tests).
"""
from __future__ import annotations

from typing import Any, Sequence


def shard(sizes: Sequence[int], world: int) -> list[list[int]]:
    """Instance indices per rank: each instance on exactly one rank, node
    counts balanced (longest-processing-time greedy), indices ascending
    within a rank.  Ranks may get no instance when world > len(sizes)."""
    if world < 1:
        raise ValueError("world must be >= 1")
    load = [0] * world
    parts: list[list[int]] = [[] for _ in range(world)]
    for i in sorted(range(len(sizes)), key=lambda k: (-int(sizes[k]), k)):
        r = min(range(world), key=lambda q: (load[q], q))
        parts[r].append(i)
        load[r] += int(sizes[i])
    return [sorted(p) for p in parts]


def job_time_ms(local_ms: float, group=None, device=None) -> float:
    """The job's time: the maximum of the ranks' own measured times."""
    import torch
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size(group) == 1:
        return float(local_ms)
    t = torch.tensor([float(local_ms)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())


def gather_by_instance(local: dict[int, Any], n_instances: int, group=None) -> list[Any] | None:
    """Per-instance results from every rank, in instance order, on rank 0
    (None on the other ranks).  Each instance must come from one rank."""
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized() or dist.get_world_size(group) == 1:
        return [local[i] for i in range(n_instances)]
    parts = [None] * dist.get_world_size(group)
    dist.all_gather_object(parts, local, group=group)
    if dist.get_rank(group) != 0:
        return None
    out: list[Any] = [None] * n_instances
    seen = set()
    for p in parts:
        for i, v in p.items():
            if i in seen:
                raise ValueError(f"instance {i} reported by two ranks")
            seen.add(i)
            out[i] = v
    if len(seen) != n_instances:
        raise ValueError(f"{n_instances - len(seen)} instances missing")
    return out


def run_shard(sets, n_steps: int, rank: int, world: int, device: int = 0, diag_every: int = 0,
              **solver_opts) -> dict[int, dict]:
    """Runs this rank's shard of ``sets`` for n_steps on ``device`` in one
    handle; returns {instance: {"u": ..., "diag": ...}} for its instances."""
    from .api import Solver
    mine = shard([s.n_nodes for s in sets], world)[rank]
    if not mine:
        return {}
    out: dict[int, dict] = {}
    with Solver([sets[i] for i in mine], device=device, **solver_opts) as sv:
        sv.step(n_steps, diag_every=diag_every)
        for k, i in enumerate(mine):
            out[i] = {"u": sv.download(k)["u"], "diag": sv.read_diag(k) if diag_every else None}
    return out
