"""Replica plumbing for runs on several GPUs of one node (one process per GPU).

The solve does not exchange data between GPUs: each rank owns whole problems (a replica of the
benchmark solve, or its share of the serving requests). What ranks share is host bookkeeping:
which requests a rank serves, the slowest rank's device time (the job's time), and the per-request
records for latency percentiles. These helpers work with any torch.distributed backend (nccl on
GPUs, gloo on CPU) and degrade to the single-process case when no process group is initialised.
"""

from __future__ import annotations

import torch


def _dist():
    import torch.distributed as dist

    return dist if dist.is_available() and dist.is_initialized() else None


def rank_world() -> tuple[int, int]:
    d = _dist()
    return (d.get_rank(), d.get_world_size()) if d else (0, 1)


def shard_requests(requests, rank: int, world: int):
    """Requests dealt round-robin by request id: rank r serves ids with id % world == r."""
    return [r for r in requests if r.rid % world == rank]


def max_over_ranks(value: float, device: torch.device | str = "cpu") -> float:
    """The largest value over all ranks (device times: the slowest rank sets the job's time)."""
    d = _dist()
    if d is None:
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    d.all_reduce(t, op=d.ReduceOp.MAX)
    return float(t.item())


def gather_records(records: list) -> list:
    """Every rank's list of picklable records, concatenated in rank order (on every rank)."""
    d = _dist()
    if d is None:
        return list(records)
    out = [None] * d.get_world_size()
    d.all_gather_object(out, list(records))
    return [x for part in out for x in part]


def serving_totals(records: list, arrivals_start: float = 0.0) -> dict:
    """Job-level serving numbers from (rid, nrhs, latency, finished, error) records of all ranks."""
    import numpy as np

    ok = [t for t in records if t[4] is None]
    makespan = max((t[3] for t in records), default=0.0) - arrivals_start
    rhs = sum(t[1] for t in ok)
    lat = np.array([t[2] for t in ok]) if ok else np.zeros(1)
    return {
        "completed": len(ok),
        "failed": len(records) - len(ok),
        "rhs_solves": rhs,
        "makespan_s": makespan,
        "solves_per_s": rhs / makespan if makespan > 0 else 0.0,
        "latency_p50_s": float(np.percentile(lat, 50)),
        "latency_p99_s": float(np.percentile(lat, 99)),
    }
