"""Multi-rank host logic on CPU (gloo, world size 2): request sharding, the slowest rank's time as
the job's time, and job-level serving totals gathered from every rank."""

from __future__ import annotations

import json
import os
import socket
import time

import numpy as np
import torch.distributed as dist
import torch.multiprocessing as mp

from yasf_b200.replicas import gather_records, max_over_ranks, rank_world, serving_totals, shard_requests
from yasf_b200.serve import RequestResult, ServeConfig, Server
from yasf_b200.workloads import Aggregate, Request


def _free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _req(rid, arrival, R):
    agg = Aggregate(f"r{rid}", np.zeros((5, 3)), np.full(5, 0.1), 1.5 + 0j, 0.5, 3, rid)
    return Request(rid, arrival, agg, np.zeros(R), np.zeros(R), np.ones(R, dtype=int))


def _fake_solve(req, cfg, device):
    time.sleep(0.01 * (1 + req.rid % 3))
    agg = req.aggregate
    if req.rid == 7:
        raise RuntimeError("solver did not converge")
    return RequestResult(req.rid, agg.n, agg.lmax, len(req.pol), c_ext=np.ones(len(req.pol)))


def _worker(rank, world, port, out_dir):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        assert rank_world() == (rank, world)
        reqs = [_req(i, 0.005 * i, R=1 + i % 4) for i in range(10)]
        mine = shard_requests(reqs, rank, world)
        assert all(r.rid % world == rank for r in mine)
        t = max_over_ranks(10.0 * (rank + 1))
        srv = Server(ServeConfig(max_slots=2, hbm_budget_bytes=10**9), device="cpu", solve_fn=_fake_solve,
                     footprint_fn=lambda r, c: 1)
        res = srv.run(mine, realtime=True)
        recs = gather_records([(r.rid, r.nrhs, r.latency, r.finished, r.error) for r in res])
        tot = serving_totals(recs, 0.0)
        with open(os.path.join(out_dir, f"rank{rank}.json"), "w") as f:
            json.dump({"t": t, "rids": sorted(r[0] for r in recs), "tot": tot,
                       "mine": [r.rid for r in mine]}, f)
        dist.barrier()
    finally:
        dist.destroy_process_group()


def test_two_rank_serving_and_timing(tmp_path):
    world = 2
    mp.spawn(_worker, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True)
    outs = [json.loads((tmp_path / f"rank{r}.json").read_text()) for r in range(world)]
    for o in outs:
        assert o["t"] == 10.0 * world                      # the slowest rank's time on every rank
        assert o["rids"] == list(range(10))                # every request, each exactly once
        assert o["tot"]["failed"] == 1 and o["tot"]["completed"] == 9
        assert o["tot"]["rhs_solves"] == sum(1 + i % 4 for i in range(10) if i != 7)
        assert o["tot"]["latency_p99_s"] >= o["tot"]["latency_p50_s"] > 0
    assert sorted(outs[0]["mine"] + outs[1]["mine"]) == list(range(10))
    assert not set(outs[0]["mine"]) & set(outs[1]["mine"])


def test_single_process_fallbacks():
    assert rank_world() == (0, 1)
    assert max_over_ranks(3.5) == 3.5
    assert gather_records([1, 2]) == [1, 2]
