"""The serving loop's admission logic on the host (no GPU): arrivals, slot limit, HBM budget,
rejection of requests that can never fit, latency accounting. The solve is a stand-in that only
records concurrency; the device solve itself is covered by tests/test_gpu_serve.py."""

from __future__ import annotations

import threading
import time

import numpy as np

from yasf_b200.serve import RequestResult, ServeConfig, Server, inner_kind, summarize
from yasf_b200.workloads import Aggregate, Request


def _req(rid, arrival, n=10, lmax=3, R=1):
    agg = Aggregate(f"r{rid}", np.zeros((n, 3)), np.full(n, 0.1), 1.5 + 0j, 0.5, lmax, rid)
    return Request(rid, arrival, agg, np.zeros(R), np.zeros(R), np.ones(R, dtype=int))


class Recorder:
    def __init__(self, dt=0.05):
        self.dt = dt
        self.active = 0
        self.peak = 0
        self.lock = threading.Lock()
        self.order = []

    def __call__(self, req, cfg, device):
        with self.lock:
            self.active += 1
            self.peak = max(self.peak, self.active)
            self.order.append(req.rid)
        time.sleep(self.dt)
        with self.lock:
            self.active -= 1
        agg = req.aggregate
        return RequestResult(req.rid, agg.n, agg.lmax, len(req.pol), c_ext=np.zeros(len(req.pol)))


def test_slots_and_arrivals():
    rec = Recorder()
    reqs = [_req(i, 0.02 * i) for i in range(8)]
    srv = Server(ServeConfig(max_slots=3, hbm_budget_bytes=10**12), device="cpu", solve_fn=rec,
                 footprint_fn=lambda r, c: 1)
    res = srv.run(reqs)
    assert [r.rid for r in res] == list(range(8))
    assert rec.peak <= 3 and rec.peak >= 2
    for r in res:
        assert r.error is None
        assert r.finished >= r.arrival + rec.dt * 0.9  # latency counts from arrival
    s = summarize(res)
    assert s["completed"] == 8 and s["rhs_solves"] == 8 and s["latency_p99_s"] >= s["latency_p50_s"]


def test_memory_budget_limits_concurrency():
    rec = Recorder(dt=0.03)
    reqs = [_req(i, 0.0) for i in range(6)]
    srv = Server(ServeConfig(max_slots=6, hbm_budget_bytes=100), device="cpu", solve_fn=rec,
                 footprint_fn=lambda r, c: 45)  # only two fit at a time
    srv.run(reqs)
    assert rec.peak == 2


def test_request_larger_than_budget_is_rejected():
    rec = Recorder(dt=0.01)
    reqs = [_req(0, 0.0), _req(1, 0.0, n=99), _req(2, 0.01)]
    srv = Server(ServeConfig(max_slots=2, hbm_budget_bytes=100), device="cpu", solve_fn=rec,
                 footprint_fn=lambda r, c: 1000 if r.aggregate.n == 99 else 10)
    res = srv.run(reqs)
    assert res[1].error is not None and "budget" in res[1].error
    assert res[0].error is None and res[2].error is None
    assert 1 not in rec.order


def test_failed_request_does_not_stop_the_loop():
    def solve(req, cfg, device):
        if req.rid == 1:
            raise FloatingPointError("non-finite right-hand side")
        return Recorder(0.0)(req, cfg, device)

    srv = Server(ServeConfig(max_slots=2, hbm_budget_bytes=10**9), device="cpu", solve_fn=solve,
                 footprint_fn=lambda r, c: 1)
    res = srv.run([_req(i, 0.0) for i in range(3)], realtime=False)
    assert res[1].error.startswith("FloatingPointError")
    assert res[0].error is None and res[2].error is None


def test_inner_kind_rule():
    assert [inner_kind(6, r) for r in (1, 2, 3, 64)] == ["c64", "c64", "tf32", "tf32"]
    assert [inner_kind(7, r) for r in (4, 5)] == ["c64", "tf32"]
    assert [inner_kind(8, r) for r in (3, 4, 64)] == ["c64", "tf32", "tf32"]


def test_admission_never_exceeds_the_budget():
    """Random footprints and durations: at every moment the footprints of the requests in flight
    sum to at most the budget, and every request that fits alone is served."""
    rng = np.random.default_rng(4)
    budget = 1000
    fp = {i: int(rng.integers(50, 600)) for i in range(40)}
    lock = threading.Lock()
    state = {"used": 0, "peak": 0}

    def solve(req, cfg, device):
        with lock:
            state["used"] += fp[req.rid]
            state["peak"] = max(state["peak"], state["used"])
            assert state["used"] <= budget
        time.sleep(float(rng.uniform(0.0, 0.01)))
        with lock:
            state["used"] -= fp[req.rid]
        agg = req.aggregate
        return RequestResult(req.rid, agg.n, agg.lmax, len(req.pol), c_ext=np.zeros(len(req.pol)))

    reqs = [_req(i, 0.001 * i) for i in range(40)]
    srv = Server(ServeConfig(max_slots=8, hbm_budget_bytes=budget), device="cpu", solve_fn=solve,
                 footprint_fn=lambda r, c: fp[r.rid])
    res = srv.run(reqs)
    assert all(r.error is None for r in res)
    assert state["peak"] <= budget and state["peak"] > 600  # several in flight at once


def test_cycle_length_by_columns():
    """Requests with few columns get long GMRES cycles (their basis is cheap), wide ones the base
    cycle; the admission footprint is sized with the same cycle length."""
    cfg = ServeConfig()
    assert [cfg.restart_for(R) for R in (1, 2, 4, 5, 16, 17, 64)] == [100, 100, 100, 60, 60, 30, 30]
    cfg = ServeConfig(restart=40, restart_few=())
    assert cfg.restart_for(1) == 40


def test_unconverged_request_is_an_error():
    """A stand-in solve that reports unconverged columns is not counted as completed."""

    def solve(req, cfg, device):
        agg = req.aggregate
        r = RequestResult(req.rid, agg.n, agg.lmax, len(req.pol), c_ext=np.zeros(len(req.pol)))
        if req.rid == 1:
            r.error = "not converged: 1 of 1 columns"
        return r

    srv = Server(ServeConfig(max_slots=2, hbm_budget_bytes=100), device="cpu", solve_fn=solve,
                 footprint_fn=lambda r, c: 1)
    out = srv.run([_req(0, 0.0), _req(1, 0.0), _req(2, 0.0)], realtime=False)
    s = summarize(out)
    assert s["completed"] == 2 and s["failed"] == 1 and s["rhs_solves"] == 2
