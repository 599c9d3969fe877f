"""Serving: a continuous-batching request loop for T-matrix solves of different sizes.

Each request carries an aggregate (spheres, refractive index, wavelength, lmax) and a set of
incidences (directions x polarisations = R right-hand sides). The loop:

- admits a request once its arrival time has passed, a slot is free and its device footprint
  (the library's own workspace query for its batched solve, plus its vectors) fits in the HBM
  budget that the requests in flight leave; a request that can never fit is rejected with an error;
- runs every admitted request on its own CUDA stream, so the kernels of in-flight solves
  interleave on the device while their GMRES state stays resident there;
- solves in mixed precision: the batched refined solve (yasf_batched_solve) with the tensor-core
  TF32 panel as the inner operator (complex64 coupling kernel for one or two columns; with
  ``ServeConfig.tuner`` set, whichever of the two the autotuner measured cheaper for the request's
  (lmax, N, R)), float64 residuals, stopping at rtol (1e-6 by default, which keeps the extinction
  cross section well inside 1e-6 of the float64 solution); GMRES cycles of 100 steps for up to 4
  columns, 60 up to 16, 30 beyond (``ServeConfig.restart_for``); a request whose columns do not
  reach rtol within max_refine cycles is reported as an error, not as a completed solve;
- packs the small requests whose inner operator is the complex64 kernel (up to
  ``group_max_spheres`` spheres) that have arrived, with the same lmax, into one grouped solve
  (yasf_grouped_solve): every operator application of the group is one persistent work-queue
  contraction for all of them, instead of a launch sequence per request; a group is admitted by
  the grouped solve's own size query (yasf_grouped_workspace_size) plus its requests' vectors;
- reports per-request latency (completion - arrival, queueing included), p50/p99 and solves/s.

The kernels are deterministic (no atomics in any reduction), so a request's result does not depend
on what else is in flight: ``solve_request`` alone and inside the loop give the same numbers.
"""

from __future__ import annotations

import threading
import time
from collections import deque
from concurrent.futures import FIRST_COMPLETED, ThreadPoolExecutor, wait
from dataclasses import dataclass, field

import numpy as np
import torch

from yasf_b200._lib import call
from yasf_b200.device import CouplingDevice
from yasf_b200.mie import mie_tmatrix_per_sphere
from yasf_b200.numerics import cached_translation_table
from yasf_b200.workloads import Request


@dataclass
class ServeConfig:
    max_slots: int = 4
    hbm_budget_bytes: int | None = None   # default: 80 % of the free device memory at start
    rtol: float = 1e-6
    restart: int = 30                     # GMRES cycle length of requests with many columns
    restart_few: tuple = ((4, 100), (16, 60))  # (up to R columns, cycle length): longer cycles
    max_refine: int = 8
    inner_rtol: float = 1e-3

    def restart_for(self, nrhs: int) -> int:
        """GMRES cycle length of a request with nrhs columns. Unpreconditioned restarted GMRES
        stagnates on dense aggregates with short cycles; a long cycle costs R (restart + 1) vectors
        of basis, cheap for a few columns, so requests with few columns get the longer cycles."""
        for cols, restart in self.restart_few:
            if nrhs <= cols:
                return int(restart)
        return int(self.restart)
    keep_solutions: bool = False
    tuner: object | None = None           # an autotune.Autotuner: inner operator by measurement
    group_small: bool = True              # small complex64-inner requests share one grouped solve
    group_max_spheres: int = 600          # a request joins a group up to this many spheres
    group_max_requests: int = 16          # requests per group


@dataclass
class RequestResult:
    rid: int
    n_spheres: int
    lmax: int
    nrhs: int
    c_ext: np.ndarray | None = None
    stats: dict = field(default_factory=dict)
    arrival: float = 0.0
    admitted: float = 0.0
    finished: float = 0.0
    error: str | None = None
    x: np.ndarray | None = None

    @property
    def latency(self) -> float:
        return self.finished - self.arrival


# Columns from which one TF32 panel step is cheaper than complex64 column applications: one panel
# step at 1000 spheres costs 1.7 (lmax 6), 4.9 (lmax 7) and 3.1 (lmax 8) complex64 columns (both
# grow like N^2, so the ratio holds across sizes).
_PANEL_MIN_COLUMNS = {7: 5, 8: 4}


def inner_kind(lmax: int, nrhs: int) -> str:
    """Inner operator of a request's refined solve: the TF32 tensor-core panel once the request has
    enough columns to amortise one panel step (3 up to lmax 6, 5 at lmax 7, 4 at lmax 8), else the
    complex64 coupling kernel column by column."""
    return "tf32" if lmax <= 8 and nrhs >= _PANEL_MIN_COLUMNS.get(lmax, 3) else "c64"


def footprint_bytes(req: Request, cfg: ServeConfig, device: torch.device | None = None) -> int:
    """Device bytes a request holds while in flight, from the library's own size query.

    The workspace of its refined batched solve is what ``yasf_batched_workspace_size`` returns for
    the request's plan, sphere count, columns and restart length, taking the larger of the two inner
    operators (TF32 panel, complex64 columns) when the autotuner may choose either; then its device
    vectors: T (n), the incident coefficients, the right-hand sides and the solution (R n each,
    complex128), the positions, the incidences' mode factors and wave vectors. Each allocation is
    rounded up to the caching allocator's 2 MiB granularity. The translation plan is shared by every
    request of the same lmax and not counted here."""
    import ctypes

    from yasf_b200.device import Plan

    agg = req.aggregate
    nmax = 2 * agg.lmax * (agg.lmax + 2)
    n = agg.n * nmax
    R = len(req.pol)
    restart = int(max(1, min(cfg.restart_for(R), 512, n)))
    device = device if device is not None else torch.device("cuda", torch.cuda.current_device())
    plan = Plan.get(agg.lmax, cached_translation_table(agg.lmax), device)
    kinds = ("tf32", "c64") if cfg.tuner is not None else (inner_kind(agg.lmax, R),)
    ws = 0
    for kind in kinds:
        nb = ctypes.c_size_t()
        call("yasf_batched_workspace_size", plan.handle, agg.n, R, restart,
             CouplingDevice.INNER_KINDS[kind], ctypes.byref(nb))
        ws = max(ws, nb.value)
    return _rounded(ws) + _vector_bytes(req)


_GRAN = 2 << 20  # the caching allocator's block granularity


def _rounded(b: int) -> int:
    return (int(b) + _GRAN - 1) // _GRAN * _GRAN


def _vector_bytes(req: Request) -> int:
    """A request's device vectors besides the solve's workspace: T (n), the incident coefficients,
    right-hand sides and solution (R n each, complex128), positions, mode factors, wave vectors."""
    agg = req.aggregate
    nmax = 2 * agg.lmax * (agg.lmax + 2)
    n = agg.n * nmax
    R = len(req.pol)
    return (_rounded(n * 16) + 3 * _rounded(R * n * 16) + _rounded(agg.n * 24) + _rounded(R * nmax * 16)
            + _rounded(R * 24) + _rounded(R * 16) + _rounded(256))


def group_restart(reqs: list[Request], cfg: ServeConfig) -> int:
    return min(cfg.restart_for(max(len(r.pol) for r in reqs)), 512)


def group_footprint_bytes(reqs: list[Request], cfg: ServeConfig, device: torch.device | None = None) -> int:
    """Device bytes a grouped solve of `reqs` holds: the library's yasf_grouped_workspace_size for
    the group (which reads only the sphere and column counts), plus every request's vectors."""
    import ctypes

    from yasf_b200 import _lib
    from yasf_b200.device import Plan

    lmax = reqs[0].aggregate.lmax
    device = device if device is not None else torch.device("cuda", torch.cuda.current_device())
    plan = Plan.get(lmax, cached_translation_table(lmax), device)
    probs = (_lib.YasfProblem * len(reqs))()
    for i, req in enumerate(reqs):
        probs[i] = _lib.YasfProblem(req.aggregate.n, None, req.aggregate.k, None, None, None, len(req.pol))
    nb = ctypes.c_size_t()
    call("yasf_grouped_workspace_size", plan.handle, len(reqs), probs, group_restart(reqs, cfg), ctypes.byref(nb))
    return _rounded(nb.value) + sum(_vector_bytes(r) for r in reqs)


def solve_request(req: Request, cfg: ServeConfig, device: torch.device) -> RequestResult:
    """One request, start to finish, on the current stream of the calling thread."""
    agg = req.aggregate
    R = len(req.pol)
    res = RequestResult(req.rid, agg.n, agg.lmax, R)
    table = cached_translation_table(agg.lmax)
    tm = mie_tmatrix_per_sphere(agg.lmax, agg.k, agg.radii, agg.refractive_index)
    dev = CouplingDevice(agg.lmax, table, agg.positions, agg.k, device)
    tmat = torch.from_numpy(tm).to(device)
    # incident coefficients and right-hand sides of the R incidences, formed on the device
    A, Bt = dev.plane_wave_rhs(tmat, req.polar, req.azimuthal, req.pol)
    decision = cfg.tuner.decide(dev, tmat, R) if cfg.tuner is not None else None
    inner = decision.inner if decision is not None else inner_kind(agg.lmax, R)
    if decision is not None:
        decision.apply_tiles()  # tile shapes for this thread's launches
    try:
        X, st = dev.batched_solve(tmat, Bt, rtol=cfg.rtol, restart=min(cfg.restart_for(R), 512, dev.n),
                                  max_refine=cfg.max_refine, inner_rtol=cfg.inner_rtol, inner=inner)
    finally:
        if decision is not None:
            from yasf_b200._lib import set_tiles

            set_tiles(0, 0, 0)
    res.c_ext = (-torch.real((A.conj() * X).sum(dim=1)) / agg.k**2 * np.pi).cpu().numpy()
    st.pop("column_residuals", None)
    st["inner"] = inner
    st["restart"] = min(cfg.restart_for(R), 512, dev.n)
    if decision is not None:
        st["tiles"] = dict(decision.tiles)
    res.stats = st
    if st.get("unconverged", 0):
        res.error = (f"not converged: {st['unconverged']} of {R} columns, relative residual "
                     f"{st['worst_relative_residual']:.3e} after {st['inner_steps']} inner steps")
    if cfg.keep_solutions:
        res.x = X.cpu().numpy()
    return res


def groupable(req: Request, cfg: ServeConfig) -> bool:
    """A request joins a grouped solve when its inner operator is the complex64 kernel (few
    columns: the tensor-core panel does not pay) and it is small enough that launches, not
    arithmetic, dominate its own solve."""
    agg = req.aggregate
    return (cfg.group_small and cfg.tuner is None and agg.n <= cfg.group_max_spheres
            and inner_kind(agg.lmax, len(req.pol)) == "c64")


def solve_group(reqs: list[Request], cfg: ServeConfig, device: torch.device) -> list[RequestResult]:
    """Several small requests of one lmax in one grouped solve (yasf_grouped_solve): every
    operator application of the group is one persistent work-queue contraction for all of them."""
    from yasf_b200.device import grouped_solve

    items, As, out = [], [], []
    for req in reqs:
        agg = req.aggregate
        tm = mie_tmatrix_per_sphere(agg.lmax, agg.k, agg.radii, agg.refractive_index)
        dev = CouplingDevice(agg.lmax, cached_translation_table(agg.lmax), agg.positions, agg.k, device)
        tmat = torch.from_numpy(tm).to(device)
        A, B = dev.plane_wave_rhs(tmat, req.polar, req.azimuthal, req.pol)
        items.append((dev, tmat, B))
        As.append(A)
    Xs, st = grouped_solve(items, rtol=cfg.rtol, restart=group_restart(reqs, cfg), max_refine=cfg.max_refine,
                           inner_rtol=cfg.inner_rtol, inner="c64")
    colres = st.pop("column_residuals")
    c0 = 0
    for req, A, X in zip(reqs, As, Xs):
        agg = req.aggregate
        R = len(req.pol)
        res = RequestResult(req.rid, agg.n, agg.lmax, R)
        res.c_ext = (-torch.real((A.conj() * X).sum(dim=1)) / agg.k**2 * np.pi).cpu().numpy()
        res.stats = dict(st, inner="c64 grouped", group_size=len(reqs), restart=group_restart(reqs, cfg),
                         worst_relative_residual=max(colres[c0:c0 + R]))
        if max(colres[c0:c0 + R]) > cfg.rtol:
            res.error = f"not converged: relative residual {max(colres[c0:c0 + R]):.3e}"
        if cfg.keep_solutions:
            res.x = X.cpu().numpy()
        out.append(res)
        c0 += R
    return out


class Server:
    """Continuous-batching loop over a request stream on one GPU."""

    def __init__(self, cfg: ServeConfig | None = None, device: torch.device | str | None = None,
                 solve_fn=None, footprint_fn=None):
        self.cfg = cfg or ServeConfig()
        self.device = torch.device(device) if device is not None else torch.device("cuda", torch.cuda.current_device())
        if self.cfg.hbm_budget_bytes is None:
            free, _ = torch.cuda.mem_get_info(self.device)
            self.cfg.hbm_budget_bytes = int(0.8 * free)
        self._solve = solve_fn or solve_request
        self._footprint = footprint_fn or (lambda r, c: footprint_bytes(r, c, self.device))
        self._tls = threading.local()

    def _worker(self, req: Request, t0: float) -> RequestResult:
        if self.device.type != "cuda":  # host-only solve functions (tests of the loop itself)
            try:
                res = self._solve(req, self.cfg, self.device)
            except Exception as e:
                agg = req.aggregate
                res = RequestResult(req.rid, agg.n, agg.lmax, len(req.pol), error=f"{type(e).__name__}: {e}")
            res.finished = time.perf_counter() - t0
            return res
        stream = getattr(self._tls, "stream", None)
        if stream is None:
            stream = torch.cuda.Stream(device=self.device)
            self._tls.stream = stream
        with torch.cuda.device(self.device), torch.cuda.stream(stream):
            try:
                res = self._solve(req, self.cfg, self.device)
            except Exception as e:  # a failed request reports its error, the loop goes on
                agg = req.aggregate
                res = RequestResult(req.rid, agg.n, agg.lmax, len(req.pol), error=f"{type(e).__name__}: {e}")
            stream.synchronize()
        res.finished = time.perf_counter() - t0
        return res

    def _worker_group(self, reqs: list[Request], t0: float) -> list[RequestResult]:
        stream = getattr(self._tls, "stream", None)
        if stream is None:
            stream = torch.cuda.Stream(device=self.device)
            self._tls.stream = stream
        with torch.cuda.device(self.device), torch.cuda.stream(stream):
            try:
                out = solve_group(reqs, self.cfg, self.device)
            except Exception as e:  # the group's requests report the error, the loop goes on
                out = [RequestResult(q.rid, q.aggregate.n, q.aggregate.lmax, len(q.pol),
                                     error=f"{type(e).__name__}: {e}") for q in reqs]
            stream.synchronize()
        fin = time.perf_counter() - t0
        for r in out:
            r.finished = fin
        return out

    def run(self, requests: list[Request], realtime: bool = True) -> list[RequestResult]:
        """Serve the requests (arrival times in seconds from the start); returns results by rid."""
        for lmax in sorted({r.aggregate.lmax for r in requests}):
            cached_translation_table(lmax)  # tables are host setup shared by all requests
        pending = deque(sorted(requests, key=lambda r: r.arrival))
        inflight: dict = {}
        used = 0
        results: list[RequestResult] = []
        budget = self.cfg.hbm_budget_bytes
        t0 = time.perf_counter()
        with ThreadPoolExecutor(max_workers=self.cfg.max_slots) as pool:
            while pending or inflight:
                now = time.perf_counter() - t0
                while pending and (not realtime or pending[0].arrival <= now) and len(inflight) < self.cfg.max_slots:
                    req = pending[0]
                    fp = self._footprint(req, self.cfg)
                    if fp > budget:
                        pending.popleft()
                        agg = req.aggregate
                        r = RequestResult(req.rid, agg.n, agg.lmax, len(req.pol),
                                          error=f"needs {fp} bytes, budget {budget}")
                        r.arrival = req.arrival
                        r.finished = now
                        results.append(r)
                        continue
                    if used + fp > budget:
                        break  # wait for memory to free up
                    pending.popleft()
                    if self.device.type == "cuda" and groupable(req, self.cfg):
                        # gather the arrived small requests of the same lmax into one grouped solve
                        # (admitted by the grouped solve's own size query)
                        group, gfp = [req], fp
                        for other in list(pending):
                            if realtime and other.arrival > now:
                                break
                            if len(group) >= self.cfg.group_max_requests:
                                break
                            if other.aggregate.lmax != req.aggregate.lmax or not groupable(other, self.cfg):
                                continue
                            tfp = group_footprint_bytes(group + [other], self.cfg, self.device)
                            if used + tfp > budget:
                                continue
                            pending.remove(other)
                            group.append(other)
                            gfp = tfp
                        used += gfp
                        fut = pool.submit(self._worker_group, group, t0)
                        inflight[fut] = (group, gfp, now)
                        continue
                    used += fp
                    fut = pool.submit(self._worker, req, t0)
                    inflight[fut] = (req, fp, now)
                if pending and realtime and pending[0].arrival > now:
                    timeout = pending[0].arrival - now
                else:
                    timeout = 0.05
                if not inflight:
                    time.sleep(max(0.0, min(timeout, 0.05)))
                    continue
                done, _ = wait(list(inflight.keys()), timeout=max(0.0, timeout), return_when=FIRST_COMPLETED)
                for f in done:
                    req, fp, admitted = inflight.pop(f)
                    used -= fp
                    got = f.result()
                    reqs = req if isinstance(req, list) else [req]
                    for q, r in zip(reqs, got if isinstance(got, list) else [got]):
                        r.arrival = q.arrival if realtime else 0.0
                        r.admitted = admitted
                        results.append(r)
        return sorted(results, key=lambda r: r.rid)


def summarize(results: list[RequestResult]) -> dict:
    ok = [r for r in results if r.error is None]
    lat = np.array([r.latency for r in ok]) if ok else np.array([0.0])
    makespan = max((r.finished for r in results), default=0.0) - min((r.arrival for r in results), default=0.0)
    rhs = sum(r.nrhs for r in ok)
    return {
        "requests": len(results),
        "completed": len(ok),
        "failed": len(results) - len(ok),
        "rhs_solves": rhs,
        "makespan_s": makespan,
        "solves_per_s": rhs / makespan if makespan > 0 else 0.0,
        "requests_per_s": len(ok) / makespan if makespan > 0 else 0.0,
        "latency_p50_s": float(np.percentile(lat, 50)),
        "latency_p99_s": float(np.percentile(lat, 99)),
    }
