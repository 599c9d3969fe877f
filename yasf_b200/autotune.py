"""Autotuner for batched solves, keyed on (lmax, N, R).

A refined batched solve spends almost all of its time in inner-operator applications, and which
operator is cheapest depends on the shape of the problem: the TF32 tensor-core panel costs about the
same for 1 to 64 columns (and is available up to lmax 8), the complex64 coupling kernel costs one
application per column, and both scale differently with the number of spheres. The tuner times
one application of each candidate on the problem's own operator (random columns, CUDA events on the
current stream), picks the cheapest per inner step, and caches the decision under
(lmax, N bucket, R) so that requests of a similar shape are not timed again. N is bucketed to
about 10 % (costs grow like N^2, so a neighbouring N decides the same way).

The cache can be persisted as JSON (``Autotuner(path=...)``); entries record the measured
milliseconds so a decision can be audited.
"""

from __future__ import annotations

import json
import math
import threading
from dataclasses import asdict, dataclass
from pathlib import Path

import torch

from yasf_b200.device import YASF_C64, CouplingDevice


@dataclass
class Decision:
    inner: str                 # "tf32" or "c64" (the inner_kind of yasf_batched_solve)
    ms_per_step: dict          # measured milliseconds of one inner step per candidate
    key: tuple

    def to_json(self) -> dict:
        d = asdict(self)
        d["key"] = list(self.key)
        return d


def n_bucket(n: int) -> int:
    """Sphere counts within about 10 % share a bucket."""
    return int(round(math.log(max(n, 1)) / math.log(1.1)))


def _time_ms(fn, reps: int = 2) -> float:
    fn()  # warm-up (workspace, plan set-up)
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        fn()
    e1.record()
    e1.synchronize()
    return e0.elapsed_time(e1) / reps


def measure_step_costs(dev: CouplingDevice, tmat: torch.Tensor, nrhs: int) -> dict:
    """Milliseconds of one inner step of a batched solve with nrhs columns, per inner operator."""
    g = torch.Generator(device=dev.device).manual_seed(0)
    x1 = torch.randn(dev.n, dtype=torch.complex128, device=dev.device, generator=g)
    costs = {"c64": nrhs * _time_ms(lambda: dev.coupling(x1, YASF_C64))}
    if dev.lmax <= 8 and nrhs >= 1:
        X = torch.randn(nrhs, dev.n, dtype=torch.complex128, device=dev.device, generator=g)
        costs["tf32"] = _time_ms(lambda: dev.panel(X, tmat))
    return costs


def choose(costs: dict) -> str:
    return min(costs, key=costs.get)


class Autotuner:
    """Thread-safe cache of inner-operator decisions keyed on (lmax, N bucket, R)."""

    def __init__(self, path: str | Path | None = None, measure=measure_step_costs):
        self.path = Path(path) if path else None
        self._measure = measure
        self._lock = threading.Lock()
        self._cache: dict[tuple, Decision] = {}
        if self.path and self.path.exists():
            for e in json.loads(self.path.read_text()):
                k = tuple(e["key"])
                self._cache[k] = Decision(e["inner"], e["ms_per_step"], k)

    def key(self, lmax: int, n_spheres: int, nrhs: int) -> tuple:
        return (int(lmax), n_bucket(n_spheres), int(nrhs))

    def decide(self, dev: CouplingDevice, tmat: torch.Tensor, nrhs: int) -> Decision:
        k = self.key(dev.lmax, dev.n_particles, nrhs)
        with self._lock:
            hit = self._cache.get(k)
        if hit is not None:
            return hit
        costs = self._measure(dev, tmat, nrhs)
        d = Decision(choose(costs), costs, k)
        with self._lock:
            self._cache.setdefault(k, d)
            d = self._cache[k]
            if self.path:
                self.path.parent.mkdir(parents=True, exist_ok=True)
                self.path.write_text(json.dumps([v.to_json() for v in self._cache.values()], indent=1))
        return d

    def decisions(self) -> list[Decision]:
        with self._lock:
            return list(self._cache.values())
