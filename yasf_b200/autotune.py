"""Autotuner for batched solves, keyed on (lmax, N, R): inner operator and tile shapes.

A refined batched solve spends almost all of its time in inner-operator applications, and which
operator is cheapest depends on the shape of the problem: the TF32 tensor-core panel costs about the
same for 1 to 64 columns (and is available up to lmax 8), the complex64 coupling kernel costs one
application per column, and both scale differently with the number of spheres. The tile shapes
matter too: how many waves of resident blocks the contraction's source chunks fill (1, 2 or 4:
fewer chunks write fewer partial sums, more balance the blocks better), how many 64-column groups
share one tensor-core panel block (1 or 2), and the float64 dense panel's column tile (32 or 64) for
the float64 residuals. The tuner times one application of every candidate (operator x tile shape) on
the problem's own operator (random columns, CUDA events on the current stream), keeps the cheapest
inner step and the cheaper residual tile, and caches the decision under (lmax, N bucket, R), so
requests of a similar shape are not timed again. N is bucketed to about 10 % (costs grow like N^2,
so a neighbouring N decides the same way). The tile shapes take effect through yasf_set_tiles on the
thread that runs the solve (``Decision.apply_tiles``).

The cache can be persisted as JSON (``Autotuner(path=...)``); entries record the measured
milliseconds so a decision can be audited.
"""

from __future__ import annotations

import json
import math
import threading
from dataclasses import asdict, dataclass, field
from pathlib import Path

import torch

from yasf_b200.device import YASF_C64, CouplingDevice


@dataclass
class Decision:
    inner: str                 # "tf32" or "c64" (the inner_kind of yasf_batched_solve)
    ms_per_step: dict          # measured milliseconds per candidate ("c64/w2", "tf32/g1", "f64/c32", ...)
    key: tuple
    tiles: dict = field(default_factory=dict)  # contract_waves, panel_groups, dpanel_cols (0: rule)

    def to_json(self) -> dict:
        d = asdict(self)
        d["key"] = list(self.key)
        return d

    def apply_tiles(self) -> None:
        """Set this decision's tile shapes for the calling thread's next launches."""
        from yasf_b200._lib import set_tiles

        set_tiles(self.tiles.get("contract_waves", 0), self.tiles.get("dpanel_cols", 0),
                  self.tiles.get("panel_groups", 0))


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


WAVES = (1, 2, 4)


def measure_step_costs(dev: CouplingDevice, tmat: torch.Tensor, nrhs: int) -> dict:
    """Milliseconds per candidate: one inner step of a batched solve with nrhs columns for every
    (inner operator, tile shape) ("c64/w<waves>", "tf32/g<groups>"), and one float64 residual pass
    of the dense panel per column tile ("f64/c<cols>", when that kernel serves the shape)."""
    from yasf_b200._lib import set_tiles

    g = torch.Generator(device=dev.device).manual_seed(0)
    x1 = torch.randn(dev.n, dtype=torch.complex128, device=dev.device, generator=g)
    costs = {}
    try:
        for w in WAVES:
            set_tiles(w, 0, 0)
            costs[f"c64/w{w}"] = nrhs * _time_ms(lambda: dev.coupling(x1, YASF_C64))
        if dev.lmax <= 8:
            X = torch.randn(nrhs, dev.n, dtype=torch.complex128, device=dev.device, generator=g)
            for grp in ((1, 2) if nrhs > 64 and dev.lmax <= 7 else (0,)):
                set_tiles(0, 0, grp)
                costs[f"tf32/g{grp}"] = _time_ms(lambda: dev.panel(X, tmat))
            if nrhs >= 12 and dev.lmax <= 6:
                for cols in (32, 64):
                    set_tiles(0, cols, 0)
                    costs[f"f64/c{cols}"] = _time_ms(lambda: dev.dpanel(X, tmat))
    finally:
        set_tiles(0, 0, 0)
    return costs


def choose(costs: dict) -> str:
    """The cheapest inner-step candidate (the float64 residual candidates are chosen apart)."""
    inner = {k: v for k, v in costs.items() if not k.startswith("f64")}
    return min(inner, key=inner.get)


def decision_from(costs: dict, key: tuple) -> Decision:
    best = choose(costs)
    inner, _, shape = best.partition("/")
    tiles = {}
    if shape.startswith("w"):
        tiles["contract_waves"] = int(shape[1:])
    elif shape.startswith("g") and int(shape[1:]) > 0:
        tiles["panel_groups"] = int(shape[1:])
    f64 = {k: v for k, v in costs.items() if k.startswith("f64")}
    if f64:
        tiles["dpanel_cols"] = int(min(f64, key=f64.get).split("/c")[1])
    return Decision(inner, costs, key, tiles)


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
                self._cache[k] = Decision(e["inner"], e["ms_per_step"], k, e.get("tiles", {}))

    def key(self, lmax: int, n_spheres: int, nrhs: int) -> tuple:
        return (int(lmax), n_bucket(n_spheres), int(nrhs))

    def decide(self, dev: CouplingDevice, tmat: torch.Tensor, nrhs: int) -> Decision:
        k = self.key(dev.lmax, dev.n_particles, nrhs)
        with self._lock:
            hit = self._cache.get(k)
        if hit is not None:
            return hit
        costs = self._measure(dev, tmat, nrhs)
        d = decision_from(costs, k)
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
