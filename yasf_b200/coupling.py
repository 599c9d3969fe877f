"""Coupling backends (mirror of yasfpy/coupling/backends.py:36-66 and yasfpy/coupling/ops.py:22-49).

``B200CouplingBackend`` is the drop-in ``"b200"`` backend: ``requires_pairwise_lookups = False``
(no O(N^2) tables, yasfpy/simulation.py:160-167), ``multiply(x, idx)`` returns ``W @ x`` with
the reference's shape conventions: ``idx`` selects one wavelength channel and returns a squeezed
``(jmax,)`` array; ``idx=None`` evaluates every channel of an ``(jmax, channels)`` input (or a 1-D
input against every channel) and returns ``(jmax, channels)`` (yasfpy/coupling/cpu_dense.py:66-120).
"""

from __future__ import annotations

from typing import TYPE_CHECKING

import numpy as np
import torch

from yasf_b200.device import PRECISIONS

if TYPE_CHECKING:
    from yasf_b200.simulation import Simulation


class CouplingBackend:
    requires_pairwise_lookups: bool = False

    def multiply(self, x: np.ndarray, idx: int | None = None) -> np.ndarray:  # pragma: no cover
        raise NotImplementedError


class B200CouplingBackend(CouplingBackend):
    """On-the-fly coupling matvec on a B200 (C ABI ``yasf_coupling_matvec``)."""

    requires_pairwise_lookups: bool = False

    def __init__(self, simulation: "Simulation"):
        self._sim = simulation

    def multiply(self, x: np.ndarray, idx: int | None = None) -> np.ndarray:
        sim = self._sim
        prec = PRECISIONS[sim.numerics.b200_precision]
        jmax = sim.parameters.particles.number * sim.numerics.nmax
        channels = sim.parameters.k_medium.shape[0]
        x = np.asarray(x, dtype=np.complex128)
        if idx is not None:
            dev = sim.device_state(idx)
            xt = torch.from_numpy(np.ascontiguousarray(x.reshape(jmax))).to(dev.device)
            return dev.coupling(xt, prec).cpu().numpy()
        out = np.zeros((jmax, channels), dtype=np.complex128)
        for w in range(channels):
            xw = x[:, w] if x.ndim == 2 else x
            dev = sim.device_state(w)
            xt = torch.from_numpy(np.ascontiguousarray(xw.reshape(jmax))).to(dev.device)
            out[:, w] = dev.coupling(xt, prec).cpu().numpy()
        return out


class B200NearFieldCouplingBackend(B200CouplingBackend):
    """The reference's ``nearfar`` semantics (yasfpy/coupling/backends.py:259-459) on the B200:
    only pairs at most ``numerics.coupling_near_field_radius`` apart contribute (self pairs
    excluded), the rest of W is dropped; C ABI ``yasf_coupling_matvec_nearfield``. The reference's
    version is CPU-only and needs the radius set; so does this one (``ValueError`` otherwise)."""

    def multiply(self, x: np.ndarray, idx: int | None = None) -> np.ndarray:
        sim = self._sim
        radius = getattr(sim.numerics, "coupling_near_field_radius", None)
        if radius is None:
            raise ValueError("nearfar backend requires numerics.coupling_near_field_radius to be set.")
        prec = PRECISIONS[sim.numerics.b200_precision]
        jmax = sim.parameters.particles.number * sim.numerics.nmax
        channels = sim.parameters.k_medium.shape[0]
        x = np.asarray(x, dtype=np.complex128)
        ws = [idx] if idx is not None else list(range(channels))
        out = np.zeros((jmax, len(ws)), dtype=np.complex128)
        for c, w in enumerate(ws):
            xw = x if (idx is not None or x.ndim == 1) else x[:, w]
            dev = sim.device_state(w)
            xt = torch.from_numpy(np.ascontiguousarray(xw.reshape(jmax))).to(dev.device)
            out[:, c] = dev.coupling_nearfield(xt, float(radius), prec).cpu().numpy()
        return out[:, 0] if idx is not None else out
