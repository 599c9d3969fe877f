"""``Simulation``: orchestration of the solve (mirror of yasfpy/simulation.py:33-249).

Backend selection keeps the reference's string switch (yasfpy/simulation.py:95-106) and adds
``"b200"``; the O(N^2) pairwise lookup tables are never formed (``requires_pairwise_lookups`` is
False, yasfpy/simulation.py:160-167), so ``sph_j``, ``sph_h``, ``e_j_dm_phi`` and ``plm`` stay
``None``. ``compute_scattered_field_coefficients`` keeps the per-wavelength loop and initial-guess
policy of yasfpy/scattered_field_coefficients.py:43-156 (guess, warm start, else the right-hand
side) but runs the whole GMRES on the device through the C ABI: no vector crosses to the host
between iterations.
"""

from __future__ import annotations

import logging
import os

import numpy as np
import torch

from yasf_b200.coupling import B200CouplingBackend, B200NearFieldCouplingBackend
from yasf_b200.device import CouplingDevice
from yasf_b200.incident import compute_initial_field_coefficients
from yasf_b200.mie import compute_mie_coefficients
from yasf_b200.numerics import Numerics
from yasf_b200.parameters import Parameters
from yasf_b200.solver import MasterOperator, Solver


def compute_idx_lookups(lmax: int, particle_number: int) -> np.ndarray:
    """(s, n, tau, l, m) rows for every unknown (yasfpy/functions/cpu_numba.py:371-407)."""
    nmax = 2 * lmax * (lmax + 2)
    rows = []
    for tau in (1, 2):
        for l in range(1, lmax + 1):
            for m in range(-l, l + 1):
                rows.append(((tau - 1) * lmax * (lmax + 2) + (l - 1) * (l + 1) + l + m, tau, l, m))
    rows.sort()
    base = np.array(rows, dtype=np.int64)  # (nmax, 4)
    idx = np.zeros((particle_number * nmax, 5), dtype=np.int64)
    idx[:, 0] = np.repeat(np.arange(particle_number), nmax)
    idx[:, 1:] = np.tile(base, (particle_number, 1))
    return idx


class Simulation:
    def __init__(self, parameters: Parameters, numerics: Numerics, device: str | torch.device | None = None):
        self.parameters = parameters
        self.numerics = numerics
        self.log = logging.getLogger(self.__class__.__module__)
        self._matvec_detail_enabled = bool(int(os.environ.get("YASF_MATVEC_DETAIL", "0")))
        self._matvec_detail: dict = {}
        backend_name = str(getattr(self.numerics, "coupling_backend", "b200")).lower()
        if backend_name in {"b200"}:
            self.coupling_backend = B200CouplingBackend(self)
        elif backend_name in {"nearfar", "near_far", "near-far"}:
            self.coupling_backend = B200NearFieldCouplingBackend(self)
        else:
            raise ValueError(
                f"Unsupported coupling backend: {backend_name!r}. Expected 'b200' or 'nearfar' "
                "(the reference's 'dense' and 'tiled_dense' backends compute what 'b200' computes)."
            )
        if device is None:
            if not torch.cuda.is_available():
                raise RuntimeError("the b200 backend needs a CUDA device")
            device = torch.device("cuda", torch.cuda.current_device())
        self.device = torch.device(device)
        self.idx_lookup = compute_idx_lookups(numerics.lmax, parameters.particles.number)
        self.sph_j = None
        self.sph_h = None
        self.e_j_dm_phi = None
        self.plm = None
        self._dev_states: dict[int, CouplingDevice] = {}
        self._tmats: dict[int, torch.Tensor] = {}
        self.solver_stats: list[dict] = []

    # -- device state ------------------------------------------------------------------------
    def _table(self) -> np.ndarray:
        if self.numerics.translation_ab5 is None:
            self.numerics.compute_translation_table()
        return self.numerics.translation_ab5

    def device_state(self, channel: int = 0) -> CouplingDevice:
        st = self._dev_states.get(channel)
        if st is None:
            st = CouplingDevice(self.numerics.lmax, self._table(), self.parameters.particles.position,
                                self.parameters.k_medium[channel], self.device)
            self._dev_states[channel] = st
        return st

    def device_tmat(self, channel: int = 0) -> torch.Tensor:
        t = self._tmats.get(channel)
        if t is None:
            if not hasattr(self, "mie_coefficients"):
                self.compute_mie_coefficients()
            sidx = self.parameters.particles.single_unique_array_idx
            tm = np.ascontiguousarray(self.mie_coefficients[sidx, :, channel].ravel(order="C"))
            t = torch.from_numpy(tm).to(self.device)
            self._tmats[channel] = t
        return t

    # -- setup (host, once per run) ------------------------------------------------------------
    def compute_mie_coefficients(self) -> None:
        p = self.parameters
        self.mie_coefficients, self.scatter_to_internal = compute_mie_coefficients(
            self.numerics.lmax, p.omega, p.k_medium, p.particles.unique_radius_index_pairs)
        self._tmats = {}

    def compute_initial_field_coefficients(self) -> None:
        p = self.parameters
        self.initial_field_coefficients = compute_initial_field_coefficients(
            self.numerics.lmax, p.particles.position, p.k_medium, p.initial_field)

    def compute_right_hand_side(self) -> None:
        self.right_hand_side = (
            self.mie_coefficients[self.parameters.particles.single_unique_array_idx, :]
            * self.initial_field_coefficients
        )

    # -- operators ---------------------------------------------------------------------------
    def coupling_matrix_multiply(self, x: np.ndarray, idx: int | None = None):
        return self.coupling_backend.multiply(x, idx)

    def master_matrix_multiply(self, value: np.ndarray, idx: int):
        op = MasterOperator(self.device_state(idx), self.device_tmat(idx), self.numerics.b200_precision)
        return op.matvec(np.asarray(value, dtype=np.complex128))

    # -- the solve -----------------------------------------------------------------------------
    def compute_scattered_field_coefficients(self, guess: np.ndarray | None = None) -> None:
        solver: Solver = self.numerics.solver
        if solver is None:
            raise ValueError("numerics.solver is not set")
        if isinstance(self.coupling_backend, B200NearFieldCouplingBackend):
            raise NotImplementedError("the device solve applies the exact coupling operator; the near-field "
                                      "backend provides coupling products (coupling_matrix_multiply)")
        W = self.parameters.wavelengths_number
        self.scattered_field_coefficients = np.zeros_like(self.initial_field_coefficients)
        self.scattered_field_err_codes = np.zeros(W)
        self.solver_stats = []
        prev = None
        for w in range(W):
            dev = self.device_state(w)
            op = MasterOperator(dev, self.device_tmat(w), self.numerics.b200_precision)
            b = torch.from_numpy(np.ascontiguousarray(self.right_hand_side[:, :, w].ravel())).to(dev.device)
            if guess is not None:
                x0 = torch.from_numpy(np.ascontiguousarray(guess[:, :, w].ravel())).to(dev.device)
            elif solver.warm_start and prev is not None:
                x0 = prev.clone()
            else:
                x0 = b.clone()
            x, err = solver.run(op, b, x0)
            self.scattered_field_coefficients[:, :, w] = x.cpu().numpy().reshape(
                self.right_hand_side.shape[:2])
            self.scattered_field_err_codes[w] = err
            self.solver_stats.append(dict(solver.last_stats or {}))
            prev = x
