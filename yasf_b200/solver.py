"""``Solver``: iterative-solver settings and the device GMRES (mirror of yasfpy/solver.py:27-231).

Keeps the reference constructor (``solver_type``, ``tolerance``, ``max_iter``, ``restart``,
``preconditioner``, ``warm_start``). ``run(A, b, x0)`` solves on the device when ``A`` is a
``MasterOperator`` (what ``Simulation`` builds); the semantics are SciPy's restarted GMRES with
left preconditioning (see ``include/yasf_b200.h``: yasf_gmres_solve). Only ``"gmres"`` runs on the
device; other solver types raise ``NotImplementedError``.
"""

from __future__ import annotations

import logging
from dataclasses import dataclass

import numpy as np
import torch

from yasf_b200.device import PRECISIONS, CouplingDevice


@dataclass
class MasterOperator:
    """(I - T W) for one aggregate and wavelength channel, resident on the device."""

    device_state: CouplingDevice
    tmat: torch.Tensor  # (N*nmax,) complex128
    precision: str = "c128"

    @property
    def shape(self):
        n = self.device_state.n
        return (n, n)

    def matvec(self, x):
        dev = self.device_state
        if isinstance(x, np.ndarray):
            xt = torch.from_numpy(np.ascontiguousarray(x, dtype=np.complex128)).to(dev.device)
            return dev.master(xt, self.tmat, PRECISIONS[self.precision]).cpu().numpy()
        return dev.master(x, self.tmat, PRECISIONS[self.precision])


class Solver:
    def __init__(self, solver_type: str = "gmres", tolerance: float = 1e-4, max_iter: float = 1e4,
                 restart: float = 1e2, preconditioner=None, *, warm_start: bool = True):
        self.type = solver_type.lower()
        self.tolerance = tolerance
        self.max_iter = int(max_iter)
        self.restart = int(restart)
        self.preconditioner = preconditioner
        self.warm_start = bool(warm_start)
        self.log = logging.getLogger(self.__class__.__module__)
        self.last_stats: dict | None = None

    def run(self, a: MasterOperator, b, x0=None, precision: str | None = None):
        """Solve a x = b on the device. Returns (x, err_code) as SciPy does (0 = converged)."""
        if self.type != "gmres":
            raise NotImplementedError(f"solver type {self.type!r} is not available on the b200 backend")
        if not isinstance(a, MasterOperator):
            raise TypeError("the b200 Solver runs on a MasterOperator built by yasf_b200.Simulation")
        dev = a.device_state
        numpy_io = isinstance(b, np.ndarray)
        bt = torch.from_numpy(np.ascontiguousarray(b, dtype=np.complex128)).to(dev.device) if numpy_io else b
        if x0 is None:
            xt = bt.clone()
        elif isinstance(x0, np.ndarray):
            xt = torch.from_numpy(np.ascontiguousarray(x0, dtype=np.complex128)).to(dev.device)
        else:
            xt = x0.clone()
        if not torch.isfinite(torch.view_as_real(bt)).all():
            raise FloatingPointError("right-hand side contains NaN or Inf")
        prec = precision or a.precision
        pc = None
        if self.preconditioner is not None:
            pc = self.preconditioner.device_handle(dev)
        stats = dev.gmres(a.tmat, bt, xt, self.tolerance, self.restart, self.max_iter,
                          PRECISIONS[prec], pc)
        self.last_stats = stats
        self.log.debug("gmres stats: %s", stats)
        x = xt.cpu().numpy() if numpy_io else xt
        return x, stats["info"]


class GMResCounter:
    """Iteration counter with the reference's interface (yasfpy/solver.py:184-231)."""

    def __init__(self, disp: bool = False, callback_type: str = "pr_norm"):
        self._disp = disp
        self.niter = 0
        self.header = " Iteration \t        Residual" if callback_type == "pr_norm" else " Iteration \t Current Iterate"

    def __call__(self, rk=None):
        self.niter += 1
        if self._disp:
            print(self.header)
            print(f"{self.niter:10} \t {rk}")
