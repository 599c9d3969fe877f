"""The ``"b200"`` coupling backend inside the reference's own ``yasfpy`` objects.

yasfpy chooses its coupling backend with a fixed string switch in ``Simulation.__init__``
(yasfpy/simulation.py:95-106) that raises ``ValueError`` for names it does not know; there is no
registry. This module supplies, for an importable ``yasfpy``:

- ``B200CouplingBackend``: a subclass of yasfpy's ``CouplingBackend``
  (yasfpy/coupling/backends.py:36-66). ``requires_pairwise_lookups`` is False, so the reference's
  ``Simulation`` never builds its O(N^2) ``plm`` / ``sph_h`` / ``e_j_dm_phi`` tables
  (yasfpy/simulation.py:160-167). ``multiply(x, idx)`` returns ``W @ x`` with the reference's shape
  rules (yasfpy/coupling/cpu_dense.py:66-120): ``idx`` selects one wavelength channel and the result
  is squeezed to ``(jmax,)``; ``idx=None`` evaluates every channel and returns ``(jmax, channels)``.
  Each product runs the on-the-fly coupling kernel of this library through its C ABI
  (``yasf_coupling_matvec``); geometry and translation plan stay resident on the GPU per channel.
- ``B200Simulation``: a subclass of yasfpy's ``Simulation`` whose backend switch also accepts
  ``numerics.coupling_backend == "b200"``; every other name goes to the reference's own switch.
  Everything else (Mie coefficients, incident field, right-hand side, ``Solver.run`` with SciPy's
  GMRES, ``Optics``) is the reference's code, calling the backend once per GMRES step exactly as it
  calls its dense backend (yasfpy/matrix_apply.py:66-120).

``yasfpy`` is imported only when ``reference_classes()`` is called, so this module loads without it.
"""

from __future__ import annotations

import logging
import os

import numpy as np
import torch

_classes = None


def reference_classes():
    """(B200CouplingBackend, B200Simulation) built on the importable ``yasfpy``."""
    global _classes
    if _classes is not None:
        return _classes
    from yasfpy.coupling.backends import CouplingBackend
    from yasfpy.simulation import Simulation

    from yasf_b200.device import PRECISIONS, CouplingDevice

    class B200CouplingBackend(CouplingBackend):
        """On-the-fly coupling matvec on a B200 behind yasfpy's backend contract."""

        requires_pairwise_lookups: bool = False

        def __init__(self, simulation, device: torch.device | str | None = None,
                     precision: str = "c128"):
            self._sim = simulation
            self._device = torch.device(device) if device is not None else None
            self._precision = PRECISIONS[precision]
            self._states: dict[int, CouplingDevice] = {}

        def _state(self, channel: int) -> CouplingDevice:
            st = self._states.get(channel)
            if st is None:
                sim = self._sim
                device = self._device
                if device is None:
                    device = torch.device("cuda", torch.cuda.current_device())
                table = sim.numerics.translation_ab5
                if table is None:
                    raise RuntimeError("compute the translation table (Numerics.compute_translation_table) "
                                       "before the first coupling product")
                st = CouplingDevice(sim.numerics.lmax, table, sim.parameters.particles.position,
                                    sim.parameters.k_medium[channel], device)
                self._states[channel] = st
            return st

        def _apply(self, channel: int, x: np.ndarray) -> np.ndarray:
            st = self._state(channel)
            xt = torch.from_numpy(np.ascontiguousarray(x.reshape(st.n), dtype=np.complex128)).to(st.device)
            return st.coupling(xt, self._precision).cpu().numpy()

        def multiply(self, x: np.ndarray, idx: int | None = None) -> np.ndarray:
            x = np.asarray(x, dtype=np.complex128)
            if idx is not None:
                return self._apply(idx, x)
            channels = np.atleast_1d(self._sim.parameters.k_medium).shape[0]
            jmax = self._sim.parameters.particles.number * self._sim.numerics.nmax
            out = np.zeros((jmax, channels), dtype=np.complex128)
            for w in range(channels):
                out[:, w] = self._apply(w, x[:, w] if x.ndim == 2 else x)
            return out

    class B200Simulation(Simulation):
        """yasfpy's ``Simulation`` with ``"b200"`` added to its backend switch."""

        def __init__(self, parameters, numerics, device: torch.device | str | None = None):
            name = str(getattr(numerics, "coupling_backend", "dense")).lower()
            if name != "b200":
                super().__init__(parameters, numerics)
                return
            # the attributes Simulation.__init__ sets (yasfpy/simulation.py:80-108), then its setup
            self.parameters = parameters
            self.numerics = numerics
            self.log = logging.getLogger(self.__class__.__module__)
            self._matvec_detail_enabled = bool(int(os.environ.get("YASF_MATVEC_DETAIL", "0")))
            self._matvec_detail = {}
            self.coupling_backend = B200CouplingBackend(self, device)
            self._Simulation__setup()

    _classes = (B200CouplingBackend, B200Simulation)
    return _classes
