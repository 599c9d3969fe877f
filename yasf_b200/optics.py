"""Cross sections from the solved coefficients (yasfpy/optics.py:55-156).

C_ext = pi/|k|^2 Re(-sum conj(a) b) and C_sca = pi/|k|^2 |sum conj(b) W_reg b| where W_reg is the
regular (j_p) translation including self pairs (yasfpy/functions/cpu_numba.py:410-457); both are
evaluated on the device. Far-field consumers (phase function, Mueller) are out of scope.
"""

from __future__ import annotations

import logging

import numpy as np
import torch


class Optics:
    def __init__(self, simulation):
        self.simulation = simulation
        self.c_ext = np.zeros_like(simulation.parameters.wavelength, dtype=complex)
        self.c_sca = np.zeros_like(simulation.parameters.wavelength, dtype=complex)
        self.log = logging.getLogger(self.__class__.__module__)

    def compute_cross_sections(self):
        sim = self.simulation
        a = sim.initial_field_coefficients
        f = sim.scattered_field_coefficients
        W = sim.parameters.wavelengths_number
        c_ext = np.zeros(W, dtype=complex)
        c_sca = np.zeros(W, dtype=complex)
        for w in range(W):
            dev = sim.device_state(w)
            at = torch.from_numpy(np.ascontiguousarray(a[:, :, w].ravel())).to(dev.device)
            bt = torch.from_numpy(np.ascontiguousarray(f[:, :, w].ravel())).to(dev.device)
            c_ext[w] = -dev.dotc(at, bt)
            c_sca[w] = dev.scattering_bilinear(bt)
        k2 = np.power(np.abs(sim.parameters.k_medium), 2)
        self.c_ext = np.real(c_ext / k2) * np.pi
        self.c_sca = np.abs(c_sca / k2) * np.pi
        self.albedo = self.c_sca / self.c_ext

    def compute_efficiencies(self):
        p = self.simulation.parameters
        self.q_sca = self.c_sca / p.particles.geometric_projection * np.abs(p.medium_refractive_index)
        self.q_ext = self.c_ext / p.particles.geometric_projection * np.abs(p.medium_refractive_index)
