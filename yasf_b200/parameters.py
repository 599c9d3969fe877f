"""``Parameters``: wavelengths, medium, particles, incident field (mirror of yasfpy/parameters.py:15-132)."""

from __future__ import annotations

import numpy as np

from yasf_b200.initial_field import InitialField
from yasf_b200.particles import Particles


class Parameters:
    def __init__(self, wavelength: np.ndarray, medium_refractive_index: np.ndarray,
                 particles: Particles, initial_field: InitialField):
        self.wavelength = np.atleast_1d(np.array(wavelength, dtype=float))
        self.medium_refractive_index = np.atleast_1d(np.asarray(medium_refractive_index))
        self.wavelengths_number = self.wavelength.size
        self.particles = particles
        self.initial_field = initial_field
        # yasfpy/parameters.py:57-59, 96-100
        self.omega = 2 * np.pi / self.wavelength
        self.k_medium = self.omega * self.medium_refractive_index
        self.k_particle = np.outer(self.particles.refractive_index, self.omega)
