"""``InitialField``: incident beam description (mirror of yasfpy/initial_field.py, file lines 14-128)."""

from __future__ import annotations

import logging

import numpy as np


class InitialField:
    def __init__(self, beam_width, focal_point, field_type: str = "gaussian", amplitude: float = 1,
                 polar_angle: float = 0, azimuthal_angle: float = 0, polarization="TE"):
        self.field_type = field_type
        self.amplitude = amplitude
        self.polar_angle = polar_angle
        self.azimuthal_angle = azimuthal_angle
        self.polarization = polarization
        self.beam_width = beam_width
        self.focal_point = np.asarray(focal_point, dtype=float)
        self.log = logging.getLogger(self.__class__.__module__)
        self._setup()

    def _setup(self) -> None:
        p = self.polarization
        if (isinstance(p, str) and p.lower() == "unp") or (isinstance(p, int) and p == 0):
            self.pol = 0
        elif (isinstance(p, str) and p.lower() == "te") or (isinstance(p, int) and p == 1):
            self.pol = 1
        elif (isinstance(p, str) and p.lower() == "tm") or (isinstance(p, int) and p == 2):
            self.pol = 2
        else:
            self.pol = 0
            self.log.warning("%s is not a valid polarization type. Reverting to unpolarized", p)
        self.normal_incidence = np.abs(np.sin(self.polar_angle)) < 1e-5

    def set_polarization(self, polarization) -> None:
        self.polarization = polarization
        self._setup()
