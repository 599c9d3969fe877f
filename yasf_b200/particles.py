"""``Particles``: sphere positions, radii and refractive indices (mirror of yasfpy/particles.py:24-247).

Only the attributes the solve path reads are derived: unique (radius, index) pairs and the map
``single_unique_array_idx`` from each sphere to its pair (yasfpy/particles.py:117-146), plus the
volume-equivalent geometric projection (yasfpy/particles.py:162-166).
"""

from __future__ import annotations

import logging

import numpy as np


class Particles:
    def __init__(self, position: np.ndarray, r: np.ndarray, refractive_index: np.ndarray,
                 refractive_index_table=None, shape_type: str = "sphere"):
        self.log = logging.getLogger(self.__class__.__module__)
        self.position = np.ascontiguousarray(np.asarray(position, dtype=float))
        self.r = np.asarray(r, dtype=float)
        refractive_index = np.asarray(refractive_index)
        if refractive_index_table is not None:
            raise NotImplementedError("material tables are out of scope; pass complex indices")
        if refractive_index.ndim > 2 or (refractive_index.ndim == 2 and refractive_index.shape[1] > 2):
            raise ValueError(
                "Refractive index should be either an integer array, complex array, or a two column float matrix!"
            )
        if refractive_index.ndim == 2 and refractive_index.shape[1] == 2:
            refractive_index = refractive_index[:, 0] + 1j * refractive_index[:, 1]
        self.refractive_index = refractive_index
        self.refractive_index_table = None
        self.type = shape_type
        if self.position.ndim != 2 or self.position.shape[1] != 3:
            raise ValueError("positions must have shape (N, 3)")
        if self.position.shape[0] != self.r.shape[0]:
            raise ValueError("positions and radii disagree on the number of particles")
        self.number = self.r.shape[0]
        self.compute_unique_radii_index_pairs()
        self.compute_volume_equivalent_area()

    def compute_unique_radii_index_pairs(self) -> None:
        self.unique_radius_index_pairs, self.single_unique_array_idx = np.unique(
            np.column_stack((self.r, self.refractive_index)), return_inverse=True, axis=0
        )
        self.single_unique_array_idx = np.asarray(self.single_unique_array_idx).reshape(-1)
        self.num_unique_pairs = self.unique_radius_index_pairs.shape[0]

    def compute_volume_equivalent_area(self) -> None:
        self.geometric_projection = np.pi * np.power(np.sum(np.power(self.r, 3)), 2 / 3)
