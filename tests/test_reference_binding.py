"""The "b200" backend inside the reference's own Simulation (host side, no GPU).

yasf_b200.reference_binding adds "b200" to yasfpy's backend switch (yasfpy/simulation.py:95-106)
through a Simulation subclass. Checked here with the reference's own classes: the switch selects
the b200 backend, the O(N^2) pairwise tables are skipped because requires_pairwise_lookups is False
(yasfpy/simulation.py:160-167), the other names still reach the reference's backends, and unknown
names still raise the reference's ValueError. No coupling product is computed (that needs a GPU).
"""

from __future__ import annotations

import numpy as np
import pytest


def _reference_sim_parts(lmax=2, backend="b200", n=4):
    from yasfpy.initial_field import InitialField
    from yasfpy.numerics import Numerics
    from yasfpy.parameters import Parameters
    from yasfpy.particles import Particles
    from yasfpy.solver import Solver

    rng = np.random.default_rng(0)
    pos = np.array([[0.0, 0.0, 0.0], [0.5, 0.0, 0.0], [0.0, 0.6, 0.1], [0.2, -0.3, 0.7]])[:n]
    particles = Particles(position=pos, r=np.full(n, 0.1), refractive_index=np.full(n, 1.5 + 0.01j))
    field = InitialField(beam_width=0, focal_point=np.zeros(3), polar_angle=0.0, azimuthal_angle=0.0,
                         polarization="TE")
    params = Parameters(wavelength=np.array([0.55]), medium_refractive_index=np.ones(1, dtype=complex),
                        particles=particles, initial_field=field)
    solver = Solver(solver_type="gmres", tolerance=1e-8, max_iter=100, restart=50)
    numerics = Numerics(lmax=lmax, sampling_points_number=np.array([10]), gpu=False, solver=solver,
                        coupling_backend=backend)
    del rng
    return params, numerics


def test_reference_switch_selects_b200_and_skips_pairwise_tables(reference_yasfpy):
    from yasfpy.coupling.backends import CouplingBackend
    from yasfpy.simulation import Simulation

    from yasf_b200.reference_binding import reference_classes

    B200CouplingBackend, B200Simulation = reference_classes()
    params, numerics = _reference_sim_parts()
    sim = B200Simulation(params, numerics)
    assert isinstance(sim, Simulation)
    assert isinstance(sim.coupling_backend, CouplingBackend)
    assert isinstance(sim.coupling_backend, B200CouplingBackend)
    assert sim.coupling_backend.requires_pairwise_lookups is False
    assert sim.sph_h is None and sim.sph_j is None and sim.plm is None and sim.e_j_dm_phi is None
    assert sim.idx_lookup.shape == (4 * numerics.nmax, 5)  # the reference's own index table


def test_other_backend_names_reach_the_reference_switch(reference_yasfpy):
    from yasfpy.coupling.backends import DenseCouplingBackend

    from yasf_b200.reference_binding import reference_classes

    _, B200Simulation = reference_classes()
    params, numerics = _reference_sim_parts(backend="dense", n=2)
    sim = B200Simulation(params, numerics)
    assert isinstance(sim.coupling_backend, DenseCouplingBackend)
    assert sim.sph_h is not None  # the reference built its pairwise tables
    params, numerics = _reference_sim_parts(backend="no-such-backend", n=2)
    with pytest.raises(ValueError, match="Unsupported coupling backend"):
        B200Simulation(params, numerics)
