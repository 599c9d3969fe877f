"""The reference's own solve path driving the b200 coupling kernel (GPU).

The reference's Simulation (with "b200" added to its backend switch by
yasf_b200.reference_binding), its Mie coefficients, plane-wave coefficients and right-hand side,
and its Solver.run (yasfpy/solver.py:65-181: SciPy GMRES, x0 = b) solve the 100-sphere lmax-4
aggregate at rtol 1e-8; every GMRES step calls B200CouplingBackend.multiply, i.e. the on-the-fly
coupling kernel through the C ABI. The scattered-field coefficients must equal the reference's
own dense-backend solve at the same tolerance (ref_solve_c1_tol1e-8.npz) to 1e-7 relative
(max-norm): both runs take the same GMRES path, their operators differ by float64 rounding; and the
reference's rtol-1e-13 solution to 1e-6 (the tolerance's reach).
"""

from __future__ import annotations

import numpy as np
import pytest
from conftest import rel_err

pytestmark = pytest.mark.gpu


def test_reference_solver_with_b200_backend_matches_reference_solve(golden, cuda_device, reference_yasfpy):
    from yasfpy.initial_field import InitialField
    from yasfpy.numerics import Numerics
    from yasfpy.parameters import Parameters
    from yasfpy.particles import Particles
    from yasfpy.solver import Solver

    from yasf_b200.reference_binding import reference_classes

    B200CouplingBackend, B200Simulation = reference_classes()
    g = golden("ref_solve_c1_tol1e-8.npz")
    exact = golden("ref_solve_c1_tol1e-13.npz")["scattered"]
    n = g["positions"].shape[0]
    particles = Particles(position=g["positions"], r=g["radii"],
                          refractive_index=np.full(n, complex(g["refractive_index"])))
    field = InitialField(beam_width=0, focal_point=np.zeros(3), polar_angle=0.0, azimuthal_angle=0.0,
                         polarization="TE")
    params = Parameters(wavelength=np.array([float(g["wavelength"])]),
                        medium_refractive_index=np.ones(1, dtype=complex), particles=particles,
                        initial_field=field)
    solver = Solver(solver_type="gmres", tolerance=1e-8, max_iter=1000, restart=100)
    numerics = Numerics(lmax=int(g["lmax"]), sampling_points_number=np.array([10]), gpu=False,
                        solver=solver, coupling_backend="b200")
    numerics.compute_translation_table()
    sim = B200Simulation(params, numerics, device=cuda_device)
    assert isinstance(sim.coupling_backend, B200CouplingBackend) and sim.sph_h is None
    sim.compute_mie_coefficients()
    sim.compute_initial_field_coefficients()
    sim.compute_right_hand_side()
    sim.compute_scattered_field_coefficients()
    assert sim.scattered_field_err_codes[0] == 0
    x = sim.scattered_field_coefficients[:, :, 0]
    assert rel_err(x, g["scattered"]) < 1e-7
    assert rel_err(x, exact) < 1e-6
    # C_ext from the reference's formula (yasfpy/optics.py:55-156) on both solutions
    k = 2 * np.pi / float(g["wavelength"])
    a = sim.initial_field_coefficients[:, :, 0]
    c_ext = -np.real(np.vdot(a, x)) / k**2 * np.pi
    assert abs(c_ext - float(g["c_ext"])) <= 1e-7 * abs(float(g["c_ext"]))
