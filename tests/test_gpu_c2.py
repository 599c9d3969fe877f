"""The benchmark configuration's own solve, pinned to the oracle.

Workload: 2000 spheres by seeded random sequential addition in a ball at volume fraction 0.20,
lognormal radii (median 0.1 um, sigma_ln 0.2, clipped to [0.04, 0.25] um), m = 1.6+0.005i,
wavelength 0.6 um, lmax 6 (192,000 unknowns), one plane wave (+z, TE), GMRES rtol 1e-8: the
solve the benchmark times, run through the drop-in Simulation / Solver / Optics API, with and
without the block-Jacobi preconditioner on 4x4x4 cells.

The oracle (the plain-C restatement of the reference's particle_interaction_scalar,
yasfpy/functions/cpu_numba.py:22-95, with the master operator of yasfpy/matrix_apply.py:66-120)
applies (I - T W) to the device solution on all host threads, and the true relative residual
||(I - T W) x - b|| / ||b|| must meet the solve's tolerance (1.01 x rtol: the oracle's own float64
rounding differs from the device's). C_ext is recomputed from x on the host
(yasfpy/optics.py:55-156) and C_sca from the oracle's bilinear form (yasfpy/functions/
cpu_numba.py:410-457), both to 1e-10 relative.
"""

from __future__ import annotations

import numpy as np
import pytest

from oracle import restate as R
from yasf_b200 import BlockDiagonalPreconditioner, InitialField, Numerics, Optics, Parameters
from yasf_b200 import Particles, Simulation, Solver
from yasf_b200.workloads import aggregate_c2

pytestmark = pytest.mark.gpu

RTOL = 1e-8


@pytest.fixture(scope="module")
def c2_aggregate():
    return aggregate_c2(seed=0)


def _solve(agg, device, preconditioned: bool):
    n = agg.n
    particles = Particles(agg.positions, agg.radii, np.full(n, agg.refractive_index))
    field = InitialField(beam_width=0, focal_point=np.zeros(3), polar_angle=0.0, azimuthal_angle=0.0,
                         polarization="TE")
    params = Parameters(np.array([agg.wavelength]), np.array([1.0 + 0j]), particles, field)
    pre = None
    if preconditioned:
        extent = agg.positions.max(axis=0) - agg.positions.min(axis=0)
        pre = BlockDiagonalPreconditioner((extent + 2.0) / 4)
    solver = Solver("gmres", tolerance=RTOL, max_iter=200, restart=100, preconditioner=pre)
    numerics = Numerics(lmax=agg.lmax, solver=solver)
    numerics.compute_translation_table()
    sim = Simulation(params, numerics, device=device)
    sim.compute_mie_coefficients()
    sim.compute_initial_field_coefficients()
    sim.compute_right_hand_side()
    if pre is not None:
        pre.prepare(sim)
    sim.compute_scattered_field_coefficients()
    opt = Optics(sim)
    opt.compute_cross_sections()
    return sim, opt


@pytest.mark.parametrize("preconditioned", [False, True], ids=["plain", "block-jacobi-4x4x4"])
def test_c2_solution_true_residual_and_cross_sections(c2_aggregate, cuda_device, preconditioned):
    agg = c2_aggregate
    sim, opt = _solve(agg, cuda_device, preconditioned)
    st = sim.solver_stats[0]
    assert sim.scattered_field_err_codes[0] == 0, st
    x = sim.scattered_field_coefficients[:, :, 0].ravel()
    b = sim.right_hand_side[:, :, 0].ravel()
    a = sim.initial_field_coefficients[:, :, 0].ravel()
    tmat = sim.device_tmat(0).cpu().numpy()
    table = sim.numerics.translation_ab5
    k = 2 * np.pi / agg.wavelength
    # true residual of the device solution under the oracle's operator
    ax = R.master_matvec(agg.lmax, agg.positions, k, table, tmat, x)
    res = np.linalg.norm(ax - b) / np.linalg.norm(b)
    assert res <= 1.01 * RTOL, (res, st)
    # C_ext = -pi/k^2 Re(a^H x), recomputed on the host
    c_ext = -np.real(np.vdot(a, x)) / k**2 * np.pi
    assert abs(opt.c_ext[0] - c_ext) <= 1e-10 * abs(c_ext)
    if not preconditioned:
        # C_sca from the oracle's bilinear form (regular translation, self pairs included)
        c_sca = abs(R.scattering_bilinear_rows(agg.lmax, agg.positions, k, table, x)) / k**2 * np.pi
        assert abs(opt.c_sca[0] - c_sca) <= 1e-10 * abs(c_sca)
