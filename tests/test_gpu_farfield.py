"""The scattered far field on the device (yasf_far_field): E_theta, E_phi and the Stokes parameters
on sampling directions, against the oracle (a serial restatement of
yasfpy/functions/cpu_numba.py:536-660, pinned to the reference's own output in
tests/test_oracle_golden.py), and the phase function of the drop-in Optics against the reference's
Optics on the same solved aggregate (tests/golden/ref_farfield.npz). Tolerances: 1e-11 relative
(float64 sums in another order)."""

from __future__ import annotations

import numpy as np
import pytest
import torch

from oracle import restate as R
from yasf_b200 import InitialField, Numerics, Optics, Parameters, Particles, Simulation
from yasf_b200.device import CouplingDevice
from yasf_b200.wigner import translation_table_ab5
from yasf_b200.workloads import rsa_cube

pytestmark = pytest.mark.gpu


def _rel(a, b):
    return float(np.abs(a - b).max() / np.abs(b).max())


@pytest.mark.parametrize("lmax", [1, 2, 3, 4, 5, 6, 7, 8])
def test_far_field_matches_the_oracle(cuda_device, lmax):
    rng = np.random.default_rng(100 + lmax)
    n = 37  # particles: one full warp chunk and a ragged one
    radii = rng.uniform(0.05, 0.1, size=n)
    pos = rsa_cube(radii, 0.12, rng)
    k = 2 * np.pi / 0.6
    dev = CouplingDevice(lmax, translation_table_ab5(lmax), pos, k, cuda_device)
    coef = rng.normal(size=(n, dev.nmax)) + 1j * rng.normal(size=(n, dev.nmax))
    polar = rng.uniform(0, np.pi, size=50)  # not a multiple of the 4 directions per warp
    azim = rng.uniform(0, 2 * np.pi, size=50)
    et, ep, st = dev.far_field(torch.from_numpy(coef.ravel()).to(cuda_device), polar, azim)
    ref_t, ref_p = R.far_field(lmax, pos, k, coef, polar, azim)
    assert _rel(et.cpu().numpy(), ref_t) < 1e-11
    assert _rel(ep.cpu().numpy(), ref_p) < 1e-11
    I, dop, dolp, dolq, dolu, docp = R.polarization_components(ref_t, ref_p)
    s = st.cpu().numpy()
    assert _rel(s[:, 0], I) < 1e-11
    q = -dolq * I
    assert np.abs(s[:, 1] - q).max() < 1e-11 * I.max()
    assert np.abs(s[:, 2] - dolu * I).max() < 1e-11 * I.max()
    assert np.abs(s[:, 3] - docp * I).max() < 1e-11 * I.max()


def test_phase_function_matches_the_reference(golden, cuda_device):
    """The drop-in Optics on the reference's solved coefficients: E fields, the phase function on
    the 12 x 9 grid and its azimuthal mean, the Legendre fit and the degrees of polarisation equal
    the reference's Optics output."""
    g = golden("ref_farfield.npz")
    n = g["positions"].shape[0]
    particles = Particles(g["positions"], g["radii"], np.full(n, complex(g["refractive_index"])))
    field = InitialField(beam_width=0, focal_point=np.zeros(3), polar_angle=0.0, azimuthal_angle=0.0,
                         polarization="TE")
    params = Parameters(np.array([float(g["wavelength"])]), np.array([1.0 + 0j]), particles, field)
    numerics = Numerics(lmax=int(g["lmax"]), sampling_points_number=g["grid"])
    numerics.compute_translation_table()
    sim = Simulation(params, numerics, device=cuda_device)
    sim.compute_mie_coefficients()
    sim.compute_initial_field_coefficients()
    sim.scattered_field_coefficients = g["scattered"][:, :, None].copy()
    opt = Optics(sim)
    opt.compute_cross_sections()
    assert abs(opt.c_sca[0] - g["c_sca"][0]) <= 1e-10 * abs(g["c_sca"][0])
    et, ep = opt.compute_scattered_e_field_angle_components()
    assert _rel(et[:, 0], g["e_theta"]) < 1e-11
    assert _rel(ep[:, 0], g["e_phi"]) < 1e-11
    opt.compute_phase_function(legendre_coefficients_number=8)
    assert _rel(opt.phase_function_3d[:, 0], g["phase_function_3d"]) < 1e-9
    assert _rel(opt.phase_function[:, 0], g["phase_function"]) < 1e-9
    assert _rel(opt.phase_function_legendre_coefficients[:, 0], g["legendre"]) < 1e-8
    assert np.allclose(opt.degree_of_polarization_3d[:, 0], g["dop_3d"], rtol=0, atol=1e-10)
    assert np.allclose(opt.degree_of_polarization[:, 0], g["dop"], rtol=0, atol=1e-10)
    assert np.allclose(opt.scattering_angles, g["scattering_angles"])
