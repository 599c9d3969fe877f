"""Pin the oracle (oracle/cpu_ref.c, oracle/restate.py) to the reference before trusting it.

Every check compares the oracle with outputs of the reference itself (ref_*.npz, generated by
tests/golden/make_golden.py from the upstream code) or with the MATLAB/CELES golden vectors the
reference's own tests use (celes_*.npz, from reference tests/data/*.mat), at the tolerances
those tests use.
"""

from __future__ import annotations

import numpy as np
import pytest
from conftest import rel_err
from scipy.special import spherical_jn, spherical_yn

from oracle import restate as R


@pytest.mark.parametrize("x", [1e-3, 0.05, 0.3, 0.84, 1.7, 3.2, 7.5, 12.0, 13.5, 17.0, 31.4, 48.0, 97.0])
def test_oracle_bessel_matches_scipy(x):
    j, y = R.sph_bessel(16, x)
    for p in range(17):
        ej, ey = spherical_jn(p, x), spherical_yn(p, x)
        assert abs(j[p] - ej) <= 1e-12 * abs(ej) + 1e-300
        assert abs(y[p] - ey) <= 1e-12 * abs(ey)


@pytest.mark.parametrize("fixture,lmax", [("ref_matvec_c1.npz", 4), ("ref_matvec_l6.npz", 6),
                                          ("ref_matvec_l3.npz", 3)])
def test_oracle_matvec_matches_reference(golden, fixture, lmax):
    g = golden(fixture)
    tab = golden("ref_translation.npz")[f"lmax{lmax}"]
    k = 2 * np.pi / float(g["wavelength"])
    wx = R.coupling_matvec_rows(lmax, g["positions"], k, tab, g["x"])
    assert rel_err(wx, g["wx"]) < 1e-12
    mx = R.master_matvec(lmax, g["positions"], k, tab, g["tmat"], g["x"])
    assert rel_err(mx, g["mx"]) < 1e-12


def test_oracle_row_sample_consistent(golden):
    g = golden("ref_matvec_c1.npz")
    tab = golden("ref_translation.npz")["lmax4"]
    k = 2 * np.pi / float(g["wavelength"])
    nmax = 48
    part = R.coupling_matvec_rows(4, g["positions"], k, tab, g["x"], 37, 41)
    assert rel_err(part, g["wx"][37 * nmax:41 * nmax]) < 1e-12


def test_oracle_matvec_matches_celes_golden(golden):
    g = golden("celes_coupling.npz")
    lmax = int(g["lmax"])
    tab = golden("ref_translation.npz")[f"lmax{lmax}"]
    k = 2 * np.pi / float(g["wavelength"]) * float(g["medium_index"])
    wx = R.coupling_matvec_rows(lmax, g["positions"], k, tab, g["x"])
    # the MATLAB/CELES output is single precision: reference tolerance (tests/test_comparison.py:228)
    np.testing.assert_allclose(wx, g["wx"], rtol=2e-4, atol=1e-5)


def test_reference_translation_matches_celes(golden):
    ref = golden("ref_translation.npz")["lmax3"]
    celes = golden("celes_translation_lmax3.npz")["table"]
    np.testing.assert_allclose(ref, celes, rtol=1e-5, atol=1e-7)


@pytest.mark.parametrize("fixture", ["ref_solve_c1_tol1e-13.npz"])
def test_oracle_cross_sections_match_reference(golden, fixture):
    g = golden(fixture)
    lmax = int(g["lmax"])
    tab = golden("ref_translation.npz")[f"lmax{lmax}"]
    k = 2 * np.pi / float(g["wavelength"])
    b = g["scattered"].ravel()
    a = g["initial"].ravel()
    c_ext = np.real(-np.vdot(a, b)) / k**2 * np.pi
    c_sca = abs(R.scattering_bilinear_rows(lmax, g["positions"], k, tab, b, threads=0)) / k**2 * np.pi
    assert abs(c_ext - float(g["c_ext"])) <= 1e-12 * abs(float(g["c_ext"]))
    assert abs(c_sca - float(g["c_sca"])) <= 1e-11 * abs(float(g["c_sca"]))


def test_oracle_solve_matches_reference(golden):
    g = golden("ref_solve_c1_tol1e-13.npz")
    lmax = int(g["lmax"])
    tab = golden("ref_translation.npz")[f"lmax{lmax}"]
    k = 2 * np.pi / float(g["wavelength"])
    tmat = g["mie"][g["sidx"]].ravel()
    x, info = R.scipy_gmres_solve(lmax, g["positions"], k, tab, tmat, g["rhs"].ravel(), rtol=1e-13)
    assert info == 0
    assert rel_err(x, g["scattered"].ravel()) < 1e-10


def test_oracle_precond_blocks_match_reference(golden):
    g = golden("ref_precond_blocks.npz")
    lmax = int(g["lmax"])
    tab = golden("ref_translation.npz")[f"lmax{lmax}"]
    k = 2 * np.pi / float(g["wavelength"])
    multi = 0
    for b in range(int(g["n_blocks"])):
        blk = g[f"particles{b}"]
        M = R.block_matrix(lmax, g["positions"], k, tab, g["tmat"], blk)
        assert rel_err(M, g[f"block{b}"]) < 1e-12
        multi += len(blk) > 1
    assert multi > 0, "fixture must hold at least one multi-sphere block"


def test_oracle_near_field_matches_reference_nearfar_backend(golden):
    """The oracle's near-field selection against the reference's NearFarCouplingBackend
    (yasfpy/coupling/backends.py:259-459), and without a cutoff against the reference's dense W x."""
    g = golden("ref_matvec_nearfar.npz")
    lmax = int(g["lmax"])
    k = 2 * np.pi / float(g["wavelength"])
    from yasf_b200.wigner import translation_table_ab5

    table = translation_table_ab5(lmax)
    near = R.coupling_matvec_rows(lmax, g["positions"], k, table, g["x"],
                                  near_field_radius=float(g["near_field_radius"]))
    assert rel_err(near, g["wx_near"]) < 1e-12
    dense = R.coupling_matvec_rows(lmax, g["positions"], k, table, g["x"])
    assert rel_err(dense, g["wx_dense"]) < 1e-12
    assert rel_err(near, dense) > 1e-3  # the cutoff drops pairs that matter


def test_far_field_oracle_matches_reference(golden):
    """The oracle's far field (E_theta, E_phi) and degrees of polarisation equal the reference's own
    Optics output (serial Numba loops) on a solved 24-sphere aggregate, 12 x 9 sampling grid."""
    g = golden("ref_farfield.npz")
    k = 2 * np.pi / float(g["wavelength"])
    et, ep = R.far_field(int(g["lmax"]), g["positions"], k, g["scattered"], g["polar"], g["azimuthal"])
    assert np.abs(et - g["e_theta"]).max() <= 1e-12 * np.abs(g["e_theta"]).max()
    assert np.abs(ep - g["e_phi"]).max() <= 1e-12 * np.abs(g["e_phi"]).max()
    I, dop, dolp, dolq, dolu, docp = R.polarization_components(et, ep)
    pf = I * 4 * np.pi / k**2 / g["c_sca"][0]
    assert np.abs(pf - g["phase_function_3d"]).max() <= 1e-12 * np.abs(pf).max()
    for ours, key in ((dop, "dop_3d"), (dolp, "dolp_3d"), (dolq, "dolq_3d"), (dolu, "dolu_3d"),
                      (docp, "docp_3d")):
        assert np.allclose(ours, g[key], rtol=0, atol=1e-12), key
