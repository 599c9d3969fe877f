"""GPU parity of the full solve path: device GMRES (yasf_gmres_solve), cross sections, the
block-Jacobi preconditioner, and the drop-in Simulation/Solver/Optics API."""

from __future__ import annotations

import numpy as np
import pytest
import torch
from conftest import rel_err

from yasf_b200 import BlockDiagonalPreconditioner, InitialField, Numerics, Optics, Parameters
from yasf_b200 import Particles, Simulation, Solver
from yasf_b200._lib import YASF_C64, YasfError
from yasf_b200.device import CouplingDevice, DevicePreconditioner
from yasf_b200.wigner import translation_table_ab5

pytestmark = pytest.mark.gpu


def make_sim(g, tol, restart=100, max_iter=1000, precision="c128", preconditioner=None):
    n = g["positions"].shape[0]
    particles = Particles(g["positions"], g["radii"], np.full(n, complex(g["refractive_index"])))
    field = InitialField(beam_width=0, focal_point=np.zeros(3), polar_angle=0.0, azimuthal_angle=0.0,
                         polarization="TE")
    params = Parameters(np.array([float(g["wavelength"])]), np.array([1.0 + 0j]), particles, field)
    solver = Solver("gmres", tolerance=tol, max_iter=max_iter, restart=restart,
                    preconditioner=preconditioner)
    numerics = Numerics(lmax=int(g["lmax"]), solver=solver, b200_precision=precision)
    numerics.compute_translation_table()
    sim = Simulation(params, numerics)
    sim.compute_mie_coefficients()
    sim.compute_initial_field_coefficients()
    sim.compute_right_hand_side()
    return sim


def test_solve_matches_reference_1e10(golden, cuda_device):
    """Both solves converged far below 1e-10 (rtol 1e-13): coefficients and C_ext/C_sca to 1e-10."""
    g = golden("ref_solve_c1_tol1e-13.npz")
    sim = make_sim(g, 1e-13)
    sim.compute_scattered_field_coefficients()
    assert sim.scattered_field_err_codes[0] == 0
    b = sim.scattered_field_coefficients[:, :, 0]
    assert rel_err(b, g["scattered"]) < 1e-10
    opt = Optics(sim)
    opt.compute_cross_sections()
    assert abs(opt.c_ext[0] - float(g["c_ext"])) < 1e-10 * abs(float(g["c_ext"]))
    assert abs(opt.c_sca[0] - float(g["c_sca"])) < 1e-10 * abs(float(g["c_sca"]))


def test_solve_at_reference_tolerance(golden, cuda_device):
    """At the config tolerance (1e-8) both solves land within the tolerance of the exact solution."""
    g = golden("ref_solve_c1_tol1e-8.npz")
    exact = golden("ref_solve_c1_tol1e-13.npz")["scattered"]
    sim = make_sim(g, 1e-8)
    sim.compute_scattered_field_coefficients()
    st = sim.solver_stats[0]
    assert st["info"] == 0 and st["relative_residual"] <= 1e-8
    assert rel_err(sim.scattered_field_coefficients[:, :, 0], exact) < 1e-6
    assert rel_err(g["scattered"], exact) < 1e-6


def test_cross_sections_of_reference_coefficients(golden, cuda_device):
    """C_sca kernel (regular translation, self pairs) on the reference's own coefficients."""
    g = golden("ref_solve_c1_tol1e-13.npz")
    sim = make_sim(g, 1e-13)
    sim.scattered_field_coefficients = g["scattered"][:, :, None]
    sim.initial_field_coefficients = g["initial"][:, :, None]
    opt = Optics(sim)
    opt.compute_cross_sections()
    assert abs(opt.c_sca[0] - float(g["c_sca"])) < 1e-11 * float(g["c_sca"])
    assert abs(opt.c_ext[0] - float(g["c_ext"])) < 1e-12 * float(g["c_ext"])


def test_mixed_precision_refinement(golden, cuda_device):
    g = golden("ref_solve_c1_tol1e-13.npz")
    sim = make_sim(g, 1e-10, precision="c64")
    sim.compute_scattered_field_coefficients()
    st = sim.solver_stats[0]
    assert st["info"] == 0 and st["relative_residual"] <= 1e-10
    assert st["refinement_steps"] >= 1 and st["matvecs_inner"] > st["matvecs_f64"]
    assert rel_err(sim.scattered_field_coefficients[:, :, 0], g["scattered"]) < 1e-8
    opt = Optics(sim)
    opt.compute_cross_sections()
    assert abs(opt.c_ext[0] - float(g["c_ext"])) < 1e-6 * float(g["c_ext"])


def test_preconditioner_blocks_match_reference(golden, cuda_device):
    g = golden("ref_precond_blocks.npz")
    lmax = int(g["lmax"])
    dev = CouplingDevice(lmax, translation_table_ab5(lmax), g["positions"], 2 * np.pi / float(g["wavelength"]),
                         cuda_device)
    blocks = [g[f"particles{b}"] for b in range(int(g["n_blocks"]))]
    pc = DevicePreconditioner(dev, blocks)
    tmat = torch.from_numpy(g["tmat"]).to(cuda_device)
    from yasf_b200 import _lib
    from yasf_b200.device import _ptr, _stream_ptr

    _lib.call("yasf_precond_assemble", pc.handle, _ptr(dev.pos), dev.k, _ptr(tmat), _stream_ptr())
    for b in range(len(blocks)):
        M = pc.block_matrix(b).cpu().numpy()
        assert rel_err(M, g[f"block{b}"]) < 1e-12
    with pytest.raises(YasfError):
        pc.apply(torch.zeros(dev.n, dtype=torch.complex128, device=cuda_device))  # not finalized
    pc.prepare(tmat, keep_float64=True)  # the library's block LU; complex128 factors kept
    rng = np.random.default_rng(0)
    y = rng.normal(size=dev.n) + 1j * rng.normal(size=dev.n)
    # M y block by block, then apply(M y) must return y
    My = np.zeros_like(y)
    nmax = dev.nmax
    for b, blk in enumerate(blocks):
        idx = (blk[:, None] * nmax + np.arange(nmax)[None, :]).ravel()
        My[idx] = g[f"block{b}"] @ y[idx]
    out = pc.apply(torch.from_numpy(My).to(cuda_device)).cpu().numpy()
    assert rel_err(out, y) < 1e-12
    out64 = pc.apply(torch.from_numpy(My).to(cuda_device), YASF_C64).cpu().numpy()
    assert rel_err(out64, y) < 1e-5


def test_preconditioned_solve_same_solution(golden, cuda_device):
    g = golden("ref_solve_c1_tol1e-13.npz")
    pos = g["positions"]
    edges = (pos.max(axis=0) - pos.min(axis=0) + 2.0) / 2.0
    pre = BlockDiagonalPreconditioner(edges)
    sim = make_sim(g, 1e-13, preconditioner=pre)
    pre.prepare(sim)
    assert any(len(b) > 1 for b in pre.partitioning)
    sim.compute_scattered_field_coefficients()
    assert sim.scattered_field_err_codes[0] == 0
    assert rel_err(sim.scattered_field_coefficients[:, :, 0], g["scattered"]) < 1e-10
    # host apply of a block-identity input (API parity)
    out = pre.apply(np.zeros(sim.device_state().n, dtype=complex))
    assert np.all(out == 0)


def test_singleton_blocks_are_identity(golden, cuda_device):
    """The reference's only preconditioner case (3 spheres, 3 singleton cells): M = I."""
    g = golden("celes_full_simulation.npz")
    n = 3
    particles = Particles(g["positions"], g["radii"], g["refractive_index"])
    field = InitialField(beam_width=0, focal_point=np.zeros(3), polarization="TE")
    params = Parameters(np.array([float(g["wavelength"])]), np.array([float(g["medium_index"])]),
                        particles, field)
    pre = BlockDiagonalPreconditioner(np.array([100.0, 100.0, 100.0]))
    solver = Solver("gmres", tolerance=1e-10, max_iter=100, restart=100, preconditioner=pre)
    numerics = Numerics(lmax=int(g["lmax"]), solver=solver)
    numerics.compute_translation_table()
    sim = Simulation(params, numerics)
    sim.compute_mie_coefficients()
    pre.prepare(sim)
    assert len(pre.partitioning) == n
    rhs = np.random.default_rng(0).normal(size=sim.device_state().n).astype(complex)
    np.testing.assert_allclose(pre.apply(rhs), rhs, rtol=0, atol=0)
    sim.compute_initial_field_coefficients()
    sim.compute_right_hand_side()
    sim.compute_scattered_field_coefficients()
    np.testing.assert_allclose(sim.scattered_field_coefficients[:, :, 0], g["scattered"], rtol=1e-3,
                               atol=1e-5)


def test_drop_in_api_shapes(golden, cuda_device):
    g = golden("ref_multichannel.npz")
    particles = Particles(g["positions"], g["radii"], np.full(3, 1.5 + 0j))
    field = InitialField(beam_width=0, focal_point=np.zeros(3), polarization="TE")
    params = Parameters(g["wavelengths"], np.array([1.0 + 0j, 1.0 + 0j]), particles, field)
    numerics = Numerics(lmax=2, solver=Solver("gmres", 1e-6, 20, 20))
    numerics.compute_translation_table()
    sim = Simulation(params, numerics)
    assert sim.sph_h is None and sim.plm is None and sim.e_j_dm_phi is None
    assert sim.coupling_backend.requires_pairwise_lookups is False
    wx_all = sim.coupling_matrix_multiply(g["x"])
    assert wx_all.shape == g["wx_all"].shape
    assert rel_err(wx_all, g["wx_all"]) < 1e-12
    wx_1 = sim.coupling_matrix_multiply(g["x"], idx=1)
    assert wx_1.shape == g["wx_1"].shape
    assert rel_err(wx_1, g["wx_1"]) < 1e-12


def test_errors_are_loud(cuda_device):
    particles = Particles(np.zeros((2, 3)) + [[0, 0, 0], [1, 0, 0]], np.array([0.1, 0.1]),
                          np.array([1.5, 1.5], dtype=complex))
    field = InitialField(beam_width=0, focal_point=np.zeros(3))
    params = Parameters(np.array([1.0]), np.array([1.0 + 0.1j]), particles, field)
    numerics = Numerics(lmax=2, solver=Solver())
    with pytest.raises(ValueError):
        Simulation(params, Numerics(lmax=2, coupling_backend="dense"))
    sim = Simulation(params, numerics)
    with pytest.raises(NotImplementedError):  # absorbing medium
        sim.coupling_matrix_multiply(np.zeros(2 * numerics.nmax, dtype=complex), idx=0)
    params_ok = Parameters(np.array([1.0]), np.array([1.0 + 0j]), particles, field)
    sim = Simulation(params_ok, numerics)
    sim.compute_mie_coefficients()
    sim.compute_initial_field_coefficients()
    sim.compute_right_hand_side()
    sim.right_hand_side[0, 0, 0] = np.nan
    with pytest.raises(FloatingPointError):
        sim.compute_scattered_field_coefficients()
    with pytest.raises(NotImplementedError):
        Solver("bicgstab").run(None, np.zeros(4, dtype=complex))


def test_solve_matches_celes500(golden, cuda_device):
    """The reference's tests/test_celes.py case through the drop-in API: 500 spheres (CELES export,
    three radii and refractive indices), lmax 3, medium index 1.63, TE plane wave along +z.
    CELES stopped its solver at 5e-4, so the comparison is norm-wise at the reference's 2e-3 (an
    accurate solution differs from CELES by 3.5e-4; elementwise 2e-3 fails for the smallest
    coefficients even then). The device solution also solves the oracle's system to 1e-8."""
    from oracle import restate as R

    g = golden("celes_500.npz")
    particles = Particles(g["positions"], g["radii"], g["refractive_index"])
    field = InitialField(beam_width=0, focal_point=np.zeros(3), polar_angle=float(g["polar"]),
                         azimuthal_angle=float(g["azimuthal"]), polarization=str(g["polarization"]).strip())
    params = Parameters(np.array([float(g["wavelength"])]), np.array([complex(g["medium_index"])]),
                        particles, field)
    lmax = int(g["lmax"])
    numerics = Numerics(lmax=lmax, solver=Solver("gmres", tolerance=1e-10, max_iter=100, restart=50))
    numerics.compute_translation_table()
    sim = Simulation(params, numerics)
    sim.compute_mie_coefficients()
    sim.compute_initial_field_coefficients()
    sim.compute_right_hand_side()
    sim.compute_scattered_field_coefficients()
    assert sim.scattered_field_err_codes[0] == 0
    x = sim.scattered_field_coefficients[:, :, 0]
    assert rel_err(x, g["scattered"]) < 2e-3
    tm = sim.mie_coefficients[particles.single_unique_array_idx, :, 0].ravel()
    b = sim.right_hand_side[:, :, 0].ravel()
    k = float(params.k_medium[0].real)
    r = R.master_matvec(lmax, g["positions"], k, translation_table_ab5(lmax), tm, x.ravel()) - b
    assert np.linalg.norm(r) / np.linalg.norm(b) < 1e-8
