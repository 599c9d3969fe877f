"""Generate the golden fixtures in tests/golden/ by running the upstream reference itself.

Run in a container where the reference ``yasfpy`` source tree is available (read-only); its
location must be given in ``$YASF_REFERENCE`` (there is no default):

    YASF_REFERENCE=<path to the yasfpy checkout> python tests/golden/make_golden.py [part ...]

Parts: ``tables`` (CELES goldens and translation tables lmax 1-6), ``c1``, ``l78`` (translation
tables lmax 7 and 8 and reference matvec fixtures at those orders), ``nearfar`` (the near-field
backend), ``celes500``, ``farfield`` (the scattered far field, Stokes parameters and phase function
of a solved aggregate on a 2-D sampling grid; run alone, with the reference's Numba loops on one
thread: its far-field loop adds into shared array elements from a parallel loop); no part = all.

The reference imports with the stand-ins from ``oracle/stubs`` (pywigxjpf via sympy's exact 3j,
refidxdb and pyperf as inert stand-ins). Two kinds of fixtures are written:

- ``celes_*.npz``: the MATLAB/CELES golden vectors that the reference's own tests hold
  (reference tests/data/*.mat, read by tests/test_comparison.py and tests/test_full_simulation.py,
  and the 500-sphere CELES export tests/data/celes_*.fits, read by tests/test_celes.py),
  converted to particle-major numpy arrays.
- ``ref_*.npz``: outputs of the reference code path on seeded synthetic inputs (coupling matvec,
  master operator, Mie / incident / right-hand side, GMRES solve, cross sections, and the
  preconditioner block matrices assembled column by column from the reference's own
  master_matrix_multiply).

Nothing reads the reference at test or bench time: the fixtures are committed.
"""

from __future__ import annotations

import os
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
REPO = HERE.parents[1]
if not os.environ.get("YASF_REFERENCE"):
    sys.exit("make_golden.py: set YASF_REFERENCE to the reference (yasfpy) source tree")
REF = Path(os.environ["YASF_REFERENCE"])
sys.path.insert(0, str(REPO))
sys.path.insert(0, str(REPO / "oracle" / "stubs"))
sys.path.insert(0, str(REF))
# the reference caches its translation tables under $HOME: keep that cache in a temporary directory
os.environ["HOME"] = tempfile.mkdtemp(prefix="yasf_golden_home_")
if sys.argv[1:] == ["farfield"]:  # serial Numba loops (set before numba is imported)
    os.environ["NUMBA_NUM_THREADS"] = "1"

from scipy.io import loadmat  # noqa: E402

from yasf_b200.workloads import aggregate_c1, rsa_ball, rsa_cube  # noqa: E402


def ref_modules():
    from yasfpy.initial_field import InitialField
    from yasfpy.numerics import Numerics
    from yasfpy.optics import Optics
    from yasfpy.parameters import Parameters
    from yasfpy.particles import Particles
    from yasfpy.simulation import Simulation
    from yasfpy.solver import Solver

    return InitialField, Numerics, Optics, Parameters, Particles, Simulation, Solver


def ref_simulation(positions, radii, m, wavelength, lmax, tol=1e-8, restart=100, max_iter=1000,
                   polar=0.0, azimuthal=0.0, pol="TE", wavelengths=None, sampling=(10,)):
    InitialField, Numerics, Optics, Parameters, Particles, Simulation, Solver = ref_modules()
    n = positions.shape[0]
    particles = Particles(position=positions, r=radii, refractive_index=np.full(n, m, dtype=complex))
    field = InitialField(beam_width=0, focal_point=np.zeros(3), polar_angle=polar,
                         azimuthal_angle=azimuthal, polarization=pol)
    wl = np.atleast_1d(wavelength if wavelengths is None else wavelengths).astype(float)
    params = Parameters(wavelength=wl, medium_refractive_index=np.ones(wl.size, dtype=complex),
                        particles=particles, initial_field=field)
    solver = Solver(solver_type="gmres", tolerance=tol, max_iter=max_iter, restart=restart)
    numerics = Numerics(lmax=lmax, sampling_points_number=np.array(sampling), gpu=False, solver=solver,
                        coupling_backend="dense")
    numerics.compute_translation_table()
    sim = Simulation(params, numerics)
    return sim, Optics


def save(name: str, **arrays):
    path = HERE / name
    np.savez_compressed(path, **arrays)
    print(f"wrote {path.name} ({path.stat().st_size / 1024:.0f} KiB)")


def celes_fixtures():
    data = REF / "tests" / "data"
    d = loadmat(data / "coupling_matrix_multiply_data.mat")
    lmax = int(d["lmax"][0, 0])
    nmax = 2 * lmax * (lmax + 2)
    npart = d["particles_position"].shape[0]
    to_pm = lambda v: v.flatten().reshape((nmax, npart)).T.flatten()  # noqa: E731
    save("celes_coupling.npz", lmax=lmax, wavelength=float(d["wavelength"][0, 0]),
         medium_index=float(d["mediumRefractiveIndex"][0, 0]),
         positions=d["particles_position"].astype(float),
         radii=d["particles_radius"].flatten().astype(float),
         refractive_index=d["particles_refractiveIndex"].flatten(),
         x=to_pm(d["input_x"]), wx=to_pm(d["coupling_matrix_output_Wx"]).astype(np.complex128))
    t = loadmat(data / "translation_table_ab_data.mat")
    save("celes_translation_lmax3.npz", table=t["translation_table_tta"]["ab5"][0, 0].astype(np.complex128))
    f = loadmat(data / "full_simulation_data.mat")
    save("celes_full_simulation.npz", lmax=int(f["lmax"][0, 0]), wavelength=float(f["wavelength"][0, 0]),
         medium_index=float(f["mediumRefractiveIndex"][0, 0]),
         positions=f["particles_position"].astype(float),
         radii=f["particles_radius"].flatten().astype(float),
         refractive_index=f["particles_refractiveIndex"].flatten(),
         initial=f["initial_field_coefficients"].astype(np.complex128),
         mie=f["mie_coefficients"].astype(np.complex128),
         scattered=f["scattered_field_coefficients"].astype(np.complex128))


def read_fits(path: Path) -> list[tuple[dict, list[int], bytes]]:
    """Minimal FITS reader (headers, including HIERARCH cards, and the raw big-endian data of each
    HDU): enough for the reference's CELES export, read without astropy."""
    raw = path.read_bytes()
    pos, hdus = 0, []
    while pos < len(raw):
        cards, end = {}, False
        while not end:
            block = raw[pos:pos + 2880]
            pos += 2880
            for i in range(36):
                c = block[i * 80:(i + 1) * 80].decode("ascii")
                if c[:8].strip() == "END":
                    end = True
                    break
                if c.startswith("HIERARCH"):
                    key, _, val = c[9:].partition("=")
                elif c[8:10] == "= ":
                    key, val = c[:8], c[10:]
                else:
                    continue
                val = val.strip()
                val = val.split("'")[1] if val.startswith("'") else val.split("/")[0].strip()
                cards[key.strip()] = val
        naxis = int(cards.get("NAXIS", 0))
        dims = [int(cards[f"NAXIS{i}"]) for i in range(1, naxis + 1)]
        size = (abs(int(cards.get("BITPIX", 8))) // 8 * int(np.prod(dims)) + int(cards.get("PCOUNT", 0))) if naxis else 0
        hdus.append((cards, dims, raw[pos:pos + size]))
        pos += (size + 2879) // 2880 * 2880
    return hdus


def celes_fits_fixture():
    """The 500-sphere CELES export the reference's tests/test_celes.py checks (HDU 1 particles,
    HDU 3 incident field, HDU 4 wavelength and medium, HDU 6 solver, HDU 7 lmax, HDU 8 incident and
    scattered coefficients as (4, N, nmax): re/im incident, re/im scattered)."""
    hdus = read_fits(REF / "tests" / "data" / "celes_2023-05-09_21-00-48.fits")
    part = np.frombuffer(hdus[1][2], dtype=">f8").reshape(-1, 6).astype(float)  # x y z r n k
    inp = hdus[4][2]
    wavelength = float(np.frombuffer(inp[0:8], dtype=">f8")[0])
    medium = np.frombuffer(inp[8:24], dtype=">f8").astype(float)
    c8, d8, b8 = hdus[8]
    coeff = np.frombuffer(b8, dtype=">f8").reshape(d8[::-1]).astype(float)  # (4, N, nmax)
    field = hdus[3][0]
    save("celes_500.npz", lmax=int(float(hdus[7][0]["L MAX"])), wavelength=wavelength,
         medium_index=complex(medium[0], medium[1]), positions=part[:, :3], radii=part[:, 3],
         refractive_index=part[:, 4] + 1j * part[:, 5],
         polar=float(field["POLAR ANGLE"]), azimuthal=float(field["AZIMUTHAL ANGLE"]),
         polarization=field["POLARIZATION"], tolerance=float(hdus[6][0]["TOLERANCE"]),
         initial=coeff[0] + 1j * coeff[1], scattered=coeff[2] + 1j * coeff[3])


def translation_fixtures(lmax_values=(1, 2, 3, 4, 5, 6), name="ref_translation.npz"):
    _, Numerics, *_ = ref_modules()
    out = {}
    for L in lmax_values:
        t0 = time.time()
        num = Numerics(lmax=L, sampling_points_number=np.array([10]))
        num.compute_translation_table(force_compute=True)
        out[f"lmax{L}"] = num.translation_ab5
        print(f"  translation table lmax={L}: {time.time() - t0:.1f}s", flush=True)
    save(name, **out)


def high_order_fixtures():
    """lmax 7 and 8 (the serving stream draws lmax up to 8): the reference's own translation
    tables and coupling / master matvecs of small seeded aggregates at those orders."""
    translation_fixtures((7, 8), name="ref_translation_l78.npz")
    rng = np.random.default_rng(17)
    r7 = rng.uniform(0.05, 0.2, size=10)
    p7 = rsa_cube(r7, 0.15, rng, max_attempts=200_000)
    matvec_fixture("ref_matvec_l7.npz", p7, r7, 1.7 + 0.01j, 0.45, 7, seed=14)
    rng = np.random.default_rng(19)
    r8 = rng.uniform(0.05, 0.2, size=9)
    p8 = rsa_cube(r8, 0.12, rng, max_attempts=200_000)
    matvec_fixture("ref_matvec_l8.npz", p8, r8, 1.35 + 0.05j, 0.4, 8, seed=15)


def matvec_fixture(name, positions, radii, m, wavelength, lmax, seed):
    sim, _ = ref_simulation(positions, radii, m, wavelength, lmax)
    rng = np.random.default_rng(seed)
    n = positions.shape[0] * sim.numerics.nmax
    x = rng.normal(size=n) + 1j * rng.normal(size=n)
    wx = sim.coupling_matrix_multiply(x, idx=0)
    sim.compute_mie_coefficients()
    mx = sim.master_matrix_multiply(x, 0)
    sidx = sim.parameters.particles.single_unique_array_idx
    tmat = sim.mie_coefficients[sidx, :, 0].ravel()
    save(name, lmax=lmax, wavelength=wavelength, refractive_index=m, positions=positions, radii=radii,
         x=x, wx=wx, mx=mx, tmat=tmat)


def multichannel_fixture():
    pos = np.array([[0.0, 0.0, 0.0], [1.0, 0.0, 0.0], [0.25, 0.5, 0.0]])
    radii = np.array([0.1, 0.1, 0.1])
    sim, _ = ref_simulation(pos, radii, 1.5 + 0.0j, None, 2, wavelengths=np.array([1.0, 1.3]))
    rng = np.random.default_rng(0)
    n = 3 * sim.numerics.nmax
    x = rng.normal(size=n) + 1j * rng.normal(size=n)
    save("ref_multichannel.npz", lmax=2, wavelengths=np.array([1.0, 1.3]), positions=pos, radii=radii,
         x=x, wx_all=sim.coupling_matrix_multiply(x), wx_1=sim.coupling_matrix_multiply(x, idx=1))


def solve_fixture(name, agg, tol, restart=100):
    sim, Optics = ref_simulation(agg.positions, agg.radii, agg.refractive_index, agg.wavelength, agg.lmax,
                                 tol=tol, restart=restart)
    t0 = time.time()
    sim.compute_mie_coefficients()
    sim.compute_initial_field_coefficients()
    sim.compute_right_hand_side()
    sim.compute_scattered_field_coefficients()
    t_solve = time.time() - t0
    opt = Optics(sim)
    opt.compute_cross_sections()
    sidx = sim.parameters.particles.single_unique_array_idx
    save(name, lmax=agg.lmax, wavelength=agg.wavelength, refractive_index=agg.refractive_index,
         positions=agg.positions, radii=agg.radii, tol=tol,
         mie=sim.mie_coefficients[:, :, 0], sidx=sidx,
         initial=sim.initial_field_coefficients[:, :, 0], rhs=sim.right_hand_side[:, :, 0],
         scattered=sim.scattered_field_coefficients[:, :, 0],
         err_code=sim.scattered_field_err_codes[0], c_ext=float(opt.c_ext[0]),
         c_sca=float(opt.c_sca[0]), solve_seconds=t_solve)
    print(f"  {name}: C_ext={opt.c_ext[0]:.10g} C_sca={opt.c_sca[0]:.10g} ({t_solve:.1f}s)")


def nearfar_fixture():
    """The reference's NearFarCouplingBackend (near-field pairs only, yasfpy/coupling/
    backends.py:259-459) on a seeded aggregate, with its dense W x for comparison."""
    rng = np.random.default_rng(23)
    radii = rng.uniform(0.05, 0.12, size=40)
    pos = rsa_cube(radii, 0.12, rng, max_attempts=200_000)
    lmax, wl, m, radius = 3, 0.55, 1.5 + 0.01j, 0.6
    sim, _ = ref_simulation(pos, radii, m, wl, lmax)
    sim.numerics.coupling_near_field_radius = radius
    sim.numerics.coupling_tile_size = 16
    from yasfpy.coupling.backends import NearFarCouplingBackend

    n = pos.shape[0] * sim.numerics.nmax
    x = rng.normal(size=n) + 1j * rng.normal(size=n)
    wx_dense = sim.coupling_matrix_multiply(x, idx=0)
    wx_near = NearFarCouplingBackend(sim).multiply(x, idx=0)
    save("ref_matvec_nearfar.npz", lmax=lmax, wavelength=wl, positions=pos, radii=radii,
         near_field_radius=radius, x=x, wx_near=np.asarray(wx_near).reshape(-1),
         wx_dense=np.asarray(wx_dense).reshape(-1))


def precond_fixture():
    """Reference-derived block matrices for a geometry whose cells hold several spheres."""
    from yasfpy.preconditioner import make_particle_partition

    rng = np.random.default_rng(7)
    radii = rng.uniform(0.05, 0.1, size=10)
    pos = rsa_cube(radii, 0.10, rng, max_attempts=200_000)
    lmax = 2
    sim, _ = ref_simulation(pos, radii, 1.55 + 0.02j, 0.6, lmax)
    sim.compute_mie_coefficients()
    extent = pos.max(axis=0) - pos.min(axis=0)
    edges = (extent + 2.0) / 2.0
    blocks = make_particle_partition(pos, edges)
    nmax = sim.numerics.nmax
    mats = {}
    for b, blk in enumerate(blocks):
        idx = (blk[:, None] * nmax + np.arange(nmax)[None, :]).ravel()
        M = np.zeros((idx.size, idx.size), dtype=complex)
        for c, gi in enumerate(idx):
            e = np.zeros(pos.shape[0] * nmax, dtype=complex)
            e[gi] = 1.0
            M[:, c] = sim.master_matrix_multiply(e, 0)[idx]
        mats[f"block{b}"] = M
        mats[f"particles{b}"] = blk
    sidx = sim.parameters.particles.single_unique_array_idx
    save("ref_precond_blocks.npz", lmax=lmax, wavelength=0.6, refractive_index=1.55 + 0.02j,
         positions=pos, radii=radii, edges=edges, n_blocks=len(blocks),
         tmat=sim.mie_coefficients[sidx, :, 0].ravel(), **mats)


def farfield_fixture():
    """The reference's Optics far field on a solved aggregate: E_theta, E_phi
    (compute_scattered_e_field_angle_components, yasfpy/optics.py:178-267) and the phase function
    with its degrees of polarisation (compute_phase_function, :752-1038) on a 2-D sampling grid."""
    rng = np.random.default_rng(31)
    radii = rng.uniform(0.05, 0.1, size=24)
    pos = rsa_cube(radii, 0.15, rng, max_attempts=200_000)
    lmax, wl, m = 3, 0.55, 1.5 + 0.01j
    grid = np.array([12, 9])  # azimuthal x polar sampling points
    sim, Optics = ref_simulation(pos, radii, m, wl, lmax, tol=1e-12, sampling=grid)
    sim.numerics.compute_spherical_unity_vectors()  # as yasfpy/yasf.py:172 does before optics
    sim.compute_mie_coefficients()
    sim.compute_initial_field_coefficients()
    sim.compute_right_hand_side()
    sim.compute_scattered_field_coefficients()
    opt = Optics(sim)
    opt.compute_cross_sections()
    e_theta, e_phi = opt.compute_scattered_e_field_angle_components()
    opt.compute_phase_function(legendre_coefficients_number=8)
    save("ref_farfield.npz", lmax=lmax, wavelength=wl, refractive_index=m, positions=pos, radii=radii,
         grid=grid, polar=sim.numerics.polar_angles, azimuthal=sim.numerics.azimuthal_angles,
         scattered=sim.scattered_field_coefficients[:, :, 0], c_sca=opt.c_sca, c_ext=opt.c_ext,
         e_theta=e_theta[:, 0], e_phi=e_phi[:, 0], phase_function_3d=opt.phase_function_3d[:, 0],
         phase_function=opt.phase_function[:, 0],
         legendre=opt.phase_function_legendre_coefficients[:, 0],
         dop_3d=opt.degree_of_polarization_3d[:, 0], dolp_3d=opt.degree_of_linear_polarization_3d[:, 0],
         dolq_3d=opt.degree_of_linear_polarization_q_3d[:, 0],
         dolu_3d=opt.degree_of_linear_polarization_u_3d[:, 0],
         docp_3d=opt.degree_of_circular_polarization_3d[:, 0],
         dop=opt.degree_of_polarization[:, 0], scattering_angles=opt.scattering_angles)


def main():
    t0 = time.time()
    only = set(sys.argv[1:])
    if only == {"farfield"}:
        farfield_fixture()
        return
    if not only or "tables" in only:
        celes_fixtures()
        celes_fits_fixture()
        translation_fixtures()
    if only == {"celes500"}:
        celes_fits_fixture()
        return
    if only == {"l78"}:
        high_order_fixtures()
        return
    if only == {"nearfar"}:
        nearfar_fixture()
        return
    c1 = aggregate_c1(seed=0)
    if not only or "c1" in only:
        matvec_fixture("ref_matvec_c1.npz", c1.positions, c1.radii, c1.refractive_index,
                       c1.wavelength, c1.lmax, seed=11)
    rng = np.random.default_rng(3)
    r6 = np.clip(rng.lognormal(np.log(0.1), 0.2, size=12), 0.04, 0.25)
    p6 = rsa_ball(r6, 0.08, rng, max_attempts=200_000)
    matvec_fixture("ref_matvec_l6.npz", p6, r6, 1.6 + 0.005j, 0.6, 6, seed=12)
    rng = np.random.default_rng(5)
    r3 = rng.uniform(0.05, 0.15, size=9)
    p3 = rsa_cube(r3, 0.12, rng, max_attempts=200_000)
    matvec_fixture("ref_matvec_l3.npz", p3, r3, 1.45 + 0.03j, 0.5, 3, seed=13)
    multichannel_fixture()
    nearfar_fixture()
    solve_fixture("ref_solve_c1_tol1e-8.npz", c1, 1e-8)
    solve_fixture("ref_solve_c1_tol1e-13.npz", c1, 1e-13)
    precond_fixture()
    print(f"done in {time.time() - t0:.0f}s")


if __name__ == "__main__":
    main()
