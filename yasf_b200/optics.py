"""Cross sections and far-field quantities from the solved coefficients (yasfpy/optics.py).

C_ext = pi/|k|^2 Re(-sum conj(a) b) and C_sca = pi/|k|^2 |sum conj(b) W_reg b| where W_reg is the
regular (j_p) translation including self pairs (yasfpy/functions/cpu_numba.py:410-457); both are
evaluated on the device. The scattered far field on the sampling directions (E_theta, E_phi and
the Stokes parameters) is the device kernel of yasf_far_field (yasfpy/optics.py:178-267,
cpu_numba.py:536-660); the phase function, its Legendre fit, the degrees of polarisation, the
double Henyey-Greenstein fit and the asymmetry parameter are the reference's host post-processing
of those arrays (yasfpy/optics.py:574-1038), kept as they are.
"""

from __future__ import annotations

import logging

import numpy as np
import torch


class Optics:
    def __init__(self, simulation):
        self.simulation = simulation
        self.c_ext = np.zeros_like(simulation.parameters.wavelength, dtype=complex)
        self.c_sca = np.zeros_like(simulation.parameters.wavelength, dtype=complex)
        self.log = logging.getLogger(self.__class__.__module__)

    def compute_cross_sections(self):
        sim = self.simulation
        a = sim.initial_field_coefficients
        f = sim.scattered_field_coefficients
        W = sim.parameters.wavelengths_number
        c_ext = np.zeros(W, dtype=complex)
        c_sca = np.zeros(W, dtype=complex)
        for w in range(W):
            dev = sim.device_state(w)
            at = torch.from_numpy(np.ascontiguousarray(a[:, :, w].ravel())).to(dev.device)
            bt = torch.from_numpy(np.ascontiguousarray(f[:, :, w].ravel())).to(dev.device)
            c_ext[w] = -dev.dotc(at, bt)
            c_sca[w] = dev.scattering_bilinear(bt)
        k2 = np.power(np.abs(sim.parameters.k_medium), 2)
        self.c_ext = np.real(c_ext / k2) * np.pi
        self.c_sca = np.abs(c_sca / k2) * np.pi
        self.albedo = self.c_sca / self.c_ext

    def compute_efficiencies(self):
        p = self.simulation.parameters
        self.q_sca = self.c_sca / p.particles.geometric_projection * np.abs(p.medium_refractive_index)
        self.q_ext = self.c_ext / p.particles.geometric_projection * np.abs(p.medium_refractive_index)

    # ---- far field (yasfpy/optics.py:178-267, 574-1038) --------------------------------------------
    def _far_field(self, stokes: bool):
        sim = self.simulation
        num = sim.numerics
        polar = np.asarray(num.polar_angles, dtype=float).ravel()
        azim = np.asarray(num.azimuthal_angles, dtype=float).ravel()
        W = sim.parameters.wavelengths_number
        e_t = np.zeros((polar.size, W), dtype=complex)
        e_p = np.zeros_like(e_t)
        S = np.zeros((polar.size, 4, W)) if stokes else None
        for w in range(W):
            dev = sim.device_state(w)
            coef = torch.from_numpy(np.ascontiguousarray(sim.scattered_field_coefficients[:, :, w].ravel()))
            et, ep, st = dev.far_field(coef.to(dev.device), polar, azim, stokes=stokes)
            e_t[:, w] = et.cpu().numpy()
            e_p[:, w] = ep.cpu().numpy()
            if stokes:
                S[:, :, w] = st.cpu().numpy()
        return e_t, e_p, S

    def compute_scattered_e_field_angle_components(self):
        """(e_field_theta, e_field_phi), each (sampling directions, wavelengths) complex, of the
        scattered far field (yasfpy/optics.py:178-267), from the device kernel."""
        e_t, e_p, _ = self._far_field(stokes=False)
        return e_t, e_p

    def compute_phase_function(self, legendre_coefficients_number: int = 15, c_and_b=False,
                               check_phase_function: bool = False):
        """Phase function and degrees of polarisation on the sampling grid (yasfpy/optics.py:752-1038).

        The far field and its Stokes parameters come from the device; the reference's host steps
        follow: the normalisation I 4 pi / |k|^2 / C_sca (needs compute_cross_sections first), the
        Legendre fit over cos(theta), the azimuthal means on a (azimuthal x polar) grid, and the
        optional double Henyey-Greenstein fit. ``check_phase_function`` is not supported: the
        reference's check (yasfpy/optics.py:553-572) indexes the phase function with angle values."""
        if check_phase_function:
            raise NotImplementedError("check_phase_function: the reference's check indexes the phase "
                                      "function with angle values (yasfpy/optics.py:553-572)")
        sim = self.simulation
        _, _, S = self._far_field(stokes=True)
        intensity, q, u, v = S[:, 0, :], S[:, 1, :], S[:, 2, :], S[:, 3, :]
        with np.errstate(divide="ignore", invalid="ignore"):
            dop = np.sqrt(q**2 + u**2 + v**2) / intensity
            dolp = np.sqrt(q**2 + u**2) / intensity
            dolq = -q / intensity
            dolu = u / intensity
            docp = v / intensity
        self.scattering_angles = np.asarray(sim.numerics.polar_angles, dtype=float).ravel()
        k_medium = np.asarray(sim.parameters.k_medium)
        self.phase_function_3d = intensity * 4 * np.pi / np.power(np.abs(k_medium), 2) / self.c_sca[np.newaxis, :]
        self.phase_function_legendre_coefficients = np.polynomial.legendre.legfit(
            np.cos(self.scattering_angles), self.phase_function_3d, legendre_coefficients_number)
        self.degree_of_polarization_3d = dop
        self.degree_of_linear_polarization_3d = dolp
        self.degree_of_linear_polarization_q_3d = dolq
        self.degree_of_linear_polarization_u_3d = dolu
        self.degree_of_circular_polarization_3d = docp
        spn = sim.numerics.sampling_points_number
        if spn is not None and np.asarray(spn).size == 2:
            shape = np.append(spn, k_medium.size)
            self.phase_function = np.mean(np.reshape(self.phase_function_3d, shape), axis=0)
            self.degree_of_polarization = np.mean(np.reshape(dop, shape), axis=0)
            self.degree_of_linear_polarization = np.mean(np.reshape(dolp, shape), axis=0)
            self.degree_of_linear_polarization_q = np.mean(np.reshape(dolq, shape), axis=0)
            self.degree_of_linear_polarization_u = np.mean(np.reshape(dolu, shape), axis=0)
            self.degree_of_circular_polarization = np.mean(np.reshape(docp, shape), axis=0)
            self.scattering_angles = np.reshape(self.scattering_angles, spn)[0, :]
        else:
            self.phase_function = self.phase_function_3d
            self.degree_of_polarization = dop
            self.degree_of_linear_polarization = dolp
            self.degree_of_linear_polarization_q = dolq
            self.degree_of_linear_polarization_u = dolu
            self.degree_of_circular_polarization = docp
        self.c_and_b_bounds = c_and_b
        if isinstance(c_and_b, bool):
            if c_and_b:
                self.c_and_b_bounds = ([-1, 0], [1, 1])
            else:
                return
        self._compute_c_and_b()

    def compute_asymmetry(self):
        """Asymmetry parameter by quadrature of phase_function_3d over the (azimuthal x polar)
        sampling grid (yasfpy/optics.py:574-593)."""
        num = self.simulation.numerics
        spn = np.asarray(num.sampling_points_number)
        d_phi = 2 * np.pi / spn[0]
        d_theta = np.pi / spn[1]
        theta = np.asarray(num.polar_angles, dtype=float).ravel()
        w = np.cos(theta) * d_phi * np.sin(theta) * d_theta
        self.g = (self.phase_function_3d * w[:, np.newaxis]).sum(axis=0) / (4 * np.pi)

    @staticmethod
    def compute_double_henyey_greenstein(theta: np.ndarray, cb: np.ndarray):
        """Double Henyey-Greenstein phase function with (c, b) or (c, b1, b2) (yasfpy/optics.py:682-709)."""
        cb = np.squeeze(cb)
        if cb.size < 2:
            cb = np.array([0, 0.5, 0.5])
        elif cb.size == 2:
            cb = np.append(cb, cb[1])
        elif cb.size > 3:
            cb = cb[:2]
        forward = (1 - cb[1] ** 2) / np.power(1 - 2 * cb[1] * np.cos(theta) + cb[1] ** 2, 3 / 2)
        backward = (1 - cb[2] ** 2) / np.power(1 + 2 * cb[2] * np.cos(theta) + cb[2] ** 2, 3 / 2)
        return (1 - cb[0]) / 2 * forward + (1 + cb[0]) / 2 * backward

    def _compute_c_and_b(self):
        """Least-squares double Henyey-Greenstein fit per wavelength (yasfpy/optics.py:711-750)."""
        from scipy.optimize import least_squares

        if len(self.c_and_b_bounds[0]) not in [2, 3]:
            self.c_and_b_bounds = ([-1, 0], [1, 1])
            self.log.warning("Number of parameters need to be 2 (b,c) or 3 (b1,b2,c). Reverting to two "
                             "parameters (b,c) and setting the bounds to standard: b in [0, 1] and c in [-1, 1]")
        bc0 = np.array([0, 0.5]) if len(self.c_and_b_bounds) == 2 else np.array([0, 0.5, 0.5])
        self.cb = np.empty((self.phase_function.shape[1], len(self.c_and_b_bounds)))
        for w in range(self.phase_function.shape[1]):
            fit = least_squares(
                lambda bc: Optics.compute_double_henyey_greenstein(self.scattering_angles, bc)
                - self.phase_function[:, w],
                bc0, jac="2-point", bounds=self.c_and_b_bounds)
            self.cb[w, :] = fit.x
