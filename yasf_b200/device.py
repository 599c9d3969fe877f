"""Device state behind the ``b200`` coupling backend: translation plans, operands, workspaces.

Storage is torch tensors on a CUDA device (plumbing only); every computation is a call through
the C ABI of ``include/yasf_b200.h``. Vectors are complex128, particle-major (s*nmax + n), with R
right-hand sides stored column after column (leading dimension N*nmax).
"""

from __future__ import annotations

import ctypes
import threading

import numpy as np
import torch

from yasf_b200 import _lib
from yasf_b200._lib import YASF_C64, YASF_C128, call

PRECISIONS = {"c128": YASF_C128, "c64": YASF_C64}


def _stream_ptr(stream: torch.cuda.Stream | None = None) -> ctypes.c_void_p:
    s = stream if stream is not None else torch.cuda.current_stream()
    return ctypes.c_void_p(s.cuda_stream)


def _ptr(t: torch.Tensor | None) -> ctypes.c_void_p:
    return ctypes.c_void_p(0 if t is None else t.data_ptr())


class Plan:
    """A translation plan (the a5/b5 table in the kernels' stream layout) on one device."""

    _cache: dict[tuple[int, int, int], "Plan"] = {}
    _lock = threading.Lock()

    def __init__(self, lmax: int, table: np.ndarray, device: torch.device):
        self.lmax = lmax
        self.nmax = 2 * lmax * (lmax + 2)
        self.device = device
        tab = np.ascontiguousarray(table, dtype=np.complex128)
        if tab.shape != (self.nmax, self.nmax, 2 * lmax + 1):
            raise ValueError(f"translation table has shape {tab.shape}, expected "
                             f"{(self.nmax, self.nmax, 2 * lmax + 1)}")
        handle = ctypes.c_void_p()
        with torch.cuda.device(device):
            call("yasf_plan_create", lmax, tab.ctypes.data_as(ctypes.c_void_p), ctypes.byref(handle))
        self.handle = handle
        nm = ctypes.c_int()
        ent = ctypes.c_longlong()
        terms = ctypes.c_longlong()
        call("yasf_plan_info", handle, ctypes.byref(nm), ctypes.byref(ent), ctypes.byref(terms))
        self.stream_entries = ent.value
        self.source_terms = terms.value

    @classmethod
    def get(cls, lmax: int, table: np.ndarray, device: torch.device) -> "Plan":
        idx = device.index if device.index is not None else torch.cuda.current_device()
        key = (lmax, idx, id(table))
        with cls._lock:
            plan = cls._cache.get(key)
            if plan is None:
                plan = cls(lmax, table, torch.device("cuda", idx))
                cls._cache[key] = plan
            return plan

    def __del__(self):
        h = getattr(self, "handle", None)
        if h is not None and h.value:
            try:
                _lib.load().yasf_plan_destroy(h)
            except Exception:
                pass


class Workspace:
    """A growable device byte buffer (256-byte aligned)."""

    def __init__(self, device: torch.device):
        self.device = device
        self.buf: torch.Tensor | None = None

    def get(self, nbytes: int) -> torch.Tensor:
        if self.buf is None or self.buf.numel() < nbytes:
            self.buf = torch.empty(max(int(nbytes), 256), dtype=torch.uint8, device=self.device)
        return self.buf


class CouplingDevice:
    """Geometry + translation plan of one aggregate at one wavenumber, resident on a GPU."""

    def __init__(self, lmax: int, table: np.ndarray, positions: np.ndarray, k_medium: complex,
                 device: torch.device | str | None = None):
        if device is None:
            device = torch.device("cuda", torch.cuda.current_device())
        device = torch.device(device)
        if device.type != "cuda":
            raise RuntimeError("the b200 backend runs on CUDA devices only")
        k = complex(k_medium)
        if abs(k.imag) > 0.0:
            raise NotImplementedError("the b200 backend supports a non-absorbing medium (real k) only")
        self.k = float(k.real)
        self.lmax = lmax
        self.nmax = 2 * lmax * (lmax + 2)
        self.device = device
        self.plan = Plan.get(lmax, table, device)
        pos = np.ascontiguousarray(positions, dtype=np.float64)
        self.n_particles = pos.shape[0]
        self.n = self.n_particles * self.nmax
        self.pos = torch.from_numpy(pos).to(device)
        self.ws = Workspace(device)

    # -- sizes ---------------------------------------------------------------------------------
    def coupling_ws_bytes(self, precision: int = YASF_C128, nrhs: int = 1) -> int:
        out = ctypes.c_size_t()
        call("yasf_coupling_workspace_size", self.plan.handle, self.n_particles, nrhs, precision,
             ctypes.byref(out))
        return out.value

    def _check_vec(self, x: torch.Tensor) -> int:
        if x.device != self.device or x.dtype != torch.complex128 or not x.is_contiguous():
            raise ValueError("vectors must be contiguous complex128 tensors on the plan's device")
        if x.shape[0] != self.n:
            raise ValueError(f"vector length {x.shape[0]} != N*nmax = {self.n}")
        return 1 if x.dim() == 1 else x.shape[1]

    # -- operators -------------------------------------------------------------------------------
    def coupling(self, x: torch.Tensor, precision: int = YASF_C128, out: torch.Tensor | None = None):
        """W x for x of shape (n,) or (R, n) stored row-major as R columns (see ``columns``)."""
        return self._apply("yasf_coupling_matvec", None, x, precision, out)

    def coupling_nearfield(self, x: torch.Tensor, radius: float, precision: int = YASF_C128,
                           out: torch.Tensor | None = None):
        """W x restricted to the pairs at most ``radius`` apart (near-field variant)."""
        cols = x.reshape(-1, self.n) if x.dim() > 1 else x.reshape(1, self.n)
        if x.dtype != torch.complex128 or x.device != self.device:
            raise ValueError("vectors must be complex128 tensors on the plan's device")
        cols = cols.contiguous()
        y = out if out is not None else torch.empty_like(cols)
        wsb = self.coupling_ws_bytes(precision)
        ws = self.ws.get(wsb)
        call("yasf_coupling_matvec_nearfield", self.plan.handle, self.n_particles, _ptr(self.pos), self.k,
             float(radius), _ptr(cols), _ptr(y), cols.shape[0], self.n, precision, _ptr(ws), wsb, _stream_ptr())
        return y.reshape(x.shape)

    def master(self, x: torch.Tensor, tmat: torch.Tensor, precision: int = YASF_C128,
               out: torch.Tensor | None = None):
        """x - T (.) W x."""
        return self._apply("yasf_master_matvec", tmat, x, precision, out)

    def _apply(self, name, tmat, x, precision, out):
        cols = x.reshape(-1, self.n) if x.dim() > 1 else x.reshape(1, self.n)
        if x.dtype != torch.complex128 or x.device != self.device:
            raise ValueError("vectors must be complex128 tensors on the plan's device")
        cols = cols.contiguous()
        R = cols.shape[0]
        y = out if out is not None else torch.empty_like(cols)
        wsb = self.coupling_ws_bytes(precision)
        ws = self.ws.get(wsb)
        s = _stream_ptr()
        if tmat is None:
            call(name, self.plan.handle, self.n_particles, _ptr(self.pos), self.k, _ptr(cols),
                 _ptr(y), R, self.n, precision, _ptr(ws), wsb, s)
        else:
            call(name, self.plan.handle, self.n_particles, _ptr(self.pos), self.k, _ptr(tmat),
                 _ptr(cols), _ptr(y), R, self.n, precision, _ptr(ws), wsb, s)
        return y.reshape(x.shape)

    def panel(self, x: torch.Tensor, tmat: torch.Tensor | None = None, out: torch.Tensor | None = None):
        """Tensor-core panel: (R, n) columns -> W x (or x - T W x), TF32 inputs, FP32 accumulation."""
        cols = x.reshape(-1, self.n).contiguous()
        R = cols.shape[0]
        y = out if out is not None else torch.empty_like(cols)
        nb = ctypes.c_size_t()
        call("yasf_panel_workspace_size", self.plan.handle, self.n_particles, R, ctypes.byref(nb))
        ws = self.ws.get(nb.value)
        call("yasf_panel_matvec", self.plan.handle, self.n_particles, _ptr(self.pos), self.k, _ptr(tmat),
             _ptr(cols), _ptr(y), R, self.n, self.n, _ptr(ws), nb.value, _stream_ptr())
        return y.reshape(x.shape)

    def dpanel(self, x: torch.Tensor, tmat: torch.Tensor | None = None, out: torch.Tensor | None = None):
        """Float64 dense multi-column coupling: (R, n) columns -> W x (or x - T W x)."""
        cols = x.reshape(-1, self.n).contiguous()
        R = cols.shape[0]
        y = out if out is not None else torch.empty_like(cols)
        nb = ctypes.c_size_t()
        call("yasf_dpanel_workspace_size", self.plan.handle, self.n_particles, R, ctypes.byref(nb))
        ws = self.ws.get(nb.value)
        call("yasf_dpanel_matvec", self.plan.handle, self.n_particles, _ptr(self.pos), self.k, _ptr(tmat),
             _ptr(cols), _ptr(y), R, self.n, self.n, _ptr(ws), nb.value, _stream_ptr())
        return y.reshape(x.shape)

    def plane_wave_rhs(self, tmat: torch.Tensor | None, polar, azimuthal, pol, amplitude: float = 1.0,
                       focal_point=(0.0, 0.0, 0.0), want_a: bool = True):
        """(A, B) for R plane-wave incidences on the device, each (R, n) complex128: the incident
        coefficients a (or None) and the right-hand sides b = T (.) a (or None without tmat)."""
        from yasf_b200.incident import plane_wave_mode_factors, wave_vectors

        coef = plane_wave_mode_factors(self.lmax, polar, azimuthal, pol, amplitude)
        R = coef.shape[0]
        kv = torch.from_numpy(wave_vectors(polar, azimuthal, self.k)).to(self.device)
        ct = torch.from_numpy(np.ascontiguousarray(coef)).to(self.device)
        A = torch.empty((R, self.n), dtype=torch.complex128, device=self.device) if want_a else None
        B = torch.empty((R, self.n), dtype=torch.complex128, device=self.device) if tmat is not None else None
        f = np.ascontiguousarray(np.asarray(focal_point, dtype=np.float64).reshape(3))
        call("yasf_plane_wave_rhs", self.lmax, self.n_particles, _ptr(self.pos), R, _ptr(kv), _ptr(ct),
             f.ctypes.data_as(ctypes.c_void_p), _ptr(tmat), _ptr(A), _ptr(B), self.n, _stream_ptr())
        return A, B

    def far_field_directions(self, polar, azimuthal) -> tuple:
        """Device arrays of a set of sampling directions for far_field: the angles and the angular
        functions pi_lm, tau_lm of yasfpy/functions/spherical_functions_trigon.py:11-96."""
        from yasf_b200.incident import spherical_functions_trigon

        polar = np.ascontiguousarray(np.asarray(polar, dtype=np.float64).ravel())
        azimuthal = np.ascontiguousarray(np.asarray(azimuthal, dtype=np.float64).ravel())
        pilm, taulm = spherical_functions_trigon(self.lmax, np.cos(polar), np.sin(polar))
        dv = self.device
        return (torch.from_numpy(polar).to(dv), torch.from_numpy(azimuthal).to(dv),
                torch.from_numpy(np.ascontiguousarray(pilm)).to(dv),
                torch.from_numpy(np.ascontiguousarray(taulm)).to(dv))

    def far_field(self, coef: torch.Tensor, polar, azimuthal=None, stokes: bool = True):
        """Scattered far field on sampling directions (yasf_far_field): (E_theta, E_phi) as
        complex128 device tensors (n_dirs,) and, with stokes, (n_dirs, 4) float64 I, Q, U, V.
        coef: the (N*nmax,) complex128 scattered-field coefficients, particle-major; the directions
        as (polar, azimuthal) angles or as the tuple far_field_directions returns."""
        pt, at, pl, tl = polar if isinstance(polar, tuple) else self.far_field_directions(polar, azimuthal)
        A = pt.numel()
        dv = self.device
        c = coef.reshape(-1).contiguous()
        et = torch.empty(A, dtype=torch.complex128, device=dv)
        ep = torch.empty(A, dtype=torch.complex128, device=dv)
        st = torch.empty((A, 4), dtype=torch.float64, device=dv) if stokes else None
        call("yasf_far_field", self.lmax, self.n_particles, _ptr(self.pos), float(self.k), _ptr(c), A, _ptr(pt),
             _ptr(at), _ptr(pl), _ptr(tl), _ptr(et), _ptr(ep), _ptr(st), _stream_ptr())
        return et, ep, st

    INNER_KINDS = {"tf32": 0, "c64": 1, "c128": 2}

    def batched_solve(self, tmat: torch.Tensor, B: torch.Tensor, rtol: float, restart: int = 50,
                      max_refine: int = 8, inner_rtol: float = 1e-3, inner: str = "tf32",
                      precond=None) -> tuple[torch.Tensor, dict]:
        """Refined lockstep GMRES for the columns of B (R, n); returns (X, stats)."""
        cols = B.reshape(-1, self.n).contiguous()
        R = cols.shape[0]
        kind = self.INNER_KINDS[inner]
        restart = int(max(1, min(restart, 512, self.n)))
        nb = ctypes.c_size_t()
        call("yasf_batched_workspace_size", self.plan.handle, self.n_particles, R, restart, kind,
             ctypes.byref(nb))
        ws = self.ws.get(nb.value)
        X = torch.empty_like(cols)
        stats = (ctypes.c_double * 8)()
        colres = (ctypes.c_double * R)()
        pc = precond.handle if precond is not None else ctypes.c_void_p(0)
        call("yasf_batched_solve", self.plan.handle, self.n_particles, _ptr(self.pos), self.k, _ptr(tmat), pc,
             _ptr(cols), _ptr(X), R, float(rtol), restart, int(max_refine), float(inner_rtol), kind,
             _ptr(ws), nb.value, stats, colres, _stream_ptr())
        info = {"inner_steps": int(stats[0]), "panel_matvecs": int(stats[1]),
                "column_matvecs": int(stats[2]), "matvecs_f64": int(stats[3]),
                "worst_relative_residual": float(stats[4]), "unconverged": int(stats[5]),
                "refinement_steps": int(stats[6]), "column_residuals": list(colres)}
        return X.reshape(B.shape), info

    def scattering_bilinear(self, b: torch.Tensor) -> complex:
        """sum conj(b) (W_reg b) with the regular (j_p) translation, self pairs included."""
        b = b.reshape(-1).contiguous()
        self._check_vec(b)
        out = torch.zeros(2, dtype=torch.float64, device=self.device)
        wsb = self.coupling_ws_bytes(YASF_C128)
        ws = self.ws.get(wsb)
        call("yasf_scattering_bilinear", self.plan.handle, self.n_particles, _ptr(self.pos), self.k,
             _ptr(b), _ptr(out), _ptr(ws), wsb, _stream_ptr())
        o = out.cpu().numpy()
        return complex(o[0], o[1])

    def dotc(self, a: torch.Tensor, b: torch.Tensor) -> complex:
        out = torch.zeros(2, dtype=torch.float64, device=self.device)
        ws = self.ws.get(1024 * 16)
        call("yasf_dotc", a.numel(), _ptr(a), _ptr(b), _ptr(out), _ptr(ws), ws.numel(), _stream_ptr())
        o = out.cpu().numpy()
        return complex(o[0], o[1])

    def gmres(self, tmat: torch.Tensor, b: torch.Tensor, x: torch.Tensor, rtol: float, restart: int,
              maxiter: int, precision: int = YASF_C128, precond=None) -> dict:
        """Device GMRES on (I - T W) x = b; x holds x0 on entry. Returns solve statistics."""
        self._check_vec(b)
        self._check_vec(x)
        restart = int(max(1, min(restart, 512, self.n)))
        nb = ctypes.c_size_t()
        call("yasf_gmres_workspace_size", self.plan.handle, self.n_particles, restart, precision,
             ctypes.byref(nb))
        ws = self.ws.get(nb.value)
        stats = (ctypes.c_double * 8)()
        pc = precond.handle if precond is not None else ctypes.c_void_p(0)
        call("yasf_gmres_solve", self.plan.handle, self.n_particles, _ptr(self.pos), self.k,
             _ptr(tmat), pc, _ptr(b), _ptr(x), float(rtol), restart, int(maxiter), precision,
             _ptr(ws), nb.value, stats, _stream_ptr())
        return {
            "inner_iterations": int(stats[0]),
            "matvecs_inner": int(stats[1]),
            "matvecs_f64": int(stats[2]),
            "relative_residual": float(stats[3]),
            "info": int(stats[4]),
            "refinement_steps": int(stats[5]),
        }


def grouped_solve(items, rtol: float, restart: int = 30, max_refine: int = 8, inner_rtol: float = 1e-3,
                  inner: str = "c64") -> tuple[list[torch.Tensor], dict]:
    """Solve the right-hand sides of several aggregates of one lmax together (yasf_grouped_solve).

    items: list of (CouplingDevice, tmat (n,), B (R, n)) on one device, sharing one translation
    plan. Returns the solutions (one (R, n) tensor per item, in order) and the solve statistics;
    the column residuals are listed aggregate by aggregate."""
    if not items:
        return [], {}
    dev0 = items[0][0]
    plan = dev0.plan
    probs = (_lib.YasfProblem * len(items))()
    outs, keep = [], []
    for i, (dev, tmat, B) in enumerate(items):
        if dev.plan is not plan:
            raise ValueError("a grouped solve needs one translation plan (one lmax, one table, one device)")
        cols = B.reshape(-1, dev.n).contiguous()
        X = torch.empty_like(cols)
        keep += [cols, tmat]
        outs.append(X)
        probs[i] = _lib.YasfProblem(dev.n_particles, dev.pos.data_ptr(), dev.k, tmat.data_ptr(), cols.data_ptr(),
                                    X.data_ptr(), cols.shape[0])
    restart = int(max(1, min(restart, 512)))
    nb = ctypes.c_size_t()
    call("yasf_grouped_workspace_size", plan.handle, len(items), probs, restart, ctypes.byref(nb))
    ws = dev0.ws.get(nb.value)
    C = sum(int(x.shape[0]) for x in outs)
    stats = (ctypes.c_double * 8)()
    colres = (ctypes.c_double * C)()
    call("yasf_grouped_solve", plan.handle, len(items), probs, float(rtol), restart, int(max_refine),
         float(inner_rtol), PRECISIONS[inner], _ptr(ws), nb.value, stats, colres, _stream_ptr())
    info = {"inner_steps": int(stats[0]), "inner_applications": int(stats[1]), "applications_f64": int(stats[2]),
            "worst_relative_residual": float(stats[3]), "unconverged": int(stats[4]),
            "refinement_steps": int(stats[5]), "columns": int(stats[6]), "work_items": int(stats[7]),
            "column_residuals": list(colres)}
    del keep
    return outs, info


class DevicePreconditioner:
    """Block-Jacobi factors of (I - T W) on the device (C-ABI handle + block inversion)."""

    def __init__(self, dev: CouplingDevice, blocks: list[np.ndarray]):
        self.dev = dev
        ptr = np.zeros(len(blocks) + 1, dtype=np.int32)
        ptr[1:] = np.cumsum([len(b) for b in blocks])
        parts = np.ascontiguousarray(np.concatenate(blocks).astype(np.int32))
        self.blocks = blocks
        handle = ctypes.c_void_p()
        with torch.cuda.device(dev.device):
            call("yasf_precond_create", dev.plan.handle, dev.n_particles, len(blocks),
                 ptr.ctypes.data_as(ctypes.c_void_p), parts.ctypes.data_as(ctypes.c_void_p),
                 ctypes.byref(handle))
        self.handle = handle

    def prepare(self, tmat: torch.Tensor, keep_float64: bool = False) -> dict:
        """Assemble, factor (the library's batched block LU) and finalize every block; returns the
        seconds of each phase. The factorisation runs in complex64, as the reference's; with
        keep_float64 it runs in complex128 and those factors stay beside the complex64 copy the
        solves stream."""
        import time

        s = _stream_ptr()
        t0 = time.perf_counter()
        call("yasf_precond_assemble", self.handle, _ptr(self.dev.pos), self.dev.k, _ptr(tmat), s)
        torch.cuda.synchronize(self.dev.device)
        t1 = time.perf_counter()
        call("yasf_precond_keep_float64", self.handle, 1 if keep_float64 else 0)
        call("yasf_precond_factor", self.handle, s)
        torch.cuda.synchronize(self.dev.device)
        t2 = time.perf_counter()
        call("yasf_precond_finalize", self.handle, s)
        t3 = time.perf_counter()
        return {"assemble_s": t1 - t0, "factor_s": t2 - t1, "finalize_s": t3 - t2}

    def assemble(self, tmat: torch.Tensor) -> None:
        """Only the block assembly: every block holds M_B = (I - T W)[B, B] (see ``block_matrix``)."""
        call("yasf_precond_assemble", self.handle, _ptr(self.dev.pos), self.dev.k, _ptr(tmat), _stream_ptr())

    def block_matrix(self, b: int) -> torch.Tensor:
        ptr = ctypes.c_void_p()
        dim = ctypes.c_int()
        call("yasf_precond_block", self.handle, b, ctypes.byref(ptr), ctypes.byref(dim))
        return _wrap_device_matrix(ptr.value, dim.value, self.dev.device)

    def apply(self, x: torch.Tensor, precision: int = YASF_C128) -> torch.Tensor:
        cols = x.reshape(-1, self.dev.n).contiguous()
        y = torch.empty_like(cols)
        call("yasf_precond_apply", self.handle, _ptr(cols), _ptr(y), cols.shape[0], self.dev.n,
             precision, _stream_ptr())
        return y.reshape(x.shape)

    def nbytes(self) -> int:
        out = ctypes.c_size_t()
        call("yasf_precond_bytes", self.handle, ctypes.byref(out))
        return out.value

    def __del__(self):
        h = getattr(self, "handle", None)
        if h is not None and h.value:
            try:
                _lib.load().yasf_precond_destroy(h)
            except Exception:
                pass


def _wrap_device_matrix(ptr: int, dim: int, device: torch.device) -> torch.Tensor:
    """A (dim, dim) complex128 torch view of library-owned device memory."""

    class _Holder:
        pass

    holder = _Holder()
    holder.__cuda_array_interface__ = {
        "shape": (dim, dim),
        "typestr": "<c16",
        "data": (int(ptr), False),
        "version": 3,
        "strides": None,
    }
    return torch.as_tensor(holder, device=device)
