"""ctypes binding of the C ABI declared in ``include/yasf_b200.h``.

The shared library is built in-tree (``yasf_b200/_build/libyasf_b200.so``, see
``yasf_b200/build.py``). There is no CPU fallback: if the library is missing or cannot be loaded,
importing the device layer raises ``RuntimeError``.
"""

from __future__ import annotations

import ctypes
import threading
from pathlib import Path

import torch  # noqa: F401  (loads the CUDA runtime the library links against)

LIB_PATH = Path(__file__).resolve().parent / "_build" / "libyasf_b200.so"

YASF_OK = 0
YASF_C128 = 0
YASF_C64 = 1

_STATUS_NAMES = {
    1: "YASF_ERR_INVALID_ARGUMENT",
    2: "YASF_ERR_UNSUPPORTED",
    3: "YASF_ERR_ALIGNMENT",
    4: "YASF_ERR_CUDA",
    5: "YASF_ERR_OUT_OF_MEMORY",
    6: "YASF_ERR_WORKSPACE",
    7: "YASF_ERR_NOT_FINITE",
    8: "YASF_ERR_NOT_PREPARED",
    9: "YASF_ERR_SCRATCH_LIMIT",
}


class YasfError(RuntimeError):
    """A C-ABI call returned a non-zero status."""

    def __init__(self, func: str, status: int, detail: str = ""):
        self.status = status
        name = _STATUS_NAMES.get(status, f"status {status}")
        msg = f"{func} failed: {name}"
        if detail:
            msg += f" ({detail})"
        super().__init__(msg)


_c = ctypes
_vp = _c.c_void_p
_i = _c.c_int
_ll = _c.c_longlong
_d = _c.c_double
_sz = _c.c_size_t
_dp = _c.POINTER(_c.c_double)

# name -> (argtypes)
SIGNATURES = {
    "yasf_abi_version": [],
    "yasf_status_string": [_i],
    "yasf_last_cuda_error": [],
    "yasf_kernel_launches": [],
    "yasf_test_stall": [_i, _i, _d],
    "yasf_set_tiles": [_i, _i, _i],
    "yasf_grouped_workspace_size": [_vp, _i, _vp, _i, _c.POINTER(_sz)],
    "yasf_grouped_solve": [_vp, _i, _vp, _d, _i, _i, _d, _i, _vp, _sz, _dp, _dp, _vp],
    "yasf_plane_wave_rhs": [_i, _i, _vp, _i, _vp, _vp, _vp, _vp, _vp, _vp, _ll, _vp],
    "yasf_far_field": [_i, _i, _vp, _d, _vp, _i, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp],
    "yasf_plan_create": [_i, _vp, _c.POINTER(_vp)],
    "yasf_plan_destroy": [_vp],
    "yasf_plan_info": [_vp, _c.POINTER(_i), _c.POINTER(_ll), _c.POINTER(_ll)],
    "yasf_plan_check_table": [_i, _vp],
    "yasf_coupling_workspace_size": [_vp, _i, _i, _i, _c.POINTER(_sz)],
    "yasf_coupling_matvec": [_vp, _i, _vp, _d, _vp, _vp, _i, _ll, _i, _vp, _sz, _vp],
    "yasf_coupling_matvec_nearfield": [_vp, _i, _vp, _d, _d, _vp, _vp, _i, _ll, _i, _vp, _sz, _vp],
    "yasf_master_matvec": [_vp, _i, _vp, _d, _vp, _vp, _vp, _i, _ll, _i, _vp, _sz, _vp],
    "yasf_coupling_matvec_noalloc": [_vp, _i, _vp, _d, _vp, _vp, _i, _vp],
    "yasf_panel_workspace_size": [_vp, _i, _i, _c.POINTER(_sz)],
    "yasf_panel_matvec": [_vp, _i, _vp, _d, _vp, _vp, _vp, _i, _ll, _ll, _vp, _sz, _vp],
    "yasf_dpanel_workspace_size": [_vp, _i, _i, _c.POINTER(_sz)],
    "yasf_dpanel_matvec": [_vp, _i, _vp, _d, _vp, _vp, _vp, _i, _ll, _ll, _vp, _sz, _vp],
    "yasf_batched_workspace_size": [_vp, _i, _i, _i, _i, _c.POINTER(_sz)],
    "yasf_batched_solve": [_vp, _i, _vp, _d, _vp, _vp, _vp, _vp, _i, _d, _i, _i, _d, _i, _vp, _sz,
                           _dp, _dp, _vp],
    "yasf_scattering_bilinear": [_vp, _i, _vp, _d, _vp, _vp, _vp, _sz, _vp],
    "yasf_dotc": [_ll, _vp, _vp, _vp, _vp, _sz, _vp],
    "yasf_precond_create": [_vp, _i, _i, _vp, _vp, _c.POINTER(_vp)],
    "yasf_precond_destroy": [_vp],
    "yasf_precond_assemble": [_vp, _vp, _d, _vp, _vp],
    "yasf_precond_block": [_vp, _i, _c.POINTER(_vp), _c.POINTER(_i)],
    "yasf_precond_finalize": [_vp, _vp],
    "yasf_precond_factor": [_vp, _vp],
    "yasf_precond_keep_float64": [_vp, _i],
    "yasf_precond_apply": [_vp, _vp, _vp, _i, _ll, _i, _vp],
    "yasf_precond_bytes": [_vp, _c.POINTER(_sz)],
    "yasf_gmres_workspace_size": [_vp, _i, _i, _i, _c.POINTER(_sz)],
    "yasf_gmres_solve": [
        _vp, _i, _vp, _d, _vp, _vp, _vp, _vp, _d, _i, _i, _i, _vp, _sz, _dp, _vp,
    ],
}
_RESTYPES = {
    "yasf_status_string": _c.c_char_p,
    "yasf_last_cuda_error": _c.c_char_p,
    "yasf_kernel_launches": _c.c_ulonglong,
}

_lib = None
_lock = threading.Lock()


def load(path: Path | str | None = None) -> ctypes.CDLL:
    """Load (once) and return the C library with argument types set."""
    global _lib
    with _lock:
        if _lib is not None:
            return _lib
        p = Path(path) if path else LIB_PATH
        if not p.exists():
            raise RuntimeError(
                f"yasf_b200 CUDA library not found at {p}; build it with "
                "`python -c 'import __graft_entry__ as g; g.build()'` or `python yasf_b200/build.py`"
            )
        lib = ctypes.CDLL(str(p))
        for name, args in SIGNATURES.items():
            fn = getattr(lib, name)
            fn.argtypes = args
            fn.restype = _RESTYPES.get(name, _i)
        _lib = lib
        return lib


def check(func: str, status: int) -> None:
    if status != YASF_OK:
        detail = ""
        if status == 4:
            detail = (load().yasf_last_cuda_error() or b"").decode()
        raise YasfError(func, status, detail)


def call(name: str, *args) -> None:
    """Call a status-returning entry point and raise ``YasfError`` on failure."""
    check(name, getattr(load(), name)(*args))


YASF_STALL_NONE = 0
YASF_STALL_CONTRACT = 1
YASF_STALL_PANEL = 2
YASF_STALL_DPANEL = 3
YASF_STALL_PRECOND = 4


def test_stall(role: int, contract_polls: int = 0, panel_wait_seconds: float = 0.0) -> None:
    """Failure-detection test hook (yasf_test_stall): the next launches from this host thread keep
    one producer role from delivering, with shortened wait bounds. ``YASF_STALL_NONE`` restores
    normal launches."""
    call("yasf_test_stall", int(role), int(contract_polls), float(panel_wait_seconds))


class YasfProblem(_c.Structure):
    """``yasf_problem`` of include/yasf_b200.h: one aggregate of a grouped solve."""

    _fields_ = [("n_particles", _i), ("positions", _vp), ("k_medium", _d), ("tmat", _vp), ("b", _vp),
                ("x", _vp), ("nrhs", _i)]


def set_tiles(contract_waves: int = 0, dpanel_cols: int = 0, panel_groups: int = 0) -> None:
    """Tile shapes of this host thread's next launches (yasf_set_tiles); zeros restore the rules."""
    call("yasf_set_tiles", int(contract_waves), int(dpanel_cols), int(panel_groups))
