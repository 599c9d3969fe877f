"""The C-ABI library: loads, exports every symbol include/yasf_b200.h declares, and rejects bad
arguments before touching the device (no GPU needed for these paths)."""

from __future__ import annotations

import ctypes
import re
from pathlib import Path

import pytest

REPO = Path(__file__).resolve().parents[1]
HEADER = REPO / "include" / "yasf_b200.h"


def declared_symbols() -> list[str]:
    text = HEADER.read_text()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(yasf_[a-z0-9_]+)\s*\(", text)))


@pytest.fixture(scope="module")
def lib():
    from yasf_b200 import build

    build.build()
    from yasf_b200 import _lib

    return _lib.load()


def test_library_exports_every_declared_symbol(lib):
    syms = declared_symbols()
    assert len(syms) >= 15
    for s in syms:
        assert hasattr(lib, s), f"{s} declared in the header but not exported"


def test_binding_covers_header():
    from yasf_b200 import _lib

    assert set(declared_symbols()) <= set(_lib.SIGNATURES)


def test_status_strings(lib):
    assert lib.yasf_abi_version() == 1
    assert lib.yasf_status_string(0) == b"ok"
    assert lib.yasf_status_string(6) == b"workspace too small"


def test_argument_validation_without_device(lib):
    h = ctypes.c_void_p()
    assert lib.yasf_plan_create(0, ctypes.c_void_p(1), ctypes.byref(h)) == 2  # lmax unsupported
    assert lib.yasf_plan_create(9, ctypes.c_void_p(1), ctypes.byref(h)) == 2
    assert lib.yasf_plan_create(3, None, ctypes.byref(h)) == 1
    assert lib.yasf_coupling_matvec(None, 10, None, 1.0, None, None, 1, 0, 0, None, 0, None) == 1
    assert lib.yasf_gmres_solve(None, 1, None, 1.0, None, None, None, None, 1e-8, 10, 10, 0, None, 0,
                                None, None) == 1
    assert lib.yasf_precond_apply(None, None, None, 1, 0, 0, None) == 1
    assert lib.yasf_dotc(0, None, None, None, None, 0, None) == 1
    n = ctypes.c_size_t()
    for fn in ("yasf_panel_workspace_size", "yasf_dpanel_workspace_size"):
        assert getattr(lib, fn)(None, 10, 4, ctypes.byref(n)) == 1      # no plan
    for fn in ("yasf_panel_matvec", "yasf_dpanel_matvec"):
        assert getattr(lib, fn)(None, 10, None, 1.0, None, None, None, 4, 0, 0, None, 0, None) == 1
    assert lib.yasf_batched_workspace_size(None, 10, 4, 30, 0, ctypes.byref(n)) == 1
    assert lib.yasf_batched_workspace_size(None, 10, 4, 30, 3, ctypes.byref(n)) == 1


def test_stall_hook_validates_its_arguments(lib):
    # the failure-detection test hook is host state only: no device is touched here
    assert lib.yasf_test_stall(7, 0, 0.0) == 1
    assert lib.yasf_test_stall(2, -1, 0.0) == 1
    assert lib.yasf_test_stall(2, 0, 100.0) == 1
    assert lib.yasf_test_stall(2, 0, float("nan")) == 1
    assert lib.yasf_test_stall(1, 4096, 0.05) == 0
    assert lib.yasf_test_stall(0, 0, 0.0) == 0


@pytest.mark.parametrize("lmax", range(1, 9))
def test_plan_layouts_accept_the_translation_table(lib, lmax):
    """The host-side builders a plan runs (the panel schedule with its slot tables and term windows,
    packed FP16 coefficients at lmax 7-8, the float64 dense panel's items) accept the exact table
    at every lmax: checked without a device."""
    import numpy as np

    from yasf_b200.wigner import translation_table_ab5

    tab = np.ascontiguousarray(translation_table_ab5(lmax), dtype=np.complex128)
    assert lib.yasf_plan_check_table(lmax, ctypes.c_void_p(tab.ctypes.data)) == 0


def test_plan_layouts_reject_a_broken_table(lib):
    import numpy as np

    from yasf_b200.wigner import translation_table_ab5

    tab = np.ascontiguousarray(translation_table_ab5(4), dtype=np.complex128)
    bad = tab.copy()
    bad[0, 0, 1] = 0.5  # a tau1 = tau2 term with l1 + l2 + p odd: outside the selection rules
    assert lib.yasf_plan_check_table(4, ctypes.c_void_p(bad.ctypes.data)) == 1
    bad = tab.copy()
    bad[2, 1, 3] = np.nan
    assert lib.yasf_plan_check_table(4, ctypes.c_void_p(bad.ctypes.data)) == 7
    assert lib.yasf_plan_check_table(9, ctypes.c_void_p(tab.ctypes.data)) == 2
    assert lib.yasf_plan_check_table(4, None) == 1


def test_no_cpu_fallback_in_product():
    """The product package never imports the oracle."""
    for py in (REPO / "yasf_b200").rglob("*.py"):
        text = py.read_text()
        assert "import oracle" not in text and "from oracle" not in text, py


def test_product_fails_loudly_without_a_gpu():
    """Without a CUDA device the drop-in API raises instead of computing on the host; an unknown
    backend name raises ValueError as the reference's if-chain does (yasfpy/simulation.py:95-106)."""
    import numpy as np
    import torch

    from yasf_b200 import InitialField, Numerics, Parameters, Particles, Simulation
    from yasf_b200.device import CouplingDevice
    from yasf_b200.wigner import translation_table_ab5

    particles = Particles(np.array([[0.0, 0.0, 0.0], [1.0, 0.0, 0.0]]), np.array([0.1, 0.1]),
                          np.array([1.5, 1.5], dtype=complex))
    params = Parameters(np.array([1.0]), np.array([1.0 + 0j]), particles,
                        InitialField(beam_width=0, focal_point=np.zeros(3)))
    with pytest.raises(ValueError):
        Simulation(params, Numerics(lmax=2, coupling_backend="dense"))
    if torch.cuda.is_available():
        pytest.skip("a CUDA device is present")
    with pytest.raises(RuntimeError):
        Simulation(params, Numerics(lmax=2))
    with pytest.raises(RuntimeError, match="CUDA devices only"):
        CouplingDevice(2, translation_table_ab5(2), particles.position, 1.0, torch.device("cpu"))


def test_plain_c_consumer_builds_and_runs(lib, tmp_path):
    """A C99 program includes the header, links the library and calls it (the binding a C or cgo host
    would write): ABI version, status strings, and the host-only table check on a zero table
    (zero is a valid, if useless, a5/b5 table)."""
    import shutil
    import subprocess

    gcc = shutil.which("gcc")
    if gcc is None:
        pytest.skip("no C compiler")
    src = tmp_path / "consumer.c"
    src.write_text(
        '#include <stdio.h>\n#include <stdlib.h>\n#include "yasf_b200.h"\n'
        "int main(void) {\n"
        "  const int lmax = 2, nmax = 2 * lmax * (lmax + 2), P = 2 * lmax + 1;\n"
        "  double* tab = calloc((size_t)nmax * nmax * P * 2, sizeof(double));\n"
        "  int ok = yasf_plan_check_table(lmax, tab);\n"
        '  printf("%d %d %s\\n", yasf_abi_version(), ok, yasf_status_string(YASF_ERR_WORKSPACE));\n'
        "  free(tab);\n  return 0;\n}\n")
    libdir = REPO / "yasf_b200" / "_build"
    exe = tmp_path / "consumer"
    subprocess.run([gcc, "-std=c99", "-Wall", "-Werror", str(src), "-I", str(REPO / "include"), "-L", str(libdir),
                    "-lyasf_b200", f"-Wl,-rpath,{libdir}", "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split(maxsplit=2)
    assert out[0] == "1" and out[1] == "0" and out[2].strip() == "workspace too small"
