"""Shared pytest configuration: the ``gpu`` marker, fixture loading, library/oracle access."""

from __future__ import annotations

import sys
from pathlib import Path

import numpy as np
import pytest

REPO = Path(__file__).resolve().parents[1]
GOLDEN = REPO / "tests" / "golden"
if str(REPO) not in sys.path:
    sys.path.insert(0, str(REPO))


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA device (B200) and the built library")


def load_golden(name: str) -> dict:
    path = GOLDEN / name
    if not path.exists():
        pytest.fail(f"golden fixture {name} missing; regenerate with tests/golden/make_golden.py")
    with np.load(path, allow_pickle=False) as z:
        return {k: z[k] for k in z.files}


@pytest.fixture(scope="session")
def golden():
    return load_golden


@pytest.fixture(scope="session")
def cuda_device():
    import torch

    if not torch.cuda.is_available():
        pytest.fail("GPU test run without a CUDA device")
    from yasf_b200 import _lib

    _lib.load()  # fails loudly if the CUDA library is missing
    return torch.device("cuda", 0)


def rel_err(a, b) -> float:
    a = np.asarray(a)
    b = np.asarray(b)
    return float(np.max(np.abs(a - b)) / max(np.max(np.abs(b)), 1e-300))


def reference_package_root():
    """Directory holding the reference ``yasfpy`` package: $YASF_REFERENCE, else the local
    install under baseline/_ref (git-ignored). None when neither is present."""
    import os

    for cand in (os.environ.get("YASF_REFERENCE"), str(REPO / "baseline" / "_ref")):
        if cand and (Path(cand) / "yasfpy" / "simulation.py").exists():
            return Path(cand)
    return None


@pytest.fixture(scope="session")
def reference_yasfpy(tmp_path_factory):
    """Import the reference's own ``yasfpy`` (with the oracle's stand-ins for its third-party
    modules: exact 3j for pywigxjpf, inert refidxdb / pyperf) or skip with the reason."""
    import os

    root = reference_package_root()
    if root is None:
        pytest.skip("reference yasfpy not importable here (no $YASF_REFERENCE, no baseline/_ref)")
    for p in (str(REPO / "oracle" / "stubs"), str(root)):
        if p not in sys.path:
            sys.path.insert(0, p)
    os.environ["HOME"] = str(tmp_path_factory.mktemp("yasfpy_home"))
    import yasfpy  # noqa: F401

    return root
