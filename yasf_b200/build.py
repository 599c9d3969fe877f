"""Build recipe for the in-tree CUDA library ``yasf_b200/_build/libyasf_b200.so``.

Every translation unit is compiled for sm_100a only (``-gencode arch=compute_100a,code=sm_100a``)
with ``-lineinfo``; the per-lmax coupling kernels are compiled from one source with
``-DYASF_INST_L=<lmax>`` in parallel. The library is rebuilt when any source or header is newer
than the shared object.
"""

from __future__ import annotations

import os
import shutil
import subprocess
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = BUILD / "libyasf_b200.so"
INCLUDE = PKG.parent / "include"
GEN = BUILD / "gen"  # build-time generated headers (panel_sched.h)

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = [
    "-std=c++17",
    "-O3",
    "-lineinfo",
    "-Xcompiler",
    "-fPIC",
    "--expt-relaxed-constexpr",
    *ARCH,
]
LMAX_RANGE = range(1, 9)


def _nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(cand).exists():
        raise RuntimeError("nvcc not found: the yasf_b200 CUDA library cannot be built")
    return cand


def _sources() -> list[Path]:
    return sorted(CSRC.glob("*.cu")) + sorted(CSRC.glob("*.cuh")) + sorted(CSRC.glob("*.h")) + sorted(
        INCLUDE.glob("*.h")
    ) + [PKG / "panel_sched.py"]


def _units() -> list[tuple[Path, list[str], Path]]:
    units = []
    for src in sorted(CSRC.glob("*.cu")):
        if src.name == "coupling_inst.cu":
            for L in LMAX_RANGE:
                units.append((src, [f"-DYASF_INST_L={L}"], BUILD / f"coupling_l{L}.o"))
        else:
            units.append((src, [], BUILD / (src.stem + ".o")))
    return units


def needs_build() -> bool:
    if not LIB.exists():
        return True
    t = LIB.stat().st_mtime
    return any(p.stat().st_mtime > t for p in _sources())


def build(verbose: bool = False, force: bool = False, jobs: int | None = None) -> Path:
    """Compile and link the library; returns its path."""
    if not force and not needs_build():
        return LIB
    nvcc = _nvcc()
    BUILD.mkdir(parents=True, exist_ok=True)
    from yasf_b200.panel_sched import write_header

    write_header(GEN / "panel_sched.h")
    units = _units()

    def compile_one(unit):
        src, extra, obj = unit
        cmd = [nvcc, *NVCC_FLAGS, *extra, "-I", str(INCLUDE), "-I", str(GEN), "-c", str(src), "-o", str(obj)]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"nvcc failed for {src.name} {extra}:\n{res.stderr}")
        if verbose and res.stderr:
            print(res.stderr)
        return obj

    jobs = jobs or max(1, min(len(units), os.cpu_count() or 1))
    with ThreadPoolExecutor(max_workers=jobs) as ex:
        objs = list(ex.map(compile_one, units))
    tmp = LIB.with_suffix(".so.tmp")
    rpath = []
    try:
        import nvidia.cuda_runtime as _cr  # the runtime torch itself loads

        rpath = ["-Xlinker", "-rpath", "-Xlinker", str(Path(list(_cr.__path__)[0]) / "lib")]
    except Exception:
        pass
    cmd = [nvcc, *ARCH, "-shared", "-o", str(tmp), *map(str, objs), "-lcudart", *rpath]
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"link failed:\n{res.stderr}")
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    import sys

    print(build(verbose="-v" in sys.argv, force="-f" in sys.argv))
