"""ORACLE — TEST INFRASTRUCTURE ONLY. Builds ``oracle/_build/liboracle.so`` from ``cpu_ref.c``
with gcc and OpenMP. Called by ``__graft_entry__.build()``; the product never links it."""

from __future__ import annotations

import os
import shutil
import subprocess
from pathlib import Path

HERE = Path(__file__).resolve().parent
SRC = HERE / "cpu_ref.c"
OUT = HERE / "_build" / "liboracle.so"


def build(force: bool = False) -> Path:
    if not force and OUT.exists() and OUT.stat().st_mtime >= SRC.stat().st_mtime:
        return OUT
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        raise RuntimeError("gcc not found: cannot build the oracle")
    OUT.parent.mkdir(parents=True, exist_ok=True)
    tmp = OUT.with_suffix(".so.tmp")
    cmd = [cc, "-O2", "-fopenmp", "-fPIC", "-shared", "-std=c99", str(SRC), "-o", str(tmp), "-lm"]
    subprocess.run(cmd, check=True)
    os.replace(tmp, OUT)
    return OUT


if __name__ == "__main__":
    print(build(force=True))
