"""Build the oracle's C/OpenMP loops (``oracle_kernels.c``) into
``oracle/_build/liboracle_kernels.so`` with gcc.  Test infrastructure only: the oracle
runs its NumPy forms when the library is absent."""

from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
SRC = HERE / "oracle_kernels.c"
OUT = HERE / "_build" / "liboracle_kernels.so"


def build(verbose: bool = False) -> Path | None:
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        return None
    if OUT.exists() and OUT.stat().st_mtime > SRC.stat().st_mtime:
        return OUT
    OUT.parent.mkdir(exist_ok=True)
    tmp = OUT.with_suffix(".so.tmp")
    cmd = [cc, "-O3", "-march=x86-64-v2", "-fopenmp", "-fPIC", "-shared", "-o", str(tmp), str(SRC)]
    if verbose:
        print(" ".join(cmd), flush=True)
    subprocess.run(cmd, check=True)
    os.replace(tmp, OUT)
    return OUT


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv))
