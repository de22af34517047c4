"""Build the CUDA library in-tree: jaxdd_b200/lib/libjaxdd_b200.so, for sm_100a only.

    python -m jaxdd_b200.build

nvcc cross-compiles without a GPU. The library is the package's only compute path; nothing
falls back to the CPU without it.
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
LIB_DIR = HERE / "lib"
LIB = LIB_DIR / "libjaxdd_b200.so"
SOURCES = ["dd_solve.cu", "dd_adjoint.cu", "dd_states.cu", "dd_impedance.cu", "dd_build.cu",
           "dd_transient.cu"]
FLAGS = [
    "-gencode", "arch=compute_100a,code=sm_100a", "-lineinfo", "-O3", "-std=c++17",
    "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC", "-shared",
]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is needed to build jaxdd_b200")


def build(verbose: bool = False, force: bool = False) -> Path:
    """Compile the library if any source is newer than it; returns its path."""
    LIB_DIR.mkdir(exist_ok=True)
    srcs = [CSRC / s for s in SOURCES]
    deps = (srcs + list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh"))
            + list((HERE.parent / "include").glob("*.h")))
    if not force and LIB.exists() and all(LIB.stat().st_mtime >= d.stat().st_mtime for d in deps):
        return LIB
    tmp = LIB.with_suffix(".so.tmp")
    cmd = [nvcc(), *FLAGS, *(["-Xptxas", "-v"] if verbose else []), "-o", str(tmp),
           *map(str, srcs)]
    proc = subprocess.run(cmd, capture_output=True, text=True)
    if proc.returncode != 0:
        raise RuntimeError(f"nvcc failed ({proc.returncode}):\n{proc.stderr}")
    if verbose:
        print(proc.stderr, file=sys.stderr)
    tmp.replace(LIB)
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, force=True))
