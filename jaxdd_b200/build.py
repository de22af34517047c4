"""Build the CUDA library in-tree: jaxdd_b200/lib/libjaxdd_b200.so, for sm_100a only.

    python -m jaxdd_b200.build [-v]

nvcc cross-compiles without a GPU. Each source compiles to its own object (in parallel, and
only when it or a header it may include is newer than its object); the objects link into one
shared library. The library is the package's only compute path; nothing falls back to the CPU
without it.
"""

from __future__ import annotations

import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

HERE = Path(__file__).resolve().parent
CSRC = HERE / "csrc"
LIB_DIR = HERE / "lib"
OBJ_DIR = LIB_DIR / "obj"
LIB = LIB_DIR / "libjaxdd_b200.so"
SOURCES = ["dd_solve.cu", "dd_adjoint.cu", "dd_states.cu", "dd_impedance.cu", "dd_build.cu",
           "dd_transient.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = [*ARCH, "-lineinfo", "-O3", "-std=c++17", "--expt-relaxed-constexpr",
         "-Xcompiler", "-fPIC"]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is needed to build jaxdd_b200")


def _headers() -> list[Path]:
    return (list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh"))
            + list((HERE.parent / "include").glob("*.h")))


def _compile(src: Path, verbose: bool) -> tuple[Path, str]:
    obj = OBJ_DIR / (src.stem + ".o")
    tmp = obj.with_suffix(".o.tmp")
    cmd = [nvcc(), *FLAGS, *(["-Xptxas", "-v"] if verbose else []), "-c", "-o", str(tmp),
           str(src)]
    proc = subprocess.run(cmd, capture_output=True, text=True)
    if proc.returncode != 0:
        raise RuntimeError(f"nvcc failed on {src.name} ({proc.returncode}):\n{proc.stderr}")
    tmp.replace(obj)
    return obj, proc.stderr


def build(verbose: bool = False, force: bool = False) -> Path:
    """Compile what is out of date and link the library; returns its path."""
    OBJ_DIR.mkdir(parents=True, exist_ok=True)
    newest_header = max(h.stat().st_mtime for h in _headers())
    stale = []
    for name in SOURCES:
        src = CSRC / name
        obj = OBJ_DIR / (src.stem + ".o")
        if (force or not obj.exists() or obj.stat().st_mtime < src.stat().st_mtime
                or obj.stat().st_mtime < newest_header):
            stale.append(src)
    if stale:
        with ThreadPoolExecutor(max_workers=max(1, min(len(stale), os.cpu_count() or 1))) as ex:
            for obj, err in ex.map(lambda s: _compile(s, verbose), stale):
                if verbose:
                    print(f"== {obj.name}\n{err}", file=sys.stderr)
    objs = [OBJ_DIR / (Path(n).stem + ".o") for n in SOURCES]
    if stale or not LIB.exists() or any(LIB.stat().st_mtime < o.stat().st_mtime for o in objs):
        tmp = LIB.with_suffix(".so.tmp")
        proc = subprocess.run([nvcc(), *ARCH, "-shared", "-o", str(tmp), *map(str, objs)],
                              capture_output=True, text=True)
        if proc.returncode != 0:
            raise RuntimeError(f"nvcc link failed ({proc.returncode}):\n{proc.stderr}")
        tmp.replace(LIB)
    return LIB


if __name__ == "__main__":
    print(build(verbose="-v" in sys.argv, force="-v" in sys.argv or "-f" in sys.argv))
