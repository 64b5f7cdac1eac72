"""Build recipe of the native library ``cusmic_b200/libcusmic_b200.so``.

nvcc compiles the CUDA sources for sm_100a only, with the reference's
floating-point rules (no FMA contraction on device or host: every threshold
compares values computed in the reference's operation order) and a static
CUDA runtime, into a shared object next to this file, so it travels with the
working tree.  ``python -m cusmic_b200.build`` or ``build()``.
"""

import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
ROOT = HERE.parent
CSRC = HERE / "csrc"
LIB = HERE / "libcusmic_b200.so"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc():
    return shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"


def sources():
    return sorted(CSRC.glob("*.cu"))


def _stale():
    if not LIB.exists():
        return True
    deps = [*CSRC.glob("*"), *(ROOT / "include").glob("*.h"), Path(__file__)]
    mtime = LIB.stat().st_mtime
    return any(p.stat().st_mtime > mtime for p in deps)


def build(force=False, verbose=False):
    if not force and not _stale():
        return LIB
    flags = ["-std=c++17", "-O3", "--fmad=false", "-lineinfo", "--cudart=static", *ARCH,
             "-Xcompiler=-fPIC,-ffp-contract=off,-Wall,-Wno-unknown-pragmas", "-I", str(ROOT / "include"),
             "--shared", "-o", str(LIB)]
    if verbose or os.environ.get("CUSMIC_PTXAS_VERBOSE"):
        flags.insert(0, "-Xptxas=-v")
    cmd = [nvcc(), *flags, *map(str, sources())]
    subprocess.run(cmd, check=True)
    return LIB


if __name__ == "__main__":
    print(build(force="--force" in sys.argv, verbose="-v" in sys.argv))
