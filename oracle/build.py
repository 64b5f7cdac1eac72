"""Build recipes for the test oracles (TEST INFRASTRUCTURE ONLY).

* ``build_oracle()`` compiles the plain-C restatement ``cusmic_oracle.c`` into
  ``oracle/_build/liboracle.so`` with the reference's floating-point rules
  (no contraction, IEEE division and square root; reference Makefile:92-105).
* ``build_reference()`` compiles the reference's own CUDA library from its
  sources where they lie (``src/api.cu`` and the headers it includes) into
  ``oracle/_ref/libcusmic_ref.so`` for sm_100a, with the reference's own
  flags (``-std=c++14 --fmad=false``, Makefile:100-103).  Nothing is copied:
  nvcc reads the reference tree directly.  The .so is git-ignored but travels
  with the working tree to a GPU machine, where GPU tests use it as a second,
  independent oracle.  Without the reference tree this step is skipped.

Run ``python oracle/build.py`` or call the functions; both are idempotent.
"""

import os
import shutil
import subprocess
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent
ORACLE_SO = HERE / "_build" / "liboracle.so"
REFERENCE_SO = HERE / "_ref" / "libcusmic_ref.so"
REFERENCE_SRC = Path(os.environ.get("CUSMIC_REFERENCE_SRC", "/root/reference/src"))


def _stale(target, sources):
    if not target.exists():
        return True
    mtime = target.stat().st_mtime
    return any(Path(s).stat().st_mtime > mtime for s in sources)


def build_oracle(force=False):
    src = HERE / "cusmic_oracle.c"
    if force or _stale(ORACLE_SO, [src, Path(__file__)]):
        ORACLE_SO.parent.mkdir(parents=True, exist_ok=True)
        cmd = ["gcc", "-std=c11", "-O2", "-fPIC", "-shared", "-fopenmp",
               "-ffp-contract=off", "-fno-fast-math", "-Wall", "-Wextra",
               str(src), "-o", str(ORACLE_SO), "-lm"]
        subprocess.run(cmd, check=True)
    return ORACLE_SO


def build_reference(force=False):
    """Compile the reference CUDA library; returns its path or None."""
    api = REFERENCE_SRC / "api.cu"
    if not api.exists():
        return REFERENCE_SO if REFERENCE_SO.exists() else None
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    sources = [api, *REFERENCE_SRC.glob("*.cuh"), *REFERENCE_SRC.glob("*.h")]
    if force or _stale(REFERENCE_SO, sources):
        REFERENCE_SO.parent.mkdir(parents=True, exist_ok=True)
        cmd = [nvcc, "-std=c++14", "--fmad=false", "--cudart=static", "-O2",
               "-gencode", "arch=compute_100a,code=sm_100a",
               "-Xcompiler=-fPIC,-ffp-contract=off",
               '-DCUSMIC_VERSION="reference-oracle"',
               f"-I{REFERENCE_SRC}", "--shared", str(api), "-o", str(REFERENCE_SO)]
        subprocess.run(cmd, check=True)
    return REFERENCE_SO


if __name__ == "__main__":
    print(build_oracle(force="--force" in sys.argv))
    print(build_reference(force="--force" in sys.argv))
