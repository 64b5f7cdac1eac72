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
  independent oracle.  The reference's ``src`` directory is given as an
  argument or by ``CUSMIC_REFERENCE_SRC``; without it this step is skipped.

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
REFERENCE_ENV = "CUSMIC_REFERENCE_SRC"  # the reference's src directory


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


def build_reference(src=None, force=False):
    """Compile the reference CUDA library from the reference's ``src``
    directory (argument, else $CUSMIC_REFERENCE_SRC); returns its path or None."""
    src = src or os.environ.get(REFERENCE_ENV)
    api = Path(src) / "api.cu" if src else None
    if api is None or not api.exists():
        return REFERENCE_SO if REFERENCE_SO.exists() else None
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    ref_src = api.parent
    sources = [api, *ref_src.glob("*.cuh"), *ref_src.glob("*.h")]
    if force or _stale(REFERENCE_SO, sources):
        REFERENCE_SO.parent.mkdir(parents=True, exist_ok=True)
        cmd = [nvcc, "-std=c++14", "--fmad=false", "--cudart=static", "-O2",
               "-gencode", "arch=compute_100a,code=sm_100a",
               "-Xcompiler=-fPIC,-ffp-contract=off",
               '-DCUSMIC_VERSION="reference-oracle"',
               f"-I{ref_src}", "--shared", str(api), "-o", str(REFERENCE_SO)]
        subprocess.run(cmd, check=True)
    return REFERENCE_SO


if __name__ == "__main__":
    args = [a for a in sys.argv[1:] if not a.startswith("--")]
    print(build_oracle(force="--force" in sys.argv))
    print(build_reference(args[0] if args else None, force="--force" in sys.argv))
