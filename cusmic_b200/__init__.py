"""cusmic_b200: a B200-native L.A.Cosmic cosmic-ray cleaner.

Drop-in for rndsrc/cusmic's Python API (``remove_cosmics``, ``Cleaner``,
``Image``) and C ABI (``include/cusmic.h``), computed by hand-written sm_100a
CUDA kernels in ``libcusmic_b200.so``.  The library is loaded on first use;
every entry point raises ImportError when it has not been built (there is no
CPU fallback).
"""

from .api import Cleaner, Image, remove_cosmics

__version__ = "0.1.0"

__all__ = ["Image", "Cleaner", "remove_cosmics", "__version__"]
