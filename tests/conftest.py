"""Shared fixtures.  GPU tests carry @pytest.mark.gpu; everything else runs on CPU."""

import hashlib
import sys
from pathlib import Path

import numpy as np
import pytest

ROOT = Path(__file__).resolve().parents[1]
if str(ROOT) not in sys.path:
    sys.path.insert(0, str(ROOT))

GOLDEN = Path(__file__).parent / "golden" / "fixture_512.npz"


def pytest_configure(config):
    config.addinivalue_line("markers", "gpu: needs a CUDA GPU (B200) and the native library")


@pytest.fixture(scope="session")
def golden():
    """The reference's lacosmic-1.4.0 golden scene (tests/golden/make_golden.py)."""
    g = np.load(GOLDEN)
    data = g["input"]
    mask = np.unpackbits(g["mask_bits"])[:data.size].reshape(data.shape).astype(bool)
    cleaned = data.copy()
    cleaned[mask] = g["masked_values"]
    assert hashlib.sha256(cleaned.tobytes()).digest() == bytes(g["cleaned_sha256"])
    contrast, cr, nb, maxiter = g["settings"]
    return dict(data=data, error=np.full(data.shape, float(g["error"])), mask=mask,
                cleaned=cleaned, settings=dict(contrast=contrast, cr_threshold=cr,
                                               neighbor_threshold=nb, maxiter=int(maxiter)))


@pytest.fixture(scope="session")
def oracle():
    from oracle import oracle as o
    o.lib()
    return o


@pytest.fixture(scope="session")
def cuda():
    import torch
    if not torch.cuda.is_available():
        pytest.fail("CUDA GPU unavailable", pytrace=False)
    from cusmic_b200 import _native
    _native.lib()
    return torch


def assert_bits_equal(actual, expected):
    a = np.ascontiguousarray(actual, dtype=np.float64)
    e = np.ascontiguousarray(expected, dtype=np.float64)
    assert a.shape == e.shape
    diff = a.view(np.uint64) != e.view(np.uint64)
    if diff.any():
        idx = np.argwhere(diff)[:5]
        raise AssertionError(f"{int(diff.sum())} pixels differ, first at {idx.tolist()}: "
                             f"{a[tuple(idx[0])]!r} vs {e[tuple(idx[0])]!r}")
