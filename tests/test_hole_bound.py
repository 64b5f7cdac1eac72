"""The exactness argument of prep_detect_kernel (cusmic_b200/csrc/prep_detect.cuh),
checked on the CPU with the kernel's arithmetic restated in numpy.

The kernel takes the Laplacian bound of the dense detection on the input rows
before the hole fill, with every hole (non-finite input) entering as -inf.  The
claims: a pixel that is not a hole and whose Laplacian reads no hole gets the
same bound as from the filled pixels; one that reads a hole gets +inf (which
lists it for classify_kernel to recompute); no pixel that is not a hole gets a
NaN.  The bound is the reference's Laplacian (src/filters.cuh:86-105) with
positive(v) replaced by v with its high word cleared when v is negative, from
quarter values and shared differences, as the kernel computes it.
"""

import numpy as np


def pos_ub(v):
    bits = v.view(np.uint64)
    neg = (bits >> np.uint64(63)) == 1
    return np.where(neg, (bits & np.uint64(0xFFFFFFFF)).view(np.float64), v)


def lap_bound(q):
    """The bound at the interior pixels of a 2-D array of quarter values,
    nearest-neighbour differences shared as the kernel shares them."""
    c = q[1:-1, 1:-1]
    up = c - q[:-2, 1:-1]
    down = c - q[2:, 1:-1]
    left = c - q[1:-1, :-2]
    right = c - q[1:-1, 2:]
    return (pos_ub(up + left) + pos_ub(up + right)) + (pos_ub(down + left) + pos_ub(down + right))


def test_holes_as_minus_infinity():
    rng = np.random.default_rng(5)
    for trial in range(200):
        h, w = 12, 40
        data = rng.normal(1000.0, 30.0, (h, w))
        data[rng.random((h, w)) < 0.3] = 5000.0  # rays
        holes = rng.random((h, w)) < (0.02 + 0.1 * (trial % 3))
        kinds = np.array([np.nan, np.inf, -np.inf])
        data[holes] = kinds[rng.integers(0, 3, int(holes.sum()))]
        filled = np.where(holes, rng.normal(1000.0, 30.0, (h, w)), data)  # any fill value
        with np.errstate(invalid="ignore", over="ignore"):
            fused = lap_bound(np.where(np.isfinite(data), data * 0.25, -np.inf))
            after = lap_bound(filled * 0.25)
        inner = holes[1:-1, 1:-1]
        reads = (holes[:-2, 1:-1] | holes[2:, 1:-1] | holes[1:-1, :-2] | holes[1:-1, 2:]) & ~inner
        plain = ~inner & ~reads
        assert not np.isnan(fused[~inner]).any()
        assert np.array_equal(fused[plain].view(np.uint64), after[plain].view(np.uint64))
        assert (fused[reads] == np.inf).all()
