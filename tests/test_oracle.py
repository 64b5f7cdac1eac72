"""CPU tests of the oracle: pinned to the reference's golden vectors and KATs.

The oracle (oracle/cusmic_oracle.c) restates the reference CUDA library; here
it must reproduce lacosmic 1.4.0's saved output bit for bit and the known
answers of the reference's own tests (test/test_cleaner.py, test/test_api.c,
test/test_batch.cu).
"""

import numpy as np
import pytest
from scipy import ndimage

from tests.conftest import assert_bits_equal

MODES = ("mirror", "reflect", "nearest", "wrap", "constant")
SETTINGS = dict(contrast=3, cr_threshold=5, neighbor_threshold=3)


def test_golden_fixture_bit_exact(oracle, golden):
    """reference test/test_reference.py:52-62 and test/test_reference.c:25-120."""
    clean, mask, passes = oracle.clean_frame(golden["data"], error=golden["error"],
                                             **golden["settings"])
    assert mask.sum() == 6518
    np.testing.assert_array_equal(mask, golden["mask"])
    assert_bits_equal(clean, golden["cleaned"])
    assert passes == 3


def test_window_median_matches_odd_even_transposition(oracle):
    rng = np.random.default_rng(1)
    for n in (9, 25, 49):
        for _ in range(300):
            v = rng.integers(-3, 3, n).astype(float)
            v[rng.random(n) < 0.15] = np.nan
            v[rng.random(n) < 0.1] = -0.0
            ref = oracle.oets(v)[n // 2]
            got = oracle.window_median(v)
            assert np.array([got]).view(np.uint64)[0] == np.array([ref]).view(np.uint64)[0]


def test_oets_sorts_without_nan(oracle):
    rng = np.random.default_rng(2)
    v = rng.normal(size=49)
    np.testing.assert_array_equal(oracle.oets(v), np.sort(v))


def test_bitonic32_sorts(oracle):
    rng = np.random.default_rng(3)
    for _ in range(50):
        v = rng.normal(size=32)
        v[rng.random(32) < 0.3] = np.inf
        np.testing.assert_array_equal(oracle.bitonic32(v), np.sort(v))


@pytest.mark.parametrize("mode", MODES)
def test_border_index_matches_numpy_pad(oracle, mode):
    pad = {"mirror": "reflect", "reflect": "symmetric", "nearest": "edge", "wrap": "wrap",
           "constant": "constant"}[mode]
    for n in (1, 2, 3, 5, 8):
        base = np.arange(n)
        kw = {"constant_values": -1} if pad == "constant" else {}
        padded = np.pad(base, 3 * n + 4, mode=pad, **kw)
        for x in range(-(3 * n + 4), n + 3 * n + 4):
            want = padded[x + 3 * n + 4]
            assert oracle.lib().oracle_border_index(x, n, oracle.BORDERS[mode]) == want, (n, x)


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("size", (3, 5, 7))
def test_median_filter_matches_scipy(oracle, mode, size):
    """Cross-check of the restated median against scipy.ndimage (NaN-free)."""
    rng = np.random.default_rng(size)
    for shape in ((13, 17), (1, 9), (9, 1), (2, 3)):
        a = rng.normal(size=shape)
        np.testing.assert_array_equal(oracle.median_filter(a, size, mode),
                                      ndimage.median_filter(a, size=size, mode=mode))


@pytest.mark.parametrize("mode", MODES)
def test_laplacian_borders(oracle, mode):
    """reference test/test_cleaner.py:33-47: collapsed form = replicate, convolve,
    clip and 2x2 block sum."""
    kernel = np.array([[0, -1, 0], [-1, 4, -1], [0, -1, 0]], dtype=float)
    for pixels in ([[12, -4, 20]], [[12], [-4], [20]], [[12, -4], [20, 0]]):
        image = np.asarray(pixels, dtype=float)
        sampled = np.repeat(np.repeat(image / 4, 2, axis=0), 2, axis=1)
        lap2 = np.maximum(ndimage.convolve(sampled, kernel, mode=mode), 0)
        expected = (lap2[0::2, 0::2] + lap2[0::2, 1::2]) + (lap2[1::2, 0::2] + lap2[1::2, 1::2])
        np.testing.assert_array_equal(oracle.laplacian(image, mode), expected)


def test_dense_patch(oracle):
    """reference test/test_cleaner.py:22-30."""
    image = np.full((15, 15), 10.0)
    image[5:10, 5:10] = 1000
    cleaned, mask, _ = oracle.clean_frame(image, error=np.ones_like(image), **SETTINGS)
    np.testing.assert_array_equal(cleaned, 10)
    np.testing.assert_array_equal(mask, image == 1000)


def test_zero_iterations_background(oracle):
    """reference test/test_cleaner.py:82-89."""
    image = np.full((3, 3), 0.1)
    cleaned, mask, _ = oracle.clean_frame(image, background=1e12, maxiter=0, **SETTINGS)
    assert_bits_equal(cleaned, (np.full((3, 3), 0.1) + 1e12) - 1e12)
    assert not mask.any()


def test_zero_iterations_keep_special_bits(oracle):
    """reference test/test_api.c:22-42: -0.0 and a NaN payload survive."""
    data = np.array([[1, -0.0], [3, 4]])
    data.view(np.uint64)[1, 0] = 0x7FF8000000001234
    cleaned, mask, _ = oracle.clean_frame(data, maxiter=0)
    assert_bits_equal(cleaned, data)
    assert not mask.any()


def test_nonfinite_pixels(oracle):
    """reference test/test_cleaner.py:92-112."""
    data = np.full((9, 9), 10.0)
    data[2:7, 2:7] = np.nan
    data[3, 3], data[3, 5], data[4, 4] = np.inf, -np.inf, 1000
    data.view("uint64")[2, 2] = 0x7FF8000000000001
    for maxiter in (0, 4):
        clean, mask, _ = oracle.clean_frame(data, error=np.ones_like(data), background=100,
                                            maxiter=maxiter, **SETTINGS)
        expected = data.copy()
        if maxiter:
            expected[4, 4] = 10
        assert_bits_equal(clean, expected)
        assert mask.sum() == bool(maxiter)
    nan = np.full((9, 9), np.nan)
    clean, mask, _ = oracle.clean_frame(nan, error=np.ones_like(nan), **SETTINGS)
    assert_bits_equal(clean, nan)
    assert not mask.any()


def test_independent_shapes(oracle):
    """reference test/test_cleaner.py:115-132."""
    for shape in ((9, 9), (7, 11)):
        data = np.full(shape, 10.0)
        data[3, 3] = 1000
        cleaned, mask, _ = oracle.clean_frame(data, error=np.ones(shape), **SETTINGS)
        np.testing.assert_array_equal(cleaned, 10)
        assert mask.sum() == 1


def test_replacement_expanding_window_and_midpoint(oracle):
    """reference test/test_cleaner.py:135-151."""
    data = np.array([[0.0, 1000, 1000, 1000, 1000, 1000, 60]])
    targets = (data == 1000).astype(np.uint8)
    out = data.copy()
    oracle.lib().oracle_replace(oracle._ptr(out), oracle._ptr(targets, oracle._bp),
                                oracle._ptr(np.zeros_like(targets), oracle._bp), 7, 1)
    np.testing.assert_array_equal(out, [[0, 0, 0, 30, 60, 60, 60]])
    high = np.finfo("float64").max
    out = np.array([[high, 0, high]])
    targets = np.array([[0, 1, 0]], dtype=np.uint8)
    oracle.lib().oracle_replace(oracle._ptr(out), oracle._ptr(targets, oracle._bp),
                                oracle._ptr(np.zeros_like(targets), oracle._bp), 3, 1)
    np.testing.assert_array_equal(out, np.full((1, 3), high))


@pytest.mark.parametrize("mode", MODES)
def test_singleton_borders(oracle, mode):
    """reference test/test_batch.cu:170-198: 1x9 and 9x1 frames; constant mode
    also flags pixels 0, 1, 7 and 8."""
    probe = np.where(np.arange(9) == 4, 1000.0, 10.0)
    want = np.arange(9) == 4
    if mode == "constant":
        want |= np.isin(np.arange(9), (0, 1, 7, 8))
    for shape in ((1, 9), (9, 1)):
        cleaned, mask, _ = oracle.clean_frame(probe.reshape(shape), error=np.ones(shape),
                                              border=mode)
        np.testing.assert_array_equal(cleaned.ravel(), 10)
        np.testing.assert_array_equal(mask.ravel(), want)


def test_no_donors_is_an_error(oracle):
    data = np.full((7, 7), 10.0)
    data[3, 3] = 1000
    mask = np.ones((7, 7), bool)
    mask[3, 3] = False
    with pytest.raises(oracle.OracleError, match="no finite replacement donors"):
        oracle.clean_frame(data, error=np.ones_like(data), mask=mask, **SETTINGS)


def test_thread_count_does_not_change_results(oracle, golden):
    """The CPU baseline times the oracle on one thread and on every core: both
    must compute the same bits."""
    data, err = golden["data"][:160], golden["error"][:160]
    prev = oracle.set_threads(0)
    try:
        out = []
        for n in (1, max(2, prev)):
            assert oracle.set_threads(n) == n
            out.append(oracle.clean_frame(data, error=err, **golden["settings"]))
    finally:
        oracle.set_threads(prev)
    assert_bits_equal(out[0][0], out[1][0])
    assert np.array_equal(out[0][1], out[1][1])
