"""GPU parity of libcusmic_b200.so against the CPU oracle, the reference's golden
fixture, the reference's known answers and (when built) the reference's own
CUDA library.  Pixels and masks must be bit-identical.
"""

import ctypes
import math

import numpy as np
import pytest

from tests import cabi
from tests.conftest import assert_bits_equal

pytestmark = pytest.mark.gpu

MODES = ("mirror", "reflect", "nearest", "wrap", "constant")
SETTINGS = dict(contrast=3.0, cr_threshold=5.0, neighbor_threshold=3.0)


def small_scene(seed, h, w, *, holes=0.0, masked=0.0, rays=None, sky=100.0):
    rng = np.random.default_rng(seed)
    data = sky + rng.normal(0, math.sqrt(sky + 9), (h, w))
    yy, xx = np.mgrid[0:h, 0:w]
    for _ in range(max(1, h * w // 400)):
        cy, cx = rng.uniform(0, h), rng.uniform(0, w)
        data += rng.uniform(50, 2000) * np.exp(-((yy - cy) ** 2 + (xx - cx) ** 2) / 2.0)
    for _ in range(rays if rays is not None else max(1, h * w // 150)):
        y, x = rng.integers(0, h), rng.integers(0, w)
        a = rng.uniform(200, 5000)
        data[y, x] += a
        if rng.random() < 0.4 and x + 1 < w:
            data[y, x + 1] += a / 2
    if holes:
        data[rng.random((h, w)) < holes] = np.nan
    mask = rng.random((h, w)) < masked if masked else None
    return data, mask


def check_against_oracle(oracle, frames, opts_kw, *, ragged=False):
    fr = cabi.Frames(frames)
    opts = cabi.options(**opts_kw)
    if ragged:
        st, msg = cabi.run_ragged(fr, opts)
    else:
        st, msg = cabi.run_batch(cabi._native.lib(), fr, opts)
    settings = {k: v for k, v in opts_kw.items() if k in
                ("contrast", "cr_threshold", "neighbor_threshold", "maxiter", "border")}
    want = []
    for f in frames:
        try:
            want.append(cabi.oracle_frame(oracle, f, **settings))
        except oracle.OracleError as e:
            want.append(e)
    if any(isinstance(wt, Exception) for wt in want):
        assert st == cabi._native.CUSMIC_INVALID and "no finite replacement donors" in msg
        return fr
    assert st == 0, msg
    for (want_clean, want_mask, _), (clean, mask) in zip(want, fr.outputs()):
        np.testing.assert_array_equal(mask, want_mask)
        assert_bits_equal(clean, want_clean)
    return fr


def test_golden_fixture_python_api(cuda, golden):
    from cusmic_b200 import remove_cosmics
    data = cuda.from_numpy(golden["data"]).cuda()
    error = cuda.from_numpy(golden["error"]).cuda()
    cleaned, mask = remove_cosmics(data, error=error, **golden["settings"])
    np.testing.assert_array_equal(mask.cpu().numpy(), golden["mask"])
    assert_bits_equal(cleaned.cpu().numpy(), golden["cleaned"])


def test_golden_fixture_host_api(cuda, golden):
    """The host entry point, as reference test/test_reference.c:25-120 calls it."""
    from cusmic_b200 import _native
    data = np.ascontiguousarray(golden["data"])
    error = np.ascontiguousarray(golden["error"])
    im = _native.Image(data.ctypes.data, error.ctypes.data, None, None, None, None, 512, 512)
    o = cabi.options(contrast=1.0, cr_threshold=5.0, neighbor_threshold=5.0)
    clean = np.empty_like(data)
    mask = np.empty(data.shape, np.uint8)
    msg = ctypes.create_string_buffer(256)
    st = _native.lib().remove_cosmics(ctypes.byref(im), ctypes.byref(o), clean.ctypes.data,
                                      mask.ctypes.data, msg, 256)
    assert st == 0, msg.value
    np.testing.assert_array_equal(mask.astype(bool), golden["mask"])
    assert_bits_equal(clean, golden["cleaned"])


def test_plain_512_noise_model(cuda, oracle):
    from cusmic_b200 import scenes
    sc = scenes.plain_512()
    f = sc.frames[0]
    frames = [dict(data=f.data, gain=2.0, readnoise=5.0, background=0.0)]
    check_against_oracle(oracle, frames, dict(SETTINGS, gain=2.0, readnoise=5.0, background=0.0))


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("path", ("error", "model"))
def test_modes_masks_holes_background(cuda, oracle, mode, path):
    data, mask = small_scene(MODES.index(mode) * 2 + (path == "model"), 70, 93, holes=0.01, masked=0.02)
    rng = np.random.default_rng(7)
    frame = dict(data=data, mask=mask, background=rng.uniform(0, 50, data.shape))
    if path == "error":
        frame["error"] = np.sqrt(np.abs(np.nan_to_num(data)) + 9)
    else:
        frame["gain"] = rng.uniform(0.8, 1.2, data.shape)
        frame["readnoise"] = 3.0
    check_against_oracle(oracle, [frame], dict(SETTINGS, border=mode,
                                               readnoise=frame.get("readnoise", 0.0)))


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("shape", ((1, 1), (1, 9), (9, 1), (2, 2), (3, 5), (5, 3), (2, 40),
                                   (40, 2), (33, 31), (64, 65)))
def test_small_shapes(cuda, oracle, mode, shape):
    data, _ = small_scene(shape[0] * 100 + shape[1], *shape, rays=max(1, shape[0] * shape[1] // 30))
    frame = dict(data=data, gain=1.0, readnoise=3.0)
    check_against_oracle(oracle, [frame], dict(SETTINGS, border=mode, gain=1.0, readnoise=3.0))


@pytest.mark.parametrize("thresholds", ((0.0, 0.0, 0.0), (1.0, 5.0, 5.0), (3.0, 2.0, 0.5),
                                        (2.0, 3.0, 5.0)))
def test_thresholds(cuda, oracle, thresholds):
    contrast, cr, nb = thresholds
    data, _ = small_scene(11, 48, 64)
    frame = dict(data=data, error=np.full(data.shape, 10.0))
    check_against_oracle(oracle, [frame], dict(contrast=contrast, cr_threshold=cr,
                                               neighbor_threshold=nb))


def test_ragged_batch_per_frame_scalars(cuda, oracle):
    frames = []
    rng = np.random.default_rng(5)
    for i, (h, w) in enumerate(((40, 70), (128, 33), (17, 200), (96, 96), (5, 7))):
        data, mask = small_scene(20 + i, h, w, holes=0.005, masked=0.01)
        frames.append(dict(data=data, mask=mask, gain=float(rng.uniform(1, 4)),
                           readnoise=float(rng.uniform(2, 10)),
                           background=float(rng.uniform(0, 200))))
    check_against_oracle(oracle, frames, dict(SETTINGS), ragged=True)


def test_batch_matches_single_calls(cuda):
    """reference test/test_batch.cu:46-169: a 3-frame 9x9 batch equals single calls."""
    frames = []
    for f in range(3):
        d = np.full((9, 9), 10.0 + f)
        d[4 + f % 2, 4 + f // 2] = 1000 + 100 * f
        frames.append(dict(data=d, error=np.ones((9, 9))))
    lib = cabi._native.lib()
    batch = cabi.Frames(frames)
    assert cabi.run_batch(lib, batch, cabi.options())[0] == 0
    outs = batch.outputs()
    for f, fr in enumerate(frames):
        one = cabi.Frames([fr])
        assert cabi.run_batch(lib, one, cabi.options())[0] == 0
        (c1, m1), = one.outputs()
        assert_bits_equal(outs[f][0], c1)
        np.testing.assert_array_equal(outs[f][1], m1)
        assert m1[4 + f % 2, 4 + f // 2]


def test_graph_plan_matches_plain(cuda, oracle):
    frames = []
    for i, (h, w) in enumerate(((300, 257), (64, 512), (129, 129))):
        data, mask = small_scene(40 + i, h, w, holes=0.002, masked=0.01)
        frames.append(dict(data=data, mask=mask, gain=2.0, readnoise=5.0, background=10.0 * i))
    opts = cabi.options(**SETTINGS)
    want = []
    for f in frames:
        c, m, p = cabi.oracle_frame(oracle, f, **SETTINGS)
        want.append((c, m, p))
    for flags in (0, cabi._native.PLAN_GRAPH):
        fr = cabi.Frames(frames)
        plan = cabi.Plan(fr, opts, flags)
        try:
            for _ in range(2):
                st, msg = plan.run()
                assert st == 0, msg
                for (c, m), (wc, wm, _) in zip(fr.outputs(), want):
                    np.testing.assert_array_equal(m, wm)
                    assert_bits_equal(c, wc)
                assert plan.passes() == [p for _, _, p in want]
        finally:
            plan.close()


def test_reference_known_answers(cuda):
    from cusmic_b200 import remove_cosmics
    image = np.full((15, 15), 10.0)
    image[5:10, 5:10] = 1000
    cleaned, mask = remove_cosmics(image, **SETTINGS, error=np.ones_like(image))
    np.testing.assert_array_equal(cleaned.cpu().numpy(), 10)
    np.testing.assert_array_equal(mask.cpu().numpy(), image == 1000)

    image = np.full((3, 3), 0.1)
    cleaned, mask = remove_cosmics(image, **SETTINGS, background=1e12, maxiter=0)
    assert_bits_equal(cleaned.cpu().numpy(), (np.full((3, 3), 0.1) + 1e12) - 1e12)
    assert not mask.any()

    data = np.full((9, 9), 10.0)
    data[2:7, 2:7] = np.nan
    data[3, 3], data[3, 5], data[4, 4] = np.inf, -np.inf, 1000
    data.view("uint64")[2, 2] = 0x7FF8000000000001
    for maxiter in (0, 4):
        clean, mask = remove_cosmics(data, **SETTINGS, error=np.ones_like(data), background=100,
                                     maxiter=maxiter)
        expected = data.copy()
        if maxiter:
            expected[4, 4] = 10
        assert_bits_equal(clean.cpu().numpy(), expected)
        assert int(mask.sum()) == bool(maxiter)
    data[:] = np.nan
    clean, mask = remove_cosmics(data, **SETTINGS, error=np.ones_like(data))
    assert_bits_equal(clean.cpu().numpy(), data)
    assert not mask.any()


@pytest.mark.parametrize("mode", MODES)
def test_singleton_borders(cuda, mode):
    """reference test/test_batch.cu:170-198 through the host entry point."""
    from cusmic_b200 import _native
    probe = np.where(np.arange(9) == 4, 1000.0, 10.0)
    error = np.ones(9)
    want = np.arange(9) == 4
    if mode == "constant":
        want |= np.isin(np.arange(9), (0, 1, 7, 8))
    for w, h in ((9, 1), (1, 9)):
        im = _native.Image(probe.ctypes.data, error.ctypes.data, None, None, None, None, w, h)
        o = cabi.options(border=mode)
        clean = np.empty(9)
        mask = np.empty(9, np.uint8)
        msg = ctypes.create_string_buffer(256)
        assert _native.lib().remove_cosmics(ctypes.byref(im), ctypes.byref(o), clean.ctypes.data,
                                            mask.ctypes.data, msg, 256) == 0, msg.value
        np.testing.assert_array_equal(clean, 10)
        np.testing.assert_array_equal(mask.astype(bool), want)


def test_host_api_keeps_special_bits_and_outputs_on_failure(cuda):
    """reference test/test_api.c:22-57."""
    from cusmic_b200 import _native
    data = np.array([1, -0.0, 3, 4])
    data.view(np.uint64)[2] = 0x7FF8000000001234
    before = data.copy()
    im = _native.Image(data.ctypes.data, None, None, None, None, None, 2, 2)
    o = cabi.options(maxiter=0)
    clean = np.full(4, 9.0)
    mask = np.full(4, 9, np.uint8)
    msg = ctypes.create_string_buffer(128)
    L = _native.lib()
    assert L.remove_cosmics(ctypes.byref(im), ctypes.byref(o), clean.ctypes.data,
                            mask.ctypes.data, msg, 128) == 0
    assert_bits_equal(clean, before)
    assert_bits_equal(data, before)
    assert not mask.any()
    o.cr_threshold = math.nan
    clean[:] = 9
    mask[:] = 9
    assert L.remove_cosmics(ctypes.byref(im), ctypes.byref(o), clean.ctypes.data,
                            mask.ctypes.data, msg, 128) == _native.CUSMIC_INVALID
    assert (clean == 9).all() and (mask == 9).all()


def test_no_donor_error(cuda):
    from cusmic_b200 import remove_cosmics
    data = np.full((7, 7), 10.0)
    data[3, 3] = 1000
    mask = np.ones((7, 7), bool)
    mask[3, 3] = False
    with pytest.raises(ValueError, match="no finite replacement donors"):
        remove_cosmics(data, **SETTINGS, error=np.ones_like(data), mask=mask)


def test_stream_handoff(cuda):
    """reference test/test_streams.py:7-33 with torch streams and events."""
    from cusmic_b200 import Cleaner, Image
    torch = cuda
    producer, consumer = torch.cuda.Stream(), torch.cuda.Stream()
    data = torch.empty((9, 9), dtype=torch.float64, device="cuda")
    error = torch.empty((9, 9), dtype=torch.float64, device="cuda")
    with torch.cuda.stream(producer):
        torch.cuda._sleep(10_000_000)
        data.fill_(10)
        data[4, 4] = 1000
        error.fill_(1)
    ready = producer.record_event()
    consumer.wait_event(ready)
    with torch.cuda.stream(consumer):
        clean, mask = Cleaner()(Image(data, error=error))
    np.testing.assert_array_equal(clean.cpu().numpy(), 10)
    assert int(mask.sum()) == 1


@pytest.mark.parametrize("workload", ("plain_512", "stack_1024"))
def test_reference_library_parity(cuda, workload):
    """Bit parity with the reference's own CUDA library built for sm_100a."""
    ref = cabi.reference_lib()
    if ref is None:
        pytest.skip("oracle/_ref/libcusmic_ref.so was not built")
    from cusmic_b200 import scenes
    if workload == "plain_512":
        f = scenes.plain_512().frames[0]
        frames = [dict(data=f.data)]
        kw = dict(SETTINGS, gain=2.0, readnoise=5.0, background=0.0)
    else:
        sc = scenes.stack_2048(frames=2, size=1024)
        frames = [dict(data=f.data, error=sc.error, mask=sc.mask) for f in sc.frames]
        kw = dict(SETTINGS)
    mine, theirs = cabi.Frames(frames), cabi.Frames(frames)
    assert cabi.run_batch(cabi._native.lib(), mine, cabi.options(**kw))[0] == 0
    st, msg = cabi.run_batch(ref, theirs, cabi.options(**kw))
    assert st == 0, msg
    for (c1, m1), (c2, m2) in zip(mine.outputs(), theirs.outputs()):
        np.testing.assert_array_equal(m1, m2)
        assert_bits_equal(c1, c2)


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("shape", ((1, 2), (2, 2), (5, 4), (33, 2), (31, 256), (40, 258),
                                   (70, 94), (65, 512), (37, 514), (3, 1000)))
def test_error_map_even_widths(cuda, oracle, mode, shape):
    """Even widths with an error map run the bulk-copy detection kernel (rows
    16-byte aligned); holes, a mask and a background map exercise every bit."""
    h, w = shape
    data, mask = small_scene(h * 1000 + w, h, w, holes=0.01, masked=0.02,
                             rays=max(1, h * w // 40))
    rng = np.random.default_rng(w)
    frame = dict(data=data, mask=mask, background=rng.uniform(0, 50, data.shape),
                 error=np.sqrt(np.abs(np.nan_to_num(data)) + 9))
    check_against_oracle(oracle, [frame], dict(SETTINGS, border=mode))


@pytest.mark.parametrize("mode", ("mirror", "wrap", "constant"))
def test_ragged_error_maps_mixed_alignment(cuda, oracle, mode):
    """A ragged batch whose frames alternate between the bulk kernel (even
    width, aligned offset) and the strip kernel (odd width, or an offset that
    an odd-sized frame before it left 8 bytes off a 16-byte boundary)."""
    frames = []
    for i, (h, w) in enumerate(((40, 300), (17, 33), (64, 256), (33, 130), (9, 7), (50, 514))):
        data, mask = small_scene(60 + i, h, w, holes=0.005, masked=0.01, rays=max(2, h * w // 60))
        frames.append(dict(data=data, mask=mask, error=np.sqrt(np.abs(np.nan_to_num(data)) + 9),
                           background=float(10 * i)))
    check_against_oracle(oracle, frames, dict(SETTINGS, border=mode), ragged=True)


@pytest.mark.parametrize("seed", range(12))
def test_structured_scenes_heavy_masks(cuda, oracle, seed):
    """Piecewise sky levels (dark and bright 16 x 16 patches), dense cosmic
    rays and a heavy mask, so replacements draw on far-away and darker donors
    and the per-block noise floors are lowered between passes."""
    rng = np.random.default_rng(1000 + seed)
    h, w = int(rng.integers(40, 140)), int(rng.integers(40, 140))
    levels = rng.choice([20.0, 300.0, 5000.0], size=((h + 15) // 16, (w + 15) // 16))
    sky = np.kron(levels, np.ones((16, 16)))[:h, :w]
    data = sky + rng.normal(0, 1, (h, w)) * np.sqrt(sky + 9)
    ys, xs = rng.integers(0, h, h * w // 25), rng.integers(0, w, h * w // 25)
    data[ys, xs] += rng.uniform(300, 20000, ys.size)
    mask = rng.random((h, w)) < rng.uniform(0.2, 0.6)
    mode = MODES[seed % len(MODES)]
    frame = dict(data=data, mask=mask, gain=float(rng.uniform(1, 3)), readnoise=float(rng.uniform(2, 8)))
    check_against_oracle(oracle, [frame], dict(SETTINGS, border=mode, gain=frame["gain"],
                                               readnoise=frame["readnoise"]))


@pytest.mark.parametrize("maps,message", [
    (dict(error=[1, 1, 0, 1]), "error must be finite and positive"),
    (dict(error=[1, math.inf, 1, 1]), "error must be finite and positive"),
    (dict(gain=[1, 1, -1, 1]), "gain must be finite and positive"),
    (dict(gain=[1, 1, 1, 1], readnoise=[0, -1, 0, 0]), "read noise must be finite and nonnegative"),
    (dict(gain=[1, 1, 1, 1], background=[1, 1, math.nan, 1]), "background must be finite"),
    (dict(error=[1, 0, 1, 1], background=[1, math.nan, 1, 1]), "error must be finite and positive"),
])
def test_host_api_map_contents(cuda, maps, message):
    """reference src/api.cu:107-114,161-168: map contents are validated, the
    first failing map (error, gain, read noise, background) is reported and
    the host outputs stay untouched."""
    from cusmic_b200 import _native
    keep = {k: np.ascontiguousarray(v, dtype=np.float64) for k, v in maps.items()}
    data = np.array([10.0, 11, 12, 13])
    ptr = lambda k: keep[k].ctypes.data if k in keep else None
    im = _native.Image(data.ctypes.data, ptr("error"), ptr("gain"), ptr("readnoise"),
                       ptr("background"), None, 2, 2)
    o = cabi.options(gain=1.0 if "error" not in maps else math.nan)
    clean = np.full(4, 9.0)
    mask = np.full(4, 9, np.uint8)
    msg = ctypes.create_string_buffer(128)
    st = _native.lib().remove_cosmics(ctypes.byref(im), ctypes.byref(o), clean.ctypes.data,
                                      mask.ctypes.data, msg, 128)
    assert st == _native.CUSMIC_INVALID and msg.value.decode() == message
    assert (clean == 9).all() and (mask == 9).all()


def clustered_scene(seed, h, w):
    """Cosmic-ray clusters whose halos fall off gradually, so a low
    neighbor_threshold keeps flagging pixels next to the last pass's
    replacements for several passes."""
    rng = np.random.default_rng(seed)
    data = 200 + rng.normal(0, 15, (h, w))
    for _ in range(max(1, h * w // 60)):
        y, x = int(rng.integers(0, h)), int(rng.integers(0, w))
        amp = rng.uniform(500, 20000)
        for dy in range(-3, 4):
            for dx in range(-3, 4):
                if 0 <= y + dy < h and 0 <= x + dx < w:
                    data[y + dy, x + dx] += amp * rng.uniform(0.05, 0.7) ** (abs(dy) + abs(dx))
    return data


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("path", ("error", "model"))
@pytest.mark.parametrize("shape", ((7, 9), (12, 13), (26, 30), (90, 77)))
def test_incremental_passes(cuda, oracle, mode, path, shape):
    """Passes after the first re-evaluate only the neighbourhood of the pixels
    the last replacement changed: many passes (maxiter 8), frames narrower
    than that neighbourhood (wrap folds it onto itself), every border mode."""
    h, w = shape
    seed = h * 1000 + w * 10 + MODES.index(mode) * 2 + (path == "model")
    data = clustered_scene(seed, h, w)
    frame = dict(data=data)
    opts = dict(contrast=1.0, cr_threshold=4.0, neighbor_threshold=1.5, maxiter=8, border=mode)
    if path == "error":
        frame["error"] = np.sqrt(np.abs(data) / 1.5 + 16)
    else:
        frame.update(gain=1.5, readnoise=4.0)
        opts.update(gain=1.5, readnoise=4.0)
    settings = {k: v for k, v in opts.items() if k not in ("gain", "readnoise")}
    _, _, passes = cabi.oracle_frame(oracle, frame, **settings)
    if h * w > 1000:
        assert passes >= 3  # the scene exercises the incremental passes
    check_against_oracle(oracle, [frame], opts)


def test_incremental_passes_ragged_stops(cuda, oracle):
    """A ragged batch whose frames stop after different numbers of passes."""
    frames = []
    for i, (h, w) in enumerate(((60, 70), (33, 130), (9, 7), (80, 41), (20, 200))):
        data = clustered_scene(500 + i, h, w) if i % 2 == 0 else small_scene(500 + i, h, w)[0]
        frames.append(dict(data=data, error=np.sqrt(np.abs(data) / 1.5 + 16)))
    check_against_oracle(oracle, frames, dict(contrast=1.0, cr_threshold=4.0,
                                              neighbor_threshold=1.5, maxiter=6), ragged=True)


@pytest.mark.parametrize("mode", ("mirror", "wrap", "constant"))
def test_ragged_mixed_error_maps_and_noise_model(cuda, oracle, mode):
    """Error-map and noise-model frames in one ragged batch: each kind runs its
    own candidate kernel, noise-model seeds go through the seed list and the
    error-map entries of that list stay empty."""
    frames = []
    for i, (h, w) in enumerate(((40, 300), (33, 130), (64, 96), (17, 33), (50, 514), (9, 7))):
        if i % 3 == 0:
            data = clustered_scene(700 + i, h, w)
        else:
            data = small_scene(700 + i, h, w, holes=0.005, rays=max(2, h * w // 60))[0]
        f = dict(data=data)
        if i % 2 == 0:
            f["error"] = np.sqrt(np.abs(np.nan_to_num(data)) / 1.5 + 16)
        else:
            f.update(gain=1.0 + 0.5 * i, readnoise=3.0 + i)
        frames.append(f)
    check_against_oracle(oracle, frames, dict(SETTINGS, border=mode, maxiter=5), ragged=True)


@pytest.mark.parametrize("kw,message", [
    (dict(error=np.array([[1.0, 0.0], [1.0, 1.0]])), "error must be positive"),
    (dict(error=np.array([[1.0, np.inf], [1.0, 1.0]])), "error must be finite"),
    (dict(error=np.array([[np.nan, 0.0], [1.0, 1.0]]), background=np.nan), "error must be finite"),
    (dict(effective_gain=-1.0, readnoise=1.0), "effective_gain must be positive"),
    (dict(effective_gain=np.array([[1.0, 2.0], [np.inf, 1.0]]), readnoise=-1.0),
     "effective_gain must be finite"),
    (dict(effective_gain=1.0, readnoise=np.array([[0.0, -1.0], [0.0, 0.0]])),
     "readnoise must be nonnegative"),
    (dict(effective_gain=1.0, readnoise=1.0, background=np.array([[1.0, np.nan], [1.0, 1.0]])),
     "background must be finite"),
])
def test_image_map_validation(cuda, kw, message):
    """Python Image checks every map's contents on the device and reads them
    back at once; the first failing check, in field order, raises the
    reference's error (mod/cusmic/image.py:60-65)."""
    from cusmic_b200 import Image
    with pytest.raises(ValueError, match=message):
        Image(np.ones((2, 2)), **kw)
    Image(np.ones((2, 2)), effective_gain=2.0, readnoise=1.0, background=0.5)


def test_host_api_pageable_and_pinned_buffers(cuda):
    """The host entry point copies page-locked buffers by DMA and pageable ones
    through pinned staging chunks (16 MiB, filled by host threads); both give
    the same bits.  The frame spans two chunks per float64 plane."""
    import torch
    h, w = 1100, 2048
    rng = np.random.default_rng(4242)
    data = 100 + rng.normal(0, 10, (h, w))
    ys, xs = rng.integers(0, h, 3000), rng.integers(0, w, 3000)
    data[ys, xs] += rng.uniform(200, 5000, ys.size)
    data[rng.random((h, w)) < 0.001] = np.nan
    mask = rng.random((h, w)) < 0.005
    error = np.sqrt(np.abs(np.nan_to_num(data)) + 9)
    o = cabi.options(**SETTINGS)
    outs = []
    for pinned in (False, True):
        if pinned:
            pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory()
            d, e, m = pin(data), pin(error), pin(mask.astype(np.uint8))
            c = torch.full((h, w), 7.0, dtype=torch.float64).pin_memory()
            f = torch.full((h, w), 7, dtype=torch.uint8).pin_memory()
            ptrs = (d.data_ptr(), e.data_ptr(), m.data_ptr(), c.data_ptr(), f.data_ptr())
        else:
            d, e, m = (np.ascontiguousarray(a) for a in (data, error, mask.astype(np.uint8)))
            c, f = np.full((h, w), 7.0), np.full((h, w), 7, np.uint8)
            ptrs = (d.ctypes.data, e.ctypes.data, m.ctypes.data, c.ctypes.data, f.ctypes.data)
        im = cabi._native.Image(ptrs[0], ptrs[1], None, None, None, ptrs[2], w, h)
        msg = ctypes.create_string_buffer(256)
        st = cabi._native.lib().remove_cosmics(ctypes.byref(im), ctypes.byref(o), ptrs[3], ptrs[4],
                                               msg, 256)
        assert st == 0, msg.value
        outs.append((c.numpy().copy(), f.numpy().copy()) if pinned else (c.copy(), f.copy()))
    np.testing.assert_array_equal(outs[0][1], outs[1][1])
    assert_bits_equal(outs[0][0], outs[1][0])
    assert outs[0][1].any()


@pytest.mark.parametrize("seed", range(40))
def test_seeded_random_scenes(cuda, oracle, seed):
    """Seeded random scenes against the oracle: sizes, border modes,
    thresholds, pass counts, error map or noise model, holes, masks and
    backgrounds all drawn from the seed."""
    rng = np.random.default_rng(90000 + seed)
    h, w = int(rng.integers(3, 130)), int(rng.integers(3, 130))
    data = clustered_scene(int(rng.integers(1 << 30)), h, w) if rng.random() < 0.5 else \
        small_scene(int(rng.integers(1 << 30)), h, w, rays=max(1, h * w // int(rng.integers(20, 200))))[0]
    if rng.random() < 0.4:
        data[rng.random((h, w)) < rng.uniform(0, 0.03)] = np.nan
    frame = dict(data=data)
    if rng.random() < 0.4:
        frame["mask"] = rng.random((h, w)) < rng.uniform(0, 0.2)
    if rng.random() < 0.3:
        frame["background"] = rng.uniform(0, 50, (h, w)) if rng.random() < 0.5 else float(rng.uniform(0, 50))
    cr = float(rng.uniform(2, 8))
    opts = dict(contrast=float(rng.uniform(0.5, 5)), cr_threshold=cr,
                neighbor_threshold=float(rng.uniform(0.5, cr)), maxiter=int(rng.integers(1, 9)),
                border=MODES[int(rng.integers(len(MODES)))])
    if rng.random() < 0.5:
        frame["error"] = np.sqrt(np.abs(np.nan_to_num(data)) * rng.uniform(0.3, 1.0) + 9)
    else:
        g, r = float(rng.uniform(0.8, 3)), float(rng.uniform(1, 8))
        frame.update(gain=g, readnoise=r)
        opts.update(gain=g, readnoise=r)
    if isinstance(frame.get("background"), float):
        opts["background"] = frame["background"]
    check_against_oracle(oracle, [frame], opts)


def test_host_api_concurrent_calls(cuda):
    """Host entry point calls from several threads at once (each call leases
    its own workspace; the staging threads are shared) give the same bits as
    the same calls one at a time."""
    import threading
    h, w = 700, 1500
    frames = []
    for i in range(4):
        rng = np.random.default_rng(700 + i)
        data = 100 + rng.normal(0, 10, (h, w))
        ys, xs = rng.integers(0, h, 800), rng.integers(0, w, 800)
        data[ys, xs] += rng.uniform(200, 5000, ys.size)
        frames.append((data, np.sqrt(np.abs(data) + 9)))
    o = cabi.options(**SETTINGS)

    def clean(data, error):
        out, flags = np.empty((h, w)), np.empty((h, w), np.uint8)
        im = cabi._native.Image(data.ctypes.data, error.ctypes.data, None, None, None, None, w, h)
        msg = ctypes.create_string_buffer(256)
        st = cabi._native.lib().remove_cosmics(ctypes.byref(im), ctypes.byref(o), out.ctypes.data,
                                               flags.ctypes.data, msg, 256)
        assert st == 0, msg.value
        return out, flags

    want = [clean(*f) for f in frames]
    got = [None] * len(frames)

    def work(i):
        got[i] = clean(*frames[i])

    threads = [threading.Thread(target=work, args=(i,)) for i in range(len(frames))]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    for (wc, wf), g in zip(want, got):
        assert g is not None
        np.testing.assert_array_equal(g[1], wf)
        assert_bits_equal(g[0], wc)


@pytest.mark.parametrize("mode", ("mirror", "constant"))
@pytest.mark.parametrize("path", ("error", "model"))
@pytest.mark.parametrize("shape", ((16, 16), (40, 48), (33, 80), (21, 528), (9, 1040)))
def test_bulk_prepare_widths(cuda, oracle, mode, path, shape):
    """Frames without a background map whose width is a multiple of 16 take the
    bulk-staged prepare: half-filled last bit words (w % 32 == 16), a partial
    last 512-pixel segment, holes, a mask and a scalar background; noise-model
    frames also write their row minima there."""
    h, w = shape
    data, mask = small_scene(h * 31 + w, h, w, holes=0.01, masked=0.02, rays=max(1, h * w // 40))
    frame = dict(data=data, mask=mask, background=25.0)
    opts = dict(SETTINGS, border=mode, background=25.0)
    if path == "error":
        frame["error"] = np.sqrt(np.abs(np.nan_to_num(data)) + 9)
    else:
        frame.update(gain=1.5, readnoise=4.0)
        opts.update(gain=1.5, readnoise=4.0)
    check_against_oracle(oracle, [frame], opts)


@pytest.mark.parametrize("mode", ("mirror", "wrap"))
def test_bulk_prepare_ragged_mixed(cuda, oracle, mode):
    """A ragged batch that takes the bulk-staged prepare (widths multiples of
    16, no background maps) with error-map and noise-model frames mixed: row
    minima only for the noise-model frames, per-frame scalar backgrounds."""
    frames = []
    for i, (h, w) in enumerate(((40, 48), (33, 528), (20, 16), (17, 1040), (64, 96))):
        data, mask = small_scene(900 + i, h, w, holes=0.005, masked=0.01 if i % 2 else 0.0,
                                 rays=max(2, h * w // 60))
        f = dict(data=data, background=float(5 * i))
        if mask is not None:
            f["mask"] = mask
        if i % 2 == 0:
            f["error"] = np.sqrt(np.abs(np.nan_to_num(data)) / 1.5 + 16)
        else:
            f.update(gain=1.0 + 0.5 * i, readnoise=3.0 + i)
        frames.append(f)
    check_against_oracle(oracle, frames, dict(SETTINGS, border=mode), ragged=True)


def test_prepare_unaligned_input(cuda, oracle):
    """An input 8 bytes off a 16-byte boundary (float64-aligned, so accepted)
    cannot be bulk-copied: that batch takes the register-staged prepare, with
    the same bits."""
    import torch
    h, w = 40, 64
    data, mask = small_scene(77, h, w, holes=0.01, masked=0.02, rays=30)
    frame = dict(data=data, mask=mask, error=np.sqrt(np.abs(np.nan_to_num(data)) + 9))
    fr = cabi.Frames([frame])
    buf = torch.empty(h * w + 1, dtype=torch.float64, device="cuda")
    buf[1:] = torch.from_numpy(data.ravel()).cuda()
    fr.keep.append(buf)
    fr.ims[0].data = buf.data_ptr() + 8
    assert fr.ims[0].data % 16 == 8
    st, msg = cabi.run_batch(cabi._native.lib(), fr, cabi.options(**SETTINGS))
    assert st == 0, msg
    want_clean, want_mask, _ = cabi.oracle_frame(oracle, frame, **SETTINGS)
    (clean, got_mask), = fr.outputs()
    np.testing.assert_array_equal(got_mask, want_mask)
    assert_bits_equal(clean, want_clean)


@pytest.mark.parametrize("seed", range(6))
def test_large_replacement_windows(cuda, oracle, seed):
    """Square blocks of holes (3 to 17 pixels across) and masked squares next
    to cosmic rays, on a sky of few distinct values with signed zeros, so the
    hole fill and the replacement use windows from 5 x 5 up past 16 x 16:
    every median path (a warp sort of 25, the sorted keys of up to 64 and 128
    cells, the radix select beyond) must pick the reference's ranks in key
    order, -0 below +0."""
    rng = np.random.default_rng(7100 + seed)
    h, w = int(rng.integers(48, 96)), int(rng.integers(48, 96))
    data = rng.choice(np.array([-0.0, 0.0, 1.0, -1.0, 2.0, 0.5]), size=(h, w))
    mask = np.zeros((h, w), bool)
    for size in (3, 5, 7, 9, 11, 13, 17):
        y, x = int(rng.integers(0, h - size)), int(rng.integers(0, w - size))
        data[y:y + size, x:x + size] = np.nan
    for size in (6, 10, 14):
        y, x = int(rng.integers(1, h - size - 1)), int(rng.integers(1, w - size - 1))
        mask[y:y + size, x:x + size] = True
        data[y + size // 2, x - 1] += 5000.0  # a ray at the block's edge grows into it
        data[y + size // 2, x] += 3000.0
    frame = dict(data=data, mask=mask, error=np.full((h, w), 0.3))
    if seed % 2:
        frame = dict(data=data + 3.0, mask=mask, gain=1.5, readnoise=0.5)
    opts = dict(SETTINGS, maxiter=3, border=MODES[seed % len(MODES)])
    if "gain" in frame:
        opts.update(gain=1.5, readnoise=0.5)
    check_against_oracle(oracle, [frame], opts)


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("w", (64, 61))
def test_hole_fill_signed_zero_donors(cuda, oracle, mode, w):
    """Isolated holes (2% NaN, some on edges and corners) on a field of +0, -0
    and 1.0 with masked pixels, so first fill windows hold even and odd donor
    counts whose middle values are zeros of either sign: the per-hole fill
    must give the reference's bits (the exchange network decides which zero a
    tie yields; windows with both signs are left to it), with width 64 for the
    fused prepare and 61 for the two-kernel path."""
    rng = np.random.default_rng(9100 + w + MODES.index(mode))
    h = 40
    data = rng.choice(np.array([0.0, -0.0, 1.0]), size=(h, w), p=[0.4, 0.4, 0.2])
    data[rng.random((h, w)) < 0.02] = np.nan
    data[0, 0] = data[h - 1, w - 1] = data[0, w - 1] = np.nan
    mask = rng.random((h, w)) < 0.15
    frame = dict(data=data, mask=mask, error=np.full((h, w), 0.4))
    check_against_oracle(oracle, [frame], dict(SETTINGS, maxiter=2, border=mode))
