"""remove_cosmics_device_noalloc: the entry point for callers that cannot
allocate device memory when they clean a frame (real-time acquisition loops
that allow allocation only at start-up, processes whose own allocator has
already reserved the GPU's memory).  Its scratch is one static device array
shared by every call and left holding the last call's contents, so two calls
in a row must not see each other's leftovers.  It runs a kernel sequence of its
own (strip and tile dense kernels, a per-row hole fill, no replacement
skipping), so it is checked over every border mode, the noise model with maps,
error maps with masks and holes, zero iterations, the donor error and a side
stream: each result must equal remove_cosmics_device's and the CPU oracle's
bit for bit.

This file is collected last on purpose: if it fails, a run that stops at the
first failure has already run every other test.
"""

import ctypes
import math

import numpy as np
import pytest

from cusmic_b200 import _native
from tests import cabi
from tests.conftest import assert_bits_equal

MODES = ("mirror", "reflect", "nearest", "wrap", "constant")
SETTINGS = dict(contrast=3.0, cr_threshold=5.0, neighbor_threshold=3.0)


def case(kind):
    """(frame dict for tests.cabi.Frames, option scalars) of one scene kind."""
    from cusmic_b200 import scenes
    rng = np.random.default_rng(11 + len(kind))
    if kind == "model":  # plain_512: scalar gain and read noise, zero background
        return dict(data=scenes.plain_512().frames[0].data), dict(gain=2.0, readnoise=5.0,
                                                                  background=0.0)
    data = scenes.make_frame(rng, 300, 257, n_stars=6, n_rays=80).data
    data[rng.random(data.shape) < 0.002] = np.nan
    mask = rng.random(data.shape) < 0.01
    if kind == "error":  # error map, mask, holes, odd width
        return dict(data=data, error=np.sqrt(np.abs(np.nan_to_num(data)) + 6.25), mask=mask), {}
    # gain and read-noise maps with a background map
    return dict(data=data, mask=mask, gain=rng.uniform(1.5, 2.5, data.shape),
                readnoise=rng.uniform(3.0, 6.0, data.shape),
                background=rng.uniform(0.0, 80.0, data.shape)), dict(readnoise=4.0)


def call(entry, frame, opts, stream=None):
    fr = cabi.Frames([frame])
    msg = ctypes.create_string_buffer(256)
    st = entry(fr.ims, ctypes.byref(opts), fr.clean.data_ptr(), fr.mask.data_ptr(), stream, msg,
               256)
    return st, msg.value.decode(), fr


@pytest.mark.gpu
@pytest.mark.parametrize("maxiter", (0, 1, 4))
@pytest.mark.parametrize("kind", ("model", "error", "maps"))
@pytest.mark.parametrize("mode", MODES)
def test_noalloc_matches_device_entry_point_and_oracle(cuda, oracle, mode, kind, maxiter):
    lib = _native.lib()
    frame, scalars = case(kind)
    opts = cabi.options(**SETTINGS, **scalars, maxiter=maxiter, border=mode)
    # Two calls in a row: the second starts from the first one's scratch.
    got = []
    for _ in range(2):
        st, msg, fr = call(lib.remove_cosmics_device_noalloc, frame, opts)
        assert st == 0, msg
        got.append(fr.outputs()[0])
    st, msg, fr = call(lib.remove_cosmics_device, frame, opts)
    assert st == 0, msg
    want_clean, want_mask = fr.outputs()[0]
    settings = dict(SETTINGS, maxiter=maxiter, border=mode)
    # Maps of the frame take precedence over the option scalars, as in the ABI.
    o_clean, o_mask, _ = cabi.oracle_frame(oracle, {**scalars, **frame}, **settings)
    np.testing.assert_array_equal(want_mask, o_mask)
    assert_bits_equal(want_clean, o_clean)
    if maxiter:
        assert o_mask.any()
    for clean, mask in got:
        np.testing.assert_array_equal(mask, want_mask)
        assert_bits_equal(clean, want_clean)


@pytest.mark.gpu
def test_noalloc_no_finite_donor_error(cuda):
    """A new cosmic-ray pixel with every other pixel masked: both entry points
    report the reference's "no finite replacement donors" (CUSMIC_INVALID)."""
    lib = _native.lib()
    data = np.full((7, 7), 10.0)
    data[3, 3] = 1000
    mask = np.ones((7, 7), bool)
    mask[3, 3] = False
    frame = dict(data=data, error=np.ones_like(data), mask=mask)
    opts = cabi.options(**SETTINGS)
    for entry in (lib.remove_cosmics_device_noalloc, lib.remove_cosmics_device,
                  lib.remove_cosmics_device_noalloc):
        st, msg, _ = call(entry, frame, opts)
        assert st == _native.CUSMIC_INVALID
        assert "no finite replacement donors" in msg


@pytest.mark.gpu
def test_noalloc_on_a_side_stream(cuda):
    """The call runs on the caller's stream: a producer stream fills the input
    late (behind a sleep), the call waits on its event through its stream."""
    torch = cuda
    lib = _native.lib()
    frame, scalars = case("error")
    opts = cabi.options(**SETTINGS, **scalars)
    st, msg, ref = call(lib.remove_cosmics_device, frame, opts)
    assert st == 0, msg
    want_clean, want_mask = ref.outputs()[0]
    fr = cabi.Frames([frame])
    data = fr.keep[0]
    host = data.clone()
    data.fill_(0.0)
    producer, side = torch.cuda.Stream(), torch.cuda.Stream()
    with torch.cuda.stream(producer):
        torch.cuda._sleep(5_000_000)
        data.copy_(host)
    side.wait_event(producer.record_event())
    msg = ctypes.create_string_buffer(256)
    st = lib.remove_cosmics_device_noalloc(fr.ims, ctypes.byref(opts), fr.clean.data_ptr(),
                                           fr.mask.data_ptr(), side.cuda_stream, msg, 256)
    assert st == 0, msg.value
    clean, mask = fr.outputs()[0]
    np.testing.assert_array_equal(mask, want_mask)
    assert_bits_equal(clean, want_clean)


def test_noalloc_rejects_frames_beyond_its_scratch():
    lib = _native.lib()
    data = np.zeros(4)
    o = _native.default_options()
    o.gain = 1.0
    msg = ctypes.create_string_buffer(256)
    for w, h in ((1024, 1024), (1, 20000)):
        im = _native.Image(data.ctypes.data, None, None, None, None, None, w, h)
        st = lib.remove_cosmics_device_noalloc(ctypes.byref(im), ctypes.byref(o), 8, 8, None,
                                               msg, 256)
        assert st == _native.CUSMIC_INVALID
        assert b"exceeds the static scratch" in msg.value
    o.cr_threshold = math.nan
    im = _native.Image(data.ctypes.data, None, None, None, None, None, 2, 2)
    assert lib.remove_cosmics_device_noalloc(ctypes.byref(im), ctypes.byref(o), 8, 8, None,
                                             msg, 256) == _native.CUSMIC_INVALID


def test_noalloc_rejects_misaligned_float64_buffers():
    """Validation returns before any launch: an odd address for a float64
    buffer is CUSMIC_INVALID, as for remove_cosmics_device."""
    lib = _native.lib()
    data = np.zeros(8)
    o = _native.default_options()
    o.gain = 1.0
    msg = ctypes.create_string_buffer(256)
    aligned = data.ctypes.data
    for shift in ("data", "clean"):
        im = _native.Image(aligned + (3 if shift == "data" else 0), None, None, None, None, None,
                           2, 2)
        clean = aligned + (5 if shift == "clean" else 0)
        for entry in (lib.remove_cosmics_device_noalloc, lib.remove_cosmics_device):
            st = entry(ctypes.byref(im), ctypes.byref(o), clean, aligned, None, msg, 256)
            assert st == _native.CUSMIC_INVALID
            assert b"must be 8-byte aligned" in msg.value
