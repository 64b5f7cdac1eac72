"""remove_cosmics_device_noalloc: the entry point for callers that cannot
allocate device memory when they clean a frame (code being captured into a
CUDA graph, real-time loops that forbid allocation after start-up, processes
whose allocator has already reserved the GPU).  Its scratch is a static device
array shared by every call, so consecutive calls must not see each other's
leftovers; its results must equal remove_cosmics_device's bit for bit.
"""

import ctypes
import math

import numpy as np
import pytest

from cusmic_b200 import _native
from tests import cabi
from tests.conftest import assert_bits_equal


def frames():
    from cusmic_b200 import scenes
    rng = np.random.default_rng(11)
    plain = scenes.plain_512().frames[0].data
    other = scenes.make_frame(rng, 300, 257, n_stars=6, n_rays=80).data
    other[rng.random(other.shape) < 0.002] = np.nan
    mask = rng.random(other.shape) < 0.01
    return [
        (dict(data=plain), dict(gain=2.0, readnoise=5.0, background=0.0)),
        (dict(data=other, error=np.sqrt(np.abs(np.nan_to_num(other)) + 6.25), mask=mask), {}),
        (dict(data=plain), dict(gain=2.0, readnoise=5.0, background=0.0)),
    ]


def call(entry, frame, scalars):
    fr = cabi.Frames([frame])
    opts = cabi.options(**scalars)
    msg = ctypes.create_string_buffer(256)
    st = entry(fr.ims, ctypes.byref(opts), fr.clean.data_ptr(), fr.mask.data_ptr(), None, msg,
               256)
    assert st == 0, msg.value
    return fr.outputs()[0]


@pytest.mark.gpu
def test_noalloc_matches_device_entry_point(cuda):
    lib = _native.lib()
    for frame, scalars in frames():  # consecutive calls share the static scratch
        got_clean, got_mask = call(lib.remove_cosmics_device_noalloc, frame, scalars)
        want_clean, want_mask = call(lib.remove_cosmics_device, frame, scalars)
        assert want_mask.any()
        np.testing.assert_array_equal(got_mask, want_mask)
        assert_bits_equal(got_clean, want_clean)


def test_noalloc_rejects_frames_beyond_its_scratch():
    lib = _native.lib()
    data = np.zeros(4)
    o = _native.default_options()
    o.gain = 1.0
    msg = ctypes.create_string_buffer(256)
    for w, h in ((1024, 1024), (1, 20000)):
        im = _native.Image(data.ctypes.data, None, None, None, None, None, w, h)
        st = lib.remove_cosmics_device_noalloc(ctypes.byref(im), ctypes.byref(o), 1, 1, None,
                                               msg, 256)
        assert st == _native.CUSMIC_INVALID
        assert b"exceeds the static scratch" in msg.value
    o.cr_threshold = math.nan
    im = _native.Image(data.ctypes.data, None, None, None, None, None, 2, 2)
    assert lib.remove_cosmics_device_noalloc(ctypes.byref(im), ctypes.byref(o), 1, 1, None,
                                             msg, 256) == _native.CUSMIC_INVALID
