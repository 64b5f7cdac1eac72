"""CPU checks of libcusmic_b200.so: it loads, exports every entry point that
include/*.h declares, and validates arguments exactly like the reference's C
ABI (src/api.cu:47-114) without touching a GPU."""

import ctypes
import math
import re
from pathlib import Path

import numpy as np
import pytest

from cusmic_b200 import _native

INCLUDE = Path(__file__).resolve().parents[1] / "include"


def declared_functions():
    names = set()
    for header in INCLUDE.glob("*.h"):
        text = header.read_text()
        names |= set(re.findall(r"^([a-z_][a-z0-9_]*)\(", text, re.M))
    return names


def test_exports_every_declared_symbol():
    names = declared_functions()
    assert names == set(_native.EXPORTS)
    lib = ctypes.CDLL(str(_native.LIB_PATH))
    for name in names:
        assert hasattr(lib, name), name


def test_version_and_defaults():
    L = _native.lib()
    assert L.cusmic_version()
    assert L.cusmic_cuda_version() >= 12000
    o = _native.default_options()
    assert (o.contrast, o.cr_threshold, o.neighbor_threshold) == (3, 5, 3)
    assert math.isnan(o.gain) and o.readnoise == 0 and math.isnan(o.background)
    assert (o.maxiter, o.border) == (4, _native.BORDERS["mirror"])


def call_host(data, w, h, opts=None, error=None, gain=None, background=None):
    buf = {}
    def ptr(a):
        if a is None:
            return None
        a = np.ascontiguousarray(a, dtype=np.float64)
        buf[id(a)] = a
        return a.ctypes.data
    im = _native.Image(ptr(data), ptr(error), ptr(gain), None, ptr(background), None, w, h)
    o = opts or _native.default_options()
    clean = np.full(max(w * h, 1), 9.0)
    mask = np.full(max(w * h, 1), 9, np.uint8)
    msg = ctypes.create_string_buffer(128)
    st = _native.lib().remove_cosmics(ctypes.byref(im), ctypes.byref(o), clean.ctypes.data,
                                      mask.ctypes.data, msg, 128)
    assert (clean == 9).all() and (mask == 9).all()  # outputs untouched on failure
    return st, msg.value.decode()


@pytest.mark.parametrize("field,value,message", [
    ("cr_threshold", math.nan, "invalid detection settings"),
    ("contrast", -1.0, "invalid detection settings"),
    ("neighbor_threshold", math.inf, "invalid detection settings"),
    ("maxiter", -1, "invalid detection settings"),
    ("border", 5, "invalid detection settings"),
])
def test_invalid_settings(field, value, message):
    o = _native.default_options()
    o.gain = 1.0
    setattr(o, field, value)
    st, msg = call_host(np.ones(4), 2, 2, o)
    assert st == _native.CUSMIC_INVALID and msg == message


def test_invalid_arguments():
    o = _native.default_options()
    o.gain = 1.0
    assert call_host(np.ones(4), 0, 2, o) == (_native.CUSMIC_INVALID, "invalid image dimensions")
    assert call_host(None, 2, 2, o)[1] == "frames must have data and the same shape"
    o.gain = math.nan
    assert call_host(np.ones(4), 2, 2, o)[1] == "positive gain or error is required"
    o.gain, o.readnoise = 1.0, -1.0
    assert call_host(np.ones(4), 2, 2, o)[1] == "read noise must be finite and nonnegative"
    o.readnoise, o.background = 0.0, math.inf
    assert call_host(np.ones(4), 2, 2, o)[1] == "background must be finite"
    msg = ctypes.create_string_buffer(64)
    assert _native.lib().remove_cosmics(None, None, None, None, msg, 64) == _native.CUSMIC_INVALID
    assert msg.value == b"invalid images, batch size or output buffers"


def test_ragged_validation():
    o = _native.default_options()
    o.gain = 1.0
    ims = (_native.Image * 2)()
    data = np.ones(64)
    ims[0] = _native.Image(data.ctypes.data, None, None, None, None, None, 8, 8)
    ims[1] = _native.Image(data.ctypes.data, None, None, None, None, None, 0, 3)
    msg = ctypes.create_string_buffer(64)
    st = _native.lib().cusmic_ragged_batch_device(ims, 2, ctypes.byref(o), None, 1, 1, None,
                                                  msg, 64)
    assert st == _native.CUSMIC_INVALID and msg.value == b"invalid image dimensions"
    sc = (_native.FrameScalars * 2)((math.nan, math.nan, math.nan), (-2.0, math.nan, math.nan))
    ims[1] = _native.Image(data.ctypes.data, None, None, None, None, None, 4, 4)
    st = _native.lib().cusmic_ragged_batch_device(ims, 2, ctypes.byref(o), sc, 1, 1, None,
                                                  msg, 64)
    assert st == _native.CUSMIC_INVALID and msg.value == b"positive gain or error is required"


def test_cleaner_settings():
    """reference test/test_cleaner.py:71-79 (host-only)."""
    from cusmic_b200 import Cleaner
    for settings in ({"contrast": -1}, {"cr_threshold": np.nan}, {"neighbor_threshold": np.inf},
                     {"maxiter": 1.5}, {"maxiter": True}, {"maxiter": -1},
                     {"border_mode": "invalid"}):
        with pytest.raises(ValueError):
            Cleaner(**settings)


def test_tuning_table_validation_and_lookup():
    from cusmic_b200 import _native
    saved = [_native.get_tuning(0)]
    try:
        _native.set_tuning([dict(max_pixels=1000, dense_rows=8, dense_blocks_per_sm=4,
                                 sparse_blocks_per_sm=2, row_blocks_per_sm=6),
                            dict(max_pixels=None, dense_rows=0, dense_blocks_per_sm=6,
                                 sparse_blocks_per_sm=8, row_blocks_per_sm=8)])
        assert _native.get_tuning(999)["dense_rows"] == 8
        assert _native.get_tuning(1000)["row_blocks_per_sm"] == 6
        assert _native.get_tuning(1001)["dense_blocks_per_sm"] == 6
        for bad in (dict(dense_rows=3), dict(dense_blocks_per_sm=0), dict(dense_blocks_per_sm=7),
                    dict(sparse_blocks_per_sm=9), dict(row_blocks_per_sm=0)):
            entry = dict(dict(max_pixels=None, dense_rows=0, dense_blocks_per_sm=6,
                              sparse_blocks_per_sm=8, row_blocks_per_sm=8), **bad)
            with pytest.raises(ValueError, match="invalid tuning entry"):
                _native.set_tuning([entry])
        _native.set_tuning([])
        d = _native.get_tuning(12345)
        assert (d["dense_rows"], d["dense_blocks_per_sm"]) == (0, 6)
    finally:
        _native.set_tuning(saved)


def test_inject_fault_kinds():
    """The failure-injection hook accepts its three kinds (each removed again
    at once) and rejects any other."""
    L = _native.lib()
    for kind in (_native.FAULT_PREPARE_WAIT, _native.FAULT_DETECT_WAIT, _native.FAULT_NO_MEMORY):
        assert L.cusmic_inject_fault(kind, 0) == _native.CUSMIC_OK
    assert L.cusmic_inject_fault(0, 1) == _native.CUSMIC_INVALID
    assert L.cusmic_inject_fault(99, 1) == _native.CUSMIC_INVALID


def test_host_batch_argument_checks():
    """cusmic_batch_host checks its arguments like the ragged device call,
    before any copy or device call."""
    L = _native.lib()
    o = _native.default_options()
    o.gain = 1.0
    msg = ctypes.create_string_buffer(256)
    assert L.cusmic_batch_host(None, 1, ctypes.byref(o), None, 8, 8, msg, 256) == \
        _native.CUSMIC_INVALID
    data = np.zeros(4)
    im = _native.Image(data.ctypes.data, None, None, None, None, None, 2, 2)
    o.cr_threshold = math.nan
    assert L.cusmic_batch_host(ctypes.byref(im), 1, ctypes.byref(o), None, 8, 8, msg, 256) == \
        _native.CUSMIC_INVALID
    assert msg.value == b"invalid detection settings"
