"""ctypes front end of the CPU oracle (TEST INFRASTRUCTURE ONLY).

Loads ``oracle/_build/liboracle.so`` (built from ``cusmic_oracle.c`` by
``oracle/build.py``).  Only tests, the smoke check and the CPU-baseline leg of
bench.py may import this module; the product path never does.
"""

import ctypes
import math

import numpy as np

from .build import ORACLE_SO, build_oracle

BORDERS = {"reflect": 0, "constant": 1, "nearest": 2, "mirror": 3, "wrap": 4}

_dp = ctypes.POINTER(ctypes.c_double)
_bp = ctypes.POINTER(ctypes.c_uint8)


class OracleImage(ctypes.Structure):
    _fields_ = [("data", _dp), ("error", _dp), ("gain", _dp), ("readnoise", _dp),
                ("background", _dp), ("mask", _bp), ("width", ctypes.c_size_t),
                ("height", ctypes.c_size_t)]


class OracleOptions(ctypes.Structure):
    _fields_ = [("contrast", ctypes.c_double), ("cr_threshold", ctypes.c_double),
                ("neighbor_threshold", ctypes.c_double), ("gain", ctypes.c_double),
                ("readnoise", ctypes.c_double), ("background", ctypes.c_double),
                ("maxiter", ctypes.c_int), ("border", ctypes.c_int)]


class OracleError(ValueError):
    pass


_lib = None


def lib():
    global _lib
    if _lib is None:
        path = ORACLE_SO if ORACLE_SO.exists() else build_oracle()
        _lib = ctypes.CDLL(str(path))
        _lib.oracle_clean_frame.restype = ctypes.c_int
        _lib.oracle_clean_frame.argtypes = [
            ctypes.POINTER(OracleImage), ctypes.POINTER(OracleOptions), _dp, _bp,
            ctypes.POINTER(ctypes.c_int), ctypes.c_char_p, ctypes.c_size_t]
        _lib.oracle_window_median.restype = ctypes.c_double
        _lib.oracle_window_median.argtypes = [_dp, ctypes.c_int]
        _lib.oracle_oets.argtypes = [_dp, ctypes.c_int]
        _lib.oracle_bitonic32.argtypes = [_dp]
        _lib.oracle_border_index.restype = ctypes.c_int
        _lib.oracle_border_index.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_int]
        for name in ("oracle_median_filter",):
            getattr(_lib, name).argtypes = [_dp, _dp, ctypes.c_int, ctypes.c_int,
                                            ctypes.c_int, ctypes.c_int]
        _lib.oracle_laplacian.argtypes = [_dp, _dp, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        _lib.oracle_replace.argtypes = [_dp, _bp, _bp, ctypes.c_int, ctypes.c_int]
        _lib.oracle_set_threads.restype = ctypes.c_int
        _lib.oracle_set_threads.argtypes = [ctypes.c_int]
    return _lib


def set_threads(n):
    """Host threads of the oracle's OpenMP loops (0: unchanged); returns the count in effect."""
    return lib().oracle_set_threads(int(n))


def _f64(a):
    return np.ascontiguousarray(a, dtype=np.float64)


def _ptr(a, kind=_dp):
    return None if a is None else a.ctypes.data_as(kind)


def clean_frame(data, *, error=None, mask=None, background=None, gain=None,
                readnoise=None, contrast=3.0, cr_threshold=5.0, neighbor_threshold=3.0,
                maxiter=4, border="mirror"):
    """Clean one 2-D frame; maps are arrays of its shape, scalars are floats.

    Returns (cleaned float64, mask bool, detection passes run).
    """
    data = _f64(data)
    h, w = data.shape
    maps = {}
    scal = {"gain": math.nan, "readnoise": 0.0, "background": math.nan}
    for name, value in (("gain", gain), ("readnoise", readnoise), ("background", background)):
        if value is None:
            continue
        if np.ndim(value) == 0:
            scal[name] = float(value)
        else:
            maps[name] = _f64(np.broadcast_to(value, data.shape))
    err = None if error is None else _f64(np.broadcast_to(error, data.shape))
    msk = None if mask is None else np.ascontiguousarray(np.broadcast_to(mask, data.shape),
                                                         dtype=np.uint8)
    im = OracleImage(_ptr(data), _ptr(err), _ptr(maps.get("gain")),
                     _ptr(maps.get("readnoise")), _ptr(maps.get("background")),
                     _ptr(msk, _bp), w, h)
    opts = OracleOptions(contrast, cr_threshold, neighbor_threshold, scal["gain"],
                         scal["readnoise"], scal["background"], int(maxiter),
                         BORDERS[border])
    out = np.empty_like(data)
    flags = np.empty(data.shape, dtype=np.uint8)
    passes = ctypes.c_int(0)
    msg = ctypes.create_string_buffer(256)
    status = lib().oracle_clean_frame(ctypes.byref(im), ctypes.byref(opts), _ptr(out),
                                      _ptr(flags, _bp), ctypes.byref(passes), msg, 256)
    if status:
        raise OracleError(msg.value.decode())
    return out, flags.astype(bool), passes.value


def window_median(values):
    v = _f64(values).copy()
    return lib().oracle_window_median(_ptr(v), len(v))


def oets(values):
    v = _f64(values).copy()
    lib().oracle_oets(_ptr(v), len(v))
    return v


def bitonic32(values):
    v = _f64(values).copy()
    assert v.shape == (32,)
    lib().oracle_bitonic32(_ptr(v))
    return v


def median_filter(a, size, border="mirror"):
    a = _f64(a)
    out = np.empty_like(a)
    lib().oracle_median_filter(_ptr(a), _ptr(out), a.shape[1], a.shape[0],
                               BORDERS[border], size)
    return out


def laplacian(a, border="mirror"):
    a = _f64(a)
    out = np.empty_like(a)
    lib().oracle_laplacian(_ptr(a), _ptr(out), a.shape[1], a.shape[0], BORDERS[border])
    return out


def backward(data, crmask, grad, *, mask=None, background=None):
    """CPU-index reference gradient of a frozen-mask cleaning of one frame.

    Returns (grad_data, grad_background_map or None, grad_background_scalar).
    """
    L = lib()
    if not hasattr(L.oracle_backward, "_set"):
        L.oracle_backward.argtypes = [ctypes.POINTER(OracleImage), ctypes.POINTER(OracleOptions),
                                      _bp, _dp, _dp, _dp, _dp]
        L.oracle_backward._set = True
    data = _f64(data)
    h, w = data.shape
    bgmap, bgs = None, math.nan
    if background is not None:
        if np.ndim(background) == 0:
            bgs = float(background)
        else:
            bgmap = _f64(np.broadcast_to(background, data.shape))
    msk = None if mask is None else np.ascontiguousarray(mask, dtype=np.uint8)
    im = OracleImage(_ptr(data), None, None, None, _ptr(bgmap), _ptr(msk, _bp), w, h)
    opts = OracleOptions(0, 0, 0, math.nan, 0, bgs, 1, 3)
    crm = np.ascontiguousarray(crmask, dtype=np.uint8)
    g = _f64(grad)
    gx = np.empty_like(data)
    gmap = np.empty_like(data) if bgmap is not None else None
    gs = ctypes.c_double(0.0)
    L.oracle_backward(ctypes.byref(im), ctypes.byref(opts), _ptr(crm, _bp), _ptr(g), _ptr(gx),
                      _ptr(gmap), ctypes.byref(gs))
    return gx, gmap, gs.value
