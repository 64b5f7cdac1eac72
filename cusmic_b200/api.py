"""Reference-shaped Python API: ``remove_cosmics``, ``Cleaner`` and ``Image``.

Mirrors rndsrc/cusmic ``mod/cusmic/api.py:20-63``, ``image.py:22-79`` and
``cleaner.py:26-118`` (same names, argument meaning, defaults, validation
messages and exception types), but the arrays are ``torch.Tensor`` on a CUDA
device (NumPy arrays and other ``__dlpack__`` objects are accepted and
uploaded) and the work is done by libcusmic_b200.so through its C ABI on the
input device's current stream.
"""

import ctypes
from dataclasses import dataclass
from math import isfinite, nan
from numbers import Integral, Real
from typing import Any

import numpy as np
import torch

from . import _native

Array = Any
MODES = ("mirror", "reflect", "nearest", "wrap", "constant")


def _as_tensor(value, device=None):
    """Tensor view of a tensor, a __dlpack__ object, a NumPy array or a scalar."""
    if isinstance(value, torch.Tensor):
        t = value
    elif hasattr(value, "__dlpack__") and not isinstance(value, np.ndarray):
        t = torch.from_dlpack(value)
    else:
        t = torch.as_tensor(value)
    if device is not None and t.device != device:
        t = t.to(device)
    return t


def _cuda_device(data):
    if data.is_cuda:
        return data.device
    return torch.device("cuda", torch.cuda.current_device())


@dataclass
class Image:
    """Float64 pixels with calibration validated on the input device.

    Maps match the data or one shared frame.  Gain, read noise and background
    may also be scalars.  An error map overrides gain and read noise.  See
    :func:`remove_cosmics` for units, exclusions and stream use.
    """

    data: Array
    error: Array | None = None
    mask: Array | None = None
    background: Array | float | None = None
    effective_gain: Array | float | None = None
    readnoise: Array | float | None = None

    def __post_init__(self):
        data = _as_tensor(self.data)
        if data.dtype != torch.float64:
            raise TypeError("data must contain float64 pixels")
        if data.dim() not in (2, 3) or not data.numel():
            raise ValueError("data must be a nonempty 2D frame or 3D stack")
        device = _cuda_device(data)
        self.data = data if data.is_cuda else data.to(device)
        shape, frame = tuple(self.data.shape), tuple(self.data.shape[-2:])
        fields = ("error",) if self.error is not None else ("effective_gain", "readnoise")
        # The content checks of every map run on the device and are read back
        # with one copy (one host synchronisation per Image, on the current
        # stream); the first failing check, in the reference's order, raises.
        checks = []
        with torch.cuda.device(device):
            for name in (*fields, "background"):
                value = getattr(self, name)
                if value is None:
                    continue
                value = _as_tensor(value, device)
                if value.dtype.is_complex or value.dtype == torch.bool or \
                        not (value.dtype.is_floating_point or value.dtype in (
                            torch.int8, torch.int16, torch.int32, torch.int64, torch.uint8)):
                    raise TypeError(f"{name} must be real numeric data")
                if tuple(value.shape) not in (shape, frame) and (name == "error" or value.dim() != 0):
                    raise ValueError(f"{name} has an incompatible shape")
                value = value.to(torch.float64)
                checks.append((~torch.isfinite(value).all(), f"{name} must be finite"))
                if name in ("error", "effective_gain"):
                    checks.append(((value <= 0).any(), f"{name} must be positive"))
                if name == "readnoise":
                    checks.append(((value < 0).any(), "readnoise must be nonnegative"))
                setattr(self, name, value)
            if checks:
                failed = torch.stack([flag for flag, _ in checks]).cpu().tolist()
                for bad, (_, message) in zip(failed, checks):
                    if bad:
                        raise ValueError(message)
            if self.mask is not None:
                self.mask = _as_tensor(self.mask, device).to(torch.bool)
                if tuple(self.mask.shape) not in (shape, frame):
                    raise ValueError("mask must match the data or one frame")


@dataclass(frozen=True)
class Cleaner:
    """Reusable detection settings; call with an Image to get pixels and a mask."""

    contrast: float = 3
    cr_threshold: float = 5
    neighbor_threshold: float = 3
    maxiter: int = 4
    border_mode: str = "mirror"

    def __post_init__(self):
        for name in ("contrast", "cr_threshold", "neighbor_threshold"):
            value = getattr(self, name)
            if isinstance(value, bool) or not isinstance(value, Real) or not isfinite(value) \
                    or value < 0:
                raise ValueError(f"{name} must be finite and nonnegative")
        if isinstance(self.maxiter, bool) or not isinstance(self.maxiter, Integral) or \
                self.maxiter < 0:
            raise ValueError("maxiter must be a nonnegative integer")
        if not isinstance(self.border_mode, str) or self.border_mode not in MODES:
            raise ValueError(f"border_mode must be one of {', '.join(MODES)}")

    def options(self, gain=nan, readnoise=0.0, background=nan):
        o = _native.default_options()
        o.contrast = float(self.contrast)
        o.cr_threshold = float(self.cr_threshold)
        o.neighbor_threshold = float(self.neighbor_threshold)
        o.maxiter = int(self.maxiter)
        o.border = _native.BORDERS[self.border_mode]
        o.gain, o.readnoise, o.background = gain, readnoise, background
        return o

    def __call__(self, image: Image):
        """Return new (cleaned float64, mask bool) tensors on the input device."""
        if self.maxiter and image.error is None and (
                image.effective_gain is None or image.readnoise is None):
            raise ValueError("Provide error, or both effective_gain and readnoise")
        data = image.data
        device = data.device
        stack = data if data.dim() == 3 else data.unsqueeze(0)
        stack = stack.contiguous()
        nf, h, w = stack.shape
        keep = [stack]

        def maps(value):
            if value is None or value.dim() == 0:
                return [None] * nf
            v = value.contiguous()
            keep.append(v)
            if v.dim() == 3:
                return [v[i].data_ptr() for i in range(nf)]
            return [v.data_ptr()] * nf

        def scalar(value, default):
            return float(value) if value is not None and value.dim() == 0 else default

        err = maps(image.error)
        gain = maps(image.effective_gain) if image.error is None else [None] * nf
        rn = maps(image.readnoise) if image.error is None else [None] * nf
        bg = maps(image.background)
        msk = [None] * nf
        if image.mask is not None:
            m = image.mask.to(torch.uint8).contiguous()
            keep.append(m)
            msk = [m[i].data_ptr() for i in range(nf)] if m.dim() == 3 else [m.data_ptr()] * nf
        opts = self.options(
            gain=scalar(image.effective_gain, nan) if image.error is None else nan,
            readnoise=scalar(image.readnoise, 0.0) if image.error is None else 0.0,
            background=scalar(image.background, nan))
        ims = (_native.Image * nf)()
        for i in range(nf):
            ims[i] = _native.Image(stack[i].data_ptr(), err[i], gain[i], rn[i], bg[i], msk[i], w, h)
        clean = torch.empty((nf, h, w), dtype=torch.float64, device=device)
        flags = torch.empty((nf, h, w), dtype=torch.uint8, device=device)
        msg = ctypes.create_string_buffer(512)
        with torch.cuda.device(device):
            stream = torch.cuda.current_stream(device).cuda_stream
            status = _native.lib().remove_cosmics_batch_device(
                ims, nf, ctypes.byref(opts), clean.data_ptr(), flags.data_ptr(), stream, msg,
                len(msg))
        del keep
        _native.raise_for(status, msg)
        flags = flags.to(torch.bool)
        if data.dim() == 2:
            return clean[0], flags[0]
        return clean, flags


def remove_cosmics(
    data,
    contrast,
    cr_threshold,
    neighbor_threshold,
    error=None,
    mask=None,
    background=None,
    effective_gain=None,
    readnoise=None,
    maxiter=4,
    border_mode="mirror",
):
    """Return cleaned float64 pixels and a boolean cosmic-ray mask on the GPU.

    ``data`` is a nonempty float64 frame (height, width) or stack (frames,
    height, width): a CUDA tensor (used on its device) or a host array
    (uploaded to the current device).  Frames are cleaned independently and
    outputs do not alias inputs.

    Supply a finite, positive 1-sigma ``error`` map in image units, or both
    ``effective_gain`` (electrons per image unit, positive) and ``readnoise``
    (electrons, nonnegative).  Error overrides gain and read noise.  Maps may
    match data or one shared frame; gain and read noise also accept scalars.

    ``contrast`` rejects fine structure; ``cr_threshold`` and
    ``neighbor_threshold`` set detection and growth thresholds in sigma; all
    three must be finite and nonnegative.  ``mask`` excludes seed and donor
    pixels, but neighbouring detections may grow into masked pixels.
    Non-finite input pixels are preserved and never flagged.

    ``background`` is a finite scalar or map in image units, added before
    cleaning and subtracted afterwards.  ``maxiter`` is nonnegative; zero
    disables detection and needs no noise model but still applies the
    background arithmetic.  Border modes are mirror, reflect, nearest, wrap and
    constant (zero padding).

    Work runs on the input device's current stream; the call returns after it
    completes.  A replacement with no finite, unmasked donors raises ValueError.
    """
    image = Image(data, error, mask, background, effective_gain, readnoise)
    clean = Cleaner(contrast, cr_threshold, neighbor_threshold, maxiter, border_mode)
    return clean(image)
