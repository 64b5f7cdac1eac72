"""Helpers that drive a cusmic-compatible C ABI with torch CUDA buffers.

Used by the GPU tests for libcusmic_b200.so and, as a second oracle, for the
reference's own library compiled into oracle/_ref/libcusmic_ref.so (same ABI).
"""

import ctypes
import math
from pathlib import Path

import numpy as np
import torch

from cusmic_b200 import _native

REF_SO = Path(__file__).resolve().parents[1] / "oracle" / "_ref" / "libcusmic_ref.so"


def reference_lib():
    """The reference CUDA library (oracle/_ref), or None when it was not built."""
    if not REF_SO.exists():
        return None
    L = ctypes.CDLL(str(REF_SO))
    img, opt = ctypes.POINTER(_native.Image), ctypes.POINTER(_native.Options)
    vp, sz, cp = ctypes.c_void_p, ctypes.c_size_t, ctypes.c_char_p
    L.remove_cosmics_batch_device.restype = ctypes.c_int
    L.remove_cosmics_batch_device.argtypes = [img, sz, opt, vp, vp, vp, cp, sz]
    return L


class Frames:
    """Device copies of a list of frames and their maps, plus descriptors."""

    def __init__(self, frames, device="cuda"):
        self.keep = []
        self.uploaded = {}  # id of a host array -> its device copy (shared maps stay shared)
        self.frames = frames
        self.nf = len(frames)
        self.ims = (_native.Image * self.nf)()
        self.sizes = []
        for i, f in enumerate(frames):
            data = self._dev(f["data"], device)
            h, w = f["data"].shape
            ptr = {}
            for name in ("error", "gain", "readnoise", "background"):
                v = f.get(name)
                ptr[name] = self._dev(v, device).data_ptr() if isinstance(v, np.ndarray) else None
            m = f.get("mask")
            ptr["mask"] = self._dev(m.astype(np.uint8), device).data_ptr() if m is not None else None
            self.ims[i] = _native.Image(data.data_ptr(), ptr["error"], ptr["gain"],
                                        ptr["readnoise"], ptr["background"], ptr["mask"], w, h)
            self.sizes.append((h, w))
        self.total = sum(h * w for h, w in self.sizes)
        self.clean = torch.empty(self.total, dtype=torch.float64, device=device)
        self.mask = torch.empty(self.total, dtype=torch.uint8, device=device)

    def _dev(self, a, device):
        hit = self.uploaded.get(id(a))
        if hit is not None and hit[0] is a:
            return hit[1]
        t = torch.from_numpy(np.ascontiguousarray(a)).to(device)
        self.keep.append(t)
        self.uploaded[id(a)] = (a, t)  # keeps `a` alive, so its id is not reused
        return t

    def scalars(self):
        arr = (_native.FrameScalars * self.nf)()
        for i, f in enumerate(self.frames):
            g, r, b = f.get("gain"), f.get("readnoise"), f.get("background")
            arr[i] = _native.FrameScalars(
                float(g) if g is not None and np.ndim(g) == 0 else math.nan,
                float(r) if r is not None and np.ndim(r) == 0 else math.nan,
                float(b) if b is not None and np.ndim(b) == 0 else math.nan)
        return arr

    def outputs(self):
        torch.cuda.synchronize()
        c, m = self.clean.cpu().numpy(), self.mask.cpu().numpy()
        out, o = [], 0
        for h, w in self.sizes:
            out.append((c[o:o + h * w].reshape(h, w), m[o:o + h * w].reshape(h, w).astype(bool)))
            o += h * w
        return out


def options(contrast=3.0, cr_threshold=5.0, neighbor_threshold=3.0, maxiter=4, border="mirror",
            gain=math.nan, readnoise=0.0, background=math.nan):
    o = _native.default_options()
    o.contrast, o.cr_threshold, o.neighbor_threshold = contrast, cr_threshold, neighbor_threshold
    o.maxiter, o.border = int(maxiter), _native.BORDERS[border]
    o.gain, o.readnoise, o.background = gain, readnoise, background
    return o


def run_batch(lib, fr, opts, stream=None):
    msg = ctypes.create_string_buffer(512)
    st = lib.remove_cosmics_batch_device(fr.ims, fr.nf, ctypes.byref(opts), fr.clean.data_ptr(),
                                         fr.mask.data_ptr(), stream, msg, 512)
    return st, msg.value.decode()


def run_ragged(fr, opts, scalars=True, stream=None):
    msg = ctypes.create_string_buffer(512)
    sc = fr.scalars() if scalars else None
    st = _native.lib().cusmic_ragged_batch_device(
        fr.ims, fr.nf, ctypes.byref(opts), sc, fr.clean.data_ptr(), fr.mask.data_ptr(), stream,
        msg, 512)
    return st, msg.value.decode()


class Plan:
    """cusmic_plan_* wrapper."""

    def __init__(self, fr, opts, flags, scalars=True):
        self.fr = fr
        self.handle = ctypes.c_void_p()
        msg = ctypes.create_string_buffer(512)
        sc = fr.scalars() if scalars else None
        st = _native.lib().cusmic_plan_create(ctypes.byref(self.handle), fr.ims, fr.nf,
                                              ctypes.byref(opts), sc, fr.clean.data_ptr(),
                                              fr.mask.data_ptr(), flags, msg, 512)
        if st:
            raise RuntimeError(msg.value.decode())

    def run(self, stream=None):
        msg = ctypes.create_string_buffer(512)
        L = _native.lib()
        st = L.cusmic_plan_execute(self.handle, stream, msg, 512) or \
            L.cusmic_plan_wait(self.handle, msg, 512)
        return st, msg.value.decode()

    def passes(self):
        arr = (ctypes.c_int * self.fr.nf)()
        assert _native.lib().cusmic_plan_passes(self.handle, arr) == 0
        return list(arr)

    def close(self):
        if self.handle:
            _native.lib().cusmic_plan_destroy(self.handle)
            self.handle = ctypes.c_void_p()


def oracle_frame(oracle, f, **settings):
    """Run the CPU oracle on one frame dict (maps as arrays, scalars as floats)."""
    kw = {k: f.get(k) for k in ("error", "mask", "background", "gain", "readnoise")}
    return oracle.clean_frame(f["data"], **kw, **settings)
