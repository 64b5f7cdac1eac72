"""Batches and plans over the cusmic_b200 C ABI.

``Batch`` holds device frames (a same-shaped stack or a ragged list), their
calibration maps, per-frame scalars and the output buffers, and builds the
``cusmic_image`` descriptors.  ``Plan`` wraps ``cusmic_plan_*``: one
workspace, descriptors uploaded once, and (``graph=True``) the whole cleaning
captured as a CUDA graph whose maxiter loop is a device-driven while node.
"""

import ctypes
import math

import torch

from . import _native


class Batch:
    """Device frames, maps and outputs of one batch (frames back to back)."""

    def __init__(self, frames, errors=None, masks=None, gains=None, readnoises=None,
                 backgrounds=None, scalars=None, stack=None):
        self.frames = list(frames)
        nf = len(self.frames)
        if not nf:
            raise ValueError("a batch needs at least one frame")
        self.device = self.frames[0].device
        for f in self.frames:
            if f.dtype != torch.float64 or f.dim() != 2 or not f.is_cuda or not f.is_contiguous():
                raise TypeError("frames must be contiguous 2D float64 CUDA tensors")
        self._keep = []

        def per_frame(maps, dtype):
            if maps is None:
                return [None] * nf
            if isinstance(maps, torch.Tensor):
                maps = [maps] * nf
            out = []
            for m in maps:
                if m is None:
                    out.append(None)
                    continue
                m = m.to(device=self.device, dtype=dtype).contiguous()
                self._keep.append(m)
                out.append(m)
            return out

        self.errors = per_frame(errors, torch.float64)
        self.masks = per_frame(masks, torch.uint8)
        self.gains = per_frame(gains, torch.float64)
        self.readnoises = per_frame(readnoises, torch.float64)
        self.backgrounds = per_frame(backgrounds, torch.float64)
        self.scalars = scalars
        self.sizes = [tuple(f.shape) for f in self.frames]
        self.total = sum(h * w for h, w in self.sizes)
        if stack is not None:
            self.data = stack
            self.clean = torch.empty_like(stack)
            self.mask_out = torch.empty(stack.shape, dtype=torch.uint8, device=self.device)
        else:
            self.data = None
            self.clean = torch.empty(self.total, dtype=torch.float64, device=self.device)
            self.mask_out = torch.empty(self.total, dtype=torch.uint8, device=self.device)
        self.offsets = []
        o = 0
        for h, w in self.sizes:
            self.offsets.append(o)
            o += h * w

    @classmethod
    def stack(cls, data, error=None, mask=None, gain=None, readnoise=None, background=None):
        """Same-shaped frames (nf, h, w); maps are (h, w) shared or (nf, h, w)."""
        data = data.contiguous()

        def split(m):
            if m is None or m.dim() == 2:
                return m
            return [m[i] for i in range(m.shape[0])]
        return cls([data[i] for i in range(data.shape[0])], split(error), split(mask),
                   split(gain), split(readnoise), split(background), stack=data)

    @classmethod
    def ragged(cls, frames, errors=None, masks=None, scalars=None):
        """Frames of any shapes; scalars = [(gain, readnoise, background), ...]."""
        return cls([f.contiguous() for f in frames], errors, masks, scalars=scalars)

    def images(self):
        nf = len(self.frames)
        ims = (_native.Image * nf)()
        ptr = lambda t: t.data_ptr() if t is not None else None
        for i, f in enumerate(self.frames):
            h, w = self.sizes[i]
            ims[i] = _native.Image(f.data_ptr(), ptr(self.errors[i]), ptr(self.gains[i]),
                                   ptr(self.readnoises[i]), ptr(self.backgrounds[i]),
                                   ptr(self.masks[i]), w, h)
        return ims

    def scalars_array(self):
        if self.scalars is None:
            return None
        arr = (_native.FrameScalars * len(self.frames))()
        for i, (g, r, b) in enumerate(self.scalars):
            arr[i] = _native.FrameScalars(
                math.nan if g is None else float(g), math.nan if r is None else float(r),
                math.nan if b is None else float(b))
        return arr

    def frame_clean(self, i):
        h, w = self.sizes[i]
        return self.clean.view(-1)[self.offsets[i]:self.offsets[i] + h * w].view(h, w)

    def frame_mask(self, i):
        h, w = self.sizes[i]
        return self.mask_out.view(-1)[self.offsets[i]:self.offsets[i] + h * w].view(h, w)


class Plan:
    """A reusable cleaning of one Batch (cusmic_plan_create / execute / wait)."""

    def __init__(self, batch, *, graph=True, keep=False, contrast=3.0, cr_threshold=5.0,
                 neighbor_threshold=3.0, maxiter=4, border="mirror", gain=math.nan,
                 readnoise=0.0, background=math.nan):
        self.batch = batch
        o = _native.default_options()
        o.contrast, o.cr_threshold, o.neighbor_threshold = contrast, cr_threshold, \
            neighbor_threshold
        o.maxiter, o.border = int(maxiter), _native.BORDERS[border]
        o.gain, o.readnoise, o.background = gain, readnoise, background
        self.options = o
        self._ims = batch.images()
        self._scalars = batch.scalars_array()
        self.handle = ctypes.c_void_p()
        flags = (_native.PLAN_GRAPH if graph else 0) | (_native.PLAN_KEEP if keep else 0)
        msg = ctypes.create_string_buffer(512)
        with torch.cuda.device(batch.device):
            st = _native.lib().cusmic_plan_create(
                ctypes.byref(self.handle), self._ims, len(batch.frames), ctypes.byref(o),
                self._scalars, batch.clean.data_ptr(), batch.mask_out.data_ptr(), flags, msg,
                len(msg))
        _native.raise_for(st, msg)

    def options_for(self, i):
        """The options a per-frame plain call of frame i uses (scalars folded in)."""
        o = _native.Options.from_buffer_copy(self.options)
        if self.batch.scalars is not None:
            g, r, b = self.batch.scalars[i]
            if g is not None and not math.isnan(g):
                o.gain = g
            if r is not None and not math.isnan(r):
                o.readnoise = r
            o.background = math.nan if b is None else b
        return o

    def bind(self, batch):
        """Point the plan at another batch of the same shapes and maps (same
        sharing of error maps): the workspace, tile lists and graph are kept,
        only the frame descriptors are uploaded again."""
        ims = batch.images()
        msg = ctypes.create_string_buffer(256)
        with torch.cuda.device(batch.device):
            st = _native.lib().cusmic_plan_bind(self.handle, ims, batch.clean.data_ptr(),
                                                batch.mask_out.data_ptr(), msg, 256)
        _native.raise_for(st, msg)
        self.batch, self._ims = batch, ims

    def _stream(self, stream):
        if stream is None:
            stream = torch.cuda.current_stream(self.batch.device)
        return stream.cuda_stream if hasattr(stream, "cuda_stream") else stream

    def execute(self, stream=None):
        msg = ctypes.create_string_buffer(256)
        st = _native.lib().cusmic_plan_execute(self.handle, self._stream(stream), msg, 256)
        _native.raise_for(st, msg)

    def wait(self):
        msg = ctypes.create_string_buffer(256)
        st = _native.lib().cusmic_plan_wait(self.handle, msg, 256)
        _native.raise_for(st, msg)

    def passes(self):
        arr = (ctypes.c_int * len(self.batch.frames))()
        st = _native.lib().cusmic_plan_passes(self.handle, arr)
        _native.raise_for(st, "plan has not been executed")
        return list(arr)

    def profile(self, stream=None):
        """(ms per kernel kind, launches per kernel kind) of one event-timed run."""
        n = len(_native.KERNEL_KINDS)
        ms = (ctypes.c_double * n)()
        launches = (ctypes.c_int * n)()
        msg = ctypes.create_string_buffer(256)
        st = _native.lib().cusmic_plan_profile(self.handle, self._stream(stream), ms, launches,
                                               n, msg, 256)
        _native.raise_for(st, msg)
        return (dict(zip(_native.KERNEL_KINDS, ms)), dict(zip(_native.KERNEL_KINDS, launches)))

    def backward(self, grad_clean, stream=None):
        """Adjoint of the last execution with its mask frozen.

        ``grad_clean`` is laid out like the outputs.  Returns (grad_data,
        grad_background): the latter per frame (nf values) unless the batch has
        background maps, then per pixel like the outputs.
        """
        g = grad_clean.to(device=self.batch.device, dtype=torch.float64).contiguous()
        if g.numel() != self.batch.total:
            raise ValueError("gradient must match the outputs")
        gx = torch.empty_like(self.batch.clean)
        if any(b is not None for b in self.batch.backgrounds):
            gbg = torch.empty_like(self.batch.clean)
        else:
            gbg = torch.empty(len(self.batch.frames), dtype=torch.float64,
                              device=self.batch.device)
        msg = ctypes.create_string_buffer(256)
        st = _native.lib().cusmic_plan_backward(self.handle, g.data_ptr(), gx.data_ptr(),
                                                gbg.data_ptr(), self._stream(stream), msg, 256)
        _native.raise_for(st, msg)
        return gx, gbg

    def close(self):
        if self.handle:
            _native.lib().cusmic_plan_destroy(self.handle)
            self.handle = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
