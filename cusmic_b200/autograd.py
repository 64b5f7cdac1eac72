"""Differentiable cleaning: a ``torch.autograd.Function`` over the C ABI.

Detection thresholds are neither differentiable nor relaxed: the forward pass
records its final cosmic-ray mask, and the backward is the adjoint of the
cleaning with that mask frozen (``cusmic_plan_backward``).  Replaced pixels
send their gradient to the donor(s) their replacement median selected; every
other pixel, and the background add/subtract, pass it straight through.
"""

import math
import threading

import torch

from .api import Cleaner, Image
from .plan import Batch, Plan

# Idle plans per batch signature (device, shapes, which maps are present and
# how they are shared, options).  A forward takes one (or creates it) and binds
# it to its tensors; the plan goes back when the autograd graph that holds it
# is freed, so a graph kept for a second backward keeps its frozen mask.
_IDLE = {}
_IDLE_PER_KEY = 2
_LOCK = threading.Lock()


class _Lease:
    """A plan held by one autograd graph; returned to the idle pool when the
    graph (and with it this object) is freed."""

    def __init__(self, key, plan):
        self.key, self.plan = key, plan

    def __del__(self):
        try:
            with _LOCK:
                idle = _IDLE.setdefault(self.key, [])
                if len(idle) < _IDLE_PER_KEY:
                    idle.append(self.plan)
                    return
            self.plan.close()
        except Exception:
            pass


def _signature(batch, options):
    def kind(maps):
        present = [m is not None for m in maps]
        shared = len({m.data_ptr() for m in maps if m is not None}) <= 1
        return (tuple(present), shared)
    # NaN (no value) compares unequal to itself: key it as None.
    opts = tuple(sorted((k, None if isinstance(v, float) and math.isnan(v) else v)
                        for k, v in options.items()))
    return (batch.device, tuple(batch.sizes), kind(batch.errors), kind(batch.masks),
            kind(batch.gains), kind(batch.readnoises), kind(batch.backgrounds), opts)


def _plan_for(batch, options):
    key = _signature(batch, options)
    with _LOCK:
        idle = _IDLE.get(key)
        plan = idle.pop() if idle else None
    if plan is None:
        plan = Plan(batch, graph=True, keep=True, **options)
    else:
        plan.bind(batch)
    return _Lease(key, plan)


class _Clean(torch.autograd.Function):
    @staticmethod
    def forward(ctx, data, background, image, cleaner):
        stack = data if data.dim() == 3 else data.unsqueeze(0)
        stack = stack.detach().contiguous()
        nf = stack.shape[0]
        bg = image.background
        scalar_bg = bg is not None and bg.dim() == 0
        batch = Batch.stack(stack, error=image.error,
                            mask=None if image.mask is None else image.mask.to(torch.uint8),
                            gain=image.effective_gain if _is_map(image.effective_gain) else None,
                            readnoise=image.readnoise if _is_map(image.readnoise) else None,
                            background=bg if _is_map(bg) else None)
        gain = float(image.effective_gain) if _is_scalar(image.effective_gain) else math.nan
        rn = float(image.readnoise) if _is_scalar(image.readnoise) else 0.0
        options = dict(contrast=float(cleaner.contrast),
                       cr_threshold=float(cleaner.cr_threshold),
                       neighbor_threshold=float(cleaner.neighbor_threshold),
                       maxiter=int(cleaner.maxiter), border=cleaner.border_mode,
                       gain=gain if image.error is None else math.nan,
                       readnoise=rn if image.error is None else 0.0,
                       background=float(bg) if scalar_bg else math.nan)
        lease = _plan_for(batch, options)
        plan = lease.plan
        plan.execute()
        plan.wait()
        ctx.lease = lease
        ctx.plan = plan
        ctx.shape = data.shape
        ctx.bg_shape = None if bg is None else tuple(bg.shape)
        ctx.nf = nf
        clean = batch.clean.clone()
        mask = batch.mask_out.to(torch.bool)
        if data.dim() == 2:
            clean, mask = clean[0], mask[0]
        ctx.mark_non_differentiable(mask)
        return clean, mask

    @staticmethod
    def backward(ctx, grad_clean, grad_mask):
        plan = ctx.plan
        gx, gbg = plan.backward(grad_clean.reshape(plan.batch.clean.shape))
        gx = gx.reshape(ctx.shape)
        g_background = None
        if ctx.needs_input_grad[1] and ctx.bg_shape is not None:
            if len(ctx.bg_shape) == 0:
                g_background = gbg.sum()  # one scalar shared by every frame
            else:
                per_frame = gbg.reshape(ctx.nf, *ctx.shape[-2:])
                g_background = per_frame.sum(0) if len(ctx.bg_shape) == 2 else per_frame
        return gx, g_background, None, None


def _is_map(v):
    return v is not None and isinstance(v, torch.Tensor) and v.dim() > 0


def _is_scalar(v):
    return v is not None and (not isinstance(v, torch.Tensor) or v.dim() == 0)


def remove_cosmics_differentiable(data, contrast=3, cr_threshold=5, neighbor_threshold=3,
                                  error=None, mask=None, background=None, effective_gain=None,
                                  readnoise=None, maxiter=4, border_mode="mirror"):
    """``remove_cosmics`` whose cleaned output is differentiable in ``data``
    and ``background`` (a tensor scalar or map), with the mask frozen."""
    bg_t = background if isinstance(background, torch.Tensor) else None
    image = Image(data.detach(), error, mask,
                  background.detach() if bg_t is not None else background,
                  effective_gain, readnoise)
    cleaner = Cleaner(contrast, cr_threshold, neighbor_threshold, maxiter, border_mode)
    return _Clean.apply(data, bg_t, image, cleaner)
