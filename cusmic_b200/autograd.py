"""Differentiable cleaning: a ``torch.autograd.Function`` over the C ABI.

Detection thresholds are neither differentiable nor relaxed: the forward pass
records its final cosmic-ray mask, and the backward is the adjoint of the
cleaning with that mask frozen (``cusmic_plan_backward``).  Replaced pixels
send their gradient to the donor(s) their replacement median selected; every
other pixel, and the background add/subtract, pass it straight through.
"""

import math

import torch

from .api import Cleaner, Image
from .plan import Batch, Plan


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
        plan = Plan(batch, graph=False, keep=True, contrast=float(cleaner.contrast),
                    cr_threshold=float(cleaner.cr_threshold),
                    neighbor_threshold=float(cleaner.neighbor_threshold),
                    maxiter=int(cleaner.maxiter), border=cleaner.border_mode,
                    gain=gain if image.error is None else math.nan,
                    readnoise=rn if image.error is None else 0.0,
                    background=float(bg) if scalar_bg else math.nan)
        plan.execute()
        plan.wait()
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
