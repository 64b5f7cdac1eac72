"""Bit parity with the reference's own CUDA library at the full size of every
benchmark workload.

The reference library (``oracle/_ref/libcusmic_ref.so``, compiled from the
reference's ``src/api.cu`` for sm_100a by ``oracle/build.py``) runs the same
inputs through its own batch entry point (reference src/api.cu:184-192, used as
test/test_reference.c:25-120 and test/test_batch.cu:46-158 use it).  Masks and
float64 pixels must be identical, bit for bit, for:

* stack_2048: 16 x 2048^2 frames, one shared error map, 0.5% + 2-column mask,
  0.1% NaN pixels; one batch call here, one graph-plan execution here, one
  batch call of the reference;
* ragged_64: 64 frames of log-uniform shapes in [256, 4096]^2 with per-frame
  gain, read noise and background; one ragged call and one graph plan here,
  64 single-frame calls of the reference (its scalars are batch-wide, so each
  frame gets its own options);
* large_8192: 4 x 8192^2 frames, full-size error map, 2% mask, saturated stars;
* adjoint_1024: 8 x 1024^2 noise-model frames (gain 2, read noise 5).

Comparisons run on the device (int64 views of the float64 outputs).
"""

import ctypes

import numpy as np
import pytest

from cusmic_b200 import _native
from tests import cabi

pytestmark = pytest.mark.gpu

SETTINGS = dict(contrast=3.0, cr_threshold=5.0, neighbor_threshold=3.0, maxiter=4)


@pytest.fixture(scope="module")
def ref():
    lib = cabi.reference_lib()
    if lib is None:
        pytest.fail("oracle/_ref/libcusmic_ref.so was not built (run oracle/build.py where "
                    "the reference sources are present)", pytrace=False)
    return lib


def same(torch, a_clean, a_mask, b_clean, b_mask, what):
    """Identical masks and float64 bits (on the device)."""
    bad_mask = int((a_mask != b_mask).sum())
    bad_px = int((a_clean.view(torch.int64) != b_clean.view(torch.int64)).sum())
    assert bad_mask == 0 and bad_px == 0, f"{what}: {bad_mask} mask bytes, {bad_px} pixels differ"
    assert int(a_mask.sum()) > 0, f"{what}: nothing flagged"


def run_plan(fr, opts, scalars):
    plan = cabi.Plan(fr, opts, _native.PLAN_GRAPH, scalars=scalars)
    try:
        st, msg = plan.run()
        assert st == 0, msg
        return plan.passes()
    finally:
        plan.close()


def reference_per_frame(ref, fr, frames):
    """One reference call per frame, each frame's scalars as its options."""
    clean = fr.clean.clone().fill_(0)
    mask = fr.mask.clone().fill_(0)
    msg = ctypes.create_string_buffer(512)
    off = 0
    for i, f in enumerate(frames):
        h, w = f["data"].shape
        o = cabi.options(**SETTINGS, gain=float(f["gain"]), readnoise=float(f["readnoise"]),
                         background=float(f["background"]))
        st = ref.remove_cosmics_batch_device(ctypes.byref(fr.ims[i]), 1, ctypes.byref(o),
                                             clean.data_ptr() + 8 * off, mask.data_ptr() + off,
                                             None, msg, 512)
        assert st == 0, msg.value
        off += h * w
    return clean, mask


def batch_pair(torch, ref, frames, opts):
    """This library's batch call and graph plan against the reference's batch call."""
    mine = cabi.Frames(frames)
    st, msg = cabi.run_batch(_native.lib(), mine, opts)
    assert st == 0, msg
    theirs = cabi.Frames(frames)
    st, msg = cabi.run_batch(ref, theirs, opts)
    assert st == 0, msg
    torch.cuda.synchronize()
    same(torch, mine.clean, mine.mask, theirs.clean, theirs.mask, "batch call")
    c0, m0 = mine.clean.clone(), mine.mask.clone()
    run_plan(mine, opts, scalars=False)
    torch.cuda.synchronize()
    same(torch, mine.clean, mine.mask, c0, m0, "graph plan")


def test_stack_2048_full(cuda, ref):
    from cusmic_b200 import scenes
    sc = scenes.stack_2048(seed=0)
    frames = [dict(data=f.data, error=sc.error, mask=sc.mask) for f in sc.frames]
    batch_pair(cuda, ref, frames, cabi.options(**SETTINGS))


def test_ragged_64_full(cuda, ref):
    torch = cuda
    from cusmic_b200 import scenes
    sc = scenes.ragged_64(seed=0)
    frames = [dict(data=f.data, gain=f.gain, readnoise=f.readnoise, background=f.background)
              for f in sc.frames]
    opts = cabi.options(**SETTINGS)
    mine = cabi.Frames(frames)
    st, msg = cabi.run_ragged(mine, opts)
    assert st == 0, msg
    clean, mask = reference_per_frame(ref, mine, frames)
    torch.cuda.synchronize()
    same(torch, mine.clean, mine.mask, clean, mask, "ragged call")
    passes = run_plan(mine, opts, scalars=True)
    torch.cuda.synchronize()
    same(torch, mine.clean, mine.mask, clean, mask, "graph plan")
    assert max(passes) == SETTINGS["maxiter"]


def test_adjoint_1024_forward(cuda, ref):
    from cusmic_b200 import scenes
    sc = scenes.adjoint_1024(seed=0)
    frames = [dict(data=f.data) for f in sc.frames]
    batch_pair(cuda, ref, frames, cabi.options(**SETTINGS, gain=2.0, readnoise=5.0,
                                               background=0.0))


def test_large_8192_full(cuda, ref):
    from cusmic_b200 import scenes
    sc = scenes.large_8192(seed=0)
    frames = [dict(data=f.data, error=sc.error, mask=sc.mask) for f in sc.frames]
    batch_pair(cuda, ref, frames, cabi.options(**SETTINGS))
