"""prep_detect_kernel: prepare and the first pass's dense detection in one
kernel, for batches whose frames all have an error map and no background,
widths that are multiples of 16 and 16-byte aligned buffers.

Holes enter its Laplacian as -inf, so every pixel whose Laplacian reads a hole
is listed with a bound of +inf and classified from the filled pixels; these
tests put holes (NaN, +inf and -inf) everywhere that matters: at edges and
corners, in clusters, next to masked pixels, and across item boundaries.
Pixels and masks must equal the CPU oracle's bit for bit, and the fused path
must give the same bits as the two-kernel path, which a buffer 8 bytes off a
16-byte boundary forces.
"""

import ctypes
import math

import numpy as np
import pytest

from cusmic_b200 import _native
from tests import cabi
from tests.conftest import assert_bits_equal
from tests.test_gpu_parity import MODES, SETTINGS, check_against_oracle, small_scene

pytestmark = pytest.mark.gpu


def holey_scene(seed, h, w, *, holes=0.01, masked=0.02, rays=None):
    """A scene with NaN, +inf and -inf holes, hole clusters, and holes on the
    frame's edges and corners."""
    data, mask = small_scene(seed, h, w, holes=0.0, masked=masked,
                             rays=rays if rays is not None else max(2, h * w // 40))
    rng = np.random.default_rng(seed + 1)
    kinds = np.array([np.nan, np.inf, -np.inf])
    pick = rng.random((h, w)) < holes
    data[pick] = kinds[rng.integers(0, 3, int(pick.sum()))]
    for y, x in ((0, 0), (0, w - 1), (h - 1, 0), (h - 1, w - 1), (h // 2, 0), (0, w // 2)):
        data[y, x] = kinds[(y + x) % 3]
    if h > 6 and w > 6:  # a 2 x 3 cluster near the middle
        cy, cx = h // 2, w // 2
        data[cy:cy + 2, cx - 1:cx + 2] = np.nan
    return data, mask


def error_of(data):
    return np.sqrt(np.abs(np.nan_to_num(data, posinf=0.0, neginf=0.0)) + 9)


def profile_launches(frames, opts):
    """Launch counts per kernel kind of one plan execution of the batch."""
    fr = cabi.Frames(frames)
    plan = cabi.Plan(fr, opts, 0, scalars=False)
    try:
        n = len(_native.KERNEL_KINDS)
        ms = (ctypes.c_double * n)()
        launches = (ctypes.c_int * n)()
        msg = ctypes.create_string_buffer(256)
        st = _native.lib().cusmic_plan_profile(plan.handle, None, ms, launches, n, msg, 256)
        assert st == 0, msg.value.decode()
        return dict(zip(_native.KERNEL_KINDS, launches))
    finally:
        plan.close()


def test_fused_path_is_taken(cuda):
    """An aligned error-map batch runs prepare and detection as one launch (no
    separate dense-detection launch); an unaligned one keeps the two kernels."""
    data, mask = holey_scene(5, 64, 528)
    frame = dict(data=data, mask=mask, error=error_of(data))
    got = profile_launches([frame], cabi.options(**SETTINGS))
    assert got["prepare"] == 1 and got["sigraw"] == 0 and got["classify"] == 1
    model = dict(data=data, mask=mask, gain=1.5, readnoise=4.0)
    got = profile_launches([model], cabi.options(**SETTINGS, gain=1.5, readnoise=4.0))
    assert got["sigraw"] == 1


@pytest.mark.parametrize("mode", MODES)
@pytest.mark.parametrize("shape", ((1, 16), (2, 16), (5, 32), (9, 48), (33, 80), (40, 528),
                                   (70, 1040), (3, 1536)))
def test_widths_and_borders(cuda, oracle, mode, shape):
    """Widths of one to three 512-column items (a half-filled last bit word
    when w % 32 == 16), heights down to one row, every border mode."""
    h, w = shape
    data, mask = holey_scene(h * 97 + w, h, w)
    frame = dict(data=data, mask=mask, error=error_of(data))
    check_against_oracle(oracle, [frame], dict(SETTINGS, border=mode))


@pytest.mark.parametrize("mode", ("mirror", "wrap", "constant"))
def test_holes_dense_and_no_mask(cuda, oracle, mode):
    """5% holes without a mask, and a frame whose first rows and columns are
    all holes."""
    h, w = 48, 96
    data, _ = holey_scene(31, h, w, holes=0.05, masked=0.0)
    data[:2, :] = np.nan
    data[:, :3] = np.inf
    frames = [dict(data=data, error=error_of(data))]
    check_against_oracle(oracle, frames, dict(SETTINGS, border=mode))


@pytest.mark.parametrize("thresholds", ((0.0, 0.0, 0.0), (1.0, 0.5, 0.25), (3.0, 8.0, 6.0)))
def test_thresholds(cuda, oracle, thresholds):
    """Zero thresholds list every pixel (full per-warp regions)."""
    c, cr, nb = thresholds
    data, mask = holey_scene(211, 64, 528)
    frame = dict(data=data, mask=mask, error=error_of(data))
    check_against_oracle(oracle, [frame],
                         dict(contrast=c, cr_threshold=cr, neighbor_threshold=nb, border="mirror"))


def test_error_map_with_nan_and_zeros(cuda, oracle):
    """Error maps with NaN and zero entries (a NaN floor lists a whole block)."""
    h, w = 64, 96
    data, mask = holey_scene(7, h, w)
    err = error_of(data)
    err[10:20, 40:50] = np.nan
    err[30, :] = 0.0
    check_against_oracle(oracle, [dict(data=data, mask=mask, error=err)], dict(SETTINGS))


@pytest.mark.parametrize("mode", ("mirror", "wrap"))
def test_ragged_batch_shared_map(cuda, oracle, mode):
    """A ragged batch of aligned error-map frames, two sharing one error map and
    mask, item heights below 32 rows (few items), per-frame passes differing."""
    frames = []
    shared_data, shared_mask = holey_scene(400, 64, 256)
    shared_err = error_of(shared_data)
    for i, (h, w) in enumerate(((64, 256), (64, 256), (17, 48), (130, 1040), (8, 16))):
        if (h, w) == (64, 256):
            data, _ = holey_scene(401 + i, h, w)
            frames.append(dict(data=data, mask=shared_mask, error=shared_err))
        else:
            data, mask = holey_scene(401 + i, h, w, masked=0.03 if i % 2 else 0.0)
            f = dict(data=data, error=error_of(data))
            if mask is not None:
                f["mask"] = mask
            frames.append(f)
    check_against_oracle(oracle, frames, dict(SETTINGS, border=mode), ragged=True)


def test_fused_equals_two_kernel_path(cuda):
    """The same frames through the fused path and, with the data 8 bytes off a
    16-byte boundary, through prepare + the dense kernel: identical bits."""
    import torch
    h, w = 96, 1040
    data, mask = holey_scene(17, h, w, holes=0.02, masked=0.03, rays=800)
    frame = dict(data=data, mask=mask, error=error_of(data))
    opts = cabi.options(**SETTINGS)
    a = cabi.Frames([frame])
    st, msg = cabi.run_batch(_native.lib(), a, opts)
    assert st == 0, msg
    b = cabi.Frames([frame])
    buf = torch.empty(h * w + 1, dtype=torch.float64, device="cuda")
    buf[1:] = torch.from_numpy(data.ravel()).cuda()
    b.keep.append(buf)
    b.ims[0].data = buf.data_ptr() + 8
    st, msg = cabi.run_batch(_native.lib(), b, opts)
    assert st == 0, msg
    (ca, ma), = a.outputs()
    (cb, mb), = b.outputs()
    np.testing.assert_array_equal(ma, mb)
    assert_bits_equal(ca, cb)
    assert ma.any()


def test_rebound_plan_changes_path(cuda, oracle):
    """A graph plan created on aligned buffers (fused path) and rebound to data
    8 bytes off a 16-byte boundary is captured again with the two-kernel path,
    and rebound back: every execution equals the oracle."""
    import torch
    h, w = 64, 528
    data, mask = holey_scene(23, h, w)
    frame = dict(data=data, mask=mask, error=error_of(data))
    want_clean, want_mask, _ = cabi.oracle_frame(oracle, frame, **SETTINGS)
    fr = cabi.Frames([frame])
    plan = cabi.Plan(fr, cabi.options(**SETTINGS), _native.PLAN_GRAPH, scalars=False)
    buf = torch.empty(h * w + 1, dtype=torch.float64, device="cuda")
    buf[1:] = torch.from_numpy(data.ravel()).cuda()
    aligned = fr.ims[0].data
    try:
        for ptr in (aligned, buf.data_ptr() + 8, aligned):
            fr.ims[0].data = ptr
            msg = ctypes.create_string_buffer(256)
            st = _native.lib().cusmic_plan_bind(plan.handle, fr.ims, fr.clean.data_ptr(),
                                                fr.mask.data_ptr(), msg, 256)
            assert st == 0, msg.value.decode()
            fr.clean.fill_(math.nan)
            st, m = plan.run()
            assert st == 0, m
            (clean, got_mask), = fr.outputs()
            np.testing.assert_array_equal(got_mask, want_mask)
            assert_bits_equal(clean, want_clean)
    finally:
        plan.close()
