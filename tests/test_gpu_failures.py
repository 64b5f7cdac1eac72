"""Failure paths of the C ABI (reference src/api.cu:83-105, src/device.cuh:23-30,
test/test_api.c:44-54), with the failures injected through
cusmic_inject_fault:

* a bounded device wait that runs out: one warp of the bulk-staged prepare or
  of the dense detection kernel waits, with a short bound, on a barrier that
  nothing completes.  The kernel drains its copies in flight, the loop control
  stops every frame, and the call returns CUSMIC_CUDA_ERROR; the next call on
  the same GPU is bit-exact again.
* an exhausted allocator: the next workspace reservation fails as cudaMalloc
  would, the call returns CUSMIC_NO_MEMORY and the host entry point leaves
  its outputs unchanged.

No GPU fault, trap or hang is involved: every wait is bounded and returns.
"""

import ctypes

import numpy as np
import pytest

from cusmic_b200 import _native
from tests import cabi
from tests.conftest import assert_bits_equal

pytestmark = pytest.mark.gpu

SETTINGS = dict(contrast=3.0, cr_threshold=5.0, neighbor_threshold=3.0)
WAIT_CYCLES = 1 << 20  # about half a millisecond of SM clock


@pytest.fixture
def inject():
    """Set an injected failure for the test; always removed afterwards."""
    lib = _native.lib()
    kinds = []

    def set_fault(kind, value):
        assert lib.cusmic_inject_fault(kind, value) == 0
        kinds.append(kind)

    yield set_fault
    for kind in kinds:
        lib.cusmic_inject_fault(kind, 0)


def scene(seed, h=256, w=512):
    """An error-map frame whose width suits the bulk-staged prepare."""
    from cusmic_b200 import scenes
    rng = np.random.default_rng(seed)
    data = scenes.make_frame(rng, h, w, n_stars=6, n_rays=90).data
    mask = rng.random(data.shape) < 0.01
    return dict(data=data, error=np.sqrt(np.abs(data) + 6.25), mask=mask)


def expect_exact(oracle, frame, opts_kw):
    fr = cabi.Frames([frame])
    st, msg = cabi.run_batch(_native.lib(), fr, cabi.options(**opts_kw))
    assert st == 0, msg
    want_clean, want_mask, _ = cabi.oracle_frame(oracle, frame, **opts_kw)
    clean, mask = fr.outputs()[0]
    np.testing.assert_array_equal(mask, want_mask)
    assert_bits_equal(clean, want_clean)
    assert mask.any()


@pytest.mark.parametrize("kind", (_native.FAULT_PREPARE_WAIT, _native.FAULT_DETECT_WAIT))
def test_bounded_wait_runs_out(cuda, oracle, inject, kind):
    lib = _native.lib()
    frame = scene(kind)
    inject(kind, WAIT_CYCLES)
    fr = cabi.Frames([frame])
    st, msg = cabi.run_batch(lib, fr, cabi.options(**SETTINGS))
    assert st == _native.CUSMIC_CUDA_ERROR
    assert "gave up waiting" in msg
    # The batch and ragged entry points and a graph plan report it the same way.
    two = cabi.Frames([frame, scene(7)])
    st, msg = cabi.run_ragged(two, cabi.options(**SETTINGS), scalars=False)
    assert st == _native.CUSMIC_CUDA_ERROR and "gave up waiting" in msg
    plan = cabi.Plan(two, cabi.options(**SETTINGS), _native.PLAN_GRAPH, scalars=False)
    try:
        st, msg = plan.run()
        assert st == _native.CUSMIC_CUDA_ERROR and "gave up waiting" in msg
    finally:
        plan.close()
    lib.cusmic_inject_fault(kind, 0)
    # The context stays usable: the same GPU cleans bit-exactly right after.
    expect_exact(oracle, frame, SETTINGS)
    plan = cabi.Plan(two, cabi.options(**SETTINGS), _native.PLAN_GRAPH, scalars=False)
    try:
        st, msg = plan.run()
        assert st == 0, msg
    finally:
        plan.close()


def test_host_entry_point_out_of_memory(cuda, golden, inject):
    """CUSMIC_NO_MEMORY with the host outputs unchanged, then a normal call."""
    lib = _native.lib()
    data = np.ascontiguousarray(golden["data"])
    error = np.ascontiguousarray(golden["error"])
    im = _native.Image(data.ctypes.data, error.ctypes.data, None, None, None, None, 512, 512)
    o = cabi.options(contrast=1.0, cr_threshold=5.0, neighbor_threshold=5.0)
    clean = np.full(data.shape, 7.0)
    mask = np.full(data.shape, 9, np.uint8)
    msg = ctypes.create_string_buffer(256)
    inject(_native.FAULT_NO_MEMORY, 1)
    st = lib.remove_cosmics(ctypes.byref(im), ctypes.byref(o), clean.ctypes.data,
                            mask.ctypes.data, msg, 256)
    assert st == _native.CUSMIC_NO_MEMORY
    assert b"bad_alloc" in msg.value
    assert (clean == 7.0).all() and (mask == 9).all()
    st = lib.remove_cosmics(ctypes.byref(im), ctypes.byref(o), clean.ctypes.data,
                            mask.ctypes.data, msg, 256)
    assert st == 0, msg.value
    np.testing.assert_array_equal(mask.astype(bool), golden["mask"])
    assert_bits_equal(clean, golden["cleaned"])


def test_device_entry_points_out_of_memory(cuda, oracle, inject):
    from cusmic_b200 import remove_cosmics
    lib = _native.lib()
    frame = scene(3)
    fr = cabi.Frames([frame])
    inject(_native.FAULT_NO_MEMORY, 1)
    st, msg = cabi.run_batch(lib, fr, cabi.options(**SETTINGS))
    assert st == _native.CUSMIC_NO_MEMORY and "bad_alloc" in msg
    inject(_native.FAULT_NO_MEMORY, 1)
    with pytest.raises(MemoryError):
        remove_cosmics(cuda.from_numpy(frame["data"]).cuda(), **SETTINGS,
                       error=cuda.from_numpy(frame["error"]).cuda())
    lib.cusmic_inject_fault(_native.FAULT_NO_MEMORY, 0)
    expect_exact(oracle, frame, SETTINGS)
