"""cusmic_batch_host: a ragged batch in host memory, cleaned in chunks whose
copies overlap.  Its results must equal the device ragged entry point's (and
so the oracle's) bit for bit, for shared and per-frame maps, pinned and
pageable buffers, batches of one chunk and of several, chunks that return all
pixels (with a background) and chunks that return only the flagged ones; map
checks and the donor error keep remove_cosmics's status and messages, and the
frames before a failing chunk hold their results."""

import ctypes
import math

import numpy as np
import pytest
import torch

from cusmic_b200 import _native
from tests import cabi
from tests.conftest import assert_bits_equal

pytestmark = pytest.mark.gpu

SETTINGS = dict(contrast=3.0, cr_threshold=5.0, neighbor_threshold=3.0)


def frames_of(kind, seed=0):
    from cusmic_b200 import scenes
    rng = np.random.default_rng(seed)
    if kind == "shared":  # one error map and one mask shared by every frame (the stack)
        sc = scenes.stack_2048(seed=seed, frames=6, size=1024)
        return [dict(data=f.data, error=sc.error, mask=sc.mask) for f in sc.frames]
    out = []
    for i, (h, w) in enumerate(((300, 257), (64, 1000), (1024, 1024), (1500, 900), (7, 9),
                                (512, 512))):
        f = scenes.make_frame(rng, h, w, n_stars=4, n_rays=max(3, h * w // 2000)).data
        f[rng.random(f.shape) < 0.001] = np.nan
        frame = dict(data=f, mask=rng.random(f.shape) < 0.01)
        if i % 2:
            frame["error"] = np.sqrt(np.abs(np.nan_to_num(f)) + 6.25)
        else:
            frame.update(gain=float(rng.uniform(1, 4)), readnoise=rng.uniform(2, 6, f.shape),
                         background=float(rng.uniform(0, 100)))
        if kind == "ragged_nobg":  # every chunk returns sparsely
            frame.pop("background", None)
        out.append(frame)
    return out


def host_images(frames, pinned):
    """Descriptors over host arrays (page-locked through torch when `pinned`),
    each distinct array once, so shared maps stay shared."""
    keep, seen = [], {}

    def host(a, dtype):
        if a is None or np.ndim(a) == 0:
            return None
        hit = seen.get(id(a))
        if hit is not None:
            return hit
        t = torch.from_numpy(np.ascontiguousarray(a, dtype=dtype))
        if pinned:
            t = t.pin_memory()
        keep.append(t)
        seen[id(a)] = t.data_ptr()
        return seen[id(a)]
    ims = (_native.Image * len(frames))()
    for i, f in enumerate(frames):
        h, w = f["data"].shape
        ims[i] = _native.Image(host(f["data"], np.float64), host(f.get("error"), np.float64),
                               host(f.get("gain"), np.float64), host(f.get("readnoise"), np.float64),
                               host(f.get("background"), np.float64),
                               host(f.get("mask"), np.uint8), w, h)
    total = sum(f["data"].size for f in frames)
    clean = torch.full((total,), 7.0, dtype=torch.float64)
    mask = torch.full((total,), 9, dtype=torch.uint8)
    if pinned:
        clean, mask = clean.pin_memory(), mask.pin_memory()
    return ims, clean, mask, keep


def scalars_of(frames):
    return cabi.Frames.scalars(type("F", (), {"frames": frames, "nf": len(frames)})())


def run_host(frames, opts, pinned):
    ims, clean, mask, keep = host_images(frames, pinned)
    msg = ctypes.create_string_buffer(512)
    st = _native.lib().cusmic_batch_host(ims, len(frames), ctypes.byref(opts), scalars_of(frames),
                                         clean.data_ptr(), mask.data_ptr(), msg, 512)
    return st, msg.value.decode(), clean.numpy(), mask.numpy()


@pytest.mark.parametrize("pinned", (True, False))
@pytest.mark.parametrize("kind", ("shared", "ragged", "ragged_nobg"))
def test_host_batch_matches_device_ragged(cuda, oracle, kind, pinned):
    frames = frames_of(kind)
    opts = cabi.options(**SETTINGS, readnoise=3.0)
    st, msg, clean, mask = run_host(frames, opts, pinned)
    assert st == 0, msg
    dev = cabi.Frames(frames)
    st, msg = cabi.run_ragged(dev, opts)
    assert st == 0, msg
    want = dev.outputs()
    off = 0
    for f, (wc, wm) in zip(frames, want):
        h, w = f["data"].shape
        np.testing.assert_array_equal(mask[off:off + h * w].reshape(h, w).astype(bool), wm)
        assert_bits_equal(clean[off:off + h * w].reshape(h, w), wc)
        off += h * w
    assert mask.any()
    # One small frame against the oracle as well.
    f = frames[-1] if kind != "shared" else frames[0]
    i = len(frames) - 1 if kind != "shared" else 0
    settings = dict(SETTINGS, maxiter=4)
    kw = {k: f.get(k) for k in ("error", "mask", "gain", "readnoise", "background")}
    if kw["readnoise"] is None and kw["error"] is None:
        kw["readnoise"] = 3.0
    oc, om, _ = oracle.clean_frame(f["data"], **kw, **settings)
    np.testing.assert_array_equal(want[i][1], om)
    assert_bits_equal(want[i][0], oc)


def test_host_batch_map_checks_and_donor_error(cuda):
    frames = frames_of("ragged")
    opts = cabi.options(**SETTINGS, readnoise=3.0)
    bad = [dict(f) for f in frames]
    bad[1] = dict(bad[1], error=bad[1]["error"].copy())
    bad[1]["error"][5, 5] = 0.0
    st, msg, clean, mask = run_host(bad, opts, True)
    assert st == _native.CUSMIC_INVALID and msg == "error must be finite and positive"
    bad = [dict(f) for f in frames]
    bad[0] = dict(bad[0], readnoise=bad[0]["readnoise"].copy())
    bad[0]["readnoise"][0, 0] = math.inf
    st, msg, _, _ = run_host(bad, opts, True)
    assert st == _native.CUSMIC_INVALID and msg == "read noise must be finite and nonnegative"
    # A frame without donors in a later chunk: the frames of earlier chunks
    # hold their results (the others are unspecified).  Chunks take whole
    # frames up to 64 MB of inputs, so with 2048^2 frames (32 MB each; the
    # shared maps are not counted) the first chunk is frames 0 and 1 and the
    # failing frame falls into the second.
    from cusmic_b200 import scenes
    sc = scenes.stack_2048(seed=4, frames=4, size=2048)
    ok = [dict(data=f.data, error=sc.error, mask=sc.mask) for f in sc.frames]
    data = np.full((7, 7), 10.0)
    data[3, 3] = 1000
    nodonor = dict(data=data, error=np.ones((7, 7)), mask=np.ones((7, 7), bool))
    nodonor["mask"][3, 3] = False
    batch = ok + [nodonor] + ok[:1]
    st, msg, clean, mask = run_host(batch, cabi.options(**SETTINGS), True)
    assert st == _native.CUSMIC_INVALID and "no finite replacement donors" in msg
    n = ok[0]["data"].size
    dev = cabi.Frames(ok[:2])
    assert cabi.run_ragged(dev, cabi.options(**SETTINGS))[0] == 0
    assert_bits_equal(clean[:2 * n], dev.clean.cpu().numpy())  # the first chunk
    np.testing.assert_array_equal(mask[:2 * n], dev.mask.cpu().numpy())
