"""Full-size workloads, checked through properties that do not need the CPU
oracle to run at that size:

* a batch equals per-frame calls bit for bit;
* unflagged finite pixels come back unchanged;
* every sampled flagged pixel holds the median of the donors in its clipped
  window under the final mask (the reference's replacement rule,
  src/replace.cuh:111-153, with midpoint() for an even donor count);
* the frozen-mask backward is linear in the incoming gradient.
"""


import numpy as np
import pytest

from tests import cabi

pytestmark = pytest.mark.gpu

SETTINGS = dict(contrast=3.0, cr_threshold=5.0, neighbor_threshold=3.0)


def midpoint(lo, hi):
    if abs(lo) < 1 and abs(hi) < 1:
        return (lo + hi) / 2
    return lo / 2 + hi / 2


def donor_median(clean_in, donors, y, x):
    h, w = clean_in.shape
    for r in range(2, max(h, w) + 1):
        y0, y1, x0, x1 = max(0, y - r), min(h, y + r + 1), max(0, x - r), min(w, x + r + 1)
        vals = np.sort(clean_in[y0:y1, x0:x1][donors[y0:y1, x0:x1]])
        if vals.size:
            n = vals.size
            return 0.0 + vals[(n - 1) // 2] if n % 2 else midpoint(vals[(n - 1) // 2], vals[n // 2])
    raise AssertionError("no donor")


def check_frame_properties(data, mask_in, cleaned, flagged, rng, samples=400):
    finite = np.isfinite(data)
    keep = finite & ~flagged
    assert np.array_equal(cleaned[keep].view(np.uint64), data[keep].view(np.uint64))
    assert np.array_equal(cleaned[~finite].view(np.uint64), data[~finite].view(np.uint64))
    donors = finite & ~(mask_in if mask_in is not None else False) & ~flagged
    ys, xs = np.nonzero(flagged)
    assert ys.size
    for i in rng.choice(ys.size, min(samples, ys.size), replace=False):
        want = donor_median(data, donors, ys[i], xs[i])
        assert cleaned[ys[i], xs[i]] == want


def test_stack_2048_batch_equals_single_calls_and_properties(cuda):
    from cusmic_b200 import scenes
    sc = scenes.stack_2048(seed=3)
    frames = [dict(data=f.data, error=sc.error, mask=sc.mask) for f in sc.frames]
    batch = cabi.Frames(frames)
    lib = cabi._native.lib()
    st, msg = cabi.run_batch(lib, batch, cabi.options(**SETTINGS))
    assert st == 0, msg
    outs = batch.outputs()
    rng = np.random.default_rng(0)
    for i in (0, 7, 15):
        one = cabi.Frames([frames[i]])
        assert cabi.run_batch(lib, one, cabi.options(**SETTINGS))[0] == 0
        (c1, m1), = one.outputs()
        assert np.array_equal(outs[i][0].view(np.uint64), c1.view(np.uint64))
        assert np.array_equal(outs[i][1], m1)
        check_frame_properties(frames[i]["data"], sc.mask, c1, m1, rng)


def test_large_8192_properties_and_backward_linearity(cuda):
    torch = cuda
    from cusmic_b200 import scenes
    from cusmic_b200.plan import Plan, Batch
    sc = scenes.large_8192(seed=1, frames=2)
    stack = torch.from_numpy(np.stack([f.data for f in sc.frames])).cuda()
    batch = Batch.stack(stack, error=torch.from_numpy(sc.error).cuda(),
                        mask=torch.from_numpy(sc.mask.astype(np.uint8)).cuda())
    plan = Plan(batch, graph=True, keep=True, **SETTINGS)
    try:
        plan.execute()
        plan.wait()
        cleaned, flagged = batch.clean.cpu().numpy(), batch.mask_out.cpu().numpy().astype(bool)
        rng = np.random.default_rng(1)
        for f in range(2):
            check_frame_properties(sc.frames[f].data, sc.mask, cleaned[f], flagged[f], rng,
                                   samples=200)
        gen = torch.Generator(device="cuda").manual_seed(2)
        g1 = torch.randn(stack.shape, dtype=torch.float64, device="cuda", generator=gen)
        g2 = torch.randn(stack.shape, dtype=torch.float64, device="cuda", generator=gen)
        a, b = 0.75, -1.5
        d1, _ = plan.backward(g1)
        d2, _ = plan.backward(g2)
        d12, _ = plan.backward(a * g1 + b * g2)
        err = (d12 - (a * d1 + b * d2)).abs().max().item()
        scale = (a * d1).abs().max().item() + (b * d2).abs().max().item()
        assert err <= 1e-12 * scale  # float64 atomics add in any order
        # A flagged pixel's output does not depend on it and it is never a
        # donor: its gradient is exactly zero.
        flagged_t = batch.mask_out.bool()
        assert int(torch.count_nonzero(d1[flagged_t])) == 0
        assert int(flagged_t.sum()) > 0
    finally:
        plan.close()
