"""GPU checks of the frozen-mask adjoint: against the CPU-index reference
gradient of the oracle and against central finite differences."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def scene(seed, nf=2, size=192):
    from cusmic_b200 import scenes
    rng = np.random.default_rng(seed)
    frames = [scenes.make_frame(rng, size, size, n_stars=8, n_rays=60) for _ in range(nf)]
    return np.stack([f.data for f in frames])


@pytest.mark.parametrize("bg_kind", ("none", "scalar", "map"))
def test_backward_matches_cpu_index_reference(cuda, oracle, bg_kind):
    torch = cuda
    from cusmic_b200.plan import Batch, Plan
    data = scene(1)
    nf, h, w = data.shape
    rng = np.random.default_rng(2)
    bg = {"none": None, "scalar": 25.0, "map": rng.uniform(0, 50, (h, w))}[bg_kind]
    stack = torch.from_numpy(data).cuda()
    batch = Batch.stack(stack, background=None if bg_kind != "map" else
                        torch.from_numpy(bg).cuda())
    plan = Plan(batch, graph=True, keep=True, gain=2.0, readnoise=5.0,
                background=bg if bg_kind == "scalar" else float("nan"))
    plan.execute()
    plan.wait()
    g = rng.normal(size=data.shape)
    gx, gbg = plan.backward(torch.from_numpy(g).cuda())
    masks = batch.mask_out.cpu().numpy().astype(bool)
    assert masks.any()
    for f in range(nf):
        want_clean, want_mask, _ = oracle.clean_frame(data[f], gain=2.0, readnoise=5.0,
                                                      background=bg)
        np.testing.assert_array_equal(masks[f], want_mask)
        rgx, rmap, rscalar = oracle.backward(data[f], want_mask, g[f], background=bg)
        np.testing.assert_allclose(gx[f].cpu().numpy(), rgx, rtol=1e-13, atol=1e-13)
        if bg_kind == "map":
            np.testing.assert_allclose(gbg[f].cpu().numpy(), rmap, rtol=1e-13, atol=1e-13)
        else:
            assert abs(float(gbg[f]) - rscalar) <= 1e-12
    plan.close()


def test_central_finite_differences(cuda):
    """d(sum w * cleaned)/d(data) against central differences, eps = 1e-6 max(|x|, 1)."""
    torch = cuda
    from cusmic_b200.plan import Batch, Plan
    data = scene(3, nf=1, size=160)
    rng = np.random.default_rng(4)
    wts = torch.from_numpy(rng.normal(size=data.shape)).cuda()
    stack = torch.from_numpy(data).cuda()
    batch = Batch.stack(stack)
    plan = Plan(batch, graph=True, gain=2.0, readnoise=5.0, background=0.0)
    plan.execute()
    plan.wait()
    mask0 = batch.mask_out.clone()
    gx, gbg = plan.backward(wts)
    gx = gx.cpu().numpy()
    flagged = np.argwhere(mask0.cpu().numpy())
    # pixels near flags (donors and targets) plus random ones
    picks = [tuple(p) for p in flagged[:: max(1, len(flagged) // 32)]]
    for p in flagged[:64]:
        f, y, x = p
        for dy in (-2, 0, 2):
            for dx in (-2, 0, 2):
                yy, xx = y + dy, x + dx
                if 0 <= yy < data.shape[1] and 0 <= xx < data.shape[2]:
                    picks.append((f, yy, xx))
    picks += [tuple(rng.integers(0, s) for s in data.shape) for _ in range(64)]
    picks = list(dict.fromkeys(picks))[:512]
    checked = agree = 0
    for f, y, x in picks:
        x0 = data[f, y, x]
        eps = 1e-6 * max(abs(x0), 1.0)
        vals = []
        same = True
        for sgn in (1, -1):
            stack[f, y, x] = x0 + sgn * eps
            plan.execute()
            plan.wait()
            same &= bool(torch.equal(batch.mask_out, mask0))
            vals.append(float((wts * batch.clean).sum()))
        stack[f, y, x] = x0
        if not same:
            continue
        fd = (vals[0] - vals[1]) / (2 * eps)
        checked += 1
        agree += abs(fd - gx[f, y, x]) <= 1e-5 * (1 + abs(gx[f, y, x]))
    plan.close()
    assert checked >= 0.9 * len(picks)
    assert agree >= checked - 2, (agree, checked)


def test_autograd_function(cuda):
    torch = cuda
    from cusmic_b200.autograd import remove_cosmics_differentiable
    data = torch.from_numpy(scene(5, nf=2, size=128)).cuda().requires_grad_()
    bg = torch.tensor(10.0, dtype=torch.float64, device="cuda", requires_grad=True)
    clean, mask = remove_cosmics_differentiable(data, 3, 5, 3, background=bg,
                                                effective_gain=2.0, readnoise=5.0)
    w = torch.randn_like(clean)
    (w * clean).sum().backward()
    assert data.grad is not None and bg.grad is not None
    g = data.grad
    assert mask.any()
    # flagged pixels pass nothing to themselves; every weight lands somewhere
    assert bool((g[mask] == 0).all())
    assert float(bg.grad) == pytest.approx(0.0, abs=1e-9)
    assert torch.allclose(g.sum(), w.sum(), rtol=1e-12)
