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


def test_adjoint_1024_workload(cuda, oracle):
    """The differentiation workload as specified: 8 x 1024^2 frames of the
    plain-scene generator (gain 2, read noise 5, scalar background 0),
    L = sum(w * cleaned) with w ~ N(0, 1) seeded, gradients with respect to
    the data and the scalar background with the forward mask frozen.

    * every frame's mask equals the CPU oracle's, and its gradient equals the
      oracle's CPU-index reference gradient (donor selection replayed on the
      CPU from the frozen mask);
    * central finite differences at 512 uniformly random pixels,
      eps = 1e-6 max(|x|, 1), agree with the data gradient to 1e-8 relative;
      a pixel whose two one-sided differences disagree sits on a kink of the
      piecewise-linear map (a donor rank changes within eps) and is skipped,
      as is one whose perturbation changes the mask;
    * the scalar background's gradient is zero (each replaced pixel's donor
      weights sum to one, so the per-target terms cancel; only the order of
      the additions rounds), and its central difference is zero up to the
      rounding of (x + bg) - bg.
    """
    torch = cuda
    from cusmic_b200 import scenes
    from cusmic_b200.plan import Batch, Plan
    settings = dict(contrast=3.0, cr_threshold=5.0, neighbor_threshold=3.0, maxiter=4)
    model = dict(gain=2.0, readnoise=5.0)
    sc = scenes.adjoint_1024(seed=0)
    data = np.stack([f.data for f in sc.frames])
    nf, h, w = data.shape
    stack = torch.from_numpy(data).cuda()
    batch = Batch.stack(stack)
    plan = Plan(batch, graph=True, keep=True, background=0.0, **model, **settings)
    rng = np.random.default_rng(2024)
    wts = rng.normal(size=data.shape)
    wt = torch.from_numpy(wts).cuda()
    try:
        plan.execute()
        plan.wait()
        clean0 = batch.clean.clone()
        mask0 = batch.mask_out.clone()
        gx, gbg = plan.backward(wt)
        gx = gx.cpu().numpy()
        masks = mask0.cpu().numpy().astype(bool)
        for f in range(nf):
            want_clean, want_mask, _ = oracle.clean_frame(data[f], background=0.0, **model,
                                                          **settings)
            np.testing.assert_array_equal(masks[f], want_mask)
            assert np.array_equal(clean0[f].cpu().numpy().view(np.uint64),
                                  want_clean.view(np.uint64))
            rgx, _, rscalar = oracle.backward(data[f], want_mask, wts[f], background=0.0)
            np.testing.assert_allclose(gx[f], rgx, rtol=1e-13, atol=1e-13)
            assert abs(float(gbg[f]) - rscalar) <= 1e-9 and abs(rscalar) <= 1e-9
        assert masks.any()

        def forward():
            plan.execute()
            plan.wait()
            return batch.clean.clone(), bool(torch.equal(batch.mask_out, mask0))

        picks = np.stack([rng.integers(0, s, 512) for s in (nf, h, w)], axis=1)
        checked = 0
        for f, y, x in picks:
            x0 = data[f, y, x]
            eps = 1e-6 * max(abs(x0), 1.0)
            stack[f, y, x] = x0 + eps
            cp, same_p = forward()
            stack[f, y, x] = x0 - eps
            cm, same_m = forward()
            stack[f, y, x] = x0
            if not (same_p and same_m):
                continue
            up = float((wt * (cp - clean0)).sum()) / eps
            down = float((wt * (clean0 - cm)).sum()) / eps
            if abs(up - down) > 1e-6 * (1 + abs(up)):
                continue  # a kink between x - eps and x + eps
            fd = float((wt * (cp - cm)).sum()) / (2 * eps)
            g = gx[f, y, x]
            assert abs(fd - g) <= 1e-8 * (1 + abs(g)), (f, y, x, fd, g)
            checked += 1
        assert checked >= 0.9 * len(picks), checked
        assert torch.equal(forward()[0].view(torch.int64), clean0.view(torch.int64))

        # Scalar background: analytic gradient zero; central difference zero up
        # to the rounding of (x + bg) - bg at each pixel.
        eps = 1e-6
        outs = []
        for bg in (eps, -eps):
            other = Plan(batch, graph=True, keep=True, background=bg, **model, **settings)
            try:
                other.execute()
                other.wait()
                assert torch.equal(batch.mask_out, mask0)
                outs.append(batch.clean.clone())
            finally:
                other.close()
        fd_bg = float((wt * (outs[0] - outs[1])).sum()) / (2 * eps)
        ulp = np.spacing(np.nanmax(np.abs(data)) + 1.0)
        bound = 4 * ulp * float(wt.abs().sum()) / (2 * eps)
        assert abs(fd_bg) <= bound, (fd_bg, bound)
    finally:
        plan.close()


def test_autograd_reuses_plans(cuda):
    """Forwards of one signature reuse a plan (workspace and graph) once the
    previous autograd graph is freed; results and gradients stay those of a
    fresh plan, and a graph still alive keeps its own plan and frozen mask."""
    torch = cuda
    from cusmic_b200.autograd import remove_cosmics_differentiable
    from cusmic_b200.plan import Batch, Plan
    base = torch.from_numpy(scene(6, nf=2, size=128)).cuda()
    w = torch.randn(base.shape, dtype=torch.float64, device="cuda",
                    generator=torch.Generator(device="cuda").manual_seed(3))
    handles = []
    kept = None
    for k in range(4):
        x = (base * (1 + 0.25 * k)).requires_grad_()
        clean, mask = remove_cosmics_differentiable(x, 3, 5, 3, effective_gain=2.0,
                                                    readnoise=5.0)
        handles.append(clean.grad_fn.plan.handle.value)
        (w * clean).sum().backward(retain_graph=(k == 1))
        fresh_batch = Batch.stack(x.detach().clone())
        fresh = Plan(fresh_batch, graph=False, keep=True, gain=2.0, readnoise=5.0)
        fresh.execute()
        fresh.wait()
        assert torch.equal(fresh_batch.clean.view(torch.int64), clean.detach().view(torch.int64))
        assert torch.equal(fresh_batch.mask_out.bool(), mask)
        gx, _ = fresh.backward(w)
        # The scatter adds with float64 atomics: the order of the additions,
        # and so the last bits, may differ between two backwards.
        assert torch.allclose(gx, x.grad, rtol=1e-13, atol=1e-13)
        fresh.close()
        if k == 1:  # keep this graph alive: its plan must not be handed out
            kept = (x, clean, mask, gx.clone())
        del clean, mask
    assert handles[1] == handles[0]  # the first graph was freed: its plan came back
    assert handles[2] != handles[1]  # the second graph is still alive
    x, clean, mask, g_kept = kept
    x.grad = None
    (w * clean).sum().backward()  # a second backward of the kept graph
    assert torch.allclose(x.grad, g_kept, rtol=1e-13, atol=1e-13)
