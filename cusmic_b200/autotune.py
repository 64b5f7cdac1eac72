"""Autotuner of the detection pass's launch parameters.

``python -m cusmic_b200.autotune [--out PATH] [--sweeps N]`` runs on a GPU and
writes ``cusmic_b200/tuning.json``, which the package installs through
``cusmic_set_tuning`` when it loads the library.

What is tuned (``struct cusmic_tuning``): the tile height of the dense
detection kernel (rows per 512-column item, or automatic), how many of its
blocks are launched per SM, and the grid sizes of the sparse per-pass kernels
(candidates, seeds, classification, replacement) and of the row kernels
(prepare, hole fill, growth, restore).  The selection networks are fixed by
the filter sizes of the algorithm: a 5 x 5 window is one 32-lane bitonic
network, the 7 x 7 window of 3 x 3 medians one 64-element network over two
values per lane, the 3 x 3 medians sorted column triples.

Batch-size classes, each tuned on its own workloads (seeded synthetic scenes
of cusmic_b200.scenes):

* ``small`` (at most 4 Mpx: single frames up to 2048 x 2048): one 512 x 512
  noise-model frame, one 1024 x 1024 frame with an error map, one 2048 x 2048
  frame of the stack;
* ``large`` (everything else): the 16 x 2048^2 stack and the 64-frame ragged
  batch.

Search: coordinate descent from the built-in defaults, each trial the median
of timed executions of a graph plan (CUDA events), the objective the sum over
the class's workloads.  Every trial must reproduce the default parameters'
masks and pixels bit for bit; a trial that does not is an error.
"""

import argparse
import json
import statistics
import sys
from pathlib import Path

import numpy as np

SETTINGS = dict(contrast=3.0, cr_threshold=5.0, neighbor_threshold=3.0, maxiter=4)
SPACE = {
    "dense_rows": (0, 4, 8, 16, 32),
    "dense_blocks_per_sm": (3, 4, 5, 6),
    "sparse_blocks_per_sm": (2, 4, 6, 8),
    "row_blocks_per_sm": (2, 4, 6, 8),
}
SMALL_MAX = 4 * 1024 * 1024


def _workloads(torch, dev):
    from . import scenes
    from .plan import Batch

    def stack(frames, error=None, mask=None, **kw):
        t = torch.from_numpy(np.stack(frames)).to(dev)
        return Batch.stack(t, error=None if error is None else torch.from_numpy(error).to(dev),
                           mask=None if mask is None else torch.from_numpy(mask.astype(np.uint8)).to(dev),
                           **kw), kw

    st = scenes.stack_2048(seed=0)
    small = []
    p = scenes.plain_512(seed=0).frames[0]
    small.append(("plain_512", stack([p.data]), dict(gain=2.0, readnoise=5.0, background=0.0)))
    a = scenes.adjoint_1024(seed=0, frames=1).frames[0]
    err = np.sqrt(np.abs(a.model) / 2 + 2.5 ** 2)
    small.append(("frame_1024_error", stack([a.data], error=err), {}))
    small.append(("frame_2048_stack", stack([st.frames[0].data], error=st.error, mask=st.mask), {}))
    large = [("stack_2048", stack([f.data for f in st.frames], error=st.error, mask=st.mask), {})]
    rg = scenes.ragged_64(seed=0)
    frames = [torch.from_numpy(f.data).to(dev) for f in rg.frames]
    large.append(("ragged_64", (Batch.ragged(frames, scalars=[(f.gain, f.readnoise, f.background)
                                                              for f in rg.frames]), {}), {}))
    return {"small": small, "large": large}


def _measure(torch, batch, plan_kw, reps):
    from .plan import Plan
    plan = Plan(batch, graph=True, **SETTINGS, **plan_kw)
    stream = torch.cuda.current_stream()
    try:
        for _ in range(3):
            plan.execute(stream)
        plan.wait()
        times = []
        for _ in range(reps):
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record(stream)
            plan.execute(stream)
            e.record(stream)
            plan.wait()
            times.append(s.elapsed_time(e))
        return statistics.median(times), batch.clean.clone(), batch.mask_out.clone()
    finally:
        plan.close()


def tune(sweeps=2, reps=7, log=print):
    import torch
    from . import _native
    dev = torch.device("cuda", torch.cuda.current_device())
    work = _workloads(torch, dev)
    _native.set_tuning([])
    default = {k: v for k, v in _native.get_tuning(0).items() if k != "max_pixels"}
    table, trials = [], []
    for cls, max_px in (("small", SMALL_MAX), ("large", None)):
        refs = {}

        def cost(params):
            _native.set_tuning([dict(params, max_pixels=None)])
            total = 0.0
            for name, (batch, _), plan_kw in work[cls]:
                ms, clean, mask = _measure(torch, batch, plan_kw, reps)
                if name not in refs:
                    refs[name] = (clean, mask)
                elif not (torch.equal(refs[name][1], mask) and
                          torch.equal(refs[name][0].view(torch.int64), clean.view(torch.int64))):
                    raise RuntimeError(f"{cls}/{name}: parameters {params} changed the result")
                total += ms
            trials.append({"class": cls, "params": dict(params), "ms": round(total, 4)})
            log(f"{cls:5s} {params} {total:.3f} ms")
            return total

        best = dict(default)
        best_ms = default_ms = cost(best)
        for _ in range(sweeps):
            changed = False
            for key, values in SPACE.items():
                for v in values:
                    if v == best[key]:
                        continue
                    cand = dict(best, **{key: v})
                    ms = cost(cand)
                    if ms < best_ms * 0.99:
                        best, best_ms, changed = cand, ms, True
            if not changed:
                break
        table.append(dict(best, max_pixels=max_px))
        log(f"{cls}: best {best} {best_ms:.3f} ms (defaults {default_ms:.3f} ms)")
    _native.set_tuning(table)
    props = torch.cuda.get_device_properties(dev)
    return {"device": props.name, "sms": props.multi_processor_count,
            "workloads": {c: [w[0] for w in ws] for c, ws in work.items()},
            "objective": "sum of median graph-plan execution times (ms), CUDA events",
            "defaults": default, "table": table, "trials": trials}


def main(argv=None):
    p = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    p.add_argument("--out", default=str(Path(__file__).with_name("tuning.json")))
    p.add_argument("--sweeps", type=int, default=2)
    p.add_argument("--reps", type=int, default=7)
    args = p.parse_args(argv)
    res = tune(args.sweeps, args.reps)
    Path(args.out).write_text(json.dumps(res, indent=1) + "\n")
    print(f"wrote {args.out}")


if __name__ == "__main__":
    sys.exit(main())
