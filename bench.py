#!/usr/bin/env python3
"""Throughput of the float64 L.A.Cosmic detect/replace path on B200.

Workload (one step): clean the ``stack_2048`` batch once, i.e. 16 float64
frames of 2048 x 2048 from the seeded scene generator (sky U[500, 3000],
400 stars, 1200 cosmic rays per frame, one shared error map, a 0.5% + 2-column
bad-pixel mask, 0.1% NaN pixels), contrast=3, cr_threshold=5,
neighbor_threshold=3, maxiter=4, mirror borders.  The inputs (512 MiB of
pixels) are larger than the 126 MB L2, so no flush is needed between steps.

* ``value``: Mpix/s with inputs resident in HBM, through a plan whose whole
  maxiter loop is one CUDA graph (device-side while node), timed with CUDA
  events on the launching stream, max over ranks.
* ``e2e``: the same metric through the reference-facing host entry point
  ``remove_cosmics`` (one call per frame, pinned host buffers in and out,
  every copy inside the timed region).
* ``roofline``: the dominant kernel (prepare, the largest share of kernel
  time): its algorithmic bytes per launch over its CUDA-event duration,
  against the measured HBM copy bandwidth; ``roofline_sig_bulk`` the same for
  the dense detection kernel.
* ``plain``/``ragged``: the same implementation called once per frame
  (``remove_cosmics_device``) versus one batched plan, on this stack and on
  the ragged 64-frame batch with per-frame scalars.
* ``cpu_baseline``: the CPU oracle (a restatement of the reference's
  algorithm; lacosmic 1.4.0 is not installed) on a bounded sample of the same
  workload, all host threads.

``--impl reference`` times that CPU implementation alone as the reference arm.
Multi-GPU (torchrun): every rank cleans its own stack (weak scaling); frames
are independent, so no collective touches the data path.
"""

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "Mpix/s (f64, maxiter=4, identical masks) batched vs plain; bwd/fwd time"
SETTINGS = dict(contrast=3.0, cr_threshold=5.0, neighbor_threshold=3.0, maxiter=4)
SIG_BULK_DRAM_BYTES_PER_PX = 8.62  # ncu: 144.6 MB per launch over 16.78 Mpix
# ncu, prepare_bulk_kernel, one 16-frame stack launch (this workload):
# 565.2 MB read + 514.2 MB written over 67.1 Mpix (written pixels still in
# L2 at the end of the launch are not counted).
PREPARE_DRAM_BYTES_PER_PX = 16.08


def parse_args():
    p = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=500)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", choices=("mine", "reference"), default="mine")
    p.add_argument("--frames", type=int, default=16)
    p.add_argument("--size", type=int, default=2048)
    p.add_argument("--no-extras", action="store_true", help="skip plain/ragged comparisons")
    p.add_argument("--no-large", action="store_true", help="skip the 4 x 8192^2 forward/backward run")
    p.add_argument("--cpu-sample-rows", type=int, default=1024,
                   help="rows of one frame timed for the CPU baseline")
    return p.parse_args()


class Clocks:
    """nvidia-smi samples (every 200 ms) taken while a region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200", "-i", str(index)], stdout=self.file, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        self.proc.wait()
        self.file.seek(0)
        rows = [r.split(",") for r in self.file.read().strip().splitlines() if r.strip()]
        os.unlink(self.file.name)
        sm, mx, power, reasons = [], [], [], set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for r in rows:
            try:
                sm.append(float(r[1]))
                mx.append(float(r[2]))
                power.append(float(r[3]))
            except (ValueError, IndexError):
                continue
            for name, v in zip(names, r[5:9]):
                if v.strip().lower().startswith("active"):
                    reasons.add(name)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(mx) if mx else None,
                "power_w_max": max(power) if power else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def cpu_reference(frame, error, mask, rows, threads=0):
    """Time the CPU oracle on the first `rows` rows of one frame (all host
    threads, or `threads` of them)."""
    from oracle import oracle
    sub = np.ascontiguousarray(frame[:rows])
    prev = oracle.set_threads(0)
    oracle.set_threads(threads or os.cpu_count())
    try:
        t = time.perf_counter()
        oracle.clean_frame(sub, error=np.ascontiguousarray(error[:rows]),
                           mask=np.ascontiguousarray(mask[:rows]), border="mirror", **SETTINGS)
        dt = time.perf_counter() - t
    finally:
        oracle.set_threads(prev)
    return sub.size / dt / 1e6, dt, sub.size


def cpu_single_thread(frame, error, mask, rows):
    """The CPU oracle on one host thread (a like-for-like stand-in for a
    single-threaded CPU implementation), on an eighth of the sample rows."""
    v, dt, n = cpu_reference(frame, error, mask, max(32, rows // 8), threads=1)
    return {"value": round(v, 4), "unit": "Mpix/s", "cores": 1,
            "sample": f"{n // frame.shape[1]}x{frame.shape[1]} rows of frame 0 ({n} px, {dt:.1f} s)"}


def run_reference_arm(args, world, rank):
    """The reference's algorithm on the host cores (CPU oracle, all threads)."""
    if rank != 0:
        return
    from cusmic_b200 import scenes
    sc = scenes.stack_2048(seed=0, frames=1, size=args.size)
    f = sc.frames[0]
    for _ in range(args.warmup):
        cpu_reference(f.data, sc.error, sc.mask, args.cpu_sample_rows)
    t0 = time.perf_counter()
    px = 0
    for _ in range(args.steps):
        _, _, n = cpu_reference(f.data, sc.error, sc.mask, args.cpu_sample_rows)
        px += n
    dt = time.perf_counter() - t0
    value = px / dt / 1e6
    cores = os.cpu_count()
    sample = (f"{args.cpu_sample_rows}x{args.size} rows of one {args.size}x{args.size} frame of "
              f"the stack per step, maxiter=4, OpenMP over {cores} threads")
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": round(value, 4), "unit": "Mpix/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1000 * dt / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload_config(args),
        "cpu_baseline": {"value": round(value, 4), "unit": "Mpix/s", "cores": cores,
                         "kind": "port", "sample": sample,
                         "single_thread": cpu_single_thread(f.data, sc.error, sc.mask,
                                                            args.cpu_sample_rows)},
        "e2e": {"value": round(value, 4), "unit": "Mpix/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }))


def workload_config(args):
    return {"workload": f"stack_2048: {args.frames} x {args.size}x{args.size} float64 frames, "
                        "shared error map, 0.5% + 2-column mask, 0.1% NaN, contrast=3 cr=5 "
                        "nb=3 maxiter=4, mirror",
            "frames": args.frames, "height": args.size, "width": args.size,
            "l2": "inputs larger than L2 (no flush)"}


def main():
    args = parse_args()
    world, rank, local = dist_setup(args)
    if args.impl == "reference":
        run_reference_arm(args, world, rank)
        return
    import torch
    import torch.distributed as dist
    from cusmic_b200 import _native, scenes
    from cusmic_b200.plan import Plan, Batch

    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", device_id=torch.device("cuda", local),
                                timeout=__import__("datetime").timedelta(seconds=300))
    dev = torch.device("cuda", local)
    sc = scenes.stack_2048(seed=rank, frames=args.frames, size=args.size)
    nf, h, w = args.frames, args.size, args.size
    total_px = nf * h * w
    host_stack = np.stack([f.data for f in sc.frames])
    stack = torch.from_numpy(host_stack).to(dev)
    error = torch.from_numpy(sc.error).to(dev)
    mask = torch.from_numpy(sc.mask.astype(np.uint8)).to(dev)
    batch = Batch.stack(stack, error=error, mask=mask)
    plan = Plan(batch, graph=True, **SETTINGS)
    stream = torch.cuda.current_stream(dev)

    def barrier():
        if world > 1:
            dist.barrier()
        torch.cuda.synchronize(dev)

    smi_index = os.environ.get("CUDA_VISIBLE_DEVICES", str(local)).split(",")[0]
    clocks = Clocks(smi_index if smi_index.isdigit() else local)
    for _ in range(args.warmup):
        plan.execute(stream)
    plan.wait()
    passes = plan.passes()
    ref_clean = batch.clean.clone()
    ref_mask = batch.mask_out.clone()

    barrier()
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record(stream)
    for _ in range(args.steps):
        plan.execute(stream)
    end.record(stream)
    barrier()
    clk = clocks.stop()
    plan.wait()
    ms = start.elapsed_time(end)
    ms_t = torch.tensor([ms], device=dev, dtype=torch.float64)
    if world > 1:
        dist.all_reduce(ms_t, op=dist.ReduceOp.MAX)
    ms = float(ms_t.item())
    value = world * total_px * args.steps / (ms / 1e3) / 1e6
    identical = bool(torch.equal(batch.mask_out, ref_mask)) and bool(
        torch.equal(batch.clean.view(torch.int64), ref_clean.view(torch.int64)))

    # Per-kernel CUDA-event durations (same work, launched without the graph).
    prof = [plan.profile(stream) for _ in range(3)]
    kinds = _native.KERNEL_KINDS
    kms = {k: sum(p[0][k] for p in prof) / len(prof) for k in kinds}
    klaunch = {k: prof[0][1][k] for k in kinds}
    peaks = json.loads((ROOT / "MEASURED_PEAKS.json").read_text()) \
        if (ROOT / "MEASURED_PEAKS.json").exists() else {}
    peak = peaks.get("hbm_gbs", 6650.0)
    peak_source = "measured" if peaks else "fallback"
    total_kernel_ms = sum(kms.values())

    # The dominant kernel: prepare (holes, exclusions, clean pixels and the
    # static bit planes, once per call), HBM-bound.  Per pixel it reads the
    # float64 input (8 B) and the mask byte (1 B), writes clean (8 B) and the
    # HOLE, EXCL and DONOR bit words (3/8 B).  This batch's frames (widths a
    # multiple of 16, aligned buffers, no background map) take the bulk-staged
    # variant.
    prep_px = nf * h * w * klaunch["prepare"]
    prep_bytes = prep_px * (8 + 1 + 8 + 3 / 8)
    prep_ms = kms["prepare"]
    prep_achieved = prep_bytes / (prep_ms / 1e3) / 1e9
    prep_launch_px = prep_px / max(1, klaunch["prepare"])
    roofline = {"bound": "hbm", "kernel": "prepare_bulk_kernel",
                "achieved": round(prep_achieved, 1), "peak": peak, "unit": "GB/s",
                "frac": round(prep_achieved / peak, 4),
                "traffic": round(prep_launch_px * PREPARE_DRAM_BYTES_PER_PX),
                "peak_source": peak_source,
                "algorithmic_bytes_per_launch": round(prep_bytes / max(1, klaunch["prepare"])),
                "avg_launch_ms": round(prep_ms / max(1, klaunch["prepare"]), 4),
                "kernel_ms": {k: round(v, 4) for k, v in kms.items() if v},
                "kernel_share": {k: round(v / total_kernel_ms, 4) for k, v in kms.items() if v}}

    # Dense detection kernel (sig_bulk_kernel), run by the first (full) pass
    # over every frame.  Per pixel it reads clean (8 B); its bit planes were
    # zeroed by the call's prologue memset, and its writes (the sparse pre
    # list) are a few MB.  The error map is not read there: its 32 x 32 block
    # floors are computed once per call by floor_kernel.  Later passes are
    # incremental and do not run it.
    active_px = nf * h * w * klaunch["sigraw"]
    detect_bytes = active_px * 8
    detect_ms = kms["sigraw"]
    achieved = detect_bytes / (detect_ms / 1e3) / 1e9
    # DRAM bytes per active pixel of one sig_bulk_kernel launch from an ncu
    # capture (profiles/sig_bulk_kernel_stack_2048_4frames.md), scaled to this
    # launch's active pixels.
    traffic = active_px * SIG_BULK_DRAM_BYTES_PER_PX / max(1, klaunch["sigraw"])
    roofline_sig_bulk = {"bound": "hbm", "kernel": "sig_bulk_kernel", "achieved": round(achieved, 1),
                         "peak": peak, "unit": "GB/s", "frac": round(achieved / peak, 4),
                         "traffic": round(traffic), "peak_source": peak_source,
                         "algorithmic_bytes_per_launch": round(detect_bytes / max(1, klaunch["sigraw"])),
                         "avg_launch_ms": round(detect_ms / max(1, klaunch["sigraw"]), 4)}
    # Kernels of one execution as the event profiler saw them, plus the one
    # that shares a mark with another kernel: the replacement's target
    # selection (every pass).
    launches_per_step = sum(klaunch.values()) + klaunch["sigraw"] + klaunch["dirty"]

    out = {"metric": METRIC, "value": round(value, 2), "unit": "Mpix/s", "n_gpus": world,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 4),
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
           "data": "synthetic (seeded scene generator, inputs resident in HBM)",
           "config": dict(workload_config(args), parallelism=f"frames sharded, {world} GPU(s)",
                          path="plan + CUDA graph (while node)", passes=passes,
                          repeatable=identical),
           "roofline": roofline, "roofline_sig_bulk": roofline_sig_bulk, "clocks": clk, "gpu_launches": launches_per_step * args.steps}

    # End to end through the host entry point, pinned host buffers.
    e2e_steps = max(2, min(args.steps, 5))
    L = _native.lib()
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory()
    h_data = [pin(f.data) for f in sc.frames]
    h_err, h_mask = pin(sc.error), pin(sc.mask.astype(np.uint8))
    h_clean = torch.empty((h, w), dtype=torch.float64).pin_memory()
    h_flags = torch.empty((h, w), dtype=torch.uint8).pin_memory()
    o = plan.options
    msg = ctypes.create_string_buffer(256)

    def host_step():
        for f in range(nf):
            im = _native.Image(h_data[f].data_ptr(), h_err.data_ptr(), None, None, None,
                               h_mask.data_ptr(), w, h)
            st = L.remove_cosmics(ctypes.byref(im), ctypes.byref(o), h_clean.data_ptr(),
                                  h_flags.data_ptr(), msg, 256)
            if st:
                raise RuntimeError(msg.value.decode())
    host_step()
    barrier()
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        host_step()
    barrier()
    e2e_s = time.perf_counter() - t0
    e2e_t = torch.tensor([e2e_s], device=dev, dtype=torch.float64)
    if world > 1:
        dist.all_reduce(e2e_t, op=dist.ReduceOp.MAX)
    e2e_s = float(e2e_t.item())
    out["e2e"] = {"value": round(world * total_px * e2e_steps / e2e_s / 1e6, 2), "unit": "Mpix/s",
                  "h2d_bytes_per_step": nf * h * w * (8 + 8 + 1),
                  "d2h_bytes_per_step": nf * h * w * (8 + 1),
                  "path": "remove_cosmics (host C ABI), one call per frame, pinned buffers"}
    last_frame_ok = bool(np.array_equal(h_flags.numpy(), batch.mask_out[-1].cpu().numpy()))
    out["e2e"]["identical_masks"] = last_frame_ok

    if not args.no_extras and world == 1:  # single-GPU comparisons
        out["plain"] = plain_vs_batched(plan, batch, stream, value / world, barrier)
        out["ragged"] = ragged_comparison(dev, stream, barrier)
        out["adjoint"] = adjoint_timing(dev, stream, barrier)
        if not args.no_large:
            out["large"] = large_run(dev, stream, barrier)

    if rank == 0:
        v, dt, n = cpu_reference(sc.frames[0].data, sc.error, sc.mask, args.cpu_sample_rows)
        out["cpu_baseline"] = {"value": round(v, 4), "unit": "Mpix/s", "cores": os.cpu_count(),
                               "kind": "port",
                               "sample": f"{args.cpu_sample_rows}x{w} rows of frame 0 "
                                         f"({n} px, {dt:.1f} s), maxiter=4, OpenMP threads",
                               "single_thread": cpu_single_thread(
                                   sc.frames[0].data, sc.error, sc.mask, args.cpu_sample_rows)}
        print(json.dumps(out))
    plan.close()
    if world > 1:
        dist.destroy_process_group()


def plain_vs_batched(plan, batch, stream, batched_value, barrier):
    """Per-frame remove_cosmics_device calls of the same implementation."""
    import torch
    from cusmic_b200 import _native
    L = _native.lib()
    o = plan.options
    nf, h, w = batch.data.shape
    msg = ctypes.create_string_buffer(256)
    ims = batch.images()

    def step():
        for f in range(nf):
            st = L.remove_cosmics_device(ctypes.byref(ims[f]), ctypes.byref(o),
                                         batch.clean[f].data_ptr(), batch.mask_out[f].data_ptr(),
                                         stream.cuda_stream, msg, 256)
            if st:
                raise RuntimeError(msg.value.decode())
    step()
    barrier()
    t0 = time.perf_counter()
    reps = 3
    for _ in range(reps):
        step()
    barrier()
    dt = time.perf_counter() - t0
    plain = nf * h * w * reps / dt / 1e6
    return {"plain_mpix_s": round(plain, 2), "batched_mpix_s": round(batched_value, 2),
            "batched_over_plain": round(batched_value / plain, 3),
            "plain_path": "remove_cosmics_device per frame (synchronising calls)"}


def ragged_comparison(dev, stream, barrier):
    """ragged_64: one batched plan (graph) versus 64 per-frame calls."""
    import torch
    from cusmic_b200 import _native, scenes
    from cusmic_b200.plan import Plan, Batch
    sc = scenes.ragged_64(seed=0)
    frames = [torch.from_numpy(f.data).to(dev) for f in sc.frames]
    scal = [(f.gain, f.readnoise, f.background) for f in sc.frames]
    batch = Batch.ragged(frames, scalars=scal)
    plan = Plan(batch, graph=True, **SETTINGS)
    for _ in range(3):
        plan.execute(stream)
    plan.wait()
    barrier()
    reps = 5
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s.record(stream)
    for _ in range(reps):
        plan.execute(stream)
    e.record(stream)
    barrier()
    plan.wait()
    px = sum(f.numel() for f in frames)
    batched = px * reps / (s.elapsed_time(e) / 1e3) / 1e6
    prof = [plan.profile(stream) for _ in range(2)]
    kernel_ms = {k: round(sum(p[0][k] for p in prof) / len(prof), 4)
                 for k in _native.KERNEL_KINDS if prof[0][0][k]}
    L = _native.lib()
    msg = ctypes.create_string_buffer(256)
    ims = batch.images()
    outs = [(torch.empty_like(f), torch.empty(f.shape, dtype=torch.uint8, device=dev))
            for f in frames]

    def step():
        for i, f in enumerate(frames):
            o = plan.options_for(i)
            st = L.remove_cosmics_device(ctypes.byref(ims[i]), ctypes.byref(o),
                                         outs[i][0].data_ptr(), outs[i][1].data_ptr(),
                                         stream.cuda_stream, msg, 256)
            if st:
                raise RuntimeError(msg.value.decode())
    step()
    same = all(torch.equal(outs[i][1].flatten(), batch.frame_mask(i).flatten())
               for i in range(len(frames)))
    barrier()
    t0 = time.perf_counter()
    for _ in range(3):
        step()
    barrier()
    plain = px * 3 / (time.perf_counter() - t0) / 1e6
    plan.close()
    return {"frames": len(frames), "pixels": px, "batched_mpix_s": round(batched, 2),
            "plain_mpix_s": round(plain, 2), "batched_over_plain": round(batched / plain, 3),
            "identical_masks": bool(same), "kernel_ms": kernel_ms}


# Cycles of the sleep kernel ahead of a gated interval (about 0.27 ms at
# 1.965 GHz): longer than the host's overhead for one call.
GATE_CYCLES = 1 << 19


def gated_ms(stream, call):
    """CUDA-event time of call() on `stream`.  A short sleep kernel ahead of the
    start event holds the stream while the host runs the call's Python and C
    checks, so the interval starts with the call's device work.  A call that
    synchronises on entry must get a stream other than the one its last
    execution ran on (the backward, after a forward on another stream); for a
    call that synchronises before returning (the backward) the interval ends
    with the host's return from that wait."""
    import torch
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(stream):
        torch.cuda._sleep(GATE_CYCLES)
    s.record(stream)
    out = call()
    e.record(stream)
    e.synchronize()
    return s.elapsed_time(e), out


def large_run(dev, stream, barrier):
    """large_8192: forward and frozen-mask backward of 4 x 8192^2 float64 frames
    (full-size error map, 2% mask), with the device memory the process holds."""
    import torch
    from cusmic_b200 import scenes
    from cusmic_b200.plan import Plan, Batch
    free0, total = torch.cuda.mem_get_info(dev)
    sc = scenes.large_8192(seed=0)
    stack = torch.from_numpy(np.stack([f.data for f in sc.frames])).to(dev)
    del sc.frames[:]
    batch = Batch.stack(stack, error=torch.from_numpy(sc.error).to(dev),
                        mask=torch.from_numpy(sc.mask.astype(np.uint8)).to(dev))
    plan = Plan(batch, graph=True, keep=True, **SETTINGS)
    g = torch.randn(stack.shape, dtype=torch.float64, device=dev,
                    generator=torch.Generator(device=dev).manual_seed(0))
    plan.execute(stream)
    plan.wait()
    first_mask = batch.mask_out.clone()
    plan.backward(g, stream)
    torch.cuda.synchronize(dev)
    reps = 3
    fwd = bwd = 0.0
    side = torch.cuda.Stream(device=dev)
    for _ in range(reps):
        barrier()
        t, _ = gated_ms(stream, lambda: plan.execute(stream))
        plan.wait()
        fwd += t
        t, _ = gated_ms(side, lambda: plan.backward(g, side))
        bwd += t
    free1, _ = torch.cuda.mem_get_info(dev)
    px = stack.numel()
    out = {"workload": "large_8192: 4 x 8192x8192 float64, full error map, 2% mask, 3000 rays "
                       "(10% tracks 10-40 px), 200 saturated stars, forward + frozen-mask backward",
           "fwd_ms": round(fwd / reps, 3), "bwd_ms": round(bwd / reps, 3),
           "bwd_over_fwd": round(bwd / fwd, 4), "fwd_mpix_s": round(px * reps / (fwd / 1e3) / 1e6, 1),
           "flagged": int(batch.mask_out.sum()),
           "repeatable": bool(torch.equal(first_mask, batch.mask_out)),
           "device_gb_held": round((total - free1) / 1e9, 2),
           "device_gb_before": round((total - free0) / 1e9, 2)}
    plan.close()
    del batch, stack, g
    torch.cuda.empty_cache()
    return out


def adjoint_timing(dev, stream, barrier):
    """adjoint_1024: forward (graph) versus frozen-mask backward, 8 x 1024^2."""
    import torch
    from cusmic_b200 import scenes
    from cusmic_b200.plan import Plan, Batch
    sc = scenes.adjoint_1024(seed=0)
    stack = torch.from_numpy(np.stack([f.data for f in sc.frames])).to(dev)
    batch = Batch.stack(stack)
    plan = Plan(batch, graph=True, keep=True, gain=2.0, readnoise=5.0, background=0.0,
                **{k: v for k, v in SETTINGS.items()})
    g = torch.randn(stack.shape, dtype=torch.float64, device=dev,
                    generator=torch.Generator(device=dev).manual_seed(0))
    for _ in range(3):
        plan.execute(stream)
        plan.wait()
        plan.backward(g, stream)
    reps = 10
    fwd = bwd = 0.0
    side = torch.cuda.Stream(device=dev)
    for _ in range(reps):
        barrier()
        t, _ = gated_ms(stream, lambda: plan.execute(stream))
        plan.wait()
        fwd += t
        t, _ = gated_ms(side, lambda: plan.backward(g, side))
        bwd += t
    plan.close()
    return {"workload": "adjoint_1024: 8 x 1024x1024, gain=2 rn=5 bg=0, L = sum(w * cleaned)",
            "fwd_ms": round(fwd / reps, 4), "bwd_ms": round(bwd / reps, 4),
            "bwd_over_fwd": round(bwd / fwd, 4)}


if __name__ == "__main__":
    main()
