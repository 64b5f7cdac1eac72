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
* ``e2e``: the same metric from host buffers to host buffers through the
  C ABI's batch host entry point ``cusmic_batch_host`` (pinned buffers; every
  copy inside the timed region; the shared maps cross PCIe once per step);
  ``e2e_per_frame`` beside it: the reference-facing ``remove_cosmics``, one
  call per frame, every map uploaded with every frame.
* ``roofline``: the dominant kernel (prepare, the largest share of kernel
  time; on this stack prepare and the first pass's dense detection run as one
  kernel, prep_detect_kernel): its algorithmic bytes per launch over its
  CUDA-event duration, against the measured HBM copy bandwidth;
  ``roofline_sig_bulk`` the same for the dense detection kernel where it runs
  on its own (the ragged batch, noise model).
* ``plain``/``ragged``: the same implementation called once per frame
  (``remove_cosmics_device``) versus one batched plan, on this stack and on
  the ragged 64-frame batch with per-frame scalars.
* ``reference_gpu``: the reference's own CUDA library, compiled from its
  sources for sm_100a, on the same resident inputs (a baseline leg, run after
  this arm's timed region): its batch call on the stack, 64 per-frame calls on
  the ragged batch, and whether its masks and pixels equal this library's on
  every workload.
* ``cpu_baseline``: the CPU oracle (a restatement of the reference's
  algorithm; lacosmic 1.4.0 is not installed) on one full frame of the same
  workload, all host threads, with a single-thread figure beside it.

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
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "Mpix/s (f64, maxiter=4, identical masks) batched vs plain; bwd/fwd time"
SETTINGS = dict(contrast=3.0, cr_threshold=5.0, neighbor_threshold=3.0, maxiter=4)
# ncu, sig_bulk_kernel, 4-frame stack launch: 144.6 MB over 16.78 Mpix.
SIG_BULK_DRAM_BYTES_PER_PX = 8.62
# ncu, prepare_bulk_kernel, one 16-frame stack launch (this workload):
# 565.2 MB read + 514.2 MB written over 67.1 Mpix (written pixels still in
# L2 at the end of the launch are not counted).
PREPARE_DRAM_BYTES_PER_PX = 16.08
# ncu, prep_detect_kernel (prepare with the dense detection), one 16-frame
# stack launch (this workload): 601.2 MB read + 525.2 MB written over
# 67.1 Mpix.
PREP_DETECT_DRAM_BYTES_PER_PX = 16.79
REF_GPU_SO = ROOT / "oracle" / "_ref" / "libcusmic_ref.so"


def parse_args():
    p = argparse.ArgumentParser(description=__doc__.split("\n")[0])
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=500)
    p.add_argument("--warmup", type=int, default=5,
                   help="warm-up executions at least (the warm-up also lasts at least "
                        "--warm-seconds, so the clock sampler sees the GPU under load)")
    p.add_argument("--warm-seconds", type=float, default=1.0)
    p.add_argument("--impl", choices=("mine", "reference"), default="mine")
    p.add_argument("--frames", type=int, default=16)
    p.add_argument("--size", type=int, default=2048)
    p.add_argument("--no-extras", action="store_true",
                   help="skip the plain/ragged/adjoint/large comparisons and the reference "
                        "library leg")
    p.add_argument("--no-large", action="store_true", help="skip the 4 x 8192^2 forward/backward run")
    p.add_argument("--cpu-sample-rows", type=int, default=0,
                   help="rows of one frame timed for the CPU baseline (0: the whole frame)")
    p.add_argument("--workload", choices=("stack_2048", "ragged_64"), default="stack_2048",
                   help="ragged_64: time only the noise-model ragged batch (its first "
                        "--ragged-frames frames), a short run for profiling its kernels")
    p.add_argument("--ragged-frames", type=int, default=64)
    p.add_argument("--no-e2e", action="store_true", help="skip the host-buffer runs")
    p.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline")
    return p.parse_args()


class Clocks:
    """SM clock, power and throttle reasons sampled every few milliseconds by a
    thread (NVML), or every 100 ms by nvidia-smi where NVML is not loadable;
    mark() brackets the timed region so its own samples are reported."""

    REASONS = (("hw_slowdown", "nvmlClocksEventReasonHwSlowdown"),
               ("hw_thermal_slowdown", "nvmlClocksEventReasonHwThermalSlowdown"),
               ("sw_thermal_slowdown", "nvmlClocksEventReasonSwThermalSlowdown"),
               ("sw_power_cap", "nvmlClocksEventReasonSwPowerCap"))

    def __init__(self, torch_device, period_s=0.002):
        self.samples = []  # (time, sm MHz, max MHz, power W, reasons)
        self.window = [None, None]
        self.stop_flag = threading.Event()
        self.proc = None
        self.source = "nvml"
        try:
            import pynvml as nv
            import torch
            nv.nvmlInit()
            props = torch.cuda.get_device_properties(torch_device)
            bus = f"{props.pci_domain_id:08x}:{props.pci_bus_id:02x}:{props.pci_device_id:02x}.0"
            self.nv, self.handle = nv, nv.nvmlDeviceGetHandleByPciBusId(bus)
            self.max_mhz = nv.nvmlDeviceGetMaxClockInfo(self.handle, nv.NVML_CLOCK_SM)
            self.thread = threading.Thread(target=self._poll, args=(period_s,), daemon=True)
            self.thread.start()
        except Exception:
            self.source = "nvidia-smi"
            self._start_smi(torch_device)

    def _poll(self, period_s):
        nv, h = self.nv, self.handle
        masks = [(name, getattr(nv, attr, 0)) for name, attr in self.REASONS]
        while not self.stop_flag.is_set():
            try:
                sm = nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)
                pw = nv.nvmlDeviceGetPowerUsage(h) / 1000.0
                bits = nv.nvmlDeviceGetCurrentClocksEventReasons(h)
                self.samples.append((time.perf_counter(), sm, self.max_mhz, pw,
                                     [n for n, m in masks if bits & m]))
            except Exception:
                pass
            time.sleep(period_s)

    def _start_smi(self, torch_device):
        fields = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,"
                  "clocks_event_reasons.hw_thermal_slowdown,"
                  "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        index = os.environ.get("CUDA_VISIBLE_DEVICES", str(torch_device.index or 0)).split(",")[0]
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={fields}", "--format=csv,noheader,nounits",
                 "-lms", "100", "-i", index], stdout=self.file, stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def mark(self, which):
        self.window[which] = time.perf_counter()

    def stop(self):
        if self.source == "nvml":
            self.stop_flag.set()
            self.thread.join()
        elif self.proc is not None:
            self.proc.terminate()
            self.proc.wait()
            self.file.seek(0)
            for row in self.file.read().strip().splitlines():
                r = [c.strip() for c in row.split(",")]
                try:
                    self.samples.append((None, float(r[0]), float(r[1]), float(r[2]),
                                         [n for (n, _), v in zip(self.REASONS, r[3:7])
                                          if v.lower().startswith("active")]))
                except (ValueError, IndexError):
                    continue
            os.unlink(self.file.name)
        else:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no clock source"],
                    "samples": 0}
        t0, t1 = self.window
        timed = [s for s in self.samples if s[0] is not None and t0 <= s[0] <= t1]
        under = timed or self.samples[-max(1, len(self.samples) // 2):]
        reasons = sorted({r for s in under for r in s[4]})
        return {"sm_mhz": statistics.median(s[1] for s in under) if under else None,
                "sm_max_mhz": max(s[2] for s in under) if under else None,
                "power_w_max": max(s[3] for s in under) if under else None,
                "reasons": reasons, "samples": len(self.samples),
                "samples_in_timed_region": len(timed), "source": self.source}


def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def cpu_reference(frame, error, mask, rows, threads=0):
    """Time the CPU oracle on the first `rows` rows of one frame (0: all rows),
    with all host threads or `threads` of them."""
    from oracle import oracle
    rows = rows or frame.shape[0]
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
    rows = rows or frame.shape[0]
    v, dt, n = cpu_reference(frame, error, mask, max(32, rows // 8), threads=1)
    return {"value": round(v, 4), "unit": "Mpix/s", "cores": 1,
            "sample": f"{n // frame.shape[1]}x{frame.shape[1]} rows of frame 0 ({n} px, {dt:.1f} s)"}


def run_reference_arm(args, world, rank):
    """The reference's algorithm on the host cores (CPU oracle, all threads),
    one full frame of the stack per step."""
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
    rows = args.cpu_sample_rows or args.size
    sample = (f"{rows}x{args.size} rows of one {args.size}x{args.size} frame of the stack per "
              f"step, maxiter=4, OpenMP over {cores} threads")
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
    if args.workload == "ragged_64":
        ragged_only(args, world, rank, dev)
        if world > 1:
            dist.destroy_process_group()
        return
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

    clocks = Clocks(dev)
    # Warm-up: at least --warmup executions and --warm-seconds of GPU work, so
    # the clocks have settled under load when the timed region starts.
    warm, t_warm = 0, time.perf_counter()
    while warm < args.warmup or time.perf_counter() - t_warm < args.warm_seconds:
        plan.execute(stream)
        warm += 1
        if warm % 64 == 0:
            stream.synchronize()
    plan.wait()
    passes = plan.passes()
    ref_clean = batch.clean.clone()
    ref_mask = batch.mask_out.clone()

    barrier()
    clocks.mark(0)
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    start.record(stream)
    for _ in range(args.steps):
        plan.execute(stream)
    end.record(stream)
    barrier()
    clocks.mark(1)
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
    # HOLE, EXCL and DONOR bit words (3/8 B).  This batch's frames (error
    # maps, widths a multiple of 16, aligned buffers, no background) take
    # prep_detect_kernel, which also runs the first pass's dense detection on
    # the input rows (no separate dense-detection launch, no re-read of the
    # clean pixels; its pre-list writes, 16 B per listed pixel, about 1% of
    # the pixels, are not counted); other batches the bulk-staged prepare.
    fused = klaunch["sigraw"] == 0
    prep_px = nf * h * w * klaunch["prepare"]
    prep_bytes = prep_px * (8 + 1 + 8 + 3 / 8)
    prep_ms = kms["prepare"]
    prep_achieved = prep_bytes / (prep_ms / 1e3) / 1e9
    prep_launch_px = prep_px / max(1, klaunch["prepare"])
    dram_px = PREP_DETECT_DRAM_BYTES_PER_PX if fused else PREPARE_DRAM_BYTES_PER_PX
    roofline = {"bound": "hbm", "kernel": "prep_detect_kernel" if fused else "prepare_bulk_kernel",
                "achieved": round(prep_achieved, 1), "peak": peak, "unit": "GB/s",
                "frac": round(prep_achieved / peak, 4),
                "traffic": round(prep_launch_px * dram_px) if dram_px else None,
                "peak_source": peak_source,
                "algorithmic_bytes_per_launch": round(prep_bytes / max(1, klaunch["prepare"])),
                "avg_launch_ms": round(prep_ms / max(1, klaunch["prepare"]), 4),
                "kernel_ms": {k: round(v, 4) for k, v in kms.items() if v},
                "kernel_share": {k: round(v / total_kernel_ms, 4) for k, v in kms.items() if v}}

    # Dense detection kernel (sig_bulk_kernel), run by the first (full) pass
    # over every frame of batches that prep_detect_kernel does not serve (on
    # this stack it is part of prepare; see roofline_sig_bulk_ragged).  Per
    # pixel it reads clean (8 B); its bit planes were zeroed by the call's
    # prologue memset, and its writes (the sparse pre list) are a few MB.  The
    # error map is not read there: its 32 x 32 block floors are computed once
    # per call by floor_kernel.  Later passes are incremental and do not run it.
    roofline_sig_bulk = None
    if not fused:
        active_px = nf * h * w * klaunch["sigraw"]
        detect_bytes = active_px * 8
        detect_ms = kms["sigraw"]
        achieved = detect_bytes / (detect_ms / 1e3) / 1e9
        # DRAM bytes per active pixel of one launch from an ncu capture of the
        # 4-frame stack, scaled to this launch's active pixels.
        traffic = active_px * SIG_BULK_DRAM_BYTES_PER_PX / max(1, klaunch["sigraw"])
        roofline_sig_bulk = {"bound": "hbm", "kernel": "sig_bulk_kernel",
                             "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                             "frac": round(achieved / peak, 4), "traffic": round(traffic),
                             "peak_source": peak_source,
                             "algorithmic_bytes_per_launch": round(
                                 detect_bytes / max(1, klaunch["sigraw"])),
                             "avg_launch_ms": round(detect_ms / max(1, klaunch["sigraw"]), 4)}
    # Kernels of one execution as the event profiler saw them, plus the one
    # that shares a mark with another kernel: the replacement's target
    # selection (every pass, as the loop control).
    launches_per_step = sum(klaunch.values()) + klaunch["control"]

    out = {"metric": METRIC, "value": round(value, 2), "unit": "Mpix/s", "n_gpus": world,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms / args.steps, 4),
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
           "data": "synthetic (seeded scene generator, inputs resident in HBM)",
           "config": dict(workload_config(args), parallelism=f"frames sharded, {world} GPU(s)",
                          path="plan + CUDA graph (while node)", passes=passes,
                          repeatable=identical, warmup_executions=warm),
           "roofline": roofline, "roofline_sig_bulk": roofline_sig_bulk, "clocks": clk,
           "gpu_launches": launches_per_step * args.steps}

    if not args.no_e2e:
        out["e2e"], out["e2e_per_frame"] = end_to_end(sc, plan, batch, args, world, barrier)

    if not args.no_extras and world == 1:  # single-GPU comparisons
        out["plain"] = plain_vs_batched(plan, batch, stream, value / world, barrier)
        ragged, ragged_ctx = ragged_comparison(dev, stream, barrier)
        out["ragged"] = ragged
        if out["roofline_sig_bulk"] is None and ragged["kernel_ms"].get("sigraw"):
            # The dense kernel on the ragged batch (noise model): 8 B per pixel.
            rb = ragged["pixels"] * 8
            ach = rb / (ragged["kernel_ms"]["sigraw"] / 1e3) / 1e9
            out["roofline_sig_bulk"] = {
                "bound": "hbm", "kernel": "sig_bulk_kernel", "workload": "ragged_64",
                "achieved": round(ach, 1), "peak": peak, "unit": "GB/s",
                "frac": round(ach / peak, 4), "traffic": None, "peak_source": peak_source,
                "algorithmic_bytes_per_launch": rb,
                "avg_launch_ms": ragged["kernel_ms"]["sigraw"]}
        out["adjoint"], adjoint_ctx = adjoint_timing(dev, stream, barrier)
        out["reference_gpu"] = reference_gpu(plan, batch, ragged_ctx, adjoint_ctx, value,
                                             ragged["batched_mpix_s"], stream, dev)
        if not args.no_large:
            out["large"] = large_run(dev, stream, barrier, out["reference_gpu"])
        ragged_ctx["plan"].close()
        adjoint_ctx["plan"].close()

    if rank == 0 and args.no_cpu:
        print(json.dumps(out))
    elif rank == 0:
        v, dt, n = cpu_reference(sc.frames[0].data, sc.error, sc.mask, args.cpu_sample_rows)
        out["cpu_baseline"] = {"value": round(v, 4), "unit": "Mpix/s", "cores": os.cpu_count(),
                               "kind": "port",
                               "sample": f"{n // w}x{w} rows of frame 0 "
                                         f"({n} px, {dt:.1f} s), maxiter=4, OpenMP threads",
                               "single_thread": cpu_single_thread(
                                   sc.frames[0].data, sc.error, sc.mask, args.cpu_sample_rows)}
        print(json.dumps(out))
    plan.close()
    if world > 1:
        dist.destroy_process_group()


def ragged_only(args, world, rank, dev):
    """The noise-model ragged batch (per-frame gain, read noise, background)
    timed alone through a graph plan: a short run for profiling its kernels."""
    import torch
    from cusmic_b200 import _native, scenes
    from cusmic_b200.plan import Plan, Batch
    sc = scenes.ragged_64(seed=rank)
    fr = sc.frames[:args.ragged_frames]
    frames = [torch.from_numpy(f.data).to(dev) for f in fr]
    batch = Batch.ragged(frames, scalars=[(f.gain, f.readnoise, f.background) for f in fr])
    plan = Plan(batch, graph=True, **SETTINGS)
    stream = torch.cuda.current_stream(dev)
    for _ in range(args.warmup):
        plan.execute(stream)
    plan.wait()
    torch.cuda.synchronize(dev)
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s.record(stream)
    for _ in range(args.steps):
        plan.execute(stream)
    e.record(stream)
    e.synchronize()
    plan.wait()
    ms = s.elapsed_time(e) / args.steps
    prof = plan.profile(stream)
    if rank == 0:
        print(json.dumps({"metric": METRIC, "workload": f"ragged_64, first {len(fr)} frames",
                          "value": round(batch.total / (ms / 1e3) / 1e6, 2), "unit": "Mpix/s",
                          "ms_per_step": round(ms, 4), "steps": args.steps,
                          "kernel_ms": {k: round(v, 4) for k, v in prof[0].items() if v}}))
    plan.close()


def end_to_end(sc, plan, batch, args, world, barrier):
    """Host buffers in, host buffers out, every copy inside the timed region:
    the batch host entry point (the headline), and the reference-facing
    single-frame host call once per frame beside it."""
    import torch
    from cusmic_b200 import _native
    nf, h, w = args.frames, args.size, args.size
    total_px = nf * h * w
    dev = batch.clean.device
    L = _native.lib()
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory()
    h_stack = pin(np.stack([f.data for f in sc.frames]))
    h_err, h_mask = pin(sc.error), pin(sc.mask.astype(np.uint8))
    h_clean = torch.empty((nf, h, w), dtype=torch.float64).pin_memory()
    h_flags = torch.empty((nf, h, w), dtype=torch.uint8).pin_memory()
    o = plan.options
    msg = ctypes.create_string_buffer(256)
    ims = (_native.Image * nf)()
    for f in range(nf):
        ims[f] = _native.Image(h_stack[f].data_ptr(), h_err.data_ptr(), None, None, None,
                               h_mask.data_ptr(), w, h)

    def batch_step():
        st = L.cusmic_batch_host(ims, nf, ctypes.byref(o), None, h_clean.data_ptr(),
                                 h_flags.data_ptr(), msg, 256)
        if st:
            raise RuntimeError(msg.value.decode())

    def frame_step():
        for f in range(nf):
            st = L.remove_cosmics(ctypes.byref(ims[f]), ctypes.byref(o),
                                  h_clean[f].data_ptr(), h_flags[f].data_ptr(), msg, 256)
            if st:
                raise RuntimeError(msg.value.decode())

    def timed(step, reps):
        step()
        barrier()
        t0 = time.perf_counter()
        for _ in range(reps):
            step()
        barrier()
        t = torch.tensor([time.perf_counter() - t0], device=dev, dtype=torch.float64)
        if world > 1:
            import torch.distributed as dist
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
        return world * total_px * reps / float(t.item()) / 1e6

    reps = max(3, min(args.steps, 10))
    v_batch = timed(batch_step, reps)
    same_batch = bool(torch.equal(h_flags.to(dev), batch.mask_out)) and bool(
        torch.equal(h_clean.to(dev).view(torch.int64), batch.clean.view(torch.int64)))
    v_frame = timed(frame_step, max(2, min(args.steps, 5)))
    same_frame = bool(torch.equal(h_flags.to(dev), batch.mask_out)) and bool(
        torch.equal(h_clean.to(dev).view(torch.int64), batch.clean.view(torch.int64)))
    flagged = int(batch.mask_out.sum())
    e2e = {"value": round(v_batch, 2), "unit": "Mpix/s",
           "h2d_bytes_per_step": total_px * 8 + h * w * (8 + 1),
           "d2h_bytes_per_step": flagged * 16,
           "path": "cusmic_batch_host (host C ABI, whole stack per call: chunks of frames, "
                   "inbound copy and cleaning of neighbouring chunks overlapped; shared error "
                   "map and mask uploaded once; no background, so each chunk returns its "
                   "flagged pixels' positions and values (16 B each) and host threads copy "
                   "the inputs to the outputs), pinned buffers",
           "identical_to_resident": same_batch}
    per_frame = {"value": round(v_frame, 2), "unit": "Mpix/s",
                 "h2d_bytes_per_step": total_px * (8 + 8 + 1),
                 "d2h_bytes_per_step": total_px * (8 + 1),
                 "path": "remove_cosmics (host C ABI, the reference's single-frame call), one "
                         "call per frame, pinned buffers",
                 "identical_to_resident": same_frame}
    return e2e, per_frame


def plain_vs_batched(plan, batch, stream, batched_value, barrier):
    """Per-frame remove_cosmics_device calls of the same implementation."""
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
    return ({"frames": len(frames), "pixels": px, "batched_mpix_s": round(batched, 2),
             "plain_mpix_s": round(plain, 2), "batched_over_plain": round(batched / plain, 3),
             "identical_masks_plain_vs_batched": bool(same), "kernel_ms": kernel_ms},
            {"plan": plan, "batch": batch, "frames": frames})


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


def reference_lib():
    """The reference's CUDA library built from its own sources (oracle/build.py)
    for the baseline leg, or None when it was not built."""
    if not REF_GPU_SO.exists():
        return None
    from cusmic_b200 import _native
    L = ctypes.CDLL(str(REF_GPU_SO))
    vp, sz = ctypes.c_void_p, ctypes.c_size_t
    L.remove_cosmics_batch_device.restype = ctypes.c_int
    L.remove_cosmics_batch_device.argtypes = [ctypes.POINTER(_native.Image), sz,
                                              ctypes.POINTER(_native.Options), vp, vp, vp,
                                              ctypes.c_char_p, sz]
    return L


def same_outputs(torch, a_clean, a_mask, b_clean, b_mask):
    return bool(torch.equal(a_mask, b_mask)) and bool(
        torch.equal(a_clean.view(torch.int64), b_clean.view(torch.int64)))


def reference_gpu(plan, batch, ragged, adjoint, value, ragged_value, stream, dev):
    """Baseline leg: the reference's own CUDA library on the same resident
    inputs, after this arm's timed region.  Its device calls allocate their
    scratch and synchronise per pass, as its stock path does; each call is
    timed with CUDA events on the stream it runs on.  Also records whether
    its outputs equal this library's bit for bit."""
    import torch
    L = reference_lib()
    if L is None:
        return {"unavailable": "oracle/_ref/libcusmic_ref.so was not built"}
    msg = ctypes.create_string_buffer(512)
    out = {"library": "reference src/api.cu compiled for sm_100a (--fmad=false, -O2)"}

    def call(ims, nf, opts, clean, mask):
        st = L.remove_cosmics_batch_device(ims, nf, ctypes.byref(opts), clean, mask,
                                           stream.cuda_stream, msg, 512)
        if st:
            raise RuntimeError("reference library: " + msg.value.decode())

    def events(fn, reps):
        fn()
        torch.cuda.synchronize(dev)
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        t0 = time.perf_counter()
        s.record(stream)
        for _ in range(reps):
            fn()
        e.record(stream)
        e.synchronize()
        return s.elapsed_time(e) / reps, (time.perf_counter() - t0) * 1e3 / reps

    # stack_2048: one batch call per step.
    nf = len(batch.frames)
    ims = batch.images()
    r_clean, r_mask = torch.empty_like(batch.clean), torch.empty_like(batch.mask_out)
    ms, wall = events(lambda: call(ims, nf, plan.options, r_clean.data_ptr(), r_mask.data_ptr()),
                      3)
    px = batch.total
    out["stack_2048"] = {"mpix_s": round(px / (ms / 1e3) / 1e6, 2), "ms_per_step": round(ms, 3),
                         "wall_ms_per_step": round(wall, 3),
                         "mine_over_reference": round(value / (px / (ms / 1e3) / 1e6), 2),
                         "identical": same_outputs(torch, r_clean, r_mask, batch.clean,
                                                   batch.mask_out)}
    # ragged_64: its scalars are batch-wide, so one call per frame.
    rb, rp = ragged["batch"], ragged["plan"]
    rims = rb.images()
    rc, rm = torch.empty_like(rb.clean), torch.empty_like(rb.mask_out)
    opts = [rp.options_for(i) for i in range(len(rb.frames))]

    def per_frame():
        for i in range(len(rb.frames)):
            call(ctypes.byref(rims[i]), 1, opts[i], rc.data_ptr() + 8 * rb.offsets[i],
                 rm.data_ptr() + rb.offsets[i])
    ms, wall = events(per_frame, 2)
    rp.execute(stream)
    rp.wait()
    out["ragged_64"] = {"mpix_s": round(rb.total / (ms / 1e3) / 1e6, 2),
                        "ms_per_step": round(ms, 3), "wall_ms_per_step": round(wall, 3),
                        "calls_per_step": len(rb.frames),
                        "mine_over_reference": round(ragged_value / (rb.total / (ms / 1e3) / 1e6), 2),
                        "identical": same_outputs(torch, rc, rm, rb.clean, rb.mask_out)}
    # adjoint_1024 forward: identity of the outputs only.
    ab, ap = adjoint["batch"], adjoint["plan"]
    ap.execute(stream)
    ap.wait()
    ac, am = torch.empty_like(ab.clean), torch.empty_like(ab.mask_out)
    call(ab.images(), len(ab.frames), ap.options, ac.data_ptr(), am.data_ptr())
    out["adjoint_1024"] = {"identical": same_outputs(torch, ac, am, ab.clean, ab.mask_out)}
    return out


def large_run(dev, stream, barrier, reference_out=None):
    """large_8192: forward and frozen-mask backward of 4 x 8192^2 float64 frames
    (full-size error map, 2% mask), with the device memory the process holds;
    the reference library's forward on the same inputs is compared once."""
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
    L = reference_lib()
    if reference_out is not None and L is not None:
        msg = ctypes.create_string_buffer(512)
        rc, rm = torch.empty_like(batch.clean), torch.empty_like(batch.mask_out)
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        st = L.remove_cosmics_batch_device(batch.images(), len(batch.frames),
                                           ctypes.byref(plan.options), rc.data_ptr(),
                                           rm.data_ptr(), stream.cuda_stream, msg, 512)
        ms = (time.perf_counter() - t0) * 1e3
        reference_out["large_8192"] = (
            {"error": msg.value.decode()} if st else
            {"wall_ms": round(ms, 1), "mpix_s": round(px / (ms / 1e3) / 1e6, 1),
             "identical": same_outputs(torch, rc, rm, batch.clean, batch.mask_out)})
        del rc, rm
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
    return ({"workload": "adjoint_1024: 8 x 1024x1024, gain=2 rn=5 bg=0, L = sum(w * cleaned)",
             "fwd_ms": round(fwd / reps, 4), "bwd_ms": round(bwd / reps, 4),
             "bwd_over_fwd": round(bwd / fwd, 4)},
            {"plan": plan, "batch": batch})


if __name__ == "__main__":
    main()
