"""Frame sharding across GPUs, one process per GPU.

Frames are independent (the reference processes a stack with one grid row
per frame, src/device.cuh:69-75, and never mixes frames), so a batch splits
across ranks with no collective on the data path: each rank cleans the frames
assigned to it on its own GPU, reading only its own memory.  The only
communication is host metadata — per-frame flagged-pixel counts and passes —
gathered with torch.distributed over whatever backend the process group uses.
"""

import torch
import torch.distributed as dist


def partition(sizes, world):
    """Assign frames to ranks balancing pixels (largest first, least loaded).

    ``sizes`` are per-frame pixel counts.  Returns ``world`` sorted lists of
    frame indices; every frame appears exactly once.
    """
    if world < 1:
        raise ValueError("world must be positive")
    load = [0] * world
    parts = [[] for _ in range(world)]
    for i in sorted(range(len(sizes)), key=lambda i: (-sizes[i], i)):
        r = min(range(world), key=lambda r: (load[r], r))
        parts[r].append(i)
        load[r] += sizes[i]
    return [sorted(p) for p in parts]


def world_rank():
    if dist.is_available() and dist.is_initialized():
        return dist.get_world_size(), dist.get_rank()
    return 1, 0


def gather_metadata(indices, values, nf):
    """All-gather per-frame host values (e.g. flagged counts) into one list."""
    world, _ = world_rank()
    mine = list(zip(indices, values))
    if world == 1:
        pairs = [mine]
    else:
        pairs = [None] * world
        dist.all_gather_object(pairs, mine)
    out = [None] * nf
    for part in pairs:
        for i, v in part:
            out[i] = v
    return out


def clean_sharded(frames, cleaner, scalars=None, errors=None, masks=None, device=None):
    """Clean this rank's share of ``frames`` (2D float64 arrays or tensors).

    Returns ({frame index: (cleaned, mask)} for the local frames, per-frame
    flagged counts of the whole batch).  ``scalars`` holds per-frame
    (gain, readnoise, background) tuples.
    """
    from .plan import Batch, Plan

    world, rank = world_rank()
    sizes = [int(f.shape[0]) * int(f.shape[1]) for f in frames]
    mine = partition(sizes, world)[rank]
    results = {}
    if mine:
        dev = device or torch.device("cuda", torch.cuda.current_device())
        as_dev = lambda a: torch.as_tensor(a, dtype=torch.float64).to(dev).contiguous()
        batch = Batch.ragged(
            [as_dev(frames[i]) for i in mine],
            errors=None if errors is None else [None if errors[i] is None else as_dev(errors[i])
                                                for i in mine],
            masks=None if masks is None else [None if masks[i] is None else
                                              torch.as_tensor(masks[i]).to(dev) for i in mine],
            scalars=None if scalars is None else [scalars[i] for i in mine])
        plan = Plan(batch, graph=False, contrast=float(cleaner.contrast),
                    cr_threshold=float(cleaner.cr_threshold),
                    neighbor_threshold=float(cleaner.neighbor_threshold),
                    maxiter=int(cleaner.maxiter), border=cleaner.border_mode)
        plan.execute()
        plan.wait()
        for k, i in enumerate(mine):
            results[i] = (batch.frame_clean(k).clone(), batch.frame_mask(k).to(torch.bool).clone())
        plan.close()
    counts = [int(results[i][1].sum()) for i in mine]
    return results, gather_metadata(mine, counts, len(frames))
