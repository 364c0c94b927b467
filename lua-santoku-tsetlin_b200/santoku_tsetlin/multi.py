"""Multi-GPU plumbing: one process per GPU, torch.distributed for the host
side.  The reference has no distributed code; its units -- 8-clause chunks
of one class of one machine -- are independent, so the path shards with no
data-path collective:

* training: machines (search trials) or replicas are partitioned across
  ranks by cost (`partition_lpt`); nothing is exchanged while they train;
* predict of one machine too large for a GPU: each rank holds a contiguous
  range of classes and computes their per-class vote sums
  (`Machine.predict_scores`); one all-gather of those sums, then the
  reference's argmax (strict >, ties to the lowest class, capi.c:934-942) or
  sign bits (capi.c:982-990) -- `gather_predict`;
* timing: the max over ranks of each rank's device time (`max_over_ranks`).
"""
import numpy as np


def partition_lpt(costs, world):
    """Longest-processing-time-first assignment of items to `world` ranks.
    Returns a list of index lists, one per rank; deterministic (ties by
    index), so every rank computes the same assignment."""
    order = sorted(range(len(costs)), key=lambda i: (-costs[i], i))
    loads = [0.0] * world
    parts = [[] for _ in range(world)]
    for i in order:
        r = min(range(world), key=lambda k: (loads[k], k))
        parts[r].append(i)
        loads[r] += costs[i]
    return [sorted(p) for p in parts]


def class_range(classes, world, rank):
    """Contiguous class range [lo, hi) held by `rank` when one machine's
    classes are split over `world` ranks."""
    base, extra = divmod(classes, world)
    lo = rank * base + min(rank, extra)
    return lo, lo + base + (1 if rank < extra else 0)


def max_over_ranks(value, group=None, device=None):
    """Max of a float over all ranks (the bench's device-time reduction)."""
    import torch
    import torch.distributed as dist
    if not dist.is_available() or not dist.is_initialized():
        return float(value)
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX, group=group)
    return float(t.item())


def gather_predict(local_scores, classes, kind="classifier", group=None, device=None):
    """All-gather the per-class vote sums of every rank's class range and
    finish predict: argmax for a classifier (ties to the lowest class), sign
    bits for an encoder (LSB-first, ceil(classes/8) bytes per sample).
    `local_scores` is int64 (n, hi - lo) for this rank's class range."""
    import torch
    import torch.distributed as dist
    local = torch.as_tensor(np.ascontiguousarray(local_scores, dtype=np.int64), device=device)
    world = dist.get_world_size(group) if dist.is_initialized() else 1
    if world > 1:
        n = local.shape[0]
        widest = max(class_range(classes, world, r)[1] - class_range(classes, world, r)[0]
                     for r in range(world))
        pad = torch.zeros((n, widest), dtype=torch.int64, device=local.device)
        pad[:, :local.shape[1]] = local
        parts = [torch.empty_like(pad) for _ in range(world)]
        dist.all_gather(parts, pad, group=group)
        full = torch.cat([parts[r][:, :class_range(classes, world, r)[1] -
                                   class_range(classes, world, r)[0]] for r in range(world)],
                         dim=1)
    else:
        full = local
    full = full.cpu().numpy()
    if kind == "classifier":
        # strict > from the lowest class: numpy argmax returns the first max
        return np.argmax(full, axis=1).astype(np.int64), full
    bits = full > 0
    return np.packbits(bits, axis=1, bitorder="little").ravel(), full
