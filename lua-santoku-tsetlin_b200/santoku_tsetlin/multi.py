"""Multi-GPU plumbing: one process per GPU, torch.distributed for the host
side.  The reference has no distributed code; its units -- 8-clause chunks
of one class of one machine -- are independent, so the path shards with no
data-path collective:

* training: machines (search trials) or replicas are partitioned across
  ranks by cost (`partition_lpt`); nothing is exchanged while they train;
* training one machine on several GPUs: each rank trains a contiguous class
  range (its units; every draw is keyed, so the units do not depend on
  each other) and the ranks then all-gather those classes' automata, after
  which every rank holds exactly the single-GPU result -- `train_sharded`;
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


def train_sharded(machine, tbl, group=None, device=None):
    """Train one machine across the ranks of `group`: rank r trains the
    units of its class range (`class_range`) -- nothing is exchanged while
    training -- then one all-gather of each range's action and count-plane
    bytes (the reference's per-class byte blocks, `Machine.export_classes`)
    leaves the full trained machine on every rank, bit-identical to training
    it on one GPU.  `device`: a CUDA device for NCCL, where the slices are
    exported, exchanged and imported device to device; None for gloo (host
    buffers).  A rank whose range is empty (more ranks than classes) trains
    nothing but joins the exchange, so no rank waits for it."""
    import torch
    import torch.distributed as dist
    world = dist.get_world_size(group) if dist.is_initialized() else 1
    rank = dist.get_rank(group) if dist.is_initialized() else 0
    info = machine.info()
    if info["individualized"]:
        raise ValueError("train_sharded: individualized machines have uneven class blocks")
    classes = info["classes"]
    lo, hi = class_range(classes, world, rank)
    if hi > lo:
        t = dict(tbl)
        t["class_range"] = (lo, hi)
        machine.train(t)
    if world == 1:
        return machine
    ranges = [class_range(classes, world, r) for r in range(world)]
    width = max(h - l for l, h in ranges)
    slot = sum(machine.class_bytes(0, width))
    local = torch.zeros(slot, dtype=torch.uint8, device=device)
    if hi > lo:
        machine.export_classes(lo, hi, local)
    parts = [torch.empty_like(local) for _ in range(world)]
    dist.all_gather(parts, local, group=group)
    for r, ((l, h), part) in enumerate(zip(ranges, parts)):
        if r != rank and h > l:
            a, st = machine.class_bytes(l, h)
            machine.import_classes(l, h, part[:a + st])
    return machine
