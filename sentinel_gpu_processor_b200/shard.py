"""Burst pairs of a frame spread over GPUs, one process per GPU.

Burst pairs are independent, so a frame (or a stack's batch) shards over
ranks with no collective on the data path: each rank processes the pairs of
its shard with its own ``BatchedFrameChain``.  This is how the reference
spreads pairs over GPUs (one consumer per GPU on a shared queue,
csrc/src/crossmul_daemon.cu:990-1126), made static and balanced: the shards
are a longest-processing-time-first (LPT) assignment of the pairs by their
pixel count (Graham, "Bounds on multiprocessing timing anomalies", 1969: the
largest load is within 4/3 of the optimum).  Every rank computes the same
assignment from the same sizes, so no rank needs to tell another anything.
"""
from __future__ import annotations


def lpt_shards(weights, n_ranks):
    """Indices of ``weights`` per rank: items in order of decreasing weight
    (ties by index), each to the rank with the smallest load so far (ties by
    rank).  Deterministic; every index appears in exactly one shard, and each
    shard lists its indices in increasing order."""
    if n_ranks < 1:
        raise ValueError("n_ranks must be >= 1")
    w = [float(x) for x in weights]
    if any(x < 0 for x in w):
        raise ValueError("weights must be non-negative")
    loads = [0.0] * n_ranks
    shards = [[] for _ in range(n_ranks)]
    for i in sorted(range(len(w)), key=lambda k: (-w[k], k)):
        r = min(range(n_ranks), key=lambda q: (loads[q], q))
        shards[r].append(i)
        loads[r] += w[i]
    return [sorted(s) for s in shards]


def pair_pixels(ref_acqs):
    """Work of each burst pair: lines x samples of its reference burst (the
    unit the throughput is counted in)."""
    return [a.radar.lines_per_burst * a.radar.samples_per_burst for a in ref_acqs]


def frame_shard(ref_acqs, sec_acqs, rank, world):
    """This rank's burst pairs of a frame: (pair indices, their reference
    acquisitions, their secondary acquisitions)."""
    idx = lpt_shards(pair_pixels(ref_acqs), world)[rank]
    return idx, [ref_acqs[k] for k in idx], [sec_acqs[k] for k in idx]


def shard_loads(weights, shards):
    """Total weight of each shard."""
    return [sum(float(weights[i]) for i in s) for s in shards]


def gather_pairs(products, n_pairs, world, dst=0):
    """Collect per-pair products of every rank on rank ``dst``, in pair order:
    the one step that needs them together is stitching a subswath, whose
    bursts the split may have put on different ranks.  ``products`` maps this
    rank's pair indices to tensors (or tuples of tensors); they travel through
    ``torch.distributed.gather_object`` (NCCL or gloo), leaving as host
    copies.  Returns the list of ``n_pairs`` products on ``dst``, None
    elsewhere; with ``world == 1`` no process group is needed."""
    import torch

    def host(x):
        if isinstance(x, torch.Tensor):
            return x.detach().cpu()
        if isinstance(x, (tuple, list)):
            return type(x)(host(y) for y in x)
        return x

    mine = {int(k): host(v) for k, v in products.items()}
    if world == 1:
        parts = [mine]
    else:
        import torch.distributed as dist
        parts = [None] * world if dist.get_rank() == dst else None
        dist.gather_object(mine, parts, dst=dst)
        if dist.get_rank() != dst:
            return None
    out = [None] * n_pairs
    for part in parts:
        for k, v in part.items():
            if out[k] is not None:
                raise ValueError(f"pair {k} came from two ranks")
            out[k] = v
    missing = [k for k, v in enumerate(out) if v is None]
    if missing:
        raise ValueError(f"pairs {missing} came from no rank")
    return out
