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
