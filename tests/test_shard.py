"""Burst pairs of a frame spread over ranks (``shard.lpt_shards``): every
pair lands on exactly one rank, the largest load is within Graham's 4/3
bound of the optimum, and ranks agree on the assignment without talking
(gloo, world size 2, each rank computing its own shard of the seeded frame)."""
import itertools
import os
import socket
import sys

import torch.multiprocessing as mp

from sentinel_gpu_processor_b200 import shard, synth

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _check_partition(shards, n):
    flat = sorted(i for s in shards for i in s)
    assert flat == list(range(n))


def test_lpt_partition_and_bound_against_brute_force():
    import random
    rnd = random.Random(7)
    for trial in range(40):
        n, m = rnd.randint(1, 9), rnd.randint(1, 4)
        w = [rnd.randint(1, 100) for _ in range(n)]
        s = shard.lpt_shards(w, m)
        assert len(s) == m
        _check_partition(s, n)
        best = min(max(sum(w[i] for i in range(n) if a[i] == r) for r in range(m))
                   for a in itertools.product(range(m), repeat=n))
        assert max(shard.shard_loads(w, s)) <= (4 / 3 - 1 / (3 * m)) * best + 1e-9


def test_gather_pairs_single_rank_and_errors():
    import torch
    out = shard.gather_pairs({1: torch.ones(2), 0: (torch.zeros(1), torch.ones(1))}, 2, 1)
    assert torch.equal(out[1], torch.ones(2)) and torch.equal(out[0][1], torch.ones(1))
    try:
        shard.gather_pairs({0: torch.ones(1)}, 2, 1)
    except ValueError as e:
        assert "no rank" in str(e)
    else:
        raise AssertionError("a missing pair was accepted")


def test_lpt_is_deterministic_and_handles_edges():
    assert shard.lpt_shards([], 3) == [[], [], []]
    assert shard.lpt_shards([5, 5, 5, 5], 2) == [[0, 2], [1, 3]]  # ties by index, then by rank
    assert shard.lpt_shards([1, 2, 3], 1) == [[0, 1, 2]]
    for bad in (([1], 0), ([-1, 2], 2)):
        try:
            shard.lpt_shards(*bad)
        except ValueError:
            continue
        raise AssertionError("accepted " + repr(bad))


def test_frame_pairs_balance():
    sc = synth.make_frame(slc_pairs=0, with_dem=False)
    w = shard.pair_pixels(sc.ref)
    for m in (2, 4, 8):
        s = shard.lpt_shards(w, m)
        _check_partition(s, len(sc.ref))
        loads = shard.shard_loads(w, s)
        # list scheduling: no rank exceeds the mean load by more than one pair
        assert max(loads) <= sum(loads) / m + max(w)
        if m <= 4:  # with several pairs per rank the uneven sizes even out
            assert max(loads) / (sum(loads) / m) < 1.05


def _free_port():
    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        return so.getsockname()[1]


def _worker(rank, world, port, q):
    sys.path.insert(0, ROOT)
    import datetime

    import torch
    import torch.distributed as dist

    from sentinel_gpu_processor_b200 import shard as sh, synth as sy
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), RANK=str(rank), WORLD_SIZE=str(world))
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    try:
        sc = sy.make_frame(slc_pairs=0, with_dem=False)
        idx, refs, secs = sh.frame_shard(sc.ref, sc.sec, rank, world)
        assert [a.radar.lines_per_burst for a in refs] == [sc.ref[k].radar.lines_per_burst for k in idx]
        mine = torch.zeros(len(sc.ref), dtype=torch.int64)
        mine[idx] = rank + 1
        seen = [torch.zeros_like(mine) for _ in range(world)]
        dist.all_gather(seen, mine)  # test only: the data path itself has no collective
        # per-pair products (a stand-in interferogram per pair) gathered on rank 0 for stitching
        prods = {k: torch.full((2, 3), float(k)) for k in idx}
        allp = sh.gather_pairs(prods, len(sc.ref), world, dst=0)
        ok = None if allp is None else all(torch.equal(t, torch.full((2, 3), float(k))) for k, t in enumerate(allp))
        q.put((rank, ([t.tolist() for t in seen], ok)))
    finally:
        dist.destroy_process_group()


def test_ranks_agree_on_disjoint_complete_shards():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(180)
        assert p.exitcode == 0
    got = dict(q.get(timeout=10) for _ in range(2))
    assert got[0][1] is True and got[1][1] is None  # rank 0 holds every pair's product, in order
    got = {r: v[0] for r, v in got.items()}
    assert got[0] == got[1]  # both ranks see the same assignment
    a, b = got[0]
    n = len(a)
    assert all((x > 0) != (y > 0) for x, y in zip(a, b))  # each pair on exactly one rank
    assert sum(x > 0 for x in a) + sum(y > 0 for y in b) == n
