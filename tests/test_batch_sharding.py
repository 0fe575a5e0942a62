"""Host logic of the batched solver that needs no GPU: the work estimate, the rank partition
of the systems (every rank computes it alone; run as two gloo ranks), and the loud failure
of the batch entry points when no GPU is present."""
import os

import numpy as np
import pytest

from project_xplus_b200.batch import shard_systems, system_work


def test_shard_partition_properties():
    from project_xplus_b200 import generators as g
    sides, _ = g.batch_sides(512, 45, 256, seed=3)
    works = [system_work(int(s) ** 2, 7 * int(s) ** 2) for s in sides]
    for world in (1, 2, 3, 8):
        parts = [shard_systems(works, world, r) for r in range(world)]
        flat = sorted(k for p in parts for k in p)
        assert flat == list(range(len(works)))  # a partition
        loads = [sum(works[k] for k in p) for p in parts]
        # greedy LPT: no rank exceeds the mean by more than the heaviest system
        assert max(loads) - sum(loads) / world <= max(works) + 1e-9
    with pytest.raises(ValueError):
        shard_systems(works, 2, 2)


def _rank_main(rank, world, port, works, q):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    mine = shard_systems(works, world, rank)
    gathered = [None] * world
    dist.all_gather_object(gathered, mine)
    dist.destroy_process_group()
    q.put((rank, gathered))


def test_two_rank_shards_agree():
    import multiprocessing as mp
    import socket
    works = [float(w) for w in np.random.default_rng(1).uniform(1, 100, 37)]
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, works, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = dict(q.get(timeout=120) for _ in procs)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    # both ranks saw the same partition, and it covers every system exactly once
    assert out[0] == out[1]
    flat = sorted(k for part in out[0] for k in part)
    assert flat == list(range(len(works)))


def test_batch_fails_loudly_without_gpu():
    from project_xplus_b200 import XplusError, device_count
    from project_xplus_b200 import generators as g
    from project_xplus_b200.batch import BatchSolver
    if device_count() > 0:
        pytest.skip("a GPU is present")
    d, _ = g.fem2d(8)
    with pytest.raises(XplusError) as e:
        BatchSolver([(d.row_ptr, d.col_idx, d.values)])
    assert e.value.code == 11  # XPLUS_ERR_CUDA


def _solve_rank(rank, world, port, q):
    """One rank of the sharded batch as bench.py runs it: every rank builds the same system
    list, solves only its shard (here with the oracle's FP64 golden standing in for the GPU
    batch kernel, which needs a GPU), times it, and the job's time is the max over ranks."""
    import time

    import torch
    import torch.distributed as dist

    from oracle import oracle as O
    from project_xplus_b200 import generators as g
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    sides, sigmas = g.batch_sides(12, 6, 24, seed=5)
    works = [system_work(int(s) ** 2, 7 * int(s) ** 2) for s in sides]
    mine = shard_systems(works, world, rank)
    t0 = time.perf_counter()
    xs = {}
    for k in mine:
        d, _ = g.fem2d(int(sides[k]), sigma=float(sigmas[k]), seed=1000 + k, x_seed=1000 + k)
        tau_rr = (1e-8 * float(np.linalg.norm(d.b))) ** 2
        xs[k] = O.golden(d, tau_rr)["x"]
    dt = torch.tensor([time.perf_counter() - t0], dtype=torch.float64)
    dist.all_reduce(dt, op=dist.ReduceOp.MAX)
    gathered = [None] * world
    dist.all_gather_object(gathered, xs)
    dist.destroy_process_group()
    q.put((rank, float(dt.item()), gathered))


def test_two_ranks_solve_their_shards():
    """Two gloo ranks each solve their shard of a batch; the gathered solutions cover every
    system once and equal a one-process solve of the whole batch bit for bit, every solution
    meets the FP64 true-residual tolerance, and both ranks report the same max-over-ranks time."""
    import multiprocessing as mp
    import socket

    from oracle import oracle as O
    from project_xplus_b200 import generators as g
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    procs = [ctx.Process(target=_solve_rank, args=(r, 2, port, q)) for r in range(2)]
    for p in procs:
        p.start()
    out = {}
    for _ in procs:
        rank, t, gathered = q.get(timeout=300)
        out[rank] = (t, gathered)
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    assert out[0][0] == out[1][0] > 0.0
    merged = {}
    for part in out[0][1]:
        assert not set(part) & set(merged)
        merged.update(part)
    sides, sigmas = g.batch_sides(12, 6, 24, seed=5)
    assert sorted(merged) == list(range(len(sides)))
    for k in range(len(sides)):
        d, _ = g.fem2d(int(sides[k]), sigma=float(sigmas[k]), seed=1000 + k, x_seed=1000 + k)
        ref = O.golden(d, (1e-8 * float(np.linalg.norm(d.b))) ** 2)["x"]
        np.testing.assert_array_equal(merged[k], ref)
        assert O.residual_norm(d, merged[k]) <= 1e-8 * np.linalg.norm(d.b)
