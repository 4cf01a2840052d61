"""Multi-GPU split of a Ferret extension (cuot_b200/shard.py), tested with
world_size 2 `gloo` ranks on CPU: the tree/row plan, the set-up broadcasts,
and that the ranks' shares concatenate to the unsplit result.  On CPU the
per-rank compute is the oracle; the GPU row-range kernel itself is checked
against the same property in test_gpu_parity.py."""
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

import oracle
from cuot_b200.shard import ShardPlan


def test_plan_matches_gpu_task_division():
    # ferret_cot.hpp:55-63 with t = 1280, 3 GPUs -> 427, 427, 426
    p = ShardPlan(1280, 13, 3)
    assert [p.trees(r) for r in range(3)] == [427, 427, 426]
    assert p.rows(0) == (0, 427 << 13) and p.rows(2)[1] == p.n
    assert all(p.rows(r)[1] == p.rows(r + 1)[0] for r in range(2))


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    port = s.getsockname()[1]
    s.close()
    return port


def _rank_main(rank, world, port, t, h, k, q):
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    plan = ShardPlan(t, h, world)
    rng = np.random.default_rng(5 + rank)
    # rank 0 owns the set-up material; the broadcast must deliver it everywhere
    seed = torch.from_numpy(rng.integers(0, 256, 16, dtype=np.uint8)) if rank == 0 else torch.zeros(16, dtype=torch.uint8)
    kk = torch.from_numpy(rng.integers(0, 256, (k, 16), dtype=np.uint8)) if rank == 0 else torch.zeros((k, 16), dtype=torch.uint8)
    dist.broadcast(seed, 0)
    dist.broadcast(kk, 0)
    # every rank derives the whole instance's roots from a common seed and takes its trees
    g = np.random.default_rng(99)
    roots_all = g.integers(0, 256, (t, 16), dtype=np.uint8)
    delta = g.integers(0, 256, 16, dtype=np.uint8)
    delta[0] |= 1
    f = plan.first_tree(rank)
    mine = roots_all[f:f + plan.trees(rank)]
    leaves, _, _, _ = oracle.ferret_pprf_sender(mine, h, delta)
    # rows [lo, hi) of the n-row LPN: the oracle computes the unsplit LPN on a
    # zero vector except this rank's rows, whose result rows are then taken
    lo, hi = plan.rows(rank)
    full = np.zeros((plan.n, 16), np.uint8)
    full[lo:hi] = leaves
    out = oracle.lpn_primal(seed.numpy(), kk.numpy(), full)[lo:hi]
    # all_gather needs equal sizes: pad every share to the largest
    mx = max(plan.trees(r) for r in range(world)) << h
    padded = torch.zeros((mx, 16), dtype=torch.uint8)
    padded[: out.shape[0]] = torch.from_numpy(np.ascontiguousarray(out))
    parts = [torch.zeros((mx, 16), dtype=torch.uint8) for _ in range(world)]
    dist.all_gather(parts, padded)
    if rank == 0:
        whole, _, _, _ = oracle.ferret_pprf_sender(roots_all, h, delta)
        exp = oracle.lpn_primal(seed.numpy(), kk.numpy(), whole)
        got = torch.cat([parts[r][: plan.trees(r) << h] for r in range(world)]).numpy()
        q.put(bool(np.array_equal(got, exp)))
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_split_equals_unsplit():
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_rank_main, args=(r, 2, port, 7, 6, 301, q)) for r in range(2)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=120)
    assert all(p.exitcode == 0 for p in procs)
    assert q.get(timeout=5) is True
