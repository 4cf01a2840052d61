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


# ---------------------------------------------------------------- SOT plane re-sharding
def _sot_rank_main(rank, world, port, t, h, q):
    from cuot_b200.shard import owners_to_rows, plane_range, planes_to_owners
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    plan = ShardPlan(t, h, world)
    n = plan.n
    g = np.random.default_rng(1234)
    rows_all = g.integers(0, 256, (n, 16), dtype=np.uint8)
    a = oracle.qc_gen_a(g.integers(0, 256, 16, dtype=np.uint8), n)
    lo, hi = plan.rows(rank)
    nr = hi - lo
    # this rank's rows -> 128 partial planes -> owners (all-to-all)
    local = oracle.bit_transpose(rows_all[lo:hi].copy(), nr, 16, 0, 128).reshape(128, nr // 8)
    mine = planes_to_owners(torch.from_numpy(np.ascontiguousarray(local)), plan, rank)
    p_lo, p_hi = plane_range(world, rank)
    P = p_hi - p_lo
    assert tuple(mine.shape) == (P, n // 8)
    # the owner holds exactly planes [p_lo, p_hi) of the whole vector
    whole = oracle.bit_transpose(rows_all, n, 16, 0, 128).reshape(128, n // 8)
    ok = bool(np.array_equal(mine.numpy(), whole[p_lo:p_hi]))
    enc = oracle.qc_encode(a, mine.numpy().view(np.uint64).reshape(P, n // 64).copy(), n)
    back = owners_to_rows(torch.from_numpy(np.ascontiguousarray(enc).view(np.uint8).reshape(P, n // 8)), plan, rank)
    out = oracle.bit_transpose(np.ascontiguousarray(back.numpy()), 128, nr // 8, 0, nr).reshape(nr, 16)
    # gather every rank's rows on rank 0 and compare with the unsplit encode
    mx = max(plan.rows(r)[1] - plan.rows(r)[0] for r in range(world))
    padded = torch.zeros((mx, 16), dtype=torch.uint8)
    padded[:nr] = torch.from_numpy(out)
    parts = [torch.zeros((mx, 16), dtype=torch.uint8) for _ in range(world)]
    dist.all_gather(parts, padded)
    oks = [torch.zeros(1, dtype=torch.uint8) for _ in range(world)]
    dist.all_gather(oks, torch.tensor([int(ok)], dtype=torch.uint8))
    if rank == 0:
        got = torch.cat([parts[r][: plan.rows(r)[1] - plan.rows(r)[0]] for r in range(world)]).numpy()
        exp = oracle.sot_dual_lpn(a, rows_all, n)
        q.put(bool(np.array_equal(got, exp)) and all(int(o) == 1 for o in oks))
    dist.barrier()
    dist.destroy_process_group()


@pytest.mark.parametrize("world,t,h", [(2, 4, 8), (3, 8, 7)])
def test_sot_plane_resharding_equals_unsplit(world, t, h):
    """Trees split over the ranks, one all-to-all to plane owners (uneven
    plane counts for 3 ranks), encode, reverse all-to-all: the ranks' rows
    concatenate to the unsplit dual-LPN output."""
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_sot_rank_main, args=(r, world, port, t, h, q)) for r in range(world)]
    for p in procs:
        p.start()
    for p in procs:
        p.join(timeout=180)
    assert all(p.exitcode == 0 for p in procs)
    assert q.get(timeout=5) is True


def test_sot_plane_ranges_cover_128():
    from cuot_b200.shard import plane_range
    for world in (1, 2, 3, 4, 8):
        rs = [plane_range(world, r) for r in range(world)]
        assert rs[0][0] == 0 and rs[-1][1] == 128
        assert all(rs[i][1] == rs[i + 1][0] for i in range(world - 1))
