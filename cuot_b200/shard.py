"""Splitting one OT extension over the GPUs of a node.

Ferret
------

One process per GPU (torch.distributed).  Trees are split as FerretCOT's
gpu_task_division (ferret_cot.hpp:55-63: t / G trees each, the first t % G
ranks one more); each rank expands its own trees and computes the LPN rows of
its own leaves, so rank g holds rows [sum of earlier ranks' rows, + its own).
The LPN of those rows is bit-identical to the unsplit computation
(cuot_lpn_primal_range).  The only collectives are set-up broadcasts of the
LPN seed and of kk (k blocks, replicated on every GPU as the reference copies
kk to every GPU, dev_layer.cu:174); there is no data-path exchange.
The per-level sums and secret sums of each rank go to the host, as in the
reference (dev_layer.cu:40-41,50).

SOT
---
The GGM trees split the same way, but the quasi-cyclic encode works on whole
bit planes (n bits each), so the one real exchange of the path sits between
the two: every rank transposes its own rows into 128 partial planes, one
all-to-all moves the planes to their owners (rank g owns planes
[128g/G, 128(g+1)/G)), each owner encodes its planes over all n bits, and the
reverse all-to-all returns every rank the encoded bits of its own rows.  Each
rank sends (G-1)/G of its 16 n/G bytes each way.  The reference avoids the
exchange by re-expanding every tree on every GPU (silent/sender.cu:113-115).
The exchange functions are plain torch.distributed collectives on tensors
of the process group's device (NCCL on GPUs, gloo on CPU).
"""
from __future__ import annotations

from contextlib import contextmanager
from dataclasses import dataclass


@contextmanager
def _on_stream(stream, device):
    """Runs the body with `stream` (default: the current stream) as torch's
    current stream, after it has waited for the work already queued on the
    caller's current stream (which produced the inputs).  Everything in a
    shard function -- the library calls, torch's own kernels and NCCL's
    collectives, which order themselves after the current stream -- then
    runs in one order on one stream.  Yields None for CPU tensors."""
    import torch
    if device.type != "cuda":
        yield None
        return
    cur = torch.cuda.current_stream(device)
    s = cur if stream is None else stream
    if s != cur:
        s.wait_stream(cur)
    with torch.cuda.stream(s):
        yield s


@dataclass(frozen=True)
class ShardPlan:
    t: int           # trees in the whole instance
    h: int           # tree depth
    world: int       # ranks (GPUs)

    def trees(self, rank: int) -> int:
        """Trees of `rank` (ferret_cot.hpp:58-60)."""
        return self.t // self.world + (1 if rank < self.t % self.world else 0)

    def first_tree(self, rank: int) -> int:
        return sum(self.trees(r) for r in range(rank))

    def rows(self, rank: int) -> tuple[int, int]:
        """[row_lo, row_hi) of the n = t * 2^h LPN rows held by `rank`."""
        lo = self.first_tree(rank) << self.h
        return lo, lo + (self.trees(rank) << self.h)

    @property
    def n(self) -> int:
        return self.t << self.h


def broadcast_setup(seed, kk, src: int = 0):
    """Broadcasts the LPN seed (16 bytes) and kk (k x 16 bytes) from `src` to
    every rank, in place (tensors of the process group's device)."""
    import torch.distributed as dist
    dist.broadcast(seed, src)
    dist.broadcast(kk, src)


def ferret_extend_rank(ctx, plan: ShardPlan, rank: int, roots, delta, choice, seed, kk_s, kk_r, stream=None):
    """Both roles of this rank's share of one Ferret extension on its GPU:
    sender MPCOT -> (ideal OT of the sums) -> receiver MPCOT -> LPN of this
    rank's rows on both roles (kk_s / kk_r: the two roles' LPN inputs).
    Returns (v, w): this rank's rows of the sender's and the receiver's
    outputs, written in order on `stream` (default: the current stream)."""
    import torch
    t, h = plan.trees(rank), plan.h
    n_r = t << h
    dev = roots.device
    with _on_stream(stream, dev) as s:
        emp = lambda m: torch.empty((m, 16), dtype=torch.uint8, device=dev)
        v, w = emp(n_r), emp(n_r)
        lsum, rsum, ss, mc = emp(t * h), emp(t * h), emp(t), emp(t * h)
        ctx.ferret_pprf_sender(roots, h, delta, v, lsum, rsum, ss, stream=s)
        torch.where(choice.view(-1, 1).bool(), rsum, lsum, out=mc)
        ctx.ferret_pprf_recver(mc, choice, ss, h, w, stream=s)
        lo, hi = plan.rows(rank)
        ctx.lpn_primal_range(seed, kk_s, v, lo, hi, plan.n, stream=s)
        ctx.lpn_primal_range(seed, kk_r, w, lo, hi, plan.n, stream=s)
    return v, w


# ---------------------------------------------------------------------------
# SOT: plane ownership


def plane_range(world: int, rank: int) -> tuple[int, int]:
    """[lo, hi) of the 128 bit planes owned by `rank`."""
    return 128 * rank // world, 128 * (rank + 1) // world


def _check_rows(plan: ShardPlan):
    for r in range(plan.world):
        lo, hi = plan.rows(r)
        if lo % 64 or hi % 64:
            raise ValueError("SOT sharding needs every rank's row range on a 64-row boundary (depth >= 6)")


def planes_to_owners(local, plan: ShardPlan, rank: int):
    """local: uint8 (128, rows_r / 8), the 128 bit planes of this rank's rows
    [plan.rows(rank)).  Returns uint8 (P, n / 8): the P planes this rank owns,
    over all n rows, assembled from every rank's share (one all-to-all)."""
    import torch
    import torch.distributed as dist
    _check_rows(plan)
    world, n = plan.world, plan.n
    lo_r, hi_r = plan.rows(rank)
    nb = (hi_r - lo_r) // 8
    if tuple(local.shape) != (128, nb):
        raise ValueError(f"expected planes of shape (128, {nb}), got {tuple(local.shape)}")
    p_lo, p_hi = plane_range(world, rank)
    P = p_hi - p_lo
    ins = [(plane_range(world, j)[1] - plane_range(world, j)[0]) * nb for j in range(world)]
    outs = [P * (plan.rows(i)[1] - plan.rows(i)[0]) // 8 for i in range(world)]
    recv = torch.empty(sum(outs), dtype=torch.uint8, device=local.device)
    dist.all_to_all_single(recv, local.contiguous().view(-1), outs, ins)
    mine = torch.empty((P, n // 8), dtype=torch.uint8, device=local.device)
    off = 0
    for i in range(world):
        lo, hi = plan.rows(i)
        mine[:, lo // 8:hi // 8] = recv[off:off + outs[i]].view(P, (hi - lo) // 8)
        off += outs[i]
    return mine


def owners_to_rows(mine, plan: ShardPlan, rank: int):
    """Inverse of planes_to_owners: mine is uint8 (P, n / 8), this rank's
    (encoded) planes; returns uint8 (128, rows_r / 8), all planes of this
    rank's rows (the reverse all-to-all)."""
    import torch
    import torch.distributed as dist
    world = plan.world
    p_lo, p_hi = plane_range(world, rank)
    P = p_hi - p_lo
    lo_r, hi_r = plan.rows(rank)
    nb = (hi_r - lo_r) // 8
    send = torch.cat([mine[:, plan.rows(i)[0] // 8:plan.rows(i)[1] // 8].reshape(-1) for i in range(world)])
    ins = [P * (plan.rows(i)[1] - plan.rows(i)[0]) // 8 for i in range(world)]
    outs = [(plane_range(world, j)[1] - plane_range(world, j)[0]) * nb for j in range(world)]
    recv = torch.empty(sum(outs), dtype=torch.uint8, device=mine.device)
    dist.all_to_all_single(recv, send, outs, ins)
    return recv.view(128, nb)


def sot_dual_lpn_rank(ctx, plan: ShardPlan, rank: int, a, rows, stream=None):
    """Rate-1 dual LPN of one SOT instance split over the ranks: `rows` holds
    this rank's noise blocks (rows_r x 16 bytes, the expansion of its own
    trees); returns its rows of out = a * e mod (x^n - 1) per bit plane,
    bit-identical to the unsplit cuot_sot_dual_lpn, written in order on
    `stream` (default: the current stream; the all-to-alls wait for it)."""
    import torch
    lo, hi = plan.rows(rank)
    nr = hi - lo
    dev = rows.device
    with _on_stream(stream, dev) as s:
        local = torch.empty((128, nr // 8), dtype=torch.uint8, device=dev)
        ctx.bit_transpose(rows, nr, 16, 0, 128, local, stream=s)
        mine = planes_to_owners(local, plan, rank)
        p_lo, p_hi = plane_range(plan.world, rank)
        if p_hi > p_lo:
            ctx.qc_encode(a, mine.view(torch.int64), plan.n, p_hi - p_lo, stream=s)
        back = owners_to_rows(mine, plan, rank)
        out = torch.empty((nr, 16), dtype=torch.uint8, device=dev)
        ctx.bit_transpose(back, 128, nr // 8, 0, nr, out, stream=s)
    return out
