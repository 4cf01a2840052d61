"""Splitting one Ferret extension over the GPUs of a node.

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
"""
from __future__ import annotations

from dataclasses import dataclass


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
    outputs."""
    import torch
    t, h = plan.trees(rank), plan.h
    n_r = t << h
    dev = roots.device
    emp = lambda m: torch.empty((m, 16), dtype=torch.uint8, device=dev)
    v, w = emp(n_r), emp(n_r)
    lsum, rsum, ss, mc = emp(t * h), emp(t * h), emp(t), emp(t * h)
    ctx.ferret_pprf_sender(roots, h, delta, v, lsum, rsum, ss, stream=stream)
    torch.where(choice.view(-1, 1).bool(), rsum, lsum, out=mc)
    ctx.ferret_pprf_recver(mc, choice, ss, h, w, stream=stream)
    lo, hi = plan.rows(rank)
    ctx.lpn_primal_range(seed, kk_s, v, lo, hi, plan.n, stream=stream)
    ctx.lpn_primal_range(seed, kk_r, w, lo, hi, plan.n, stream=stream)
    return v, w
