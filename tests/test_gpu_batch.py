"""Batched engine: a mixed batch (Ferret-style and SOT instances of uneven n
and depth) run as one device program (CUDA graph) must give, for every
instance, exactly the single-instance path's outputs and the oracle's."""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

from cuot_b200 import CuotError  # noqa: E402
from cuot_b200.batch import (FORK_FERRET, FORK_SIZES, KIND_FERRET, KIND_SOT, SERIAL, Batch, Instance,  # noqa: E402
                             mixed_workload)


def oracle_outputs(inst):
    if inst.kind == KIND_FERRET:
        lv, ls, rs, ss = oracle.ferret_pprf_sender(inst.roots, inst.h, inst.delta, threads=8)
        mc = np.where(inst.choice[:, None] == 0, ls, rs)
        rl = oracle.ferret_pprf_recver(mc, inst.choice, ss, inst.h, threads=8)
        return (oracle.lpn_primal(inst.seed, inst.kk_s, lv, d=inst.d, threads=8),
                oracle.lpn_primal(inst.seed, inst.kk_r, rl, d=inst.d, threads=8), None)
    lv, m0, m1 = oracle.sot_pprf_sender(inst.roots, inst.h, inst.delta, inst.base0, inst.base1, threads=8)
    rl = oracle.sot_pprf_recver(m0, m1, inst.mc, inst.choice, inst.t, inst.h, threads=8)
    a = inst.a.cpu().numpy().view(np.uint64)
    return (oracle.sot_dual_lpn(a, lv, inst.n, threads=8), oracle.sot_dual_lpn(a, rl, inst.n, threads=8),
            oracle.qc_encode_sparse(a, inst.punct.astype(np.uint64), inst.n))


def snapshot(insts):
    torch.cuda.synchronize()
    return [(i.v.cpu().numpy().copy(), i.w.cpu().numpy().copy(),
             None if i.kind == KIND_FERRET else i.cbits.cpu().numpy().view(np.uint64).copy()) for i in insts]


@pytest.mark.parametrize("schedule", [SERIAL, FORK_FERRET, FORK_SIZES])
def test_mixed_batch_equals_plain_and_oracle(ctx, schedule):
    """Every schedule of the batched program (one chain; the Ferret branch
    beside the SOT chain; every SOT size on its own stream) gives the same
    outputs."""
    specs = [(KIND_FERRET, 8, 10, 1000), (KIND_SOT, 4, 10, 0), (KIND_FERRET, 3, 12, 77), (KIND_SOT, 16, 10, 0),
             (KIND_FERRET, 64, 10, 8192), (KIND_SOT, 2, 11, 0), (KIND_FERRET, 5, 1, 9), (KIND_SOT, 1, 12, 0)]
    insts = [Instance(ctx, kd, t, h, 100 + i, k=k) for i, (kd, t, h, k) in enumerate(specs)]
    stream = torch.cuda.Stream()
    b = Batch(ctx, insts, use_graph=True, schedule=schedule)
    b.run(stream)        # captures the graph and runs it
    b.run(stream)        # replays: a second run must give the same outputs
    got = snapshot(insts)
    assert b.kernels_per_run() > 0
    for inst in insts:   # clobber the outputs before the plain run
        inst.v.zero_(); inst.w.zero_()
    b.run_plain(stream)
    plain = snapshot(insts)
    for inst, g, p in zip(insts, got, plain):
        ev, ew, ec = oracle_outputs(inst)
        assert np.array_equal(g[0], ev) and np.array_equal(g[1], ew)
        assert np.array_equal(p[0], ev) and np.array_equal(p[1], ew)
        if ec is not None:
            assert np.array_equal(g[2], ec) and np.array_equal(p[2], ec)
    b.close()


def test_configs3_shaped_mix_is_a_cot_everywhere(ctx):
    """A smaller mix shaped like the 64-instance batch (log2 n in [12, 16]); every instance's
    outputs satisfy the COT correlation against its own delta."""
    insts = mixed_workload(ctx, count=10, seed=7, lo=12, hi=16)
    stream = torch.cuda.Stream()
    b = Batch(ctx, insts, use_graph=True)
    b.run(stream)
    torch.cuda.synchronize()
    for inst in insts:
        v, w = inst.v.cpu().numpy(), inst.w.cpu().numpy()
        ev, ew, ec = oracle_outputs(inst)
        assert np.array_equal(v, ev) and np.array_equal(w, ew)
    b.close()


def test_large_sot_batch_equals_plain_and_is_a_cot(ctx):
    """SOT instances at n = 2^21 and 2^22 (the direct FFT: 512 x 4096, and
    1024 x 4096 with centred planes against the lighter of a and ~a in
    4-column CTAs) beside a small Ferret instance: the graph-captured batched
    program gives the plain path's outputs (the one-shot entry points, checked
    against the oracle by the QC tests), and each SOT instance's outputs form
    a COT, w_j = v_j ^ c_j * delta."""
    specs = [(KIND_SOT, 512, 12, 0), (KIND_SOT, 1024, 12, 0), (KIND_FERRET, 8, 10, 1000)]
    insts = [Instance(ctx, kd, t, h, 300 + i, k=k) for i, (kd, t, h, k) in enumerate(specs)]
    stream = torch.cuda.Stream()
    b = Batch(ctx, insts, use_graph=True)
    b.run(stream)
    got = snapshot(insts)
    for inst in insts:
        inst.v.zero_(); inst.w.zero_()
    b.run_plain(stream)
    plain = snapshot(insts)
    for inst, g, p in zip(insts, got, plain):
        assert np.array_equal(g[0], p[0]) and np.array_equal(g[1], p[1])
        if inst.kind == KIND_SOT:
            assert np.array_equal(g[2], p[2])
            cbits = np.unpackbits(g[2].view(np.uint8), bitorder="little").astype(bool)
            diff = g[0] ^ g[1]
            assert not diff[~cbits].any()
            assert (diff[cbits] == inst.delta).all()
            assert 0.4 < cbits.mean() < 0.6
    b.close()


def test_unknown_schedule_is_rejected(ctx):
    insts = [Instance(ctx, KIND_FERRET, 4, 8, 500, k=300), Instance(ctx, KIND_SOT, 2, 10, 501)]
    for bad in (-1, 3):
        with pytest.raises(CuotError):
            Batch(ctx, insts, use_graph=True, schedule=bad)
    b = Batch(ctx, insts, use_graph=True, schedule=SERIAL)  # the context stays usable
    b.run(torch.cuda.Stream())
    torch.cuda.synchronize()
    for inst in insts:
        ev, ew, _ = oracle_outputs(inst)
        assert np.array_equal(inst.v.cpu().numpy(), ev) and np.array_equal(inst.w.cpu().numpy(), ew)
    b.close()


@pytest.mark.parametrize("use_graph,schedule", [(True, SERIAL), (False, SERIAL), (True, FORK_FERRET),
                                                (True, FORK_SIZES), (False, FORK_SIZES)])
def test_item_completion_points(ctx, use_graph, schedule):
    """cuot_batch_wait_item: a copy stream that waits for each instance's
    completion point (rank order: Ferret after the LPN, then the SOT sizes
    largest first) and copies its outputs right away gets the final outputs,
    though the run has not ended when the first copies start.  The outputs
    are zeroed on the compute stream before the run, so a copy that ran early
    would see zeros or a partial result.  The forked schedules record the
    points on their own streams (inside the graph when captured)."""
    specs = [(KIND_SOT, 16, 10, 0), (KIND_FERRET, 8, 10, 1000), (KIND_SOT, 64, 10, 0), (KIND_FERRET, 3, 12, 77),
             (KIND_SOT, 4, 10, 0), (KIND_SOT, 2, 12, 0)]
    insts = [Instance(ctx, kd, t, h, 700 + i, k=k) for i, (kd, t, h, k) in enumerate(specs)]
    b = Batch(ctx, insts, use_graph=use_graph, schedule=schedule)
    ranks = [b.item_rank(i) for i in range(len(insts))]
    assert ranks == [2, 0, 1, 0, 4, 3]  # 2^14, Ferret, 2^16, Ferret, 2^12, 2^13
    with pytest.raises(IndexError):
        b.item_rank(len(insts))
    stream, cs = torch.cuda.Stream(), torch.cuda.Stream()
    expect = [oracle_outputs(inst) for inst in insts]
    for rep in range(2):
        with torch.cuda.stream(stream):
            for inst in insts:
                inst.v.zero_(); inst.w.zero_()
                if inst.kind != KIND_FERRET:
                    inst.cbits.zero_()
        b.run(stream)
        host = {}
        with torch.cuda.stream(cs):
            for ix in sorted(range(len(insts)), key=lambda j: ranks[j]):
                b.wait_item(ix, cs)
                inst = insts[ix]
                outs = [inst.v, inst.w] + ([] if inst.kind == KIND_FERRET else [inst.cbits])
                host[ix] = [torch.empty_like(o, device="cpu").pin_memory() for o in outs]
                for h, o in zip(host[ix], outs):
                    h.copy_(o, non_blocking=True)
        cs.synchronize()
        for ix, (ev, ew, ec) in enumerate(expect):
            assert np.array_equal(host[ix][0].numpy(), ev) and np.array_equal(host[ix][1].numpy(), ew), (rep, ix)
            if ec is not None:
                assert np.array_equal(host[ix][2].numpy().view(np.uint64), ec), (rep, ix)
        torch.cuda.synchronize()
    b.close()
