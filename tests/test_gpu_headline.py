"""The headline configuration itself, instance by instance.

The batched mix that bench.py times by default (64 instances, half SOT and
half Ferret-style, log2 n uniform over [16, 22], depth 10-14, seed 2024:
`mixed_workload(ctx)`), run as one CUDA-graph program with the batch
configuration bench.py's autotuner picks on B200 and with the defaults, and
through the plain path.  Every instance is checked against the oracle:
  * Ferret-style: both roles' LPN outputs in full (GGM sender + receiver +
    primal LPN, which the oracle restates from emp-ot and the emp-ot pin
    tests tie to the reference's own code);
  * SOT: the receiver's choice bits in full (encode_sparse), the COT
    correlation w_j = v_j ^ c_j * delta on every block, and the dual-LPN
    planes in full for n <= 2^19 and on a seeded sample of 8 planes per role
    above (the oracle's exact GF(2) product takes about a second per plane
    at 2^22).
"""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

from cuot_b200.batch import KIND_FERRET, Batch, mixed_workload  # noqa: E402

THREADS = 8


def planes_of(blocks: np.ndarray, idx) -> np.ndarray:
    """Bit planes `idx` of n 16-byte blocks as (len(idx), n/64) uint64 words
    (bit j of plane r = bit r of block j, LSB-first)."""
    out = []
    for r in idx:
        bits = (blocks[:, r // 8] >> (r % 8)) & 1
        out.append(np.packbits(bits, bitorder="little").view(np.uint64))
    return np.stack(out)


def check_ferret(inst, v, w):
    lv, ls, rs, ss = oracle.ferret_pprf_sender(inst.roots, inst.h, inst.delta, threads=THREADS)
    mc = np.where(inst.choice[:, None] == 0, ls, rs)
    rl = oracle.ferret_pprf_recver(mc, inst.choice, ss, inst.h, threads=THREADS)
    assert np.array_equal(v, oracle.lpn_primal(inst.seed, inst.kk_s, lv, d=inst.d, threads=THREADS))
    assert np.array_equal(w, oracle.lpn_primal(inst.seed, inst.kk_r, rl, d=inst.d, threads=THREADS))


def check_sot(inst, v, w, cbits, sample_seed):
    n = inst.n
    a = inst.a.cpu().numpy().view(np.uint64)
    assert np.array_equal(cbits, oracle.qc_encode_sparse(a, inst.punct.astype(np.uint64), n))
    c = np.unpackbits(cbits.view(np.uint8), bitorder="little").astype(bool)
    diff = v ^ w
    assert not diff[~c].any()
    assert (diff[c] == inst.delta).all()
    lv, m0, m1 = oracle.sot_pprf_sender(inst.roots, inst.h, inst.delta, inst.base0, inst.base1, threads=THREADS)
    rl = oracle.sot_pprf_recver(m0, m1, inst.mc, inst.choice, inst.t, inst.h, threads=THREADS)
    if n <= 1 << 19:
        assert np.array_equal(v, oracle.sot_dual_lpn(a, lv, n, threads=THREADS))
        assert np.array_equal(w, oracle.sot_dual_lpn(a, rl, n, threads=THREADS))
        return
    idx = sorted(np.random.default_rng(sample_seed).choice(128, 8, replace=False).tolist())
    for leaves, out in ((lv, v), (rl, w)):
        exp = oracle.qc_encode(a, planes_of(leaves, idx), n, threads=THREADS)
        assert np.array_equal(planes_of(out, idx), exp), idx


def snapshot(insts):
    torch.cuda.synchronize()
    return [(i.v.cpu().numpy().copy(), i.w.cpu().numpy().copy(),
             None if i.kind == KIND_FERRET else i.cbits.cpu().numpy().view(np.uint64).copy()) for i in insts]


def test_mixed64_every_instance(ctx):
    insts = mixed_workload(ctx)
    assert len(insts) == 64 and sum(i.kind != KIND_FERRET for i in insts) == 32
    stream = torch.cuda.Stream()
    tuned = Batch(ctx, insts, pprf_threads=128, ctas_per_sm=3, lpn_rows_per_task=16384, use_graph=True)
    tuned.run(stream)
    tuned.run(stream)  # a replay of the captured graph
    got = snapshot(insts)
    tuned.close()
    for inst in insts:
        inst.v.zero_(); inst.w.zero_()
    dflt = Batch(ctx, insts, use_graph=True)
    dflt.run(stream)
    assert all(np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1]) for a, b in zip(got, snapshot(insts)))
    for inst in insts:
        inst.v.zero_(); inst.w.zero_()
    dflt.run_plain(stream)
    assert all(np.array_equal(a[0], b[0]) and np.array_equal(a[1], b[1]) for a, b in zip(got, snapshot(insts)))
    dflt.close()
    for i, (inst, (v, w, cb)) in enumerate(zip(insts, got)):
        if inst.kind == KIND_FERRET:
            check_ferret(inst, v, w)
        else:
            check_sot(inst, v, w, cb, sample_seed=i)
