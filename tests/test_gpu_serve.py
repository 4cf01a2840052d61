"""Serving on the GPU: requests run concurrently (continuous batching over
several slots) give exactly the results they give alone (one slot), and
those results are the oracle's."""
import numpy as np
import pytest

import oracle

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

from cuot_b200.serve import KIND_FERRET, Server, make_stream, request_scalars  # noqa: E402


def oracle_result(r):
    t, h, n = r.t, r.h, r.n
    sc = request_scalars(r.seed)
    off = 0

    def take(m):
        nonlocal off
        x = oracle.prg(np.frombuffer(r.seed, np.uint8), m, offset=off)
        off += m
        return x
    roots = take(t)
    choice = (take((t * h + 15) // 16).reshape(-1)[: t * h] & 1).astype(np.uint8)
    if r.kind == KIND_FERRET:
        kk_s, kk_r = take(r.k), take(r.k)
        lv, ls, rs, ss = oracle.ferret_pprf_sender(roots, h, sc["delta"], threads=8)
        mc = np.where(choice[:, None] == 0, ls, rs)
        rl = oracle.ferret_pprf_recver(mc, choice, ss, h, threads=8)
        return (oracle.lpn_primal(sc["lpn_seed"], kk_s, lv, threads=8),
                oracle.lpn_primal(sc["lpn_seed"], kk_r, rl, threads=8), None)
    b0, b1 = take(h * t), take(h * t)
    mc = np.where(choice[:, None] == 0, b0, b1)
    lv, m0, m1 = oracle.sot_pprf_sender(roots, h, sc["delta"], b0, b1, threads=8)
    rl = oracle.sot_pprf_recver(m0, m1, mc, choice, t, h, threads=8)
    a = oracle.qc_gen_a(sc["akey"], n)
    chm = choice.reshape(h, t)
    pos = np.zeros(t, np.int64)
    for d in range(h):
        pos = pos * 2 + 1 - chm[d].astype(np.int64)
    pos += np.arange(t) * (1 << h)
    return (oracle.sot_dual_lpn(a, lv, n, threads=8), oracle.sot_dual_lpn(a, rl, n, threads=8),
            oracle.qc_encode_sparse(a, pos.astype(np.uint64), n))


def test_results_same_alone_and_in_the_mix():
    reqs = make_stream(14, rate=0.0, seed=11, lo=11, hi=15)
    mix = Server(slots=4, max_log_n=15, keep_outputs=True, budget_bytes=8e9, high_priority_below_n=1 << 13)
    rep = mix.run(reqs)
    mix.close()
    assert rep["done"] == len(reqs)
    in_mix = [r.result for r in reqs]
    alone = Server(slots=1, max_log_n=15, keep_outputs=True, budget_bytes=8e9)
    alone.run(reqs)
    alone.close()
    for r, m in zip(reqs, in_mix):
        a = r.result
        assert np.array_equal(a[0], m[0]) and np.array_equal(a[1], m[1])
        if a[2] is not None:
            assert np.array_equal(a[2], m[2])
    for r in (reqs[0], reqs[1], reqs[-1]):
        ev, ew, ec = oracle_result(r)
        assert np.array_equal(r.result[0], ev) and np.array_equal(r.result[1], ew)
        if ec is not None:
            assert np.array_equal(r.result[2].view(np.uint64), ec)


def test_both_kinds_checked_and_big_limit_on_device():
    """One Ferret and one SOT request against the oracle, served with the
    big-request limit on and arrivals spread out."""
    reqs = make_stream(12, rate=400.0, seed=21, lo=11, hi=14)
    kinds = {r.kind for r in reqs}
    assert kinds == {0, 1}
    srv = Server(slots=3, max_log_n=14, keep_outputs=True, budget_bytes=8e9, big_n=1 << 13, max_big=1)
    rep = srv.run(reqs)
    srv.close()
    assert rep["done"] == len(reqs)
    for kind in (0, 1):
        r = next(x for x in reqs if x.kind == kind)
        ev, ew, ec = oracle_result(r)
        assert np.array_equal(r.result[0], ev) and np.array_equal(r.result[1], ew)
        if ec is not None:
            assert np.array_equal(r.result[2].view(np.uint64), ec)
