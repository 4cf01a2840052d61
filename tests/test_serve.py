"""Serving loop scheduling (cuot_server_* in libcuot through
cuot_b200/serve.py) in its host-only mode: HBM budget admission, FIFO
order, queue timeouts, cancellation, rejection, the big-request limit.  No
GPU: with dry_run_service_s every request takes that long and no device
work is done."""
import threading
import time

import numpy as np

import oracle
from cuot_b200.serve import KIND_FERRET, KIND_SOT, Request, Server, footprint, make_stream, request_scalars


def req(rid, arrival, e=14):
    return Request(rid, KIND_FERRET, (1 << e) >> 10, 10, bytes(16), arrival, k=100)


def admit_order(reqs):
    return [r.rid for r in sorted((r for r in reqs if r.t_admit == r.t_admit), key=lambda r: r.t_admit)]


def test_budget_limits_concurrency_and_order_is_fifo():
    reqs = [req(i, 0.0) for i in range(8)]
    fp = footprint(reqs[0])
    srv = Server(slots=8, budget_bytes=2.5 * fp, dry_run_service_s=0.01)
    rep = srv.run(reqs)
    assert rep["done"] == 8
    assert 0 < srv.max_used_bytes <= 2.5 * fp          # never more than 2 admitted at once
    assert admit_order(reqs) == list(range(8))
    # requests 2 and 3 wait for the first two
    assert reqs[2].t_admit >= min(reqs[0].t_done, reqs[1].t_done) - 1e-4


def test_queue_timeout_cancel_and_reject():
    reqs = [req(i, 0.0) for i in range(6)]
    big = Request(99, KIND_FERRET, 1 << 10, 10, bytes(16), 0.0, k=10)     # n = 2^20: above the budget
    bad = Request(98, KIND_SOT, 3, 10, bytes(16), 0.0)                    # SOT n not a power of two
    srv = Server(slots=1, budget_bytes=10 * footprint(reqs[0]), max_queue_wait=0.12, dry_run_service_s=0.05)
    srv.cancel(5)
    rep = srv.run(reqs + [big, bad])
    assert big.status == "rejected" and bad.status == "rejected"
    assert reqs[5].status == "cancelled"
    assert rep["timeout"] >= 1 and any(r.status == "timeout" for r in reqs)
    assert reqs[0].status == "done"
    assert rep["done"] + rep["timeout"] + rep["cancelled"] + rep["rejected"] == 8


def test_cancel_from_another_thread_during_run():
    reqs = [req(i, 0.0) for i in range(6)]
    srv = Server(slots=1, dry_run_service_s=0.05)
    th = threading.Timer(0.02, srv.cancel, args=(4,))
    th.start()
    srv.run(reqs)
    th.join()
    assert reqs[4].status == "cancelled"
    assert sum(r.status == "done" for r in reqs) == 5


def test_latency_includes_queueing():
    reqs = [req(i, 0.0) for i in range(4)]
    srv = Server(slots=1, dry_run_service_s=0.02)
    rep = srv.run(reqs)
    lat = sorted(r.latency for r in reqs)
    assert lat[-1] >= 4 * 0.02 * 0.9 and rep["p99_ms"] >= rep["p50_ms"]


def test_arrivals_are_respected():
    reqs = [req(0, 0.0), req(1, 0.08)]
    t0 = time.perf_counter()
    Server(slots=2, dry_run_service_s=0.01).run(reqs)
    assert reqs[1].t_admit >= 0.08 - 1e-3 and time.perf_counter() - t0 >= 0.09


def test_stream_shape():
    s = make_stream(200, rate=100.0, seed=3)
    assert all(14 <= (r.n.bit_length() - 1) <= 24 and 10 <= r.h <= 14 for r in s)
    assert sorted(r.arrival for r in s) == [r.arrival for r in s]
    assert 0.3 < sum(r.kind for r in s) / len(s) < 0.7


def test_big_request_limit_lets_small_ones_pass():
    """At most one request with n >= big_n runs at a time; small requests
    queued behind a waiting big one are admitted meanwhile."""
    big = [Request(i, KIND_FERRET, 1 << 6, 10, bytes(16), 0.0, k=10) for i in range(2)]     # n = 2^16
    small = [req(10 + i, 0.0) for i in range(3)]                                            # n = 2^14
    srv = Server(slots=4, budget_bytes=1e12, big_n=1 << 16, max_big=1, dry_run_service_s=0.03)
    rep = srv.run(big + small)
    assert rep["done"] == 5
    order = admit_order(big + small)
    assert order[0] == 0 and order.index(1) > order.index(12)   # the second big waits for the first
    assert big[1].t_admit >= big[0].t_done - 1e-3
    assert all(s.t_admit < big[0].t_done for s in small)


def test_request_scalars_are_prg_blocks():
    """delta, LPN seed and QC key = blocks 2^40 + {0, 1, 2} of the seed's
    PRNG stream (delta with its LSB set)."""
    seed = bytes(range(16))
    sc = request_scalars(seed)
    ref = oracle.prg(np.frombuffer(seed, np.uint8), 3, offset=1 << 40)
    ref[0, 0] |= 1
    assert np.array_equal(sc["delta"], ref[0]) and np.array_equal(sc["lpn_seed"], ref[1])
    assert np.array_equal(sc["akey"], ref[2])


def test_footprint_formula():
    r = req(0, 0.0, e=16)
    n, t, h = r.n, r.t, r.h
    assert footprint(r) == 2 * 16 * n + 16 * t + t * h + 2 * 16 * r.k + 4 * 16 * t * h + 16 * t
