"""Serving loop host logic (cuot_b200/serve.py) with a fake executor: HBM
budget admission, FIFO order, queue timeouts, cancellation, rejection.  No
GPU: the fake executor's requests finish after a fixed wall time."""
import time

from cuot_b200.serve import KIND_FERRET, Request, Server, footprint, make_stream


class FakeExecutor:
    def __init__(self, slots, service_s=0.01, reserved=0):
        self.slots, self.service_s, self.reserved = slots, service_s, reserved
        self.started = {}
        self.log = []          # (event, rid, time)
        self.live_bytes = 0
        self.max_live_bytes = 0

    def reserved_bytes(self):
        return self.reserved

    def start(self, slot, r):
        self.started[slot] = (r, time.perf_counter())
        self.live_bytes += footprint(r)
        self.max_live_bytes = max(self.max_live_bytes, self.live_bytes)
        self.log.append(("start", r.rid))

    def poll(self, slot):
        return time.perf_counter() - self.started[slot][1] >= self.service_s

    def finish(self, slot):
        r, _ = self.started.pop(slot)
        self.live_bytes -= footprint(r)
        return r.rid


def req(rid, arrival, e=14):
    return Request(rid, KIND_FERRET, (1 << e) >> 10, 10, bytes(16), arrival, k=100)


def test_budget_limits_concurrency_and_order_is_fifo():
    reqs = [req(i, 0.0) for i in range(8)]
    fp = footprint(reqs[0])
    ex = FakeExecutor(slots=8)
    rep = Server(ex, budget_bytes=2.5 * fp).run(reqs)
    assert rep["done"] == 8
    assert ex.max_live_bytes <= 2.5 * fp          # never more than 2 admitted at once
    assert [rid for ev, rid in ex.log if ev == "start"] == list(range(8))
    assert all(r.result == r.rid for r in reqs)


def test_queue_timeout_cancel_and_reject():
    reqs = [req(i, 0.0) for i in range(6)]
    big = Request(99, KIND_FERRET, 1 << 20, 10, bytes(16), 0.0, k=10)
    ex = FakeExecutor(slots=1, service_s=0.05)
    srv = Server(ex, budget_bytes=10 * footprint(reqs[0]), max_queue_wait=0.12)
    srv.cancel(5)
    rep = srv.run(reqs + [big])
    assert big.status == "rejected"
    assert reqs[5].status == "cancelled"
    assert rep["timeout"] >= 1 and any(r.status == "timeout" for r in reqs)
    assert reqs[0].status == "done"
    assert rep["done"] + rep["timeout"] + rep["cancelled"] + rep["rejected"] == 7


def test_latency_includes_queueing():
    reqs = [req(i, 0.0) for i in range(4)]
    ex = FakeExecutor(slots=1, service_s=0.02)
    rep = Server(ex).run(reqs)
    lat = sorted(r.latency for r in reqs)
    assert lat[-1] >= 4 * 0.02 * 0.9 and rep["p99_ms"] >= rep["p50_ms"]


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
    ex = FakeExecutor(slots=4, service_s=0.03)
    rep = Server(ex, budget_bytes=1e12, big_n=1 << 16, max_big=1).run(big + small)
    assert rep["done"] == 5
    order = [rid for ev, rid in ex.log if ev == "start"]
    assert order[0] == 0 and order.index(1) > order.index(12)   # the second big waits for the first
    assert big[1].t_admit >= big[0].t_done - 1e-3
    assert all(s.t_admit < big[0].t_done for s in small)
