"""Serving loop: continuous batching of OT-extension session requests.

Each request is one OT extension (Ferret-style or SOT) with both roles.  The
server keeps `slots` executors busy (one CUDA stream and one libcuot context
each); a request that arrives while others run is admitted as soon as a slot
is free and its device footprint fits the HBM budget, so requests overlap on
the GPU.  A request's inputs are derived on the device from its seed (the
cryptoTools PRNG stream, cuot_prg_fill) and its state (roots, delta, trees,
level sums, outputs) stays resident on the device across the PPRF -> LPN /
quasi-cyclic encode -> transpose stages; nothing returns to the host between
stages.  Latency = completion (outputs in device memory, observed by the
loop) - arrival.

Scheduling: requests are admitted in arrival order; optionally at most
`max_big` requests with n >= `big_n` run at once (one such request already
fills the GPU, two only time-slice it and both finish late) while smaller
requests may pass a big one that waits for that reason.  The executor can
launch small requests on a higher-priority stream so their blocks are
scheduled ahead of a running big request's.

Host-side failure handling: a request waiting in the queue longer than
`max_queue_wait` seconds times out; a request can be cancelled while
queued; a request whose footprint can never fit the budget is rejected.  No
device-side waits are involved (completion is polled with event queries).
"""
from __future__ import annotations

import collections
import hashlib
import math
import time
from dataclasses import dataclass, field

import numpy as np

KIND_FERRET, KIND_SOT = 0, 1
K_RATIO = 452000 / 10485760  # ferret_b13's k / n


@dataclass
class Request:
    rid: int
    kind: int
    t: int
    h: int
    seed: bytes
    arrival: float                      # seconds from the start of the stream
    k: int = 0
    status: str = "pending"             # queued, running, done, timeout, cancelled, rejected
    t_admit: float = math.nan
    t_done: float = math.nan
    result: object = field(default=None, repr=False)

    @property
    def n(self) -> int:
        return self.t << self.h

    @property
    def latency(self) -> float:
        return self.t_done - self.arrival


def request_scalars(seed: bytes) -> dict:
    """Per-request values passed by value (derived on the host so starting a
    request never reads device memory): delta (LSB set, as Ferret's Delta,
    ferret_cot.hpp:29-31), the LPN seed and the key of the QC polynomial."""
    d = lambda tag: np.frombuffer(hashlib.sha256(seed + tag).digest()[:16], np.uint8).copy()
    delta = d(b"delta")
    delta[0] |= 1
    return {"delta": delta, "lpn_seed": d(b"lpn"), "akey": d(b"a")}


def footprint(req: Request) -> int:
    """Device bytes one request holds while admitted (its inputs, both roles'
    outputs and per-request intermediates); the per-slot scratch arenas are
    accounted separately by the executor."""
    n, t, h = req.n, req.t, req.h
    b = 2 * 16 * n + 16 * t + t * h          # v, w, roots, choices
    if req.kind == KIND_FERRET:
        b += 2 * 16 * req.k + 4 * 16 * t * h + 16 * t
    else:
        b += 3 * 16 * h * t + 2 * 16 * (h + 1) * t + n // 8 + n // 8 + 8 * t
    return b


def make_stream(count: int, rate: float, seed: int = 1, lo: int = 14, hi: int = 24,
                sot_fraction: float = 0.5) -> list[Request]:
    """Poisson arrivals at `rate` requests/s, log2 n uniform over [lo, hi],
    depth 10-14 (t = n / 2^h), kind SOT with probability sot_fraction."""
    rng = np.random.default_rng(seed)
    t_arr = np.cumsum(rng.exponential(1.0 / rate, count)) if rate > 0 else np.zeros(count)
    out = []
    for i in range(count):
        e = int(rng.integers(lo, hi + 1))
        h = int(rng.integers(10, min(14, e) + 1))
        kind = KIND_SOT if rng.random() < sot_fraction else KIND_FERRET
        k = math.ceil((1 << e) * K_RATIO) if kind == KIND_FERRET else 0
        out.append(Request(i, kind, (1 << e) >> h, h, rng.bytes(16), float(t_arr[i]), k=k))
    return out


class Server:
    """Continuous-batching loop over an executor (GpuExecutor, or a fake with
    the same interface for host-only tests)."""

    def __init__(self, executor, budget_bytes: float = 120e9, max_queue_wait: float | None = None,
                 poll_s: float = 20e-6, big_n: int | None = None, max_big: int = 1):
        self.ex = executor
        self.budget = float(budget_bytes) - float(executor.reserved_bytes())
        self.max_queue_wait = max_queue_wait
        self.poll_s = poll_s
        self.big_n, self.max_big = big_n, max_big
        self.cancelled: set[int] = set()

    def _is_big(self, r: Request) -> bool:
        return self.big_n is not None and r.n >= self.big_n

    def cancel(self, rid: int):
        self.cancelled.add(rid)

    def run(self, requests: list[Request], clock=time.perf_counter) -> dict:
        pending = sorted(requests, key=lambda r: r.arrival)
        queue: collections.deque[Request] = collections.deque()
        free_slots = list(range(self.ex.slots))
        busy: dict[int, Request] = {}
        used = 0.0
        i = 0
        t0 = clock()
        while i < len(pending) or queue or busy:
            now = clock() - t0
            while i < len(pending) and pending[i].arrival <= now:
                r = pending[i]
                i += 1
                if footprint(r) > self.budget:
                    r.status = "rejected"
                    continue
                r.status = "queued"
                queue.append(r)
            # completions
            for s in list(busy):
                if self.ex.poll(s):
                    r = busy.pop(s)
                    r.result = self.ex.finish(s)
                    r.t_done = clock() - t0
                    r.status = "done"
                    used -= footprint(r)
                    free_slots.append(s)
            # cancellations and queue timeouts (host side)
            if self.cancelled or self.max_queue_wait is not None:
                keep = collections.deque()
                for r in queue:
                    if r.rid in self.cancelled:
                        r.status = "cancelled"
                    elif self.max_queue_wait is not None and now - r.arrival > self.max_queue_wait:
                        r.status = "timeout"
                    else:
                        keep.append(r)
                queue = keep
            # admission in arrival order, as slots and memory free up; memory
            # is head-of-line (no request passes one that does not fit), the
            # big-request limit is not
            while queue and free_slots:
                nbig = sum(self._is_big(b) for b in busy.values())
                pick = None
                for j, r in enumerate(queue):
                    if used + footprint(r) > self.budget:
                        break
                    if self._is_big(r) and nbig >= self.max_big:
                        continue
                    pick = j
                    break
                if pick is None:
                    break
                r = queue[pick]
                del queue[pick]
                s = free_slots.pop()
                used += footprint(r)
                r.t_admit = clock() - t0
                r.status = "running"
                busy[s] = r
                self.ex.start(s, r)
            if not busy and not queue and i < len(pending):
                wait = pending[i].arrival - (clock() - t0)
                if wait > 0:
                    time.sleep(min(wait, 0.01))
            elif busy:
                time.sleep(self.poll_s)
        wall = clock() - t0
        done = [r for r in requests if r.status == "done"]
        lat = np.array([r.latency for r in done]) if done else np.array([math.nan])
        cots = sum(r.n for r in done)
        return {"requests": len(requests), "done": len(done),
                "timeout": sum(r.status == "timeout" for r in requests),
                "cancelled": sum(r.status == "cancelled" for r in requests),
                "rejected": sum(r.status == "rejected" for r in requests),
                "wall_s": wall, "cots": cots, "cots_per_s": cots / wall if wall > 0 else math.nan,
                "p50_ms": float(np.percentile(lat, 50) * 1e3), "p99_ms": float(np.percentile(lat, 99) * 1e3),
                "mean_ms": float(lat.mean() * 1e3)}


class GpuExecutor:
    """`slots` CUDA streams, each with its own libcuot context; one request
    per slot at a time.  Inputs come from the request seed's PRNG stream on
    the device (block layout in `_inputs`)."""

    def __init__(self, slots: int = 8, device: int = 0, max_log_n: int = 24, keep_outputs: bool = False,
                 high_priority_below_n: int | None = None):
        import torch
        import cuot_b200
        self.torch, self.cb = torch, cuot_b200
        self.slots = slots
        self.keep_outputs = keep_outputs
        self.high_below = high_priority_below_n
        torch.cuda.set_device(device)
        self.ctxs = [cuot_b200.Context(device) for _ in range(slots)]
        self.streams = [torch.cuda.Stream() for _ in range(slots)]
        # requests with n < high_below run on a higher-priority stream of their slot
        self.streams_hi = [torch.cuda.Stream(priority=-1) for _ in range(slots)] if self.high_below else None
        self.events = [None] * slots
        self.state = [None] * slots
        nmax = 1 << max_log_n
        # per-slot scratch: PPRF levels (16n) or dual LPN (8n ahat + 16n planes
        # + the NTT batch: up to 512 MiB, at least 4n), plus the QC twiddle
        # tables of every size
        self.scratch_per_slot = 24 * nmax + max(4 * nmax, 512 << 20) + (64 << 20)
        self.tables_per_slot = sum(16 * (1 << e) + 32 * (1 << (e // 2 + 1)) for e in range(10, max_log_n + 1))
        for c in self.ctxs:
            c.reserve(self.scratch_per_slot)
        # build the QC tables of every size once (the first use of a size synchronises)
        for e in range(10, max_log_n + 1):
            n = 1 << e
            a = torch.zeros(n // 64, dtype=torch.int64, device="cuda")
            p = torch.zeros(n // 64, dtype=torch.int64, device="cuda")
            for c in self.ctxs:
                c.qc_encode(a, p, n, 1)
        torch.cuda.synchronize()

    def reserved_bytes(self) -> int:
        return self.slots * (self.scratch_per_slot + self.tables_per_slot)

    def _inputs(self, ctx, r: Request, st):
        """Device inputs from the seed's PRNG stream: roots [0, t), then
        ceil(t*h/16) blocks whose bytes' LSBs are the choice bits, then kk_s,
        kk_r (Ferret) or base0, base1 (SOT)."""
        torch = self.torch
        t, h, n = r.t, r.h, r.n
        blocks = lambda m: torch.empty((m, 16), dtype=torch.uint8, device="cuda")
        off = 0

        def take(m):
            nonlocal off
            x = blocks(m)
            ctx.prg_fill(r.seed, x, block_offset=off, stream=st)
            off += m
            return x
        roots = take(t)
        choice_raw = take((t * h + 15) // 16)
        choice = (choice_raw.view(-1)[: t * h] & 1).contiguous()
        inp = {"roots": roots, "choice": choice}
        if r.kind == KIND_FERRET:
            inp["kk_s"], inp["kk_r"] = take(r.k), take(r.k)
        else:
            inp["base0"], inp["base1"] = take(h * t), take(h * t)
        return inp

    def start(self, slot: int, r: Request):
        torch = self.torch
        ctx, st = self.ctxs[slot], self.streams[slot]
        if self.streams_hi is not None and r.n < self.high_below:
            st = self.streams_hi[slot]
        with torch.cuda.stream(st):
            inp = self._inputs(ctx, r, st)
            t, h, n = r.t, r.h, r.n
            emp = lambda m: torch.empty((m, 16), dtype=torch.uint8, device="cuda")
            v, w = emp(n), emp(n)
            sc = request_scalars(r.seed)
            delta = sc["delta"]
            if r.kind == KIND_FERRET:
                lsum, rsum, ss, mc = emp(t * h), emp(t * h), emp(t), emp(t * h)
                ctx.ferret_pprf_sender(inp["roots"], h, delta, v, lsum, rsum, ss, stream=st)
                torch.where(inp["choice"].view(-1, 1).bool(), rsum, lsum, out=mc)
                ctx.ferret_pprf_recver(mc, inp["choice"], ss, h, w, stream=st)
                ctx.lpn_primal(sc["lpn_seed"], inp["kk_s"], v, stream=st)
                ctx.lpn_primal(sc["lpn_seed"], inp["kk_r"], w, stream=st)
                keep = (inp, v, w, lsum, rsum, ss, mc)
                out = (v, w, None)
            else:
                m0, m1 = emp((h + 1) * t), emp((h + 1) * t)
                mc = torch.where(inp["choice"].view(-1, 1).bool(), inp["base1"], inp["base0"])
                ctx.sot_pprf_sender(inp["roots"], h, delta, inp["base0"], inp["base1"], v, m0, m1, stream=st)
                ctx.sot_pprf_recver(m0, m1, mc, inp["choice"], t, h, w, stream=st)
                a = torch.empty(n // 64, dtype=torch.int64, device="cuda")
                ctx.qc_gen_a(sc["akey"], n, a, stream=st)
                ctx.sot_dual_lpn(a, v, n, stream=st)
                ctx.sot_dual_lpn(a, w, n, stream=st)
                chm = inp["choice"].view(h, t).to(torch.int64)
                pos = torch.zeros(t, dtype=torch.int64, device="cuda")
                for dd in range(h):
                    pos = pos * 2 + 1 - chm[dd]
                pos = pos + torch.arange(t, device="cuda", dtype=torch.int64) * (1 << h)
                cb = torch.empty(n // 64, dtype=torch.int64, device="cuda")
                ctx.qc_encode_sparse(a, pos, n, cb, stream=st)
                keep = (inp, v, w, m0, m1, mc, a, pos, cb)
                out = (v, w, cb)
            ev = torch.cuda.Event()
            ev.record(st)
        self.events[slot] = ev
        self.state[slot] = (keep, out)

    def poll(self, slot: int) -> bool:
        return self.events[slot].query()

    def finish(self, slot: int):
        keep, out = self.state[slot]
        self.state[slot] = None
        self.events[slot] = None
        if self.keep_outputs:
            return tuple(None if x is None else x.cpu().numpy() for x in out)
        return None


def sustained_rate(executor, probe: list[Request], headroom: float = 0.9) -> float:
    """Requests/s the server sustains: saturation throughput on `probe`
    (every request present at t = 0), times `headroom`."""
    for r in probe:
        r.arrival, r.status, r.result = 0.0, "pending", None
    rep = Server(executor, budget_bytes=1e15).run(probe)
    return headroom * rep["done"] / rep["wall_s"]
