"""Serving loop: continuous batching of OT-extension requests.

Python binding of the server in libcuot (cuot_server_* in include/cuot.h,
cuot_b200/csrc/serve.cu).  Each request is one OT extension (Ferret-style or
SOT) with both roles.  The server keeps `slots` contexts busy; a request
that arrives while others run is admitted as soon as a slot is free and its
device footprint fits the HBM budget, so requests overlap on the GPU.  A
request's inputs are derived on the device from its seed (the cryptoTools
PRNG stream) and its state stays resident on the device across the PPRF ->
LPN / quasi-cyclic encode -> transpose stages.  Latency = completion
(outputs in device memory, or in host memory with keep_outputs, observed by
the loop) - arrival.

Scheduling: requests are admitted in arrival order; optionally at most
`max_big` requests with n >= `big_n` run at once (one such request already
fills the GPU, two only time-slice it and both finish late) while smaller
requests may pass a big one that waits for that reason.  Requests with
n < `high_priority_below_n` run on a higher-priority stream so their blocks
are scheduled ahead of a running big request's.

Host-side failure handling: a request waiting in the queue longer than
`max_queue_wait` seconds times out; a queued request can be cancelled (also
from another thread during run()); a request that can never run is
rejected.  Completion is polled with event queries; nothing waits on the
device.  With `dry_run_service_s` > 0 the server does no device work (each
request takes that long), which tests the scheduling on a host without a GPU.
"""
from __future__ import annotations

import ctypes
import math
import threading
from dataclasses import dataclass, field

import numpy as np

from . import _check, load

KIND_FERRET, KIND_SOT = 0, 1
K_RATIO = 452000 / 10485760  # ferret_b13's k / n
STATUS = ("pending", "queued", "running", "done", "timeout", "cancelled", "rejected", "failed")


@dataclass
class Request:
    rid: int
    kind: int
    t: int
    h: int
    seed: bytes
    arrival: float                      # seconds from the start of the stream
    k: int = 0
    status: str = "pending"             # see STATUS
    t_admit: float = math.nan
    t_done: float = math.nan
    result: object = field(default=None, repr=False)

    @property
    def n(self) -> int:
        return self.t << self.h

    @property
    def latency(self) -> float:
        return self.t_done - self.arrival


class _Block(ctypes.Structure):
    _fields_ = [("w", ctypes.c_uint32 * 4)]


class _Request(ctypes.Structure):
    _fields_ = [("kind", ctypes.c_int), ("h", ctypes.c_int), ("t", ctypes.c_uint64), ("k", ctypes.c_int64),
                ("seed", ctypes.c_uint8 * 16), ("arrival", ctypes.c_double),
                ("v_h", ctypes.c_void_p), ("w_h", ctypes.c_void_p), ("c_h", ctypes.c_void_p),
                ("status", ctypes.c_int), ("t_admit", ctypes.c_double), ("t_done", ctypes.c_double)]


class _Config(ctypes.Structure):
    _fields_ = [("slots", ctypes.c_int), ("max_log_n", ctypes.c_int), ("budget_bytes", ctypes.c_double),
                ("max_queue_wait", ctypes.c_double), ("big_n", ctypes.c_uint64), ("max_big", ctypes.c_int),
                ("high_priority_below_n", ctypes.c_uint64), ("dry_run_service_s", ctypes.c_double)]


class _Stats(ctypes.Structure):
    _fields_ = [("wall_s", ctypes.c_double), ("max_used_bytes", ctypes.c_double)]


def _c_request(r: Request) -> _Request:
    if len(r.seed) != 16:
        raise ValueError("seed must be 16 bytes")
    c = _Request(kind=r.kind, h=r.h, t=r.t, k=r.k, arrival=r.arrival)
    ctypes.memmove(c.seed, r.seed, 16)
    return c


def request_scalars(seed: bytes) -> dict:
    """Per-request values passed by value: blocks 2^40 + {0, 1, 2} of the
    seed's AES-CTR stream -- delta (LSB set, as Ferret's Delta,
    ferret_cot.hpp:29-31), the LPN seed and the key of the QC polynomial."""
    out = (_Block * 3)()
    _check(load().cuot_request_scalars(ctypes.c_char_p(bytes(seed)), out), "cuot_request_scalars")
    raw = np.frombuffer(bytes(out), np.uint8).reshape(3, 16).copy()
    return {"delta": raw[0], "lpn_seed": raw[1], "akey": raw[2]}


def footprint(req: Request) -> int:
    """Device bytes one request holds while admitted (its inputs, both roles'
    outputs and per-request intermediates); the slots' scratch arenas are
    accounted separately."""
    out = ctypes.c_uint64()
    _check(load().cuot_request_footprint(ctypes.byref(_c_request(req)), ctypes.byref(out)), "cuot_request_footprint")
    return int(out.value)


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
    """The continuous-batching server on one device (or host-only with
    dry_run_service_s > 0).  keep_outputs copies each request's v, w (and
    SOT c) into pinned host memory as part of the request (Request.result)."""

    def __init__(self, slots: int = 8, device: int = 0, max_log_n: int = 24, budget_bytes: float = 120e9,
                 max_queue_wait: float | None = None, big_n: int | None = None, max_big: int = 1,
                 high_priority_below_n: int | None = None, keep_outputs: bool = False,
                 dry_run_service_s: float = 0.0):
        self.lib = load()
        self.slots, self.device, self.keep_outputs = slots, device, keep_outputs
        self.dry = dry_run_service_s > 0
        self.cfg = _Config(slots=slots, max_log_n=max_log_n, dry_run_service_s=dry_run_service_s)
        self.configure(budget_bytes, max_queue_wait, big_n, max_big, high_priority_below_n, _apply=False)
        if not self.dry:
            import torch
            torch.cuda.set_device(device)
        self._h = ctypes.c_void_p()
        _check(self.lib.cuot_server_create(ctypes.c_int(device), ctypes.byref(self.cfg), ctypes.byref(self._h)),
               "cuot_server_create")
        self._lock = threading.Lock()
        self._index: dict[int, int] | None = None
        self._pre_cancel: set[int] = set()
        self.max_used_bytes = 0.0

    def configure(self, budget_bytes: float = 120e9, max_queue_wait: float | None = None,
                  big_n: int | None = None, max_big: int = 1, high_priority_below_n: int | None = None,
                  _apply: bool = True):
        """Scheduling policy for later run() calls."""
        c = self.cfg
        c.budget_bytes = float(budget_bytes)
        c.max_queue_wait = float(max_queue_wait or 0.0)
        c.big_n = int(big_n or 0)
        c.max_big = int(max_big)
        c.high_priority_below_n = int(high_priority_below_n or 0)
        if _apply:
            _check(self.lib.cuot_server_configure(self._h, ctypes.byref(c)), "cuot_server_configure")

    def reserved_bytes(self) -> int:
        out = ctypes.c_uint64()
        _check(self.lib.cuot_server_reserved_bytes(self._h, ctypes.byref(out)), "cuot_server_reserved_bytes")
        return int(out.value)

    def cancel(self, rid: int):
        """Cancels request `rid` if it is queued (now, or when the next run() starts)."""
        with self._lock:
            if self._index is None:
                self._pre_cancel.add(rid)
            elif rid in self._index:
                _check(self.lib.cuot_server_cancel(self._h, ctypes.c_int(self._index[rid])), "cuot_server_cancel")

    def run(self, requests: list[Request]) -> dict:
        arr = (_Request * len(requests))()
        outs = []
        for i, r in enumerate(requests):
            arr[i] = _c_request(r)
            r.status, r.result, r.t_admit, r.t_done = "pending", None, math.nan, math.nan
            if self.keep_outputs and not self.dry:
                import torch
                v = torch.empty((r.n, 16), dtype=torch.uint8, pin_memory=True)
                w = torch.empty((r.n, 16), dtype=torch.uint8, pin_memory=True)
                c = torch.empty(r.n // 64, dtype=torch.int64, pin_memory=True) if r.kind == KIND_SOT else None
                arr[i].v_h, arr[i].w_h = v.data_ptr(), w.data_ptr()
                arr[i].c_h = c.data_ptr() if c is not None else None
                outs.append((v, w, c))
            else:
                outs.append(None)
        with self._lock:
            self._index = {r.rid: i for i, r in enumerate(requests)}
            for rid in self._pre_cancel:
                if rid in self._index:
                    self.lib.cuot_server_cancel(self._h, ctypes.c_int(self._index[rid]))
            self._pre_cancel.clear()
        stats = _Stats()
        try:
            st = self.lib.cuot_server_run(self._h, arr, ctypes.c_int(len(requests)), ctypes.byref(stats))
        finally:
            with self._lock:
                self._index = None
        for r, c, o in zip(requests, arr, outs):
            r.status = STATUS[c.status]
            r.t_admit = c.t_admit if c.t_admit >= 0 else math.nan
            r.t_done = c.t_done if c.t_done >= 0 else math.nan
            if o is not None and r.status == "done":
                r.result = tuple(None if x is None else x.numpy() for x in o)
        _check(st, "cuot_server_run")
        self.max_used_bytes = stats.max_used_bytes
        return report(requests, stats.wall_s)

    def close(self):
        if self._h:
            self.lib.cuot_server_destroy(self._h)
            self._h = ctypes.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def report(requests: list[Request], wall: float) -> dict:
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


def saturation(server: Server, probe: list[Request]) -> dict:
    """Saturation throughput of the server under its current policy: every
    request of `probe` present at t = 0.  Returns {"req_per_s", "cots_per_s",
    "requests", "wall_s"}."""
    for r in probe:
        r.arrival = 0.0
    rep = server.run(probe)
    return {"req_per_s": rep["done"] / rep["wall_s"], "cots_per_s": rep["cots_per_s"], "requests": rep["done"],
            "wall_s": rep["wall_s"]}


def sustained_rate(server: Server, probe: list[Request], headroom: float = 0.9) -> float:
    """Requests/s the server sustains under its current policy: saturation
    throughput on `probe` (every request present at t = 0), times `headroom`."""
    return headroom * saturation(server, probe)["req_per_s"]
