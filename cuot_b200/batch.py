"""Batched engine binding (cuot_batch_* in include/cuot.h) and synthetic
instance construction for benchmarks and tests.

An instance is one OT extension with both roles: Ferret-style (GGM MPCOT +
primal LPN) or SOT (GGM PPRF + exact quasi-cyclic encode).  `make_instance`
builds one from a seed with device buffers; `Batch` runs a list of them as
one device program (or one by one, the plain path).
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _check, _ptr, _stream, load

C = ctypes
KIND_FERRET, KIND_SOT = 0, 1
# cuot_batch_config.schedule
SERIAL, FORK_FERRET, FORK_SIZES = 0, 1, 2
SCHEDULES = {"serial": SERIAL, "fork_ferret": FORK_FERRET, "fork_sizes": FORK_SIZES}


class BatchItem(C.Structure):
    _fields_ = [("kind", C.c_int), ("h", C.c_int), ("t", C.c_uint64), ("delta", C.c_uint32 * 4),
                ("roots_d", C.c_void_p), ("choice_d", C.c_void_p), ("v_d", C.c_void_p), ("w_d", C.c_void_p),
                ("k", C.c_int64), ("d", C.c_int), ("lpn_seed", C.c_uint8 * 16),
                ("kk_send_d", C.c_void_p), ("kk_recv_d", C.c_void_p),
                ("base0_d", C.c_void_p), ("base1_d", C.c_void_p), ("mc_d", C.c_void_p), ("a_d", C.c_void_p),
                ("punct_d", C.c_void_p), ("cbits_d", C.c_void_p)]


class BatchConfig(C.Structure):
    _fields_ = [("pprf_threads", C.c_int), ("ctas_per_sm", C.c_int), ("lpn_rows_per_task", C.c_int),
                ("qc_planes_per_pass", C.c_int), ("use_graph", C.c_int), ("schedule", C.c_int)]


class Instance:
    """Seeded synthetic instance; host arrays (numpy) plus device tensors."""

    def __init__(self, ctx, kind: int, t: int, h: int, seed: int, k: int = 0, d: int = 10):
        import torch
        self.kind, self.t, self.h, self.n, self.k, self.d = kind, t, h, t << h, k, d
        rng = np.random.default_rng(seed)
        blk = lambda m: rng.integers(0, 256, (m, 16), dtype=np.uint8)
        dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
        self.roots, self.delta = blk(t), blk(1)[0]
        self.delta[0] |= 1
        self.choice = rng.integers(0, 2, t * h).astype(np.uint8)
        self.d_roots, self.d_choice = dev(self.roots), dev(self.choice)
        self.v = torch.empty((self.n, 16), dtype=torch.uint8, device="cuda")
        self.w = torch.empty_like(self.v)
        self.keep = []
        if kind == KIND_FERRET:
            self.seed = blk(1)[0]
            self.kk_s, self.kk_r = blk(k), blk(k)
            self.d_kk_s, self.d_kk_r = dev(self.kk_s), dev(self.kk_r)
        else:
            self.base0, self.base1 = blk(h * t), blk(h * t)
            self.mc = np.where(self.choice[:, None] == 0, self.base0, self.base1)
            self.d_b0, self.d_b1, self.d_mc = dev(self.base0), dev(self.base1), dev(self.mc)
            self.a = torch.empty(self.n // 64, dtype=torch.int64, device="cuda")
            ctx.qc_gen_a(blk(1)[0], self.n, self.a)
            chm = self.choice.reshape(h, t)
            pos = np.zeros(t, np.int64)
            for dd in range(h):
                pos = pos * 2 + 1 - chm[dd].astype(np.int64)
            self.punct = pos + np.arange(t) * (1 << h)
            self.d_punct = dev(self.punct)
            self.cbits = torch.empty(self.n // 64, dtype=torch.int64, device="cuda")

    INPUTS = {KIND_FERRET: ("d_roots", "d_choice", "d_kk_s", "d_kk_r"),
              KIND_SOT: ("d_roots", "d_choice", "d_b0", "d_b1", "d_mc")}

    def input_copy(self, own_outputs: bool = False) -> "Instance":
        """The same instance with its own copy of the per-step device inputs
        (same polynomial; same outputs, or its own with own_outputs): a
        second batch over these copies lets host steps double-buffer their
        inputs (HostPipeline input_sets=2), and with own_outputs their
        outputs too (per_set_outputs)."""
        import copy

        import torch
        other = copy.copy(self)
        for name in self.INPUTS[self.kind]:
            setattr(other, name, getattr(self, name).clone())
        if own_outputs:
            other.v, other.w = torch.empty_like(self.v), torch.empty_like(self.w)
            if self.kind != KIND_FERRET:
                other.cbits = torch.empty_like(self.cbits)
        return other

    def item(self) -> BatchItem:
        it = BatchItem()
        it.kind, it.h, it.t = self.kind, self.h, self.t
        it.delta[:] = list(np.frombuffer(self.delta.tobytes(), "<u4"))
        it.roots_d, it.choice_d = self.d_roots.data_ptr(), self.d_choice.data_ptr()
        it.v_d, it.w_d = self.v.data_ptr(), self.w.data_ptr()
        if self.kind == KIND_FERRET:
            it.k, it.d = self.k, self.d
            it.lpn_seed[:] = list(self.seed)
            it.kk_send_d, it.kk_recv_d = self.d_kk_s.data_ptr(), self.d_kk_r.data_ptr()
        else:
            it.base0_d, it.base1_d, it.mc_d = self.d_b0.data_ptr(), self.d_b1.data_ptr(), self.d_mc.data_ptr()
            it.a_d, it.punct_d, it.cbits_d = self.a.data_ptr(), self.d_punct.data_ptr(), self.cbits.data_ptr()
        return it


class Batch:
    def __init__(self, ctx, instances, pprf_threads: int = 0, ctas_per_sm: int = 0, lpn_rows_per_task: int = 0,
                 qc_planes_per_pass: int = 0, use_graph: bool = True, schedule: int = 0):
        self.lib, self.ctx, self.instances = load(), ctx, list(instances)
        arr = (BatchItem * len(self.instances))(*[i.item() for i in self.instances])
        cfg = BatchConfig(pprf_threads, ctas_per_sm, lpn_rows_per_task, qc_planes_per_pass, int(use_graph),
                          int(schedule))
        h = C.c_void_p()
        _check(self.lib.cuot_batch_create(ctx.h, arr, C.c_int(len(self.instances)), C.byref(cfg), C.byref(h)),
               "cuot_batch_create")
        self.h = h

    def run(self, stream=None):
        _check(self.lib.cuot_batch_run(self.h, _stream(stream)), "cuot_batch_run")

    def run_plain(self, stream=None):
        _check(self.lib.cuot_batch_run_plain(self.h, _stream(stream)), "cuot_batch_run_plain")

    def run_phases(self, stream=None):
        """Diagnostic un-graphed run; returns [sender PPRF + select,
        receiver PPRF, LPN, SOT encodes] in ms."""
        ms = (C.c_float * 4)()
        _check(self.lib.cuot_batch_run_phases(self.h, _stream(stream), ms), "cuot_batch_run_phases")
        return list(ms)

    def kernels_per_run(self) -> int:
        return int(self.lib.cuot_batch_kernels_per_run(self.h))

    def item_rank(self, i: int) -> int:
        """Completion point of instance i: 0 for Ferret instances (after the
        LPN), then 1, 2, ... for the SOT sizes, largest first."""
        r = int(self.lib.cuot_batch_item_rank(self.h, C.c_int(i)))
        if r < 0:
            raise IndexError(f"batch has no instance {i}")
        return r

    def wait_item(self, i: int, stream) -> None:
        """Makes `stream` wait until instance i's outputs of the last run()
        are final (earlier than the end of the run for all but the last
        size)."""
        _check(self.lib.cuot_batch_wait_item(self.h, C.c_int(i), _stream(stream)), "cuot_batch_wait_item")

    def close(self):
        if getattr(self, "h", None):
            self.lib.cuot_batch_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def mixed_shapes(count: int = 64, seed: int = 2024, lo: int = 16, hi: int = 22):
    """Shapes of the mixed batch: `count` (kind, t, h, k) tuples, half SOT
    and half Ferret-style, log2(n) uniform over [lo, hi], depth in [10, 14]
    with t = n / 2^h; Ferret k = ceil(n * 452000 / 10485760) (ferret_b13's
    ratio).  Needs no device."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(count):
        kind = KIND_SOT if i % 2 == 0 else KIND_FERRET
        e = int(rng.integers(lo, hi + 1))
        h = int(rng.integers(10, min(14, e) + 1))
        t = (1 << e) >> h
        k = -(-(1 << e) * 452000 // 10485760) if kind == KIND_FERRET else 0
        out.append((kind, t, h, k))
    return out


def mixed_workload(ctx, count: int = 64, seed: int = 2024, lo: int = 16, hi: int = 22):
    """The mixed batch of `mixed_shapes`, each instance seeded with
    seed * 1000 + its index, with device buffers."""
    return [Instance(ctx, kind, t, h, seed * 1000 + i, k=k)
            for i, (kind, t, h, k) in enumerate(mixed_shapes(count, seed, lo, hi))]
