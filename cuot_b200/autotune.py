"""Autotuner for the launch configuration of the hot path.

Measures candidate configurations on the caller's own shapes with CUDA
events and keeps the fastest, persisted as a JSON table keyed by
(kind, n, depth) for single instances and by the batch's shape signature for
batches.  Knobs:
  pprf_threads        threads per tree CTA (128 / 256)
  ctas_per_sm         persistent-grid CTAs per SM of the batched PPRF / LPN
  lpn_rows_per_task   LPN work-queue granularity (the LPN tile)
  qc_planes_per_pass  planes per QC transform pass
The GGM expansion runs all levels of a tree in one kernel, so there is no
separate levels-per-pass knob.
"""
from __future__ import annotations

import hashlib
import itertools
import json
import os

DEFAULT_TABLE = os.environ.get("CUOT_TUNING_TABLE",
                               os.path.join(os.path.expanduser("~"), ".cache", "cuot_b200", "tuning.json"))


class TuningTable:
    def __init__(self, path: str = DEFAULT_TABLE):
        self.path = path
        self.data: dict = {}
        if os.path.exists(path):
            try:
                with open(path) as f:
                    self.data = json.load(f)
            except (OSError, ValueError):
                self.data = {}

    def get(self, key: str):
        return self.data.get(key)

    def put(self, key: str, value: dict):
        self.data[key] = value

    def save(self):
        os.makedirs(os.path.dirname(self.path) or ".", exist_ok=True)
        tmp = self.path + ".tmp"
        with open(tmp, "w") as f:
            json.dump(self.data, f, indent=1, sort_keys=True)
        os.replace(tmp, self.path)


def shape_key(kind: int, n: int, h: int) -> str:
    return f"{'sot' if kind == 1 else 'ferret'}:{n}:{h}"


def batch_key(instances) -> str:
    sig = sorted((i.kind, i.n, i.h) for i in instances)
    return "batch:" + hashlib.sha256(json.dumps(sig).encode()).hexdigest()[:16]


def _time(fn, stream, reps: int) -> float:
    import torch
    fn(stream)
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    for _ in range(reps):
        fn(stream)
    b.record(stream)
    b.synchronize()
    return a.elapsed_time(b) / reps


def tune_batch(ctx, instances, table: TuningTable | None = None, reps: int = 2, candidates=None):
    """Tries candidate batch configurations; returns (best kwargs for Batch,
    {config: ms}).  Cached by the batch's shape signature."""
    import torch
    from .batch import Batch
    table = table or TuningTable()
    key = batch_key(instances)
    hit = table.get(key)
    if hit:
        return hit["config"], hit.get("results", {})
    if candidates is None:
        candidates = [dict(pprf_threads=p, ctas_per_sm=c, lpn_rows_per_task=r)
                      for p, c, r in itertools.product((128, 256), (2, 3), (16384, 65536))]
    stream = torch.cuda.Stream()
    results = {}
    best, best_ms = None, float("inf")
    for cfg in candidates:
        b = Batch(ctx, instances, use_graph=True, **cfg)
        ms = _time(b.run, stream, reps)
        b.close()
        results[json.dumps(cfg, sort_keys=True)] = ms
        if ms < best_ms:
            best, best_ms = cfg, ms
    table.put(key, {"config": best, "ms": best_ms, "results": results})
    table.save()
    return best, results


def tune_single(ctx, inst, table: TuningTable | None = None, reps: int = 3):
    """Tunes the single-instance knobs for one instance shape (threads per
    tree for the PPRF; planes per QC transform pass for SOT), applies the winners to
    `ctx` and records them under (kind, n, depth)."""
    import torch
    table = table or TuningTable()
    key = shape_key(inst.kind, inst.n, inst.h)
    hit = table.get(key)
    if hit is None:
        stream = torch.cuda.Stream()
        t, h = inst.t, inst.h
        emp = lambda m: torch.empty((m, 16), dtype=torch.uint8, device="cuda")
        lsum, rsum, ss = emp(t * h), emp(t * h), emp(t)
        res = {}
        for thr in (128, 256):
            ctx.set_tuning(ctx.TUNE_PPRF_THREADS, thr)
            res[thr] = _time(lambda st: ctx.ferret_pprf_sender(inst.d_roots, h, inst.delta, inst.v, lsum, rsum, ss,
                                                               stream=st), stream, reps)
        hit = {"pprf_threads": min(res, key=res.get), "pprf_ms": res}
        if inst.kind == 1:
            base = max(1, (512 << 20) // (4 * inst.n))  # the library's default batch
            qres = {}
            for planes in sorted({max(1, base // 4), max(1, min(128, base // 2)), min(128, base)}):
                ctx.set_tuning(ctx.TUNE_QC_PLANES, planes)
                qres[planes] = _time(lambda st: ctx.sot_dual_lpn(inst.a, inst.v, inst.n, stream=st), stream, reps)
            hit["qc_planes_per_pass"] = min(qres, key=qres.get)
            hit["qc_ms"] = qres
        table.put(key, hit)
        table.save()
    ctx.set_tuning(ctx.TUNE_PPRF_THREADS, int(hit["pprf_threads"]))
    if "qc_planes_per_pass" in hit:
        ctx.set_tuning(ctx.TUNE_QC_PLANES, int(hit["qc_planes_per_pass"]))
    return hit
