"""Benchmark: COTs/sec of the silent-OT hot path on B200.

A step produces one full COT correlation on the GPU: both roles (sender and
receiver) of one OT-extension instance, seeded synthetic inputs of the named
shape.

Workloads (--workload):
  mixed64     batched mix (the headline line): 64 instances, half SOT and
              half Ferret-style, log2 n uniform in [16, 22], depth 10-14; run
              as one CUDA-graph device program (value) and one instance at a
              time through the plain entry points (plain.value).
  mixed64_small  the same mix with log2 n in [12, 16]: launch-bound
              instances, where one device program pays off most.
  sot_n20     plain SOT, n = 2^20: 256 GGM trees of depth 12 (both roles),
              exact quasi-cyclic encode of the 128 bit planes of the n noise
              blocks, transposes both ways, plus the
              receiver's choice-bit encode.
  sot_n20_r2  SOT rate-1/2 form with n = 2^20 outputs: 512 trees of depth
              12 give 2n noise blocks e = (e0, e1) per role, encoded as
              e0 ^ a * e1 (the flagged second SOT configuration).
  sot_n21, sot_n22  plain SOT at n = 2^21 and 2^22 (512 / 1024 trees of
              depth 12), the largest sizes of the batched mix.
  ferret_b13  plain Ferret at full size (ferret_b13): n = 10,485,760,
              t = 1280 trees of depth 13, k = 452,000, d = 10 (both roles:
              MPCOT + primal LPN).
  ferret_b13_mal  ferret_b13 plus the per-tree GF(2^128) check values of the
              malicious consistency check on both roles (stage "chi").
  ferret_c1   plain Ferret small: t = 64, h = 10, k = 8192.
  ferret_rcot FerretCOT's extension loop at ferret_b13 parameters (cuot_b200.ferret):
              one extension per step, pre-COTs carried over on the device,
              usable COTs (ot_limit per extension) per second.

Multi-GPU: one process per GPU (torchrun), each rank runs its own instance
(the path shards by independent instances; no data-path collective):
"scaling": "weak", value = COTs of all ranks / max-over-ranks time.

--impl reference: the reference's CPU implementation of the path timed on
all host threads on a bounded sample of the same workload: the Ferret GGM
and LPN by the reference's own emp-ot headers (compiled over an emp-tool shim
into oracle/_ref/libempref.so, where the reference tree was present at build
time), the SOT PPRF and QC encode by the oracle's restatement (the reference
has no CPU SOT code).  For the batched mix every one of its 64 instances is
sampled (CpuMix).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

import numpy as np

WORKLOADS = {
    "mixed64": dict(kind="batch", count=64, lo=16, hi=22),
    "mixed64_small": dict(kind="batch", count=64, lo=12, hi=16),
    "sot_n20": dict(kind="sot", t=256, h=12),
    "sot_n20_r2": dict(kind="sot", t=512, h=12, r2=True),
    "sot_n21": dict(kind="sot", t=512, h=12),
    "sot_n22": dict(kind="sot", t=1024, h=12),
    "ferret_b13": dict(kind="ferret", t=1280, h=13, k=452000, d=10),
    "ferret_b13_mal": dict(kind="ferret", t=1280, h=13, k=452000, d=10, mal=True),
    "ferret_c1": dict(kind="ferret", t=64, h=10, k=8192, d=10),
    "ferret_rcot": dict(kind="session", t=1280, h=13, k=452000, d=10),
    "aes_ecb": dict(kind="aes", n=1 << 26),
}
CONFIG_TEXT = {
    "mixed64": "batched mix: 64 instances (32 SOT, 32 Ferret-style), log2 n uniform in [16,22], depth 10-14, "
               "both roles, one CUDA-graph program vs the plain one-instance-at-a-time path",
    "mixed64_small": "batched mix of small instances: 64 instances (32 SOT, 32 Ferret-style), log2 n uniform in "
                     "[12,16], depth 10-14, both roles, one CUDA-graph program vs the plain one-instance-at-a-time path",
    "sot_n20": "plain SOT n=2^20: 256 GGM trees depth 12, exact QC encode of 128 planes, transposes (both roles)",
    "sot_n20_r2": "plain SOT rate-1/2, n=2^20 outputs: 512 GGM trees depth 12 (2n noise blocks), "
                  "out = e0 ^ a*e1 exact on 128 planes, transposes (both roles)",
    "sot_n21": "plain SOT n=2^21: 512 GGM trees depth 12, exact QC encode of 128 planes, transposes (both roles)",
    "sot_n22": "plain SOT n=2^22 (the mix's largest size): 1024 GGM trees depth 12, exact QC encode of 128 "
               "planes, transposes (both roles)",
    "ferret_b13": "plain Ferret ferret_b13: n=10485760, t=1280, h=13, k=452000, d=10 (both roles)",
    "ferret_b13_mal": "ferret_b13 plus the malicious consistency check's per-tree GF(2^128) sums of both roles "
                      "(seeds given; their SHA-256 derivation is host protocol)",
    "ferret_c1": "plain Ferret small: n=65536, t=64, h=10, k=8192, d=10 (both roles)",
    "aes_ecb": "diagnostic: AES-128 ECB of 2^26 blocks (1 GiB) in place, the shared-memory T-table kernel "
               "against the bitsliced register kernel",
    "ferret_rcot": "Ferret rcot session at ferret_b13 parameters: one extension per step (both roles), its M = "
                   "k + t*h + 128 pre-COTs carried over on the device; value counts the ot_limit = 10,016,992 "
                   "usable COTs per extension",
}


def metric_name(workload: str) -> str:
    if WORKLOADS[workload]["kind"] == "aes":
        return "AES-128 blocks/sec on 1 B200 (T-table vs bitsliced)"
    if WORKLOADS[workload]["kind"] == "batch":
        return "COTs/sec on 1 B200, batched vs plain path (bit-exact)"
    return "COTs/sec on 1 B200 (plain path, bit-exact)"


def log(*a):
    print(*a, file=sys.stderr, flush=True)


# --------------------------------------------------------------------------
class ClockSampler:
    """nvidia-smi clocks/throttle sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index, self.proc, self.lines = index, None, []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.th = threading.Thread(target=self._read, daemon=True)
            self.th.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return d, "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


# --------------------------------------------------------------------------
class Instance:
    """Seeded synthetic inputs + device buffers for one workload instance."""

    def __init__(self, name: str, seed: int, torch, cuot_b200):
        self.name, self.spec = name, WORKLOADS[name]
        self.torch, self.cb = torch, cuot_b200
        s = self.spec
        self.t, self.h = s["t"], s["h"]
        self.r2 = bool(s.get("r2"))
        self.nleaves = self.t << self.h
        self.n = self.nleaves // 2 if self.r2 else self.nleaves  # COTs per role
        rng = np.random.default_rng(seed)
        blk = lambda m: rng.integers(0, 256, (m, 16), dtype=np.uint8)
        dev = lambda a: torch.from_numpy(np.ascontiguousarray(a)).cuda()
        emp = lambda m: torch.empty((m, 16), dtype=torch.uint8, device="cuda")
        t, h, n = self.t, self.h, self.n
        self.roots = blk(t)
        self.delta = blk(1)[0]
        self.delta[0] |= 1
        self.choice = rng.integers(0, 2, t * h).astype(np.uint8)
        # device buffers
        self.sctx = new_context(cuot_b200, torch.cuda.current_device())
        self.rctx = new_context(cuot_b200, torch.cuda.current_device())
        self.d_roots = dev(self.roots)
        self.d_choice = dev(self.choice)
        self.leaves_s, self.leaves_r = emp(self.nleaves), emp(self.nleaves)
        self.mal = False
        if s["kind"] == "ferret":
            k = s["k"]
            self.k, self.d = k, s["d"]
            self.kk_s = blk(k)
            self.kk_r = blk(k)
            self.d_kk_s, self.d_kk_r = dev(self.kk_s), dev(self.kk_r)
            self.lsum, self.rsum, self.ss = emp(t * h), emp(t * h), emp(t)
            self.mc = emp(t * h)
            self.seed = blk(1)[0]
            self.mal = bool(s.get("mal"))
            if self.mal:
                self.d_chiseed = dev(blk(t))
                self.chi_v, self.chi_w = emp(t), emp(t)
        else:
            self.base0, self.base1 = blk(h * t), blk(h * t)
            self.d_b0, self.d_b1 = dev(self.base0), dev(self.base1)
            self.mc_np = np.where(self.choice[:, None] == 0, self.base0, self.base1)
            self.d_mc = dev(self.mc_np)
            self.m0, self.m1 = emp((h + 1) * t), emp((h + 1) * t)
            self.a = torch.empty(n // 64, dtype=torch.int64, device="cuda")
            self.sctx.qc_gen_a(blk(1)[0], n, self.a)
            self.plan_s = self.sctx.qc_plan(self.a, n)
            self.plan_r = self.rctx.qc_plan(self.a, n)
            chm = self.choice.reshape(h, t)
            pos = np.zeros(t, np.int64)
            for dd in range(h):
                pos = pos * 2 + 1 - chm[dd].astype(np.int64)
            self.d_pos = dev(pos + np.arange(t) * (1 << h))
            self.cbits = torch.empty(n // 64, dtype=torch.int64, device="cuda")
        torch.cuda.synchronize()

    # one step on the device (inputs resident); stage events optional
    def step(self, ev=None):
        torch = self.torch
        mark = (lambda k: ev[k].record()) if ev is not None else (lambda k: None)
        if self.spec["kind"] == "ferret":
            t, h = self.t, self.h
            mark("pprf0")
            self.sctx.ferret_pprf_sender(self.d_roots, h, self.delta, self.leaves_s, self.lsum, self.rsum, self.ss)
            # ideal OT of the per-level sums (OTIdeal, emp-ot/ideal.h): mc = choice ? rsum : lsum
            torch.where(self.d_choice.view(-1, 1).bool(), self.rsum, self.lsum, out=self.mc)
            self.rctx.ferret_pprf_recver(self.mc, self.d_choice, self.ss, h, self.leaves_r)
            mark("pprf1")
            if self.mal:
                self.sctx.ferret_chi_sum(self.leaves_s, h, self.d_chiseed, self.chi_v)
                self.rctx.ferret_chi_sum(self.leaves_r, h, self.d_chiseed, self.chi_w)
            mark("chi1")
            # both roles' LPN share the public seed: one dual-role launch
            self.sctx.lpn_primal_dual(self.seed, self.d_kk_s, self.d_kk_r, self.leaves_s, self.leaves_r, d=self.d)
            mark("lpn1")
        else:
            t, h, n = self.t, self.h, self.n
            mark("pprf0")
            self.sctx.sot_pprf_sender(self.d_roots, h, self.delta, self.d_b0, self.d_b1, self.leaves_s,
                                      self.m0, self.m1)
            self.rctx.sot_pprf_recver(self.m0, self.m1, self.d_mc, self.d_choice, t, h, self.leaves_r)
            mark("pprf1")
            mark("chi1")
            if self.r2:
                self.plan_s.dual_lpn_r2(self.leaves_s, self.leaves_s[:n])
                self.plan_r.dual_lpn_r2(self.leaves_r, self.leaves_r[:n])
                self.rctx.qc_encode_sparse_r2(self.a, self.d_pos, n, self.cbits)
            else:
                self.plan_s.dual_lpn(self.leaves_s)
                self.plan_r.dual_lpn(self.leaves_r)
                self.rctx.qc_encode_sparse(self.a, self.d_pos, n, self.cbits)
            mark("lpn1")

    def launches_per_step(self) -> int:
        before = self.cb.launch_count()
        self.step()
        self.torch.cuda.synchronize()
        return self.cb.launch_count() - before


# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of the dominant
# stage's kernels per step, from ncu captures of the same bench command, one
# kernel and one to three launches per capture (ncu starts every launch with
# cold caches, so intermediate that steady state keeps in L2 is counted):
# ferret_b13: the dual-role LPN launch (profiles/pprf_lpn_ferret_b13.md);
# sot_n20: gather, 16 launches of each transform pass and scatter per role
# (profiles/qc_fft_sot_n20.md); sot_n20_ntt: the same workload on the NTT
# backend, which scales the SOT encodes of NTT sizes (profiles/qc_ntt_sot_n20.md);
# sot_n22: 32 transforms of 251.8 MB per role plus gather and scatter
# (profiles/qc_fft_sot_n22.md).
NCU_TRAFFIC_PER_STEP = {
    "ferret_b13:lpn": 631.83e6,
    "sot_n20:dual_lpn": 2 * (16.79e6 + 16 * 88.24e6 + 16.86e6),
    "sot_n20_ntt:dual_lpn": 2 * (509.60e6 + 1024.36e6 + 563.98e6 + 33.58e6),
    "sot_n22:dual_lpn": 2 * (32 * 251.75e6 + 84.17e6 + 82.25e6),
}

QC_FFT_MAX_LOG_N = 22  # the fp64 FFT encodes n <= 2^22 (exactness bound)
QC_KARA_MAX_LOG_N = 24  # dual LPNs up to 2^24: GF(2) Karatsuba over 2^22 FFTs; the NTT above


def qc_leaves(lg: int) -> int:
    """FFT dual LPNs (of at most 2^22 points) behind one dual LPN of n = 2^lg
    (0: NTT)."""
    if lg <= QC_FFT_MAX_LOG_N:
        return 1
    if lg <= QC_KARA_MAX_LOG_N:
        return 3 ** (lg - QC_FFT_MAX_LOG_N)
    return 0
QC_BACKENDS = {"auto": 0, "ntt": 1, "fft": 2}
_qc_backend = 0


def new_context(cuot_b200, device: int):
    """A libcuot context with the QC backend chosen on the command line."""
    c = cuot_b200.Context(device)
    if _qc_backend:
        c.set_tuning(c.TUNE_QC_BACKEND, _qc_backend)
    return c


def qc_transform_work(ns) -> dict:
    """Arithmetic of the SOT dual LPNs of one step (both roles, 128 planes
    each) for instance sizes `ns`: fp64 flops of the FFT backend (4 planes per
    complex transform: 32 forward + 32 inverse n-point transforms per role at
    the standard 5 n log2 n flops, plus 6n per pointwise product) and radix-2
    butterflies of the NTT backend (128 forward + 128 inverse per role)."""
    flops = bfly = 0
    for n in ns:
        lg = n.bit_length() - 1
        leaves = qc_leaves(lg)
        if leaves:
            m, lm = min(n, 1 << QC_FFT_MAX_LOG_N), min(lg, QC_FFT_MAX_LOG_N)
            flops += leaves * 2 * 32 * (2 * 5 * m * lm + 6 * m)
        else:
            bfly += 2 * 128 * 2 * (n // 2) * lg
    return {"fft_fp64_flops": flops, "ntt_butterflies": bfly}


def qc_transform_report(ns, ms: float, fp64_peak: float | None = None) -> dict:
    """fp64_peak: the device's measured FMA rate in TFLOP/s
    (Context.measure_fp64_tflops), the denominator of frac_of_measured."""
    w = qc_transform_work(ns)
    out = {"backend": "fft (n <= 2^22) / karatsuba over 2^22 ffts (2^23, 2^24) / ntt (larger n)", "stage_ms": ms, **w,
           "model": "fft: 5 m log2 m flops per complex m-point transform + 6m per product, 3^L leaves of "
                    "m = 2^22 for the Karatsuba sizes; ntt: n/2 log2 n butterflies"}
    if w["fft_fp64_flops"] and not w["ntt_butterflies"]:
        out["fp64_tflops"] = w["fft_fp64_flops"] / (ms / 1e3) / 1e12
        out["fp64_peak_nominal_tflops"] = 37.0
        out["frac_of_nominal"] = out["fp64_tflops"] / 37.0
        if fp64_peak:
            out["fp64_peak_measured_tflops"] = fp64_peak
            out["frac_of_measured"] = out["fp64_tflops"] / fp64_peak
            out["fp64_peak_method"] = ("cuot_measure_fp64_tflops: 8 independent FMA chains per thread, 2048 "
                                       "threads per SM, best of 5 launches of ~9 ms, 2 flops per FMA")
    return out


def fp64_roofline(qct: dict) -> dict | None:
    """The FFT encode stage against the fp64 pipe (measured FMA rate): the
    bound its exact transforms actually work against, reported beside the
    stage's HBM fraction (whose algorithmic bytes, 96n per role, are a small
    part of what an exact transform moves)."""
    if "frac_of_measured" not in qct:
        return None
    return {"achieved": qct["fp64_tflops"], "peak": qct["fp64_peak_measured_tflops"], "unit": "TFLOP/s",
            "frac": qct["frac_of_measured"], "peak_source": "measured (cuot_measure_fp64_tflops)",
            "work": "fft_fp64_flops of qc_transform per step"}


AES_PEAK_MODEL = ("T-table AES: 160 shared-memory lookups per block (10 rounds x 16), one conflict-free "
                  "32-lane lookup wavefront per clock per SM; peak = SMs x 32 x median SM clock / 160")


LPN_L1_MODEL = ("L1 wavefronts per LPN row pair (the dual-role kernel: one index computation for the two "
                "parties' rows): index-AES table lookups (145 per block for d = 10 blocks of a 4-row group "
                "plus 15 shared round-1 lookups, i.e. (145 d + 15) / 4 per row, 32 lanes per wavefront) + 2d "
                "random 16-byte kk gathers (one line, one wavefront each) + both rows' 16-byte read and write "
                "(1/8 wavefront each); rows counted per role, peak rows/s = SMs x median SM clock / "
                "wavefronts per role row")


def lpn_l1_roofline(rows: int, d: int, ms: float, clocks: dict, props) -> dict:
    """LPN rows per second against the L1 wavefront bound the index AES and
    the kk gathers share (both go through the L1/shared data pipe)."""
    mhz = clocks.get("sm_mhz") or clocks.get("sm_max_mhz") or 1965.0
    per_row = ((145 * d + 15) / 4 / 32 + 2 * d + 0.5) / 2  # per role row
    peak = props.multi_processor_count * mhz * 1e6 / per_row
    achieved = rows / (ms / 1e3)
    return {"rows_per_step": rows, "rows_per_s": achieved, "peak_rows_per_s": peak, "frac": achieved / peak,
            "wavefronts_per_row": per_row, "model": LPN_L1_MODEL}


def transpose_roofline(inst: Instance, flush, peaks: dict, peak_kind: str, reps: int = 10) -> dict:
    """The 128-plane bit transpose (cuot_bit_transpose, blocks -> planes and
    back) of the instance's n blocks against HBM: 32n algorithmic bytes per
    direction (16n read + 16n write), L2 flushed before each timed call."""
    torch = inst.torch
    res = {}
    for tag, n in (("config", inst.n), ("streaming_2^24", 1 << 24)):
        src = inst.leaves_s[:n] if n <= inst.leaves_s.shape[0] else \
            torch.randint(0, 256, (n, 16), dtype=torch.uint8, device="cuda")
        planes = torch.empty((n, 16), dtype=torch.uint8, device="cuda")
        back = torch.empty_like(planes)
        for name, fn in (("blocks_to_planes", lambda: inst.sctx.bit_transpose(src, n, 16, 0, 128, planes)),
                         ("planes_to_blocks", lambda: inst.sctx.bit_transpose(planes, 128, n // 8, 0, n, back))):
            fn()
            ms = 0.0
            for _ in range(reps):
                flush.zero_()
                # keep the GPU busy (~100 us) while the host enqueues the call, so the events
                # bracket the kernel and not the host's launch latency
                torch.cuda._sleep(200_000)
                a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a.record()
                fn()
                b.record()
                torch.cuda.synchronize()
                ms += a.elapsed_time(b) / reps
            gbs = 32 * n / (ms / 1e3) / 1e9
            res[f"{tag}:{name}"] = {"n": n, "ms": ms, "achieved_gbs": gbs, "frac": gbs / peaks["hbm_gbs"]}
        del planes, back, src
    res.update({"algorithmic_bytes": "32n per direction", "peak_gbs": peaks["hbm_gbs"],
                "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)",
                "note": "the standalone transpose of the reference's operator surface; the FFT dual LPN uses "
                        "its own gather/scatter into the column-tile layout instead"})
    return res


def aes_roofline(inst: Instance, stages: dict, clocks: dict, props) -> dict:
    """AES blocks per second of the AES-bound stages against the T-table
    lookup roofline (the integer-pipe figure that bounds the PPRF and the
    LPN index generation)."""
    mhz = clocks.get("sm_mhz") or clocks.get("sm_max_mhz") or 1965.0
    peak = props.multi_processor_count * 32 * mhz * 1e6 / 160
    t, h = inst.t, inst.h
    counts = {"pprf": 4 * t * ((1 << h) - 1)}  # 2 AES per internal node, both roles
    if inst.spec["kind"] == "ferret":
        counts["lpn"] = inst.n * inst.d // 4  # d index blocks per 4 rows, computed once for both roles
    res = {"peak_aes_per_s": peak, "model": AES_PEAK_MODEL}
    for k, cnt in counts.items():
        a = cnt / (stages[k][0] / 1e3)
        res[k] = {"aes_per_step": cnt, "aes_per_s": a, "frac": a / peak}
    if "lpn" in counts and inst.d == 10:
        res["lpn_l1_roofline"] = lpn_l1_roofline(2 * inst.n, inst.d, stages["lpn"][0], clocks, props)
    return res


def device_inputs(inst: Instance, slot: int = 0) -> dict:
    """Device input buffers of input set `slot`: set 0 is the instance's own,
    set 1 a second copy for double-buffered host steps (HostPipeline
    input_sets=2)."""
    names = ["roots", "choice"] + (["kk_s", "kk_r"] if inst.spec["kind"] == "ferret" else ["b0", "b1", "mc"])
    base = {k: getattr(inst, "d_" + k) for k in names}
    if slot == 0:
        return base
    if not hasattr(inst, "_din1"):
        inst._din1 = {k: v.clone() for k, v in base.items()}
    return inst._din1


def e2e_inputs(inst: Instance, host, slot: int = 0):
    """(pinned host tensor, device tensor) pairs of one step's inputs."""
    din = device_inputs(inst, slot)
    names = ["roots", "choice"] + (["kk_s", "kk_r"] if inst.spec["kind"] == "ferret" else ["b0", "b1", "mc"])
    return [(host[k], din[k]) for k in names]


def e2e_outputs(inst: Instance, host):
    """(device result, pinned host tensor) pairs returned by every step."""
    pairs = [(inst.leaves_s[:inst.n], host["v"]), (inst.leaves_r[:inst.n], host["w"])]
    if inst.spec["kind"] != "ferret":
        pairs.append((inst.cbits, host["c"]))
    return pairs


def e2e_compute(inst: Instance, host, stream, slot: int = 0) -> int:
    """The step's device work through the public API on `stream`, reading
    input set `slot`.  Ferret's level sums and secret sums go to the host
    inside the step, as in dev_layer.cu:40-41,50; returns those bytes."""
    torch = inst.torch
    din = device_inputs(inst, slot)
    d2h = 0
    with torch.cuda.stream(stream):
        if inst.spec["kind"] == "ferret":
            inst.sctx.ferret_pprf_sender(din["roots"], inst.h, inst.delta, inst.leaves_s, inst.lsum, inst.rsum,
                                         inst.ss, stream=stream)
            # the sums go to the host mid-step through SM stores: a DMA copy
            # would wait behind the previous step's outputs on the copy engine
            for k, d in (("lsum", inst.lsum), ("rsum", inst.rsum), ("ss", inst.ss)):
                inst.cb.copy_to_host(d, host[k], stream=stream)
                d2h += host[k].numel()
            torch.where(din["choice"].view(-1, 1).bool(), inst.rsum, inst.lsum, out=inst.mc)
            inst.rctx.ferret_pprf_recver(inst.mc, din["choice"], inst.ss, inst.h, inst.leaves_r, stream=stream)
            if inst.mal:
                inst.sctx.ferret_chi_sum(inst.leaves_s, inst.h, inst.d_chiseed, inst.chi_v, stream=stream)
                inst.rctx.ferret_chi_sum(inst.leaves_r, inst.h, inst.d_chiseed, inst.chi_w, stream=stream)
            inst.sctx.lpn_primal_dual(inst.seed, din["kk_s"], din["kk_r"], inst.leaves_s, inst.leaves_r, d=inst.d,
                                      stream=stream)
        else:
            inst.sctx.sot_pprf_sender(din["roots"], inst.h, inst.delta, din["b0"], din["b1"], inst.leaves_s,
                                      inst.m0, inst.m1, stream=stream)
            inst.rctx.sot_pprf_recver(inst.m0, inst.m1, din["mc"], din["choice"], inst.t, inst.h, inst.leaves_r,
                                      stream=stream)
            n = inst.n
            if inst.r2:
                inst.plan_s.dual_lpn_r2(inst.leaves_s, inst.leaves_s[:n], stream=stream)
                inst.plan_r.dual_lpn_r2(inst.leaves_r, inst.leaves_r[:n], stream=stream)
                inst.rctx.qc_encode_sparse_r2(inst.a, inst.d_pos, n, inst.cbits, stream=stream)
            else:
                inst.plan_s.dual_lpn(inst.leaves_s, stream=stream)
                inst.plan_r.dual_lpn(inst.leaves_r, stream=stream)
                inst.rctx.qc_encode_sparse(inst.a, inst.d_pos, n, inst.cbits, stream=stream)
    return d2h


def make_host(inst: Instance):
    torch = inst.torch
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory()
    host = {"roots": pin(inst.roots), "choice": pin(inst.choice),
            "v": torch.empty((inst.n, 16), dtype=torch.uint8).pin_memory(),
            "w": torch.empty((inst.n, 16), dtype=torch.uint8).pin_memory()}
    if inst.spec["kind"] == "ferret":
        host.update(kk_s=pin(inst.kk_s), kk_r=pin(inst.kk_r),
                    lsum=torch.empty((inst.t * inst.h, 16), dtype=torch.uint8).pin_memory(),
                    rsum=torch.empty((inst.t * inst.h, 16), dtype=torch.uint8).pin_memory(),
                    ss=torch.empty((inst.t, 16), dtype=torch.uint8).pin_memory())
    else:
        host.update(b0=pin(inst.base0), b1=pin(inst.base1), mc=pin(inst.mc_np),
                    c=torch.empty(inst.n // 64, dtype=torch.int64).pin_memory())
    return host


# --------------------------------------------------------------------------
def ref_ferret_available() -> bool:
    """True when oracle/_ref/libempref.so (the reference's own emp-ot GGM and
    LPN code) was built and travelled with the repository."""
    import oracle
    return oracle.emp_lib() is not None


def _ref_ferret_step(roots, h, delta, ch, kk, seed_b, threads: int):
    """Both roles of one Ferret MPCOT + LPN through the reference's own
    emp-ot code, threaded as emp-ot threads it: trees split over `threads`
    workers, the LPN rows over `threads` LpnF2::task ranges (each with its own
    __compute1 tail, as emp-ot's threaded LPN does)."""
    import concurrent.futures as cf
    import oracle
    t = roots.shape[0]
    cuts = [t * i // threads for i in range(threads + 1)]
    ls = np.empty((t << h, 16), np.uint8)
    lr = np.empty((t << h, 16), np.uint8)

    def trees(i):
        a, b = cuts[i], cuts[i + 1]
        if b > a:
            ls[a << h:b << h], lr[a << h:b << h] = oracle.emp_mpcot_trees(roots[a:b], h, delta, ch[a * h:b * h])

    n = t << h
    rcuts = [n * i // threads // 4 * 4 for i in range(threads)] + [n]

    def rows(i):
        for out in (ls, lr):
            oracle.emp_lpn_task(seed_b, kk, out, start=rcuts[i], end=rcuts[i + 1], inplace=True)

    with cf.ThreadPoolExecutor(max_workers=threads) as pool:
        list(pool.map(trees, range(threads)))
        list(pool.map(rows, range(threads)))
    return ls, lr


def cpu_sample(name: str, threads: int, budget_s: float = 10.0):
    """Times the CPU path on a bounded sample of the workload; returns
    (COTs/s, sample description).  Ferret: the reference's own emp-ot code
    (oracle/_ref/libempref.so) when it is built, else the oracle's
    restatement; SOT: the oracle's restatement."""
    import oracle
    spec = WORKLOADS[name]
    rng = np.random.default_rng(99)
    blk = lambda m: rng.integers(0, 256, (m, 16), dtype=np.uint8)
    t_full, h = spec["t"], spec["h"]
    if spec["kind"] == "ferret":
        t = min(t_full, max(threads, 64))
        n = t << h
        roots, delta = blk(t), blk(1)[0]
        delta[0] |= 1
        kk = blk(spec["k"])
        ch = rng.integers(0, 2, t * h).astype(np.uint8)
        use_ref = ref_ferret_available() and spec["d"] == 10
        t0 = time.perf_counter()
        reps = 0
        while True:
            if use_ref:
                _ref_ferret_step(roots, h, delta, ch, kk, blk(1)[0], threads)
            else:
                lv, ls, rs, ss = oracle.ferret_pprf_sender(roots, h, delta, threads=threads)
                mc = np.where(ch[:, None] == 0, ls, rs)
                rl = oracle.ferret_pprf_recver(mc, ch, ss, h, threads=threads)
                oracle.lpn_primal(blk(1)[0], kk, lv, d=spec["d"], threads=threads)
                oracle.lpn_primal(blk(1)[0], kk, rl, d=spec["d"], threads=threads)
            reps += 1
            el = time.perf_counter() - t0
            if el > budget_s or reps >= 3:
                break
        code = "reference emp-ot code (SPCOT_Sender/Recver, LpnF2::task)" if use_ref else "oracle restatement"
        return reps * n / el, (f"{t} of {t_full} trees (n={n}), both roles, MPCOT + LPN (k={spec['k']}), "
                               f"{reps} reps, {code}")
    # SOT: PPRF both roles on all trees; QC encode on a subset of planes, scaled
    r2 = bool(spec.get("r2"))
    nl = t_full << h
    n = nl // 2 if r2 else nl
    roots, delta = blk(t_full), blk(1)[0]
    b0, b1 = blk(h * t_full), blk(h * t_full)
    ch = rng.integers(0, 2, h * t_full).astype(np.uint8)
    mc = np.where(ch[:, None] == 0, b0, b1)
    a = oracle.qc_gen_a(blk(1)[0], n)
    nplanes = max(4, min(128, threads * 2))
    t0 = time.perf_counter()
    lv, m0, m1 = oracle.sot_pprf_sender(roots, h, delta, b0, b1, threads=threads)
    rl = oracle.sot_pprf_recver(m0, m1, mc, ch, t_full, h, threads=threads)
    t_pprf = time.perf_counter() - t0
    t0 = time.perf_counter()
    pl = oracle.bit_transpose(lv, nl, 16, 0, 128).view(np.uint64).reshape(128, nl // 64)
    enc = oracle.qc_encode(a, pl[:nplanes, nl // 64 - n // 64:].copy(), n, threads=threads)
    if r2:
        enc ^= pl[:nplanes, :n // 64]
    t_qc = (time.perf_counter() - t0) * (128 / nplanes) * 2  # both roles
    el = t_pprf + t_qc
    return n / el, f"both roles PPRF on all {t_full} trees; QC encode timed on {nplanes} of 128 planes (one role) and scaled x{128 / nplanes * 2:g}"


class CpuMix:
    """The CPU path on the batched mix's own instances (the shapes the GPU
    arm runs, `mixed_shapes` with the same seed), every instance sampled and
    scaled to its full size.  `time_step()` times one pass and returns the
    estimated COTs/s of the whole mix on `threads` host threads.

    Work units, run as independent jobs on a pool of `threads` host threads
    (each job single-threaded, so all cores are busy while any job is timed):
      * Ferret-style instance: both roles of min(t, sample_trees) trees and
        the LPN of their rows on both roles, with the instance's own k;
        scaled by t / trees.  The reference's own emp-ot code does this
        (SPCOT_Sender / SPCOT_Recver::compute, LpnF2::task, compiled from
        its headers into oracle/_ref/libempref.so); without that library the
        oracle's restatement does.
      * SOT instance: the PPRF of both roles on the same tree sample plus the
        two transposes of its rows, scaled by t / trees; and the exact QC
        product of one bit plane of the instance's own n, scaled by 256 (128
        planes x 2 roles).  The reference has no CPU SOT code, so these run
        on the oracle's restatement.
    The step time is then sum(job time x scale) / threads: the mix spread
    over every host thread, each unit costing what it cost with all threads
    busy."""

    def __init__(self, spec: dict, threads: int, seed: int = 2024, sample_trees: int = 8):
        import oracle
        from cuot_b200.batch import mixed_shapes  # the workload's shapes only; no device code
        self.threads = threads
        self.shapes = mixed_shapes(spec["count"], seed, spec["lo"], spec["hi"])
        self.use_ref = oracle.emp_lib() is not None
        self.jobs = self._jobs(seed, sample_trees)
        fer_code = ("the reference's own emp-ot code (oracle/_ref/libempref.so)" if self.use_ref
                    else "the oracle's restatement")
        self.sample = (
            f"all {len(self.shapes)} instances of the mix (seed {seed}), each sampled and scaled: Ferret-style: both "
            f"roles of {sample_trees} trees (or all, if fewer) + LPN of their rows on both roles, by {fer_code}, "
            f"x t/trees; SOT (oracle restatement; the reference has no CPU SOT code): PPRF both roles + "
            f"transposes on the same tree sample x t/trees, one bit plane's exact QC product of the instance's "
            f"own n x 256; step time = sum of job times / {threads} threads, jobs run {threads} at a time")
        # "reference" only when every leg runs the reference's own code; the
        # SOT legs never do
        self.kind = "port"

    def _jobs(self, seed: int, sample_trees: int):
        import oracle
        from cuot_b200.batch import KIND_FERRET
        use_ref = self.use_ref
        rng = np.random.default_rng(seed)
        blk = lambda m: rng.integers(0, 256, (m, 16), dtype=np.uint8)
        jobs = []  # (fn, scale)
        for kind, t, h, k in self.shapes:
            n, ts = t << h, min(t, sample_trees)
            roots, delta = blk(ts), blk(1)[0]
            delta[0] |= 1
            ch = rng.integers(0, 2, ts * h).astype(np.uint8)
            if kind == KIND_FERRET:
                kk, seed_b = blk(k), blk(1)[0]

                def fer(roots=roots, h=h, delta=delta, ch=ch, kk=kk, seed_b=seed_b):
                    if use_ref:
                        ls, lr = oracle.emp_mpcot_trees(roots, h, delta, ch)
                        oracle.emp_lpn_task(seed_b, kk, ls, inplace=True)
                        oracle.emp_lpn_task(seed_b, kk, lr, inplace=True)
                    else:
                        lv, lsum, rsum, ss = oracle.ferret_pprf_sender(roots, h, delta)
                        rl = oracle.ferret_pprf_recver(np.where(ch[:, None] == 0, lsum, rsum), ch, ss, h)
                        oracle.lpn_primal(seed_b, kk, lv)
                        oracle.lpn_primal(seed_b, kk, rl)
                jobs.append((fer, t / ts))
            else:
                b0, b1 = blk(h * ts), blk(h * ts)
                chs = rng.integers(0, 2, h * ts).astype(np.uint8)
                mc = np.where(chs[:, None] == 0, b0, b1)
                a = oracle.qc_gen_a(blk(1)[0], n)
                plane = rng.integers(0, 2**63, (1, n // 64), dtype=np.uint64)

                def sot_pprf(roots=roots, h=h, delta=delta, b0=b0, b1=b1, mc=mc, chs=chs, ts=ts):
                    lv, m0, m1 = oracle.sot_pprf_sender(roots, h, delta, b0, b1)
                    rl = oracle.sot_pprf_recver(m0, m1, mc, chs, ts, h)
                    rows = ts << h
                    for lvs in (lv, rl):
                        pl = oracle.bit_transpose(lvs, rows, 16, 0, 128)
                        oracle.bit_transpose(pl, 128, rows // 8, 0, rows)

                def sot_qc(a=a, plane=plane, n=n):
                    oracle.qc_encode(a, plane, n)
                jobs.append((sot_pprf, t / ts))
                jobs.append((sot_qc, 256.0))
        return jobs

    def time_step(self) -> float:
        import concurrent.futures as cf

        def timed(job):
            t0 = time.perf_counter()
            job[0]()
            return (time.perf_counter() - t0) * job[1]

        with cf.ThreadPoolExecutor(max_workers=self.threads) as pool:
            # the 256-scaled plane jobs (the longest) first, so the pool drains evenly
            order = sorted(range(len(self.jobs)), key=lambda j: -self.jobs[j][1])
            total = sum(pool.map(lambda j: timed(self.jobs[j]), order))
        return sum(t << h for _, t, h, _ in self.shapes) / (total / self.threads)


def reference_gpu_context(workload: str, pprf_ms: float, lpn_ms: float, reps: int = 5):
    """Speed context only: the reference's own GPU path rebuilt for sm_100a
    (oracle/_ref/librefgpu.so) on this workload's shape, beside this
    library's stage times.  The reference calls are its blocking API
    (dev_layer.h's cuda_mpcot_sender and cuda_primal_lpn, with their own host
    copies; SOTSender::dual_lpn's transpose + cuFFT encode + transpose),
    timed per role; their outputs are not bit-exact (non-FIPS AES schedule,
    racy level sums, float FFT), so this is not a parity baseline.  None
    when the library was not built or the shape is outside the reference
    kernels' safe range."""
    import oracle
    L = oracle.refgpu_lib()
    spec = WORKLOADS[workload]
    if L is None or spec["kind"] not in ("ferret", "sot") or spec.get("r2") or spec.get("mal"):
        return None
    t, h = spec["t"], spec["h"]
    n = t << h
    if spec["kind"] == "ferret":
        if n % 2048 or n > (1 << 22):
            return None
        snd = L.ref_gpu_mpcot_sender_ms(t, h, reps)
        lpn = L.ref_gpu_primal_lpn_ms(n, spec["k"], reps)
        if snd <= 0 or lpn <= 0:
            return None
        return {"what": "reference cuda_mpcot_sender and cuda_primal_lpn (dev_layer.cu), per role, blocking, "
                        "host copies included; sm_100a -O2",
                "mpcot_sender_ms_per_role": snd, "primal_lpn_ms_per_role": lpn,
                "ours_pprf_ms_per_role": pprf_ms / 2, "ours_lpn_ms_per_role": lpn_ms / 2,
                "note": "ours: device time of the stage (both roles) halved; the reference receiver "
                        "(cuda_mpcot_recver) is not run"}
    if n < (1 << 17) or n > (1 << 23):
        return None
    dl = L.ref_gpu_sot_dual_lpn_ms(n, reps)
    if dl <= 0:
        return None
    return {"what": "reference SOTSender::dual_lpn content (Mat::bit_transpose, QuasiCyclic::encode_dense with "
                    "cuFFT, Mat::bit_transpose), one role, sm_100a -O2",
            "dual_lpn_ms_per_role": dl, "ours_dual_lpn_ms_per_role": lpn_ms / 2,
            "note": "speed context only: the reference's float encode is not exact (57-64 % of its output bits "
                    "differ from a * b mod (x^n - 1) with its own a at n = 2^17 .. 2^22)"}


# --------------------------------------------------------------------------
def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    name = args.workload
    if rank != 0:
        return 0
    threads = os.cpu_count() or 1
    vals = []
    sample = ""
    spec = WORKLOADS[name]
    kind = "port"
    mix = CpuMix(spec, threads) if spec["kind"] == "batch" else None
    for i in range(args.warmup + args.steps):
        if mix is not None:
            v, sample, kind = mix.time_step(), mix.sample, mix.kind
        elif spec["kind"] == "session":
            v, sample = cpu_sample("ferret_b13", threads, budget_s=5.0)
            v *= (spec["t"] << spec["h"]) - (spec["k"] + spec["t"] * spec["h"] + 128)
            v /= spec["t"] << spec["h"]
            sample += "; usable COTs (ot_limit / n of the outputs)"
        else:
            v, sample = cpu_sample(name, threads, budget_s=5.0)
        if spec["kind"] in ("ferret", "session"):
            kind = "reference" if ref_ferret_available() else "port"
        if i >= args.warmup:
            vals.append(v)
    v = statistics.median(vals)
    unit = "COTs/s"
    print(json.dumps({
        "impl": "reference", "metric": metric_name(name), "value": v, "unit": unit,
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u8", "data": "synthetic (seeded)",
        "config": {"workload": name, "what": CONFIG_TEXT[name]},
        "cpu_baseline": {"value": v, "unit": unit, "cores": threads, "kind": kind, "sample": sample},
        "e2e": {"value": v, "unit": unit, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "reference CPU path on all host threads: Ferret GGM/LPN by the reference's own emp-ot headers "
                "(spcot_sender.h, spcot_recver.h, lpn_f2.h) compiled over an emp-tool shim into "
                "oracle/_ref/libempref.so; SOT by the oracle's restatement (the reference has no CPU SOT code)",
    }), flush=True)
    return 0


def run_batch(args):
    """The mixed batch of instances, batched (graph) vs plain."""
    import torch
    import cuot_b200
    from cuot_b200.batch import KIND_FERRET, Batch, mixed_workload

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    spec = WORKLOADS[args.workload]
    ctx = new_context(cuot_b200, local)
    insts = mixed_workload(ctx, count=spec["count"], seed=2024 + rank, lo=spec["lo"], hi=spec["hi"])
    cots = sum(i.n for i in insts)
    stream = torch.cuda.Stream()
    tuned = {}
    if not args.no_autotune:
        from cuot_b200.autotune import TuningTable, tune_batch
        tuned, _ = tune_batch(ctx, insts, table=TuningTable())  # CUOT_TUNING_TABLE sets its path
    from cuot_b200.batch import SCHEDULES
    batch = Batch(ctx, insts, use_graph=True, schedule=SCHEDULES[args.batch_schedule], **tuned)
    for _ in range(args.warmup):
        batch.run(stream)
        batch.run_plain(stream)
    torch.cuda.synchronize()
    launches = batch.kernels_per_run()
    phases = batch.run_phases(stream)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")

    def timed(fn):
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        for i in range(args.steps):
            with torch.cuda.stream(stream):
                flush.zero_()
            evs[i][0].record(stream)
            fn(stream)
            evs[i][1].record(stream)
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        ms = sum(a.elapsed_time(b) for a, b in evs) / args.steps
        if dist:
            tt = torch.tensor([ms], device="cuda", dtype=torch.float64)
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
            ms = tt.item()
        return ms

    def timed_pipelined(fn, pipe):
        """Like timed(), but one event pair around all steps, closed after
        the last step's host copy (steps overlap, so per-step events would
        not bracket a step's own work)."""
        if dist:
            dist.barrier()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(args.steps):
            fn(stream)
        pipe.join()
        b.record(stream)
        torch.cuda.synchronize()
        if dist:
            dist.barrier()
        ms = a.elapsed_time(b) / args.steps
        if dist:
            tt = torch.tensor([ms], device="cuda", dtype=torch.float64)
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
            ms = tt.item()
        return ms

    clk = ClockSampler(local)
    clk.start()
    time.sleep(0.3)
    ms = timed(batch.run)
    clocks = clk.stop()
    ms_plain = timed(batch.run_plain)

    # e2e: inputs from pinned host memory, outputs back, through the public
    # API.  Two device input sets (a second batch over copies of the inputs,
    # same outputs): step j's input copy runs during step j-1.
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory()
    insts2 = [i.input_copy(own_outputs=True) for i in insts]
    batch2 = Batch(ctx, insts2, use_graph=True, schedule=SCHEDULES[args.batch_schedule], **tuned)
    batch2.run(stream)
    batches = [batch, batch2]
    host_in, host_out = [[], []], []
    # outputs in the order they become final (Ferret after the LPN, then the
    # SOT sizes largest first); each instance's copies wait for its own
    # completion point, so all but the last sizes reach the host during the
    # step that computes them
    order = sorted(range(len(insts)), key=batch.item_rank)
    ready = [[], []]
    for ix in order:
        i, i2 = insts[ix], insts2[ix]
        names = ["roots", "choice"] + (["kk_s", "kk_r"] if i.kind == KIND_FERRET else ["base0", "base1", "mc"])
        dev = {"roots": "d_roots", "choice": "d_choice", "kk_s": "d_kk_s", "kk_r": "d_kk_r",
               "base0": "d_b0", "base1": "d_b1", "mc": "d_mc"}
        for k in names:
            hs = pin(getattr(i, k))
            host_in[0].append((hs, getattr(i, dev[k])))
            host_in[1].append((hs, getattr(i2, dev[k])))
        outs = [(torch.empty_like(i.v, device="cpu").pin_memory(), i.v, i2.v),
                (torch.empty_like(i.w, device="cpu").pin_memory(), i.w, i2.w)]
        if i.kind != KIND_FERRET:
            outs.append((torch.empty_like(i.cbits, device="cpu").pin_memory(), i.cbits, i2.cbits))
        host_out += outs
        for slot in (0, 1):
            ready[slot] += [lambda cs, b=batches[slot], ix=ix: b.wait_item(ix, cs)] + [None] * (len(outs) - 1)
    h2d = sum(hs.numel() * hs.element_size() for hs, _ in host_in[0])
    d2h = sum(hs.numel() * hs.element_size() for hs, _, _ in host_out)

    # the host copy of step i overlaps step i+1's compute (HostPipeline); the
    # two batches write their own outputs, which go to the host directly
    from cuot_b200.pipeline import HostPipeline
    pipe = HostPipeline([[d0 for _, d0, _ in host_out], [d1 for _, _, d1 in host_out]], stream=stream,
                        input_sets=2, per_set_outputs=True)

    def run_flushed(st, slot):
        with torch.cuda.stream(st):
            flush.zero_()  # L2 flush between steps, as in the device-timed loop
        batches[slot].run(st)

    def e2e(st):
        slot = pipe.slot
        pipe.step(host_in[slot], lambda s: run_flushed(s, slot), [hs for hs, _, _ in host_out], ready[slot])

    e2e(stream)
    pipe.join()
    e2e_ms = timed_pipelined(e2e, pipe)

    names = ["pprf_send", "pprf_recv", "lpn", "sot_encode"]
    stages = dict(zip(names, phases))
    n_sot = sum(i.n for i in insts if i.kind != KIND_FERRET)
    n_fer = cots - n_sot
    k_fer = sum(i.k for i in insts if i.kind == KIND_FERRET)
    alg = {"pprf_send": 16 * cots, "pprf_recv": 16 * cots, "lpn": 2 * 32 * n_fer + 2 * 16 * k_fer,
           "sot_encode": 2 * 3 * 32 * n_sot}
    dom = max(stages, key=lambda k: stages[k])
    peaks, peak_kind = measured_peaks()
    achieved = alg[dom] / (stages[dom] / 1e3) / 1e9
    # traffic: the batch is too large for a multi-metric ncu capture; the SOT
    # encode runs the same kernels as the single-instance sot_n20 / sot_n22
    # lines (FFT up to 2^22, Karatsuba over 2^22 FFTs at 2^23 and 2^24, NTT
    # above), whose captured DRAM bytes per COT (both roles) scale it: the
    # 2^22 capture for the 1024 x 4096 split of 2^22 (and the Karatsuba
    # leaves), the 2^20 capture below; other stages have no capture (null)
    traffic = None
    if dom == "sot_encode":
        fft_cot = NCU_TRAFFIC_PER_STEP["sot_n20:dual_lpn"] / (1 << 20)  # FFT dual LPN, both roles
        fft22_cot = NCU_TRAFFIC_PER_STEP["sot_n22:dual_lpn"] / (1 << 22)
        ntt_cot = NCU_TRAFFIC_PER_STEP["sot_n20_ntt:dual_lpn"] / (1 << 20)
        traffic = 0.0
        for i in insts:
            if i.kind == KIND_FERRET:
                continue
            lg = i.n.bit_length() - 1
            leaves = qc_leaves(lg)
            per = fft22_cot if lg >= QC_FFT_MAX_LOG_N else fft_cot
            traffic += per * leaves * min(i.n, 1 << QC_FFT_MAX_LOG_N) if leaves else i.n * ntt_cot
    props = torch.cuda.get_device_properties(local)
    mhz = clocks.get("sm_mhz") or clocks.get("sm_max_mhz") or 1965.0
    aes_peak = props.multi_processor_count * 32 * mhz * 1e6 / 160
    aes_counts = {"pprf_send": sum(2 * i.t * ((1 << i.h) - 1) for i in insts),
                  "pprf_recv": sum(2 * i.t * ((1 << i.h) - 1) for i in insts),
                  "lpn": sum(i.n * i.d // 4 for i in insts if i.kind == KIND_FERRET)}  # once for both roles
    aes = {"peak_aes_per_s": aes_peak, "model": AES_PEAK_MODEL}
    for k, cnt in aes_counts.items():
        a = cnt / (stages[k] / 1e3)
        aes[k] = {"aes_per_step": cnt, "aes_per_s": a, "frac": a / aes_peak}
    fer_rows = sum(2 * i.n for i in insts if i.kind == KIND_FERRET and i.d == 10)
    if fer_rows and stages.get("lpn"):
        aes["lpn_l1_roofline"] = lpn_l1_roofline(fer_rows, 10, stages["lpn"], clocks, props)
    out = {
        "metric": metric_name(args.workload),
        "value": world * cots / (ms / 1e3), "unit": "COTs/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u8", "data": "synthetic (seeded)",
        "config": {"workload": args.workload, "what": CONFIG_TEXT[args.workload], "qc_backend": args.qc_backend,
                   "schedule": args.batch_schedule, "instances": len(insts),
                   "cots_per_step_per_gpu": cots, "parallelism": f"replicas x{world}",
                   "l2": "256 MiB buffer written between timed steps (L2 flush)"},
        "plain": {"value": world * cots / (ms_plain / 1e3), "ms_per_step": ms_plain,
                  "batched_over_plain": ms_plain / ms},
        "autotuned": tuned,
        "stages_ms": stages,
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                     "frac": achieved / peaks["hbm_gbs"], "traffic": traffic,
                     "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)",
                     "algorithmic_bytes_per_step": alg[dom],
                     "basis": "stage totals per step (both roles); traffic scaled from one-kernel ncu "
                              "captures of the single-instance lines (cold cache per kernel): n = 2^22 "
                              "(profiles/qc_fft_sot_n22.md) 3,921 DRAM bytes per COT for the 2^22 instances "
                              "and, 3^L times, the Karatsuba leaves; n = 2^20 (profiles/qc_fft_sot_n20.md) "
                              "2,757 per COT for smaller FFT sizes; 4,066 per COT for NTT sizes "
                              "(profiles/qc_ntt_sot_n20.md)"},
        "aes_roofline": aes,
        "qc_transform": qc_transform_report([i.n for i in insts if i.kind != KIND_FERRET], stages["sot_encode"],
                                            ctx.measure_fp64_tflops()),
        "e2e": {"value": world * cots / (e2e_ms / 1e3), "unit": "COTs/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h, "ms_per_step": e2e_ms,
                "method": "steps back to back through Batch.run with two device input/output sets; each "
                          "step's inputs copied from pinned host memory during the previous step, each "
                          "instance's outputs copied to pinned host memory from its completion point in the "
                          "step (Batch.wait_item: Ferret after the LPN, SOT sizes largest first); one event "
                          "pair around all steps, closed after the last step's copies"},
        "gpu_launches": launches * args.steps,
        "clocks": clocks,
    }
    if dom == "sot_encode" and fp64_roofline(out["qc_transform"]):
        out["roofline"]["fp64"] = fp64_roofline(out["qc_transform"])
    batch.close()
    batch2.close()
    if args.serve_requests > 0:
        out["served"] = run_served(args, local)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        mix = CpuMix(spec, threads, seed=2024 + rank)
        vals = [mix.time_step() for _ in range(3)]
        out["cpu_baseline"] = {"value": statistics.median(vals), "unit": "COTs/s", "cores": threads,
                               "kind": mix.kind, "sample": mix.sample + "; median of 3 passes"}
    if rank == 0:
        print(json.dumps(out), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def run_aes(args):
    """Diagnostic: the two AES-128 designs on the same data, CUDA events,
    the 1 GiB buffer larger than L2 (each kernel reads and writes it once)."""
    import torch
    import cuot_b200
    spec = WORKLOADS[args.workload]
    n = spec["n"]
    torch.cuda.set_device(0)
    ctx = new_context(cuot_b200, 0)
    key = np.arange(16, dtype=np.uint8)
    buf = torch.randint(0, 256, (n, 16), dtype=torch.uint8, device="cuda")
    res = {}
    clk = ClockSampler(0)
    clk.start()
    for name, fn in (("ttable", ctx.aes128_ecb), ("bitsliced", ctx.aes128_ecb_bitsliced)):
        for _ in range(args.warmup):
            fn(key, buf)
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        for _ in range(args.steps):
            fn(key, buf)
        b.record()
        b.synchronize()
        ms = a.elapsed_time(b) / args.steps
        res[name] = {"ms": ms, "aes_per_s": n / (ms / 1e3), "hbm_gbs": 32 * n / (ms / 1e3) / 1e9}
    clocks = clk.stop()
    out = {"metric": metric_name(args.workload), "value": res["ttable"]["aes_per_s"], "unit": "AES/s",
           "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": res["ttable"]["ms"],
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8",
           "data": "synthetic (random)", "config": {"workload": args.workload, "what": CONFIG_TEXT[args.workload],
                                                     "blocks": n},
           "aes": res, "bitsliced_over_ttable": res["bitsliced"]["aes_per_s"] / res["ttable"]["aes_per_s"],
           "clocks": clocks}
    print(json.dumps(out), flush=True)
    ctx.close()
    return 0


def run_served(args, device: int) -> dict:
    """The served request stream, by the continuous-batching server and by
    plain per-request execution (one request at a time), both under the
    same policy.  Saturation: the completion rate of a stream offered at
    three times the rate the servers can take (requests arrive faster than
    they finish, so the rate measures the server, not the arrivals).  The
    10,000-request stream is then offered at 70 % of the continuous server's
    saturation, a rate at which its queue stays bounded (see the
    --serve-sweep option), and served by both."""
    from cuot_b200.serve import Server, make_stream, saturation

    lo, hi = 14, 24
    # small requests (n < 2^20) on high-priority streams; at most one request
    # with n >= 2^22 in flight (a sweep of these two knobs on this workload:
    # this pair beat plain per-request execution on p50, p99 and mean)
    big_n, prio_n = 1 << 22, 1 << 20
    cont = Server(slots=args.serve_slots, device=device, max_log_n=hi, budget_bytes=120e9,
                  high_priority_below_n=prio_n)
    cont.configure(budget_bytes=120e9, big_n=big_n, high_priority_below_n=prio_n)
    plain = Server(slots=1, device=device, max_log_n=hi, budget_bytes=120e9)
    # a first estimate: every request of a probe present at t = 0 (its wall
    # time ends with the big requests, which run one at a time)
    n_probe = min(200, args.serve_requests)
    probe = saturation(cont, make_stream(n_probe, rate=0.0, seed=5, lo=lo, hi=hi))
    over_n = min(1000, max(n_probe, args.serve_requests))

    def overload(server):
        stream = make_stream(over_n, rate=3.0 * probe["req_per_s"], seed=8, lo=lo, hi=hi)
        r = server.run(stream)
        return {"req_per_s": r["done"] / r["wall_s"], "cots_per_s": r["cots_per_s"], "requests": r["done"],
                "wall_s": r["wall_s"], "offered_rps": 3.0 * probe["req_per_s"]}
    sat, sat_plain = overload(cont), overload(plain)
    rate = 0.7 * sat["req_per_s"]
    reqs = make_stream(args.serve_requests, rate=rate, seed=6, lo=lo, hi=hi)
    rep = cont.run(reqs)
    sweep = None
    if args.serve_sweep:
        # offered rate swept as fractions of the saturation throughput; a rate
        # is sustained while requests complete as fast as they arrive
        sweep = {"requests_per_rate": args.serve_sweep_requests, "points": []}
        for j, f in enumerate(float(x) for x in args.serve_sweep.split(",")):
            offered = f * sat["req_per_s"]
            stream = make_stream(args.serve_sweep_requests, rate=offered, seed=100 + j, lo=lo, hi=hi)
            r = cont.run(stream)
            arrived = max(q.arrival for q in stream)
            point = {"fraction_of_saturation": f, "offered_rps": offered,
                     "completed_rps": r["done"] / r["wall_s"], "p50_ms": r["p50_ms"], "p99_ms": r["p99_ms"],
                     "mean_ms": r["mean_ms"], "cots_per_s": r["cots_per_s"],
                     "backlog_s": r["wall_s"] - arrived}
            sweep["points"].append(point)
        ok = [p for p in sweep["points"] if p["completed_rps"] >= 0.95 * p["offered_rps"]]
        sweep["sustained_rps"] = max((p["offered_rps"] for p in ok), default=None)
    cont.close()
    rep_plain = plain.run(reqs)
    plain.close()
    keys = ("done", "cots_per_s", "p50_ms", "p99_ms", "mean_ms", "wall_s")
    return {"requests": args.serve_requests, "slots": args.serve_slots, "budget_gb": 120,
            "log2_n": [lo, hi], "rate_rps": rate,
            "policy": {"high_priority_below_n": prio_n, "max_in_flight_with_n_ge": [big_n, 1]},
            "saturation": {"method": f"completion rate of {over_n} requests offered at 3x the probe rate",
                           "continuous": sat, "plain_per_request": sat_plain,
                           "continuous_over_plain": sat["req_per_s"] / sat_plain["req_per_s"],
                           "probe_all_at_t0": probe},
            "continuous": {k: rep[k] for k in keys},
            "plain_per_request": {k: rep_plain[k] for k in keys},
            **({"rate_sweep": sweep} if sweep else {}),
            "note": "latency = arrival -> outputs in device memory; the stream is offered at 0.7 x the "
                    "continuous server's saturation; plain per-request execution serves the same stream"}


def run_session(args):
    """Ferret extension loop (FerretSession.extend_f2k) at ferret_b13
    parameters; one replica per rank."""
    import torch
    import cuot_b200
    from cuot_b200.ferret import FERRET_B13, FerretSession
    from cuot_b200.pipeline import HostPipeline

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    p = FERRET_B13
    st = torch.cuda.Stream()
    ctx = new_context(cuot_b200, local)
    sess = FerretSession(ctx, ctx, p, seed=b"bench-session-%d" % rank, stream=st)
    for _ in range(args.warmup):
        sess.extend_f2k()
    st.synchronize()
    before = cuot_b200.launch_count()
    sess.extend_f2k()
    st.synchronize()
    launches = cuot_b200.launch_count() - before
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    clk = ClockSampler(local)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clk.start()
    time.sleep(0.3)
    for i in range(args.steps):
        with torch.cuda.stream(st):
            flush.zero_()
        evs[i][0].record(st)
        sess.extend_f2k()
        evs[i][1].record(st)
    torch.cuda.synchronize()
    clocks = clk.stop()
    ms = sum(a.elapsed_time(b) for a, b in evs) / args.steps
    # e2e: every extension's usable COTs of both roles returned to pinned host
    # memory, overlapped with the next extension (the extension's inputs are
    # the previous extension's outputs, resident on the device)
    hv = torch.empty((p.ot_limit, 16), dtype=torch.uint8).pin_memory()
    hw = torch.empty((p.ot_limit, 16), dtype=torch.uint8).pin_memory()
    pipe = HostPipeline([sess.ot_s[:p.ot_limit], sess.ot_r[:p.ot_limit]], stream=st)
    pipe.step([], lambda s: sess.extend_f2k(), [hv, hw])
    pipe.join()
    st.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(st)
    for _ in range(args.steps):
        h2d, d2h = pipe.step([], lambda s: sess.extend_f2k(), [hv, hw])
    pipe.join()
    b.record(st)
    torch.cuda.synchronize()
    e2e_ms = a.elapsed_time(b) / args.steps
    if dist:
        tt = torch.tensor([ms, e2e_ms], device="cuda", dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        ms, e2e_ms = tt.tolist()
    peaks, peak_kind = measured_peaks()
    alg = 2 * (32 * p.n + 16 * p.k) + 2 * (16 * p.n + 32 * p.t * p.h)  # LPN + PPRF, both roles
    achieved = alg / (ms / 1e3) / 1e9
    out = {
        "metric": metric_name(args.workload), "value": world * p.ot_limit / (ms / 1e3), "unit": "COTs/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u8",
        "data": "synthetic (seeded)",
        "config": {"workload": args.workload, "what": CONFIG_TEXT[args.workload], "qc_backend": args.qc_backend, "usable_cots_per_step_per_gpu":
                   p.ot_limit, "parallelism": f"replicas x{world}",
                   "l2": "256 MiB buffer written between timed steps (L2 flush)"},
        "roofline": {"bound": "hbm", "kernel": "extension (PPRF + LPN, both roles)", "achieved": achieved,
                     "peak": peaks["hbm_gbs"], "unit": "GB/s", "frac": achieved / peaks["hbm_gbs"],
                     "traffic": None, "algorithmic_bytes_per_step": alg,
                     "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)"},
        "e2e": {"value": world * p.ot_limit / (e2e_ms / 1e3), "unit": "COTs/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h, "ms_per_step": e2e_ms},
        "gpu_launches": launches * args.steps,
        "clocks": clocks,
    }
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        v, sample = cpu_sample("ferret_b13", threads)
        out["cpu_baseline"] = {"value": v * p.ot_limit / p.n, "unit": "COTs/s", "cores": threads,
                               "kind": "reference" if ref_ferret_available() else "port",
                               "sample": sample + "; scaled by ot_limit / n"}
    if rank == 0:
        print(json.dumps(out), flush=True)
    del sess
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def run_ours(args):
    import torch
    import cuot_b200

    if WORKLOADS[args.workload]["kind"] == "batch":
        return run_batch(args)
    if WORKLOADS[args.workload]["kind"] == "session":
        return run_session(args)
    if WORKLOADS[args.workload]["kind"] == "aes":
        return run_aes(args)

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))

    inst = Instance(args.workload, 1234 + rank, torch, cuot_b200)
    n = inst.n
    # warm-up
    for _ in range(args.warmup):
        inst.step()
    torch.cuda.synchronize()
    launches = inst.launches_per_step()

    # L2 flush buffer (larger than the 126 MB L2), written between steps
    flush = torch.empty(256 << 20, dtype=torch.uint8, device="cuda")
    names = ["pprf0", "pprf1", "chi1", "lpn1"]
    step_ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    stage_ev = [{k: torch.cuda.Event(enable_timing=True) for k in names} for _ in range(args.steps)]
    clk = ClockSampler(local)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clk.start()
    time.sleep(0.3)
    for i in range(args.steps):
        flush.zero_()
        step_ev[i][0].record()
        inst.step(stage_ev[i])
        step_ev[i][1].record()
    torch.cuda.synchronize()
    if dist:
        dist.barrier()
    clocks = clk.stop()
    ms_steps = [a.elapsed_time(b) for a, b in step_ev]
    ms = sum(ms_steps) / len(ms_steps)
    pprf_ms = statistics.mean(e["pprf0"].elapsed_time(e["pprf1"]) for e in stage_ev)
    chi_ms = statistics.mean(e["pprf1"].elapsed_time(e["chi1"]) for e in stage_ev)
    lpn_ms = statistics.mean(e["chi1"].elapsed_time(e["lpn1"]) for e in stage_ev)
    if dist:
        tt = torch.tensor([ms, pprf_ms, chi_ms, lpn_ms], device="cuda", dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        ms, pprf_ms, chi_ms, lpn_ms = tt.tolist()
    value = world * n / (ms / 1e3)

    # e2e through the public API with pinned host buffers: every step's inputs
    # go host -> device and its outputs device -> host inside the timed
    # region; the host copy of step i overlaps step i+1's compute
    from cuot_b200.pipeline import HostPipeline
    host = make_host(inst)
    stream = torch.cuda.Stream()
    outs = e2e_outputs(inst, host)
    # two device input sets: step j's input copy runs during step j-1
    pipe = HostPipeline([d for d, _ in outs], stream=stream, input_sets=2)

    def compute(st, extra, slot):
        with torch.cuda.stream(st):
            flush.zero_()  # L2 flush between steps, as in the device-timed loop
        extra.append(e2e_compute(inst, host, st, slot))

    def e2e_one():
        extra = []
        slot = pipe.slot
        h2d, d2h = pipe.step(e2e_inputs(inst, host, slot), lambda st: compute(st, extra, slot),
                             [h for _, h in outs])
        return h2d, d2h + extra[0]
    for _ in range(max(1, args.warmup)):
        e2e_one()
    pipe.join()
    stream.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    if dist:
        dist.barrier()
    e0.record(stream)
    for _ in range(args.steps):
        h2d, d2h = e2e_one()
    pipe.join()
    e1.record(stream)
    stream.synchronize()
    e2e_ms = e0.elapsed_time(e1) / args.steps
    if dist:
        tt = torch.tensor([e2e_ms], device="cuda", dtype=torch.float64)
        dist.all_reduce(tt, op=dist.ReduceOp.MAX)
        e2e_ms = tt.item()

    # roofline of the dominant stage
    peaks, peak_kind = measured_peaks()
    if inst.spec["kind"] == "ferret":
        k = inst.k
        # LPN: algorithmic bytes per launch = 32n (e read + y write) + 16k (kk once); 2 launches / step
        lpn_bytes = 2 * (32 * n + 16 * k)
        pprf_bytes = 2 * (16 * n + 32 * inst.t * inst.h)
        stages = {"pprf": (pprf_ms, pprf_bytes), "lpn": (lpn_ms, lpn_bytes)}
        if inst.mal:
            stages["chi"] = (chi_ms, 2 * 16 * n)  # both roles read their n leaves
    else:
        # dual LPN per role: two transposes (32 B per block each way) + encode
        # planes in/out (32n); rate-1/2: 2n blocks in (64n), e0 XOR (48n), n out (32n)
        dual = 2 * (144 * n if inst.r2 else 3 * 32 * n)
        stages = {"pprf": (pprf_ms, 2 * (16 * inst.nleaves + 32 * inst.t * (inst.h + 1))),
                  "dual_lpn": (lpn_ms, dual)}
    dom = max(stages, key=lambda s: stages[s][0])
    dms, dbytes = stages[dom]
    achieved = dbytes / (dms / 1e3) / 1e9
    traffic = NCU_TRAFFIC_PER_STEP.get(f"{args.workload}:{dom}")
    out = {
        "metric": metric_name(args.workload),
        "value": value, "unit": "COTs/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "u8", "data": "synthetic (seeded)",
        "config": {"workload": args.workload, "what": CONFIG_TEXT[args.workload], "qc_backend": args.qc_backend, "cots_per_step_per_gpu": n,
                   "parallelism": f"replicas x{world} (independent instances per GPU)",
                   "l2": "256 MiB buffer written between timed steps (L2 flush)"},
        "stages_ms": {k: v[0] for k, v in stages.items()},
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peaks["hbm_gbs"],
                     "unit": "GB/s", "frac": achieved / peaks["hbm_gbs"], "traffic": traffic,
                     "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else "fallback",
                     "algorithmic_bytes_per_step": dbytes,
                     "basis": "stage totals per step (both roles): algorithmic bytes / stage time; "
                              "traffic = ncu DRAM bytes of the stage's kernels per step"},
        "e2e": {"value": world * n / (e2e_ms / 1e3), "unit": "COTs/s", "h2d_bytes_per_step": h2d,
                "d2h_bytes_per_step": d2h, "ms_per_step": e2e_ms},
        "gpu_launches": launches * args.steps,
        "clocks": clocks,
    }
    out["aes_roofline"] = aes_roofline(inst, stages, clocks, torch.cuda.get_device_properties(local))
    if inst.spec["kind"] == "sot":
        out["transpose"] = transpose_roofline(inst, flush, peaks, peak_kind)
    if inst.spec["kind"] == "sot":
        out["qc_transform"] = qc_transform_report([inst.n], lpn_ms, inst.sctx.measure_fp64_tflops())
        if dom == "dual_lpn" and fp64_roofline(out["qc_transform"]):
            out["roofline"]["fp64"] = fp64_roofline(out["qc_transform"])
    if rank == 0 and world == 1:
        rg = reference_gpu_context(args.workload, pprf_ms, lpn_ms)
        if rg:
            out["reference_gpu"] = rg
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        v, sample = cpu_sample(args.workload, threads)
        ref = inst.spec["kind"] == "ferret" and inst.spec["d"] == 10 and ref_ferret_available()
        out["cpu_baseline"] = {"value": v, "unit": "COTs/s", "cores": threads,
                               "kind": "reference" if ref else "port", "sample": sample}
    if rank == 0:
        print(json.dumps(out), flush=True)
    del inst
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="mixed64", choices=sorted(WORKLOADS))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--serve-requests", type=int, default=10000,
                    help="requests of the served stream reported with mixed64 (0: skip; the full served configuration is 10000)")
    ap.add_argument("--serve-slots", type=int, default=8)
    ap.add_argument("--serve-sweep", default="",
                    help="comma-separated fractions of the saturation rate to serve a stream at (continuous server)")
    ap.add_argument("--serve-sweep-requests", type=int, default=2000)
    ap.add_argument("--no-autotune", action="store_true")
    ap.add_argument("--batch-schedule", default="serial", choices=["serial", "fork_ferret", "fork_sizes"],
                    help="batched mix: one chain (default), the Ferret branch beside the SOT chain, or every SOT "
                         "size on its own stream too")
    ap.add_argument("--qc-backend", default="auto", choices=sorted(QC_BACKENDS),
                    help="transform of the exact QC encode (auto: fp64 FFT for n <= 2^22, Karatsuba over it for "
                         "dual LPNs at 2^23 and 2^24, NTT above)")
    args = ap.parse_args()
    global _qc_backend
    _qc_backend = QC_BACKENDS[args.qc_backend]
    if args.impl == "reference":
        if WORKLOADS[args.workload]["kind"] == "aes":
            print(json.dumps({"impl": "reference", "unavailable": "diagnostic workload without a reference CPU path"}))
            return 0
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
