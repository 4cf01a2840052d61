"""Ferret random-COT session with device-resident state: the bootstrap
instance and the rcot buffer loop of FerretCOT (ferret_cot.hpp) over the
engine's MPCOT and primal-LPN kernels.

Both parties live on one GPU and the transport between them is ideal: the
sender's per-level sums reach the receiver as the OT would deliver them (the
message selected by the receiver's pre-COT choice bit), the secret sums and
the LPN seed are handed over directly.  What stays faithful to the reference
is the data flow of one extension (ferret_cot.hpp:83-97, 99-106):

* an extension consumes M = k + t*h + 128 pre-COTs P: P[0, t*h) feed the
  MPCOT's OTs (OTPre over the pre-COTs, preot.h:26-48: the receiver's choice
  bit of OT i is LSB(P_recv[i])), and the LPN input kk is P[128, 128 + k)
  (`lpn->compute(ot_output, expSeed, ot_input + consist_check_cot_num)`);
* its n outputs split into ot_limit = n - M usable COTs and the last M,
  which become the next extension's pre-COTs (ferret_cot.hpp:102);
* set-up (ferret_cot.hpp:132-171) runs one bootstrap extension of the
  pre-parameters (n_pre, t_pre, h_pre, k_pre) on base COTs: t_pre*h_pre for
  its MPCOT and k_pre + 128 for its LPN; its n_pre outputs are the first
  pre-COT buffer;
* rcot(num) (ferret_cot.hpp:178-210) serves COTs from the current buffer and
  extends whenever it runs dry.

Outputs keep the correlation w = v ^ x * Delta with LSB(Delta) = 1 and
LSB(v) = 0 (ferret_cot.hpp:27-31; spcot_sender.h clears the leaves' LSB), so
the receiver's choice bit of every COT is LSB(w).

Base COTs come from an ideal dealer seeded by the session (the reference
produces them with IKNP, which is host protocol).  Host scalars (Delta, the
per-extension LPN seed) are derived from the session seed with SHA-256;
tree roots are drawn on the device with the AES-CTR PRG.
"""
from __future__ import annotations

import hashlib
from dataclasses import dataclass

CONSIST_CHECK_COT_NUM = 128  # mpcot_reg.h:44


@dataclass(frozen=True)
class PrimalLPNParameter:
    """constants.h:9-25: n = t * 2^h outputs, k LPN inputs, and the set-up
    instance (n_pre, t_pre, k_pre, h_pre)."""
    n: int
    t: int
    k: int
    h: int
    n_pre: int
    t_pre: int
    k_pre: int
    h_pre: int

    def __post_init__(self):
        if (self.n != self.t << self.h or self.n_pre != self.t_pre << self.h_pre
                or self.n_pre < self.k + self.t * self.h + CONSIST_CHECK_COT_NUM):
            raise ValueError("LPN parameter not matched")

    @property
    def M(self) -> int:
        """Pre-COTs one extension consumes (ferret_cot.hpp:80)."""
        return self.k + self.t * self.h + CONSIST_CHECK_COT_NUM

    @property
    def ot_limit(self) -> int:
        """Usable COTs per extension (ferret_cot.hpp:81)."""
        return self.n - self.M

    def buf_sz(self) -> int:
        return self.n - self.t * self.h - self.k - CONSIST_CHECK_COT_NUM


FERRET_B13 = PrimalLPNParameter(10485760, 1280, 452000, 13, 470016, 918, 32768, 9)
FERRET_B12 = PrimalLPNParameter(10268672, 2507, 238000, 12, 268800, 1050, 17384, 8)
FERRET_B11 = PrimalLPNParameter(10180608, 4971, 124000, 11, 178944, 699, 17384, 8)


def session_scalar(seed: bytes, label: str, index: int = 0) -> bytes:
    """16 bytes derived from the session seed (SHA-256 of seed, label, index)."""
    return hashlib.sha256(bytes(seed) + label.encode() + index.to_bytes(8, "little")).digest()[:16]


def session_delta(seed: bytes) -> bytes:
    """Delta with its LSB set (ferret_cot.hpp:27-31)."""
    d = bytearray(session_scalar(seed, "delta"))
    d[0] |= 1
    return bytes(d)


def chi_seeds(secret_sums) -> bytes:
    """Seeds of the per-tree consistency check: the first 16 bytes of
    SHA-256 over each tree's 16-byte secret sum (Hash::hash_once in
    spcot_sender.h:91-94), concatenated."""
    raw = bytes(secret_sums)
    return b"".join(hashlib.sha256(raw[i:i + 16]).digest()[:16] for i in range(0, len(raw), 16))


class FerretSession:
    """Both roles of a Ferret random-COT generator on one GPU.

    ctx_s / ctx_r: the sender's and the receiver's contexts (they may be the
    same object).  `seed`: 16+ bytes from which every random choice of the
    session is derived (reproducible).  After construction (set-up done),
    rcot(num) returns (v, w): num COTs of each role as (num, 16) uint8 device
    tensors."""

    def __init__(self, ctx_s, ctx_r, param: PrimalLPNParameter, seed: bytes, d: int = 10, stream=None):
        import torch
        self.torch = torch
        self.ctx_s, self.ctx_r = ctx_s, ctx_r
        self.p, self.seed, self.d = param, bytes(seed), d
        self.stream = stream
        self.delta = session_delta(self.seed)
        self.extensions = 0  # extensions run, the bootstrap included
        dev = torch.device("cuda", torch.cuda.current_device())
        self.dev = dev
        emp = lambda m: torch.empty((m, 16), dtype=torch.uint8, device=dev)
        p = param
        # current output buffer of each role (n blocks) and the pre-COTs (M)
        self.ot_s, self.ot_r = emp(p.n), emp(p.n)
        self.pre_s, self.pre_r = emp(p.M), emp(p.M)
        tmax = max(p.t, p.t_pre)
        thmax = max(p.t * p.h, p.t_pre * p.h_pre)
        self._roots = emp(tmax)
        self._lsum, self._rsum, self._mc = emp(thmax), emp(thmax), emp(thmax)
        self._ss = emp(tmax)
        self._setup()
        self.ot_used = p.ot_limit

    # -- one extension (ferret_cot.hpp:83-97) ------------------------------
    def _extend(self, n, t, h, k, mp_s, mp_r, kk_s, kk_r, out_s, out_r):
        torch = self.torch
        st = self.stream
        idx = self.extensions
        roots = self._roots[:t]
        self.ctx_s.prg_fill(session_scalar(self.seed, "roots", idx), roots, stream=st)
        lsum, rsum, ss, mc = self._lsum[:t * h], self._rsum[:t * h], self._ss[:t], self._mc[:t * h]
        self.ctx_s.ferret_pprf_sender(roots, h, self.delta, out_s, lsum, rsum, ss, stream=st)
        # OTs over the pre-COTs: choice bit i = LSB(mp_r[i]); the receiver gets
        # the sum its bit selects (preot.h:58-82)
        with torch.cuda.stream(st) if st is not None else _null():
            choice = (mp_r[:, 0] & 1).contiguous()
            torch.where(choice.view(-1, 1).bool(), rsum, lsum, out=mc)
        self.ctx_r.ferret_pprf_recver(mc, choice, ss, h, out_r, stream=st)
        lpn_seed = session_scalar(self.seed, "lpn", idx)
        self.ctx_s.lpn_primal(lpn_seed, kk_s, out_s, d=self.d, stream=st)
        self.ctx_r.lpn_primal(lpn_seed, kk_r, out_r, d=self.d, stream=st)
        self.extensions += 1

    def _setup(self):
        """Bootstrap (ferret_cot.hpp:150-170) on dealer base COTs."""
        torch, p = self.torch, self.p
        nb_mp, nb_data = p.t_pre * p.h_pre, p.k_pre + CONSIST_CHECK_COT_NUM
        base_s, base_r = self.base_cots(nb_mp + nb_data)
        emp = lambda m: torch.empty((m, 16), dtype=torch.uint8, device=self.dev)
        out_s, out_r = emp(p.n_pre), emp(p.n_pre)
        data_s, data_r = base_s[nb_mp:], base_r[nb_mp:]
        c = CONSIST_CHECK_COT_NUM
        self._extend(p.n_pre, p.t_pre, p.h_pre, p.k_pre, base_s[:nb_mp], base_r[:nb_mp],
                     data_s[c:c + p.k_pre], data_r[c:c + p.k_pre], out_s, out_r)
        self.pre_s.copy_(out_s[:p.M])
        self.pre_r.copy_(out_r[:p.M])

    def base_cots(self, count: int):
        """Ideal dealer: count COTs (v, w = v ^ x * Delta) with LSB(v) = 0."""
        torch = self.torch
        emp = lambda m: torch.empty((m, 16), dtype=torch.uint8, device=self.dev)
        v, x = emp(count), emp(count)
        self.ctx_s.prg_fill(session_scalar(self.seed, "base-v"), v, stream=self.stream)
        self.ctx_s.prg_fill(session_scalar(self.seed, "base-x"), x, stream=self.stream)
        with torch.cuda.stream(self.stream) if self.stream is not None else _null():
            v[:, 0] &= 0xFE
            dl = torch.frombuffer(bytearray(self.delta), dtype=torch.uint8).to(self.dev)
            w = torch.where((x[:, :1] & 1).bool(), v ^ dl, v)
        return v, w

    def extend_f2k(self):
        """One extension into the session buffer; its last M outputs become
        the next pre-COTs (ferret_cot.hpp:99-106)."""
        p = self.p
        c = CONSIST_CHECK_COT_NUM
        th = p.t * p.h
        self._extend(p.n, p.t, p.h, p.k, self.pre_s[:th], self.pre_r[:th],
                     self.pre_s[c:c + p.k], self.pre_r[c:c + p.k], self.ot_s, self.ot_r)
        with self.torch.cuda.stream(self.stream) if self.stream is not None else _null():
            self.pre_s.copy_(self.ot_s[p.ot_limit:])
            self.pre_r.copy_(self.ot_r[p.ot_limit:])
        self.ot_used = 0

    def silent_ot_left(self) -> int:
        return self.p.ot_limit - self.ot_used

    def rcot(self, num: int):
        """num random COTs of each role (ferret_cot.hpp:178-210)."""
        torch = self.torch
        emp = lambda m: torch.empty((m, 16), dtype=torch.uint8, device=self.dev)
        v, w = emp(num), emp(num)
        done = 0
        while done < num:
            if self.silent_ot_left() == 0:
                self.extend_f2k()
            take = min(num - done, self.silent_ot_left())
            a = self.ot_used
            with torch.cuda.stream(self.stream) if self.stream is not None else _null():
                v[done:done + take].copy_(self.ot_s[a:a + take])
                w[done:done + take].copy_(self.ot_r[a:a + take])
            self.ot_used += take
            done += take
        return v, w


class _null:
    def __enter__(self):
        return None

    def __exit__(self, *a):
        return False
