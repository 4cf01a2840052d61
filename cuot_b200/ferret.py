"""Ferret random-COT session with device-resident state: the bootstrap
instance and the rcot buffer loop of FerretCOT (ferret_cot.hpp), run by the
C session of the library (cuot_ferret_session_*, ferret_session.cu); this
module is its Python binding plus the parameter sets.

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
produces them with IKNP, which is host protocol).  Every random choice comes
from the AES-CTR stream (the cryptoTools PRNG) keyed by SHA-256 of the
caller's seed: block 0 = Delta (LSB set), blocks 1 and 2 seed the dealer's
COT values and choice bits, blocks 16 + 2e and 17 + 2e are the LPN seed and
the roots seed of extension e (e = 0 is the set-up).
"""
from __future__ import annotations

import ctypes
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


def session_key(seed: bytes) -> bytes:
    """The 16-byte AES key of a session: SHA-256 of the caller's seed."""
    return hashlib.sha256(bytes(seed)).digest()[:16]


def chi_seeds(secret_sums) -> bytes:
    """Seeds of the per-tree consistency check: the first 16 bytes of
    SHA-256 over each tree's 16-byte secret sum (Hash::hash_once in
    spcot_sender.h:91-94), concatenated."""
    raw = bytes(secret_sums)
    return b"".join(hashlib.sha256(raw[i:i + 16]).digest()[:16] for i in range(0, len(raw), 16))


class _Param(ctypes.Structure):
    _fields_ = [(f, ctypes.c_int64) for f in ("n", "t", "k", "log_bin_sz", "n_pre", "t_pre", "k_pre",
                                              "log_bin_sz_pre")]


class _State(ctypes.Structure):
    _fields_ = [("M", ctypes.c_int64), ("ot_limit", ctypes.c_int64), ("ot_used", ctypes.c_int64),
                ("extensions", ctypes.c_int64), ("delta", ctypes.c_uint32 * 4)]


class FerretSession:
    """Both roles of a Ferret random-COT generator on one GPU, over the C
    session (cuot_ferret_session_*, ferret_session.cu).

    ctx_s / ctx_r: the roles' contexts; both roles run on ctx_s's context and
    `stream` (the C session orders them).  `seed`: bytes from which every
    random choice of the session is derived (reproducible).  After
    construction (set-up done), rcot(num) returns (v, w): num COTs of each
    role as (num, 16) uint8 device tensors; ot_s / ot_r are the session's
    output buffers (n blocks each)."""

    def __init__(self, ctx_s, ctx_r, param: PrimalLPNParameter, seed: bytes, d: int = 10, stream=None):
        import torch
        from . import _check, _ptr, _stream
        self.torch, self._check, self._ptr = torch, _check, _ptr
        self.ctx = ctx_s
        self.p, self.seed, self.d = param, bytes(seed), d
        self.stream = stream
        self.dev = torch.device("cuda", torch.cuda.current_device())
        emp = lambda m: torch.empty((m, 16), dtype=torch.uint8, device=self.dev)
        self.ot_s, self.ot_r = emp(param.n), emp(param.n)
        pr = _Param(param.n, param.t, param.k, param.h, param.n_pre, param.t_pre, param.k_pre, param.h_pre)
        key = (ctypes.c_uint8 * 16).from_buffer_copy(session_key(self.seed))
        h = ctypes.c_void_p()
        self.lib = ctx_s.lib
        _check(self.lib.cuot_ferret_session_create(ctx_s.h, ctypes.byref(pr), key, ctypes.c_int(d), _ptr(self.ot_s),
                                                   _ptr(self.ot_r), _stream(stream), ctypes.byref(h)),
               "cuot_ferret_session_create")
        self.h = h

    def _state(self) -> _State:
        st = _State()
        self._check(self.lib.cuot_ferret_session_info(self.h, ctypes.byref(st)), "cuot_ferret_session_info")
        return st

    @property
    def extensions(self) -> int:
        return int(self._state().extensions)

    @property
    def ot_used(self) -> int:
        return int(self._state().ot_used)

    @property
    def delta(self) -> bytes:
        return bytes(bytearray(self._state().delta))

    def extend_f2k(self):
        """One extension into ot_s / ot_r (ferret_cot.hpp:99-106)."""
        self._check(self.lib.cuot_ferret_session_extend(self.h), "cuot_ferret_session_extend")

    def silent_ot_left(self) -> int:
        st = self._state()
        return int(st.ot_limit - st.ot_used)

    def rcot(self, num: int):
        """num random COTs of each role (ferret_cot.hpp:178-210)."""
        emp = lambda m: self.torch.empty((m, 16), dtype=self.torch.uint8, device=self.dev)
        v, w = emp(num), emp(num)
        self._check(self.lib.cuot_ferret_session_rcot(self.h, ctypes.c_int64(num), self._ptr(v), self._ptr(w)),
                    "cuot_ferret_session_rcot")
        return v, w

    def close(self):
        if getattr(self, "h", None):
            self.lib.cuot_ferret_session_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
