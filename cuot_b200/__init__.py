"""cuot_b200 -- Python binding of libcuot, a B200 (sm_100a) silent-OT engine.

Thin ctypes layer over the C ABI declared in include/cuot.h.  Tensors are
torch CUDA tensors (torch is used only for device memory and streams); blocks
are uint8 tensors of shape (..., 16) with emp-tool's `block` memory image, bit
vectors are uint64 tensors.  Every call runs on the given (or current) CUDA
stream and raises CuotError on a non-zero status.  There is no CPU fallback:
importing on a machine without the built library raises.
"""
from __future__ import annotations

import ctypes
import os
import re

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libcuot.so")
HEADER = os.path.join(os.path.dirname(_HERE), "include", "cuot.h")

_lib = None


class CuotError(RuntimeError):
    def __init__(self, status: int, where: str):
        lib = load()
        msg = lib.cuot_status_string(status).decode()
        detail = lib.cuot_last_error().decode()
        super().__init__(f"{where}: {msg} ({status}) {detail}")
        self.status = status


def load() -> ctypes.CDLL:
    """Loads libcuot.so (in-tree).  Raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} not built; run `python -m cuot_b200.build`")
        lib = ctypes.CDLL(LIB_PATH)
        lib.cuot_status_string.restype = ctypes.c_char_p
        lib.cuot_last_error.restype = ctypes.c_char_p
        lib.cuot_version.restype = ctypes.c_char_p
        lib.cuot_ctx_scratch_bytes.restype = ctypes.c_uint64
        lib.cuot_launch_count.restype = ctypes.c_ulonglong
        _lib = lib
    return _lib


def launch_count() -> int:
    """Kernels launched by libcuot so far in this process."""
    return int(load().cuot_launch_count())


def declared_symbols() -> list[str]:
    """Every function name declared in include/cuot.h."""
    txt = open(HEADER).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(cuot_[a-z0-9_]+)\s*\(", txt)))


def copy_to_host(src, dst, stream=None):
    """Device tensor -> pinned host tensor through SM stores
    (cuot_copy_to_host): does not queue behind copy-engine transfers."""
    if not src.is_cuda or dst.is_cuda or not dst.is_pinned():
        raise ValueError("expected a CUDA source and a pinned host destination")
    nbytes = src.numel() * src.element_size()
    if dst.numel() * dst.element_size() < nbytes or not src.is_contiguous() or not dst.is_contiguous():
        raise ValueError("destination too small or not contiguous")
    _check(load().cuot_copy_to_host(ctypes.c_void_p(src.data_ptr()), ctypes.c_void_p(dst.data_ptr()),
                                    ctypes.c_uint64(nbytes), _stream(stream)), "cuot_copy_to_host")


def _check(status: int, where: str):
    if status != 0:
        raise CuotError(status, where)


def _ptr(t) -> ctypes.c_void_p:
    if t is None:
        return ctypes.c_void_p(0)
    if not t.is_cuda:
        raise ValueError("expected a CUDA tensor")
    if not t.is_contiguous():
        raise ValueError("expected a contiguous tensor")
    return ctypes.c_void_p(t.data_ptr())


def _stream(stream):
    import torch
    s = stream if stream is not None else torch.cuda.current_stream()
    return ctypes.c_void_p(s.cuda_stream)


def _host_block(b) -> ctypes.Array:
    import numpy as np
    if hasattr(b, "cpu"):
        b = b.cpu().numpy()
    arr = np.ascontiguousarray(np.frombuffer(bytes(b), np.uint8) if isinstance(b, (bytes, bytearray)) else np.asarray(b, np.uint8)).reshape(-1)
    assert arr.size == 16
    return (ctypes.c_uint8 * 16).from_buffer_copy(arr.tobytes())


def _nblocks(t) -> int:
    return t.numel() * t.element_size() // 16


C = ctypes


class Context:
    """A libcuot context on one CUDA device (AES tables + scratch arena)."""

    def __init__(self, device: int = 0):
        self.lib = load()
        self.device = device
        h = ctypes.c_void_p()
        _check(self.lib.cuot_ctx_create(C.c_int(device), C.byref(h)), "cuot_ctx_create")
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            self.lib.cuot_ctx_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def reserve(self, nbytes: int):
        _check(self.lib.cuot_ctx_reserve(self.h, C.c_uint64(nbytes)), "cuot_ctx_reserve")

    def scratch_bytes(self) -> int:
        return int(self.lib.cuot_ctx_scratch_bytes(self.h))

    TUNE_PPRF_THREADS, TUNE_QC_PLANES, TUNE_QC_BACKEND, TUNE_QC_STREAMS = 1, 2, 3, 4
    TUNE_QC_RECORD_MARGIN = 5

    def set_tuning(self, key: int, value: int):
        _check(self.lib.cuot_ctx_set_tuning(self.h, C.c_int(key), C.c_int64(value)), "cuot_ctx_set_tuning")

    def qc_fft_margin(self, reset: bool = True) -> float:
        """Largest |v - round(v)| rounded by this context's fp64 FFT encodes
        since recording was switched on (TUNE_QC_RECORD_MARGIN) or last reset."""
        v = C.c_double()
        _check(self.lib.cuot_qc_fft_margin(self.h, C.byref(v), C.c_int(int(reset))), "cuot_qc_fft_margin")
        return v.value

    def measure_fp64_tflops(self, reps: int = 5) -> float:
        """The device's fp64 FMA rate in TFLOP/s (independent FMA chains at
        full occupancy, best of `reps` launches; synchronises)."""
        v = C.c_double()
        _check(self.lib.cuot_measure_fp64_tflops(self.h, C.c_int(reps), C.byref(v)), "cuot_measure_fp64_tflops")
        return v.value

    # ---- AES ---------------------------------------------------------------
    def aes128_ecb(self, key, io, stream=None):
        _check(self.lib.cuot_aes128_ecb(self.h, _host_block(key), _ptr(io), C.c_uint64(_nblocks(io)),
                                        _stream(stream)), "cuot_aes128_ecb")
        return io

    def aes128_ecb_bitsliced(self, key, io, stream=None):
        _check(self.lib.cuot_aes128_ecb_bitsliced(self.h, _host_block(key), _ptr(io), C.c_uint64(_nblocks(io)),
                                                  _stream(stream)), "cuot_aes128_ecb_bitsliced")
        return io

    def prg_fill(self, seed, out, block_offset: int = 0, stream=None):
        _check(self.lib.cuot_prg_fill(self.h, _host_block(seed), C.c_uint64(block_offset), _ptr(out),
                                      C.c_uint64(_nblocks(out)), _stream(stream)), "cuot_prg_fill")
        return out

    # ---- Ferret ------------------------------------------------------------
    def ferret_chi_sum(self, leaves, h: int, seeds, out, stream=None):
        """Per-tree GF(2^128) check values sum_i seed^(i+1) * leaf_i."""
        t = _nblocks(seeds)
        _check(self.lib.cuot_ferret_chi_sum(self.h, _ptr(leaves), C.c_uint64(t), C.c_int(h), _ptr(seeds),
                                            _ptr(out), _stream(stream)), "cuot_ferret_chi_sum")

    def ferret_pprf_sender(self, roots, h: int, delta, leaves, lsum, rsum, secret_sum, stream=None):
        t = _nblocks(roots)
        _check(self.lib.cuot_ferret_pprf_sender(self.h, _ptr(roots), C.c_uint64(t), C.c_int(h),
                                                _host_block(delta), _ptr(leaves), _ptr(lsum), _ptr(rsum),
                                                _ptr(secret_sum), _stream(stream)),
               "cuot_ferret_pprf_sender")

    def ferret_pprf_recver(self, mc, choice, secret_sum, h: int, leaves, stream=None):
        t = _nblocks(secret_sum)
        _check(self.lib.cuot_ferret_pprf_recver(self.h, _ptr(mc), _ptr(choice), _ptr(secret_sum),
                                                C.c_uint64(t), C.c_int(h), _ptr(leaves), _stream(stream)),
               "cuot_ferret_pprf_recver")

    def lpn_primal(self, seed, kk, e_io, d: int = 10, stream=None):
        _check(self.lib.cuot_lpn_primal(self.h, _host_block(seed), _ptr(kk), C.c_int64(_nblocks(kk)),
                                        C.c_int(d), _ptr(e_io), C.c_int64(_nblocks(e_io)), _stream(stream)),
               "cuot_lpn_primal")

    def lpn_primal_dual(self, seed, kk_send, kk_recv, e_send, e_recv, d: int = 10, stream=None):
        """Both roles' LPN of one extension (same seed) in one launch: the
        public index matrix is generated once for the two."""
        n = _nblocks(e_send)
        if _nblocks(e_recv) != n or _nblocks(kk_recv) != _nblocks(kk_send):
            raise ValueError("the two roles need equal row and kk counts")
        _check(self.lib.cuot_lpn_primal_dual(self.h, _host_block(seed), _ptr(kk_send), _ptr(kk_recv),
                                             C.c_int64(_nblocks(kk_send)), C.c_int(d), _ptr(e_send), _ptr(e_recv),
                                             C.c_int64(n), _stream(stream)), "cuot_lpn_primal_dual")

    def lpn_primal_range(self, seed, kk, e_rows, row_lo: int, row_hi: int, n: int, d: int = 10, stream=None):
        _check(self.lib.cuot_lpn_primal_range(self.h, _host_block(seed), _ptr(kk), C.c_int64(_nblocks(kk)),
                                              C.c_int(d), _ptr(e_rows), C.c_int64(row_lo), C.c_int64(row_hi),
                                              C.c_int64(n), _stream(stream)), "cuot_lpn_primal_range")

    # ---- SOT ---------------------------------------------------------------
    def sot_pprf_sender(self, roots, h: int, delta, base0, base1, leaves, m0, m1, stream=None):
        t = _nblocks(roots)
        _check(self.lib.cuot_sot_pprf_sender(self.h, _ptr(roots), C.c_uint64(t), C.c_int(h),
                                             _host_block(delta), _ptr(base0), _ptr(base1), _ptr(leaves),
                                             _ptr(m0), _ptr(m1), _stream(stream)), "cuot_sot_pprf_sender")

    def sot_pprf_recver(self, m0, m1, mc, choice, t: int, h: int, leaves, stream=None):
        _check(self.lib.cuot_sot_pprf_recver(self.h, _ptr(m0), _ptr(m1), _ptr(mc), _ptr(choice),
                                             C.c_uint64(t), C.c_int(h), _ptr(leaves), _stream(stream)),
               "cuot_sot_pprf_recver")

    def bit_transpose(self, inp, rows: int, row_bytes: int, col_lo: int, col_hi: int, out, stream=None):
        _check(self.lib.cuot_bit_transpose(self.h, _ptr(inp), C.c_uint64(rows), C.c_uint64(row_bytes),
                                           C.c_uint64(col_lo), C.c_uint64(col_hi), _ptr(out), _stream(stream)),
               "cuot_bit_transpose")

    def qc_gen_a(self, key, n: int, a_out, stream=None):
        _check(self.lib.cuot_qc_gen_a(self.h, _host_block(key), C.c_uint64(n), _ptr(a_out), _stream(stream)),
               "cuot_qc_gen_a")

    def qc_encode(self, a, planes, n: int, nplanes: int, stream=None):
        _check(self.lib.cuot_qc_encode(self.h, _ptr(a), _ptr(planes), C.c_uint64(n), C.c_int(nplanes),
                                       _stream(stream)), "cuot_qc_encode")

    def qc_encode_sparse(self, a, pos, n: int, out, stream=None):
        _check(self.lib.cuot_qc_encode_sparse(self.h, _ptr(a), _ptr(pos), C.c_int(pos.numel()), C.c_uint64(n),
                                              _ptr(out), _stream(stream)), "cuot_qc_encode_sparse")

    def sot_dual_lpn(self, a, io, n: int, stream=None):
        _check(self.lib.cuot_sot_dual_lpn(self.h, _ptr(a), _ptr(io), C.c_uint64(n), _stream(stream)),
               "cuot_sot_dual_lpn")

    def sot_dual_lpn_r2(self, a, inp, n: int, out, stream=None):
        """Rate-1/2 form: out[:n] = inp[:n] ^ (a * inp[n:2n]) per bit plane."""
        _check(self.lib.cuot_sot_dual_lpn_r2(self.h, _ptr(a), _ptr(inp), C.c_uint64(n), _ptr(out),
                                             _stream(stream)), "cuot_sot_dual_lpn_r2")

    def qc_encode_sparse_r2(self, a, pos, n: int, out, stream=None):
        _check(self.lib.cuot_qc_encode_sparse_r2(self.h, _ptr(a), _ptr(pos), C.c_int(pos.numel()), C.c_uint64(n),
                                                 _ptr(out), _stream(stream)), "cuot_qc_encode_sparse_r2")

    def qc_plan(self, a, n: int, stream=None) -> "QcPlan":
        return QcPlan(self, a, n, stream)


class QcPlan:
    """Counterpart of cuOT's QuasiCyclic object: `a` transformed once."""

    def __init__(self, ctx: Context, a, n: int, stream=None):
        self.ctx, self.n = ctx, n
        h = ctypes.c_void_p()
        _check(ctx.lib.cuot_qc_plan_create(ctx.h, _ptr(a), C.c_uint64(n), _stream(stream), C.byref(h)),
               "cuot_qc_plan_create")
        self.h = h

    def set_batch(self, planes: int):
        _check(self.ctx.lib.cuot_qc_plan_set_batch(self.h, C.c_int(planes)), "cuot_qc_plan_set_batch")

    def encode(self, planes, nplanes: int, stream=None):
        _check(self.ctx.lib.cuot_qc_plan_encode(self.h, _ptr(planes), C.c_int(nplanes), _stream(stream)),
               "cuot_qc_plan_encode")

    def dual_lpn(self, io, stream=None):
        _check(self.ctx.lib.cuot_qc_plan_dual_lpn(self.h, _ptr(io), _stream(stream)), "cuot_qc_plan_dual_lpn")

    def dual_lpn_r2(self, inp, out, stream=None):
        _check(self.ctx.lib.cuot_qc_plan_dual_lpn_r2(self.h, _ptr(inp), _ptr(out), _stream(stream)),
               "cuot_qc_plan_dual_lpn_r2")

    def close(self):
        if getattr(self, "h", None):
            self.ctx.lib.cuot_qc_plan_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
