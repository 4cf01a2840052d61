"""CPU oracle for the silent-OT hot path -- TEST INFRASTRUCTURE ONLY.

Loaded by tests/, by __graft_entry__.smoke() and by bench.py's CPU-baseline
and reference legs as the checker.  The product (cuot_b200, libcuot.so) never
imports this package.  Arrays are numpy; blocks are uint8 arrays of shape
(..., 16) with the memory image of emp-tool's `block`.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None
_REF = None


def lib() -> ctypes.CDLL:
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "liboracle.so")
        if not os.path.exists(path):
            import subprocess
            subprocess.check_call(["make", "-s", "-C", _HERE])
        _LIB = ctypes.CDLL(path)
    return _LIB


def ref_lib():
    """oracle/_ref/libctref.so (reference cryptoTools, built from the
    reference sources) or None when it was not built."""
    global _REF
    if _REF is None:
        path = os.path.join(_HERE, "_ref", "libctref.so")
        if not os.path.exists(path):
            return None
        _REF = ctypes.CDLL(path)
    return _REF


_EMP = None


def emp_lib():
    """oracle/_ref/libempref.so: the reference's own emp-ot Ferret headers
    (twokeyprp.h, spcot_sender.h, spcot_recver.h, lpn_f2.h) compiled from the
    reference tree over the emp-tool shim (oracle/emp_shim), or None when it
    was not built."""
    global _EMP
    if _EMP is None:
        path = os.path.join(_HERE, "_ref", "libempref.so")
        if not os.path.exists(path):
            return None
        _EMP = ctypes.CDLL(path)
        _EMP.ref_lpn_task.argtypes = [C.c_void_p, C.c_void_p, C.c_int, C.c_int, C.c_void_p,
                                      C.c_int64, C.c_int64, C.c_int64]
    return _EMP


_REFGPU = None


def refgpu_lib():
    """oracle/_ref/librefgpu.so: the reference's own GPU path (gpu/*.cu,
    dev_layer.cu, silent/quasi_cyclic.cu) for sm_100a with a timing and
    transpose harness (oracle/ref_gpu_driver.cu), or None when it was not
    built.  Speed context and the transpose pin only: its other outputs are
    not the oracle's semantics."""
    global _REFGPU
    if _REFGPU is None:
        path = os.path.join(_HERE, "_ref", "librefgpu.so")
        if not os.path.exists(path):
            return None
        try:
            L = ctypes.CDLL(path)
        except OSError:  # no CUDA driver on this host (libcuda.so.1)
            return None
        L.ref_gpu_mpcot_sender_ms.restype = C.c_double
        L.ref_gpu_mpcot_sender_ms.argtypes = [C.c_int, C.c_int, C.c_int]
        L.ref_gpu_primal_lpn_ms.restype = C.c_double
        L.ref_gpu_primal_lpn_ms.argtypes = [C.c_int64, C.c_int, C.c_int]
        L.ref_gpu_sot_dual_lpn_ms.restype = C.c_double
        L.ref_gpu_sot_dual_lpn_ms.argtypes = [C.c_uint64, C.c_int]
        L.ref_gpu_bit_transpose.argtypes = [C.c_void_p, C.c_uint64, C.c_void_p]
        L.ref_gpu_mpcot_sender_leaves.argtypes = [C.c_int, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p]
        L.ref_gpu_primal_lpn_run.argtypes = [C.c_int64, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p,
                                             C.c_void_p]
        L.ref_gpu_qc_encode.argtypes = [C.c_uint64, C.c_uint, C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p]
        _REFGPU = L
    return _REFGPU


def refgpu_bit_transpose(blocks: np.ndarray) -> np.ndarray:
    """The reference's Mat::bit_transpose of n one-block rows (n a multiple
    of 256, at most 2^23): 128 planes of n/8 bytes."""
    inp = np.ascontiguousarray(blocks, np.uint8).reshape(-1, 16)
    n = inp.shape[0]
    out = np.empty((128, n // 8), np.uint8)
    rc = refgpu_lib().ref_gpu_bit_transpose(_p(inp), n, _p(out))
    assert rc == 0, f"ref_gpu_bit_transpose rejected n={n} ({rc})"
    return out


def refgpu_mpcot_sender_leaves(roots: np.ndarray, h: int, delta) -> np.ndarray:
    """Leaves (t * 2^h blocks, tree-major) of the reference's own GPU
    cuda_mpcot_sender for the given roots (t * 2^h a multiple of 1024)."""
    roots = np.ascontiguousarray(roots, np.uint8).reshape(-1, 16)
    t = roots.shape[0]
    out = np.empty((t << h, 16), np.uint8)
    rc = refgpu_lib().ref_gpu_mpcot_sender_leaves(t, h, _p(roots), _p(_u8(delta)), _p(out))
    assert rc == 0, f"ref_gpu_mpcot_sender_leaves rejected t={t} h={h} ({rc})"
    return out


def refgpu_primal_lpn(key, kk: np.ndarray, nn: np.ndarray) -> np.ndarray:
    """The reference's own GPU cuda_primal_lpn (d = 10, one GPU) on rows nn
    (n a multiple of 2048) with the 16-byte AES key it reads from LpnF2's
    expanded schedule."""
    kk = np.ascontiguousarray(kk, np.uint8).reshape(-1, 16)
    inp = np.ascontiguousarray(nn, np.uint8).reshape(-1, 16)
    out = np.empty_like(inp)
    rc = refgpu_lib().ref_gpu_primal_lpn_run(inp.shape[0], kk.shape[0], _p(_u8(key)), _p(kk), _p(inp), _p(out))
    assert rc == 0, f"ref_gpu_primal_lpn_run rejected n={inp.shape[0]} ({rc})"
    return out


def refgpu_qc_encode(planes: np.ndarray, n: int, seed: int):
    """The reference's float QuasiCyclic::encode_dense of 128 planes of n
    bits (uint64 words, shape (128, n / 64)); returns (out, key, a): the key
    its constructor drew for `a` (compat_qc_a(key, n) rebuilds it) and the
    constructor's `a` itself (n / 64 words)."""
    inp = np.ascontiguousarray(planes, np.uint64).reshape(128, n // 64)
    out = np.empty_like(inp)
    key = np.empty(16, np.uint8)
    a = np.empty(n // 64, np.uint64)
    rc = refgpu_lib().ref_gpu_qc_encode(n, seed, _p(inp), _p(out), _p(key), _p(a))
    assert rc == 0, f"ref_gpu_qc_encode rejected n={n} ({rc})"
    return out, key, a


def compat_qc_a(key, n: int) -> np.ndarray:
    """The reference GPU QuasiCyclic's `a` (silent/quasi_cyclic.cu:59-66): n
    bits = AES' (the GPU key schedule) of make_block(i) = (low 64 bits
    4 floor(i / 10), high 64 bits i mod 10), i < n / 128, as n / 64 words."""
    nb = n // 128
    i = np.arange(nb, dtype=np.uint64)
    pt = np.empty((nb, 2), np.uint64)
    pt[:, 0] = 4 * (i // 10)
    pt[:, 1] = i % 10
    ct = aes_ecb_rk(compat_key_expand(key), pt.view(np.uint8).reshape(nb, 16))
    return ct.reshape(-1).view(np.uint64).copy()


def emp_aes_ecb(key, blocks: np.ndarray):
    """AES-128 ECB through the emp-tool shim (AES_set_encrypt_key +
    AES_ecb_encrypt_blks)."""
    inp = np.ascontiguousarray(blocks, np.uint8).reshape(-1, 16)
    out = np.empty_like(inp)
    emp_lib().ref_emp_aes_ecb(_p(_u8(key)), _p(inp), _p(out), C.c_uint64(inp.shape[0]))
    return out


def emp_spcot_sender(roots, h: int, delta):
    """SPCOT_Sender::compute (spcot_sender.h:40-86) per tree, seed = root:
    (leaves [t*2^h], ot_msg_0 [t*h], ot_msg_1 [t*h], secret_sum [t]) in the
    MPCOT layout (tree-major leaves, [tree][level] messages).  h >= 2."""
    roots = np.ascontiguousarray(roots, np.uint8).reshape(-1, 16)
    t = roots.shape[0]
    leaves = np.empty((t << h, 16), np.uint8)
    m0 = np.empty((t * h, 16), np.uint8)
    m1 = np.empty((t * h, 16), np.uint8)
    ss = np.empty((t, 16), np.uint8)
    d = _u8(delta)
    L = emp_lib()
    for i in range(t):
        rc = L.ref_spcot_sender(_p(roots[i]), INT(h), _p(d), _p(leaves[i << h:(i + 1) << h]),
                                _p(m0[i * h:(i + 1) * h]), _p(m1[i * h:(i + 1) * h]), _p(ss[i]))
        assert rc == 0, f"ref_spcot_sender rejected h={h}"
    return leaves, m0, m1, ss


def emp_spcot_recver(mc, choice, secret_sum, h: int):
    """SPCOT_Recver::get_index + compute (spcot_recver.h:33-95) per tree:
    (leaves [t*2^h], punctured index [t])."""
    ss = np.ascontiguousarray(secret_sum, np.uint8).reshape(-1, 16)
    t = ss.shape[0]
    mc = np.ascontiguousarray(mc, np.uint8).reshape(t * h, 16)
    ch = np.ascontiguousarray(choice, np.uint8).reshape(t * h)
    leaves = np.empty((t << h, 16), np.uint8)
    pos = np.empty(t, np.int32)
    L = emp_lib()
    for i in range(t):
        p = C.c_int(0)
        rc = L.ref_spcot_recver(INT(h), _p(ch[i * h:(i + 1) * h]), _p(mc[i * h:(i + 1) * h]), _p(ss[i]),
                                _p(leaves[i << h:(i + 1) << h]), C.byref(p))
        assert rc == 0
        pos[i] = p.value
    return leaves, pos


def emp_mpcot_trees(roots, h: int, delta, choice):
    """Both roles of the trees `roots` through the reference's own
    SPCOT_Sender / SPCOT_Recver::compute in one single-threaded call (the
    level OT by selection: choice[i*h + l] = 1 picks ot_msg_1).  Returns
    (sender leaves, receiver leaves), tree-major.  h >= 2."""
    roots = np.ascontiguousarray(roots, np.uint8).reshape(-1, 16)
    t = roots.shape[0]
    ch = np.ascontiguousarray(choice, np.uint8).reshape(t * h)
    ls = np.empty((t << h, 16), np.uint8)
    lr = np.empty((t << h, 16), np.uint8)
    rc = emp_lib().ref_mpcot_trees(_p(roots), INT(t), INT(h), _p(_u8(delta)), _p(ch), _p(ls), _p(lr))
    assert rc == 0, f"ref_mpcot_trees rejected h={h}"
    return ls, lr


def emp_lpn_task(seed, kk, nn, d: int = 10, start: int = 0, end: int | None = None,
                 inplace: bool = False) -> np.ndarray:
    """LpnF2<IO, d>::task(nn, kk, start, end) (lpn_f2.h:46-79): one task
    over rows [start, end), default [0, n), on a copy of nn (or on nn itself,
    a C-contiguous (n, 16) uint8 array, with inplace=True)."""
    kk = np.ascontiguousarray(kk, np.uint8).reshape(-1, 16)
    if inplace:
        assert nn.dtype == np.uint8 and nn.flags["C_CONTIGUOUS"] and nn.shape[-1] == 16
        out = nn.reshape(-1, 16)
    else:
        out = np.array(nn, dtype=np.uint8, copy=True).reshape(-1, 16)
    n = out.shape[0]
    end = n if end is None else end
    rc = emp_lib().ref_lpn_task(_p(_u8(seed)), _p(kk), kk.shape[0], d, _p(out), n, start, end)
    assert rc == 0, "ref_lpn_task rejected its arguments"
    return out


def _p(a: np.ndarray):
    assert a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(ctypes.c_void_p)


def _u8(a) -> np.ndarray:
    return np.ascontiguousarray(np.frombuffer(bytes(a), dtype=np.uint8)) if isinstance(a, (bytes, bytearray)) else np.ascontiguousarray(a, dtype=np.uint8)


C = ctypes
I64, U64, SZ, INT = C.c_int64, C.c_uint64, C.c_size_t, C.c_int


def aes_key_expand(key) -> np.ndarray:
    rk = np.zeros(176, np.uint8)
    lib().or_aes128_key_expand(_p(_u8(key)), _p(rk))
    return rk


def aes_ecb(key, blocks: np.ndarray, portable: bool = False) -> np.ndarray:
    rk = aes_key_expand(key)
    inp = np.ascontiguousarray(blocks, dtype=np.uint8).reshape(-1, 16)
    out = np.empty_like(inp)
    f = lib().or_aes128_encrypt_portable if portable else lib().or_aes128_encrypt
    f(_p(rk), _p(inp), _p(out), SZ(inp.shape[0]))
    return out


def aes_ecb_rk(rk, blocks: np.ndarray) -> np.ndarray:
    """AES-128 rounds under an explicit expanded schedule (176 bytes)."""
    inp = np.ascontiguousarray(blocks, dtype=np.uint8).reshape(-1, 16)
    out = np.empty_like(inp)
    lib().or_aes128_encrypt(_p(_u8(rk)), _p(inp), _p(out), SZ(inp.shape[0]))
    return out


def prg(seed, nblocks: int, offset: int = 0) -> np.ndarray:
    out = np.empty((nblocks, 16), np.uint8)
    lib().or_prg_fill(_p(_u8(seed)), U64(offset), _p(out), SZ(nblocks))
    return out


def ferret_pprf_sender(roots, h: int, delta, threads: int = 1):
    roots = np.ascontiguousarray(roots, np.uint8).reshape(-1, 16)
    t = roots.shape[0]
    leaves = np.empty((t << h, 16), np.uint8)
    lsum = np.empty((t * h, 16), np.uint8)
    rsum = np.empty((t * h, 16), np.uint8)
    ss = np.empty((t, 16), np.uint8)
    d = _u8(delta)
    lib().or_ferret_pprf_sender(_p(roots), I64(t), INT(h), *_blk_by_value(d), _p(leaves),
                                _p(lsum), _p(rsum), _p(ss), INT(threads))
    return leaves, lsum, rsum, ss


class _Blk(C.Structure):
    _fields_ = [("lo", C.c_uint64), ("hi", C.c_uint64)]


def _blk_by_value(b: np.ndarray):
    b = _u8(b)
    return (_Blk(int.from_bytes(b[:8].tobytes(), "little"), int.from_bytes(b[8:16].tobytes(), "little")),)


def ferret_pprf_recver(mc, choice, secret_sum, h: int, threads: int = 1):
    mc = np.ascontiguousarray(mc, np.uint8).reshape(-1, 16)
    ss = np.ascontiguousarray(secret_sum, np.uint8).reshape(-1, 16)
    t = ss.shape[0]
    ch = np.ascontiguousarray(choice, np.uint8).reshape(-1)
    assert mc.shape[0] == t * h and ch.shape[0] == t * h
    leaves = np.empty((t << h, 16), np.uint8)
    lib().or_ferret_pprf_recver(_p(mc), _p(ch), _p(ss), I64(t), INT(h), _p(leaves), INT(threads))
    return leaves


def lpn_primal(seed, kk, nn, d: int = 10, threads: int = 1) -> np.ndarray:
    kk = np.ascontiguousarray(kk, np.uint8).reshape(-1, 16)
    out = np.array(nn, dtype=np.uint8, copy=True).reshape(-1, 16)
    lib().or_lpn_primal(_p(_u8(seed)), _p(kk), I64(kk.shape[0]), INT(d), _p(out),
                        I64(out.shape[0]), INT(threads))
    return out


def compat_key_expand(key) -> np.ndarray:
    """cuOT's GPU key schedule (round constants one entry early)."""
    rk = np.zeros(176, np.uint8)
    lib().or_compat_key_expand(_p(_u8(key)), _p(rk))
    return rk


def compat_ferret_sender(roots, h: int, delta, threads: int = 1):
    """cuOT's GPU Ferret sender semantics (no parent XOR, its own keys and
    schedule, no leaf mask): (leaves, secret sums)."""
    roots = np.ascontiguousarray(roots, np.uint8).reshape(-1, 16)
    t = roots.shape[0]
    leaves = np.empty((t << h, 16), np.uint8)
    ss = np.empty((t, 16), np.uint8)
    lib().or_compat_ferret_sender(_p(roots), I64(t), INT(h), *_blk_by_value(_u8(delta)), _p(leaves), _p(ss),
                                  INT(threads))
    return leaves, ss


def compat_lpn(key, kk, nn, d: int = 10, start: int = 0, threads: int = 1) -> np.ndarray:
    """cuOT's GPU primal LPN semantics (swapped index plaintext, % k)."""
    kk = np.ascontiguousarray(kk, np.uint8).reshape(-1, 16)
    out = np.array(nn, dtype=np.uint8, copy=True).reshape(-1, 16)
    lib().or_compat_lpn(_p(_u8(key)), _p(kk), I64(kk.shape[0]), INT(d), _p(out), I64(out.shape[0]), I64(start),
                        INT(threads))
    return out


def bit_transpose(inp: np.ndarray, rows: int, row_bytes: int, col_lo: int, col_hi: int) -> np.ndarray:
    inp = np.ascontiguousarray(inp, np.uint8).reshape(-1)
    out = np.empty((col_hi - col_lo) * (rows // 8), np.uint8)
    lib().or_bit_transpose(_p(inp), U64(rows), U64(row_bytes), U64(col_lo), U64(col_hi), _p(out))
    return out


def qc_gen_a(key, n: int) -> np.ndarray:
    a = np.zeros(n // 64, np.uint64)
    lib().or_qc_gen_a(_p(_u8(key)), U64(n), _p(a))
    return a


def gf2_cyclic_mul(a: np.ndarray, b: np.ndarray, n: int) -> np.ndarray:
    a = np.ascontiguousarray(a, np.uint64)
    b = np.ascontiguousarray(b, np.uint64)
    out = np.empty(n // 64, np.uint64)
    lib().or_gf2_cyclic_mul(_p(a), _p(b), U64(n), _p(out))
    return out


def qc_encode(a: np.ndarray, planes: np.ndarray, n: int, threads: int = 1) -> np.ndarray:
    out = np.array(planes, dtype=np.uint64, copy=True).reshape(-1)
    npl = out.shape[0] // (n // 64)
    lib().or_qc_encode(_p(np.ascontiguousarray(a, np.uint64)), _p(out), U64(n), INT(npl), INT(threads))
    return out.reshape(npl, n // 64)


def qc_encode_sparse(a: np.ndarray, pos, n: int) -> np.ndarray:
    pos = np.ascontiguousarray(pos, np.uint64)
    out = np.empty(n // 64, np.uint64)
    lib().or_qc_encode_sparse(_p(np.ascontiguousarray(a, np.uint64)), _p(pos), INT(pos.shape[0]),
                              U64(n), _p(out))
    return out


def sot_dual_lpn(a: np.ndarray, io: np.ndarray, n: int, threads: int = 1) -> np.ndarray:
    out = np.array(io, dtype=np.uint8, copy=True).reshape(n, 16)
    lib().or_sot_dual_lpn(_p(np.ascontiguousarray(a, np.uint64)), _p(out), U64(n), INT(threads))
    return out


def sot_pprf_sender(roots, h: int, delta, base0, base1, threads: int = 1):
    roots = np.ascontiguousarray(roots, np.uint8).reshape(-1, 16)
    t = roots.shape[0]
    b0 = np.ascontiguousarray(base0, np.uint8).reshape(h * t, 16)
    b1 = np.ascontiguousarray(base1, np.uint8).reshape(h * t, 16)
    leaves = np.empty((t << h, 16), np.uint8)
    m0 = np.empty(((h + 1) * t, 16), np.uint8)
    m1 = np.empty(((h + 1) * t, 16), np.uint8)
    lib().or_sot_pprf_sender(_p(roots), I64(t), INT(h), *_blk_by_value(_u8(delta)), _p(b0), _p(b1),
                             _p(leaves), _p(m0), _p(m1), INT(threads))
    return leaves, m0, m1


def sot_pprf_recver(m0, m1, mc, choice, t: int, h: int, threads: int = 1):
    m0 = np.ascontiguousarray(m0, np.uint8).reshape((h + 1) * t, 16)
    m1 = np.ascontiguousarray(m1, np.uint8).reshape((h + 1) * t, 16)
    mc = np.ascontiguousarray(mc, np.uint8).reshape(h * t, 16)
    ch = np.ascontiguousarray(choice, np.uint8).reshape(h * t)
    leaves = np.empty((t << h, 16), np.uint8)
    lib().or_sot_pprf_recver(_p(m0), _p(m1), _p(mc), _p(ch), I64(t), INT(h), _p(leaves), INT(threads))
    return leaves


def ref_aes_ecb(key, blocks: np.ndarray):
    r = ref_lib()
    if r is None:
        return None
    inp = np.ascontiguousarray(blocks, np.uint8).reshape(-1, 16)
    out = np.empty_like(inp)
    r.ref_aes_ecb(_p(_u8(key)), _p(inp), _p(out), C.c_ulonglong(inp.shape[0]))
    return out


def ref_prng(seed, nblocks: int):
    r = ref_lib()
    if r is None:
        return None
    out = np.empty((nblocks, 16), np.uint8)
    r.ref_prng(_p(_u8(seed)), _p(out), C.c_ulonglong(nblocks))
    return out


def gf128_mul(a, b) -> np.ndarray:
    """GF(2^128) product of 16-byte blocks (natural bit order, mod x^128 +
    x^7 + x^2 + x + 1)."""
    a = np.ascontiguousarray(a, np.uint8).reshape(16)
    b = np.ascontiguousarray(b, np.uint8).reshape(16)
    out = np.empty(16, np.uint8)
    lib().or_gf128_mul(_p(a), _p(b), _p(out))
    return out


def ferret_chi_sum(leaves, h: int, seeds, threads: int = 1) -> np.ndarray:
    """Per-tree sum_i seed^(i+1) * leaf_i over GF(2^128)."""
    seeds = np.ascontiguousarray(seeds, np.uint8).reshape(-1, 16)
    t = seeds.shape[0]
    leaves = np.ascontiguousarray(leaves, np.uint8).reshape(t << h, 16)
    out = np.empty((t, 16), np.uint8)
    lib().or_ferret_chi_sum(_p(leaves), I64(t), INT(h), _p(seeds), _p(out), INT(threads))
    return out
