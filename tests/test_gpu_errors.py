"""Argument errors come back as CUOT_EINVAL statuses (CuotError) before any
launch, and the context stays usable afterwards."""
import numpy as np
import pytest

import oracle
from tests.util import rng_blocks, to_dev, to_host

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

EINVAL = 1


def einval(fn):
    import cuot_b200
    with pytest.raises(cuot_b200.CuotError) as e:
        fn()
    assert e.value.status == EINVAL
    return str(e.value)


def test_argument_errors_leave_context_usable(ctx):
    dev = lambda m: torch.zeros((m, 16), dtype=torch.uint8, device="cuda")
    words = lambda n: torch.zeros(max(1, n // 64), dtype=torch.int64, device="cuda")
    # QC sizes: power of two in [2^10, 2^25]
    assert "power of two" in einval(lambda: ctx.qc_encode(words(3072), words(3072), 3072, 1))
    einval(lambda: ctx.qc_encode(words(1 << 26), words(1 << 26), 1 << 26, 1))
    einval(lambda: ctx.qc_encode(words(512), words(512), 512, 1))
    # GGM depth
    delta = np.ones(16, np.uint8)
    einval(lambda: ctx.ferret_pprf_sender(dev(1), 0, delta, dev(1), dev(1), dev(1), dev(1)))
    einval(lambda: ctx.ferret_pprf_sender(dev(1), 31, delta, dev(1), dev(1), dev(1), dev(1)))
    # LPN arguments: d, empty kk, unaligned row range
    seed = np.zeros(16, np.uint8)
    einval(lambda: ctx.lpn_primal(seed, dev(8), dev(16), d=0))
    einval(lambda: ctx.lpn_primal(seed, dev(0), dev(16)))
    einval(lambda: ctx.lpn_primal_range(seed, dev(8), dev(6), 2, 8, 16))
    # tuning keys and values
    einval(lambda: ctx.set_tuning(ctx.TUNE_PPRF_THREADS, 64))
    einval(lambda: ctx.set_tuning(99, 1))
    # still usable
    rng = np.random.default_rng(1)
    key, pt = rng_blocks(rng, 1)[0], rng_blocks(rng, 1000)
    d = to_dev(pt)
    ctx.aes128_ecb(key, d)
    assert np.array_equal(to_host(d), oracle.aes_ecb(key, pt))


def test_host_block_arguments_need_no_alignment(ctx):
    """A host cuot_block (delta) is only 4-byte aligned in C; the entry points
    must not assume 16 (a misaligned vector load would crash the caller)."""
    import ctypes
    from cuot_b200 import _check, _ptr, _stream
    from tests.util import delta_ferret
    rng = np.random.default_rng(4)
    t, h = 3, 5
    roots, delta = rng_blocks(rng, t), delta_ferret(rng)
    buf = (ctypes.c_uint8 * 64)()
    base = ctypes.addressof(buf)
    addr = base + (4 if base % 16 != 4 else 8)   # 4-byte aligned, not 16
    assert addr % 16 != 0
    ctypes.memmove(addr, delta.tobytes(), 16)
    e = lambda m: torch.empty((m, 16), dtype=torch.uint8, device="cuda")
    lv, ls, rs, ss = e(t << h), e(t * h), e(t * h), e(t)
    _check(ctx.lib.cuot_ferret_pprf_sender(ctx.h, _ptr(to_dev(roots)), ctypes.c_uint64(t), ctypes.c_int(h),
                                           ctypes.c_void_p(addr), _ptr(lv), _ptr(ls), _ptr(rs), _ptr(ss),
                                           _stream(None)), "cuot_ferret_pprf_sender")
    exp = oracle.ferret_pprf_sender(roots, h, delta)
    assert np.array_equal(to_host(lv), exp[0]) and np.array_equal(to_host(ss), exp[3])


def test_empty_and_degenerate_inputs(ctx):
    """Zero-size work is a no-op that launches nothing (null pointers allowed
    where there is nothing to read or write); shapes with no valid meaning
    are CUOT_EINVAL; the context stays usable."""
    import cuot_b200
    empty = torch.empty((0, 16), dtype=torch.uint8, device="cuda")
    seed = np.arange(16, dtype=np.uint8)
    kk = to_dev(rng_blocks(np.random.default_rng(2), 8))
    k0 = cuot_b200.launch_count()
    ctx.lpn_primal(seed, kk, empty)                        # n = 0 rows
    ctx.lpn_primal_dual(seed, kk, kk, empty, empty)       # both roles, n = 0
    ctx.aes128_ecb(seed, empty)                           # no blocks
    ctx.aes128_ecb_bitsliced(seed, empty)
    ctx.bit_transpose(empty, 0, 16, 0, 128, empty)        # no rows
    assert cuot_b200.launch_count() == k0                 # nothing launched
    # a tree count of zero and a plane count of zero have no meaning
    delta = np.ones(16, np.uint8)
    einval(lambda: ctx.ferret_pprf_sender(empty, 4, delta, empty, empty, empty, empty))
    words = torch.zeros(1024 // 64, dtype=torch.int64, device="cuda")
    einval(lambda: ctx.qc_encode(words, words, 1024, 0))
    from cuot_b200.batch import Batch
    einval(lambda: Batch(ctx, []))
    # one-tree, depth-1 and one-row extremes still compute
    rng = np.random.default_rng(3)
    roots = rng_blocks(rng, 1)
    e = lambda m: torch.empty((m, 16), dtype=torch.uint8, device="cuda")
    lv, ls, rs, ss = e(2), e(1), e(1), e(1)
    ctx.ferret_pprf_sender(to_dev(roots), 1, delta, lv, ls, rs, ss)
    assert np.array_equal(to_host(lv), oracle.ferret_pprf_sender(roots, 1, delta)[0])
    one = rng_blocks(rng, 1)
    d1 = to_dev(one)
    ctx.lpn_primal(seed, kk, d1)
    assert np.array_equal(to_host(d1), oracle.lpn_primal(seed, to_host(kk), one))


def test_fp64_rate_probe(ctx):
    """cuot_measure_fp64_tflops: argument checks, and a rate in a plausible
    range for B200's fp64 pipe (nominal 37 TFLOP/s)."""
    import ctypes
    from cuot_b200 import CuotError
    v = ctypes.c_double()
    assert ctx.lib.cuot_measure_fp64_tflops(ctx.h, 0, ctypes.byref(v)) == 1
    assert ctx.lib.cuot_measure_fp64_tflops(ctx.h, 1, None) == 1
    with pytest.raises(CuotError):
        ctx.measure_fp64_tflops(reps=1001)
    rate = ctx.measure_fp64_tflops(reps=3)
    print(f"fp64 FMA rate: {rate:.2f} TFLOP/s")
    assert 10.0 < rate < 100.0
