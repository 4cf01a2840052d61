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
