"""The allocation-free Ferret sender (cuot_ferret_pprf_sender_noalloc).

It exists for callers that cannot allocate device memory when they call in
(a server whose HBM belongs to its own pool allocator, or a latency-critical
path that cannot take cudaMalloc's implicit device synchronisation).  These
tests call it through the C ABI and require its outputs to equal, bit for
bit, those of the ordinary cuot_ferret_pprf_sender on the same inputs, on two
calls in a row (the calls share one scratch array, so the second call also
shows that nothing stale from the first leaks into its result).  This file is
collected last so that a run stopping at its first failure has already run
every other test.
"""
import ctypes

import numpy as np
import pytest

import cuot_b200
from tests.util import delta_ferret, rng_blocks, to_dev, to_host

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

C = ctypes


def _p(x):
    return C.c_void_p(x.data_ptr())


def _noalloc(lib, roots, t, h, delta, leaves, lsum, rsum, ss):
    d = (C.c_uint8 * 16).from_buffer_copy(delta.tobytes())
    return lib.cuot_ferret_pprf_sender_noalloc(
        _p(roots), C.c_uint64(t), C.c_int(h), d, _p(leaves), _p(lsum), _p(rsum), _p(ss),
        C.c_void_p(torch.cuda.current_stream().cuda_stream))


@pytest.fixture(scope="module")
def lib():
    lib = cuot_b200.load()
    lib.cuot_last_error.restype = C.c_char_p
    return lib


def test_noalloc_sender_equals_ordinary_sender_twice(ctx, lib):
    # calls in a row with different shapes and inputs; the last one fills the
    # scratch array to its limit, t * 2^h = 2^20 leaves
    for t, h, seed in [(64, 10, 11), (300, 9, 12), (1024, 10, 13)]:
        rng = np.random.default_rng(seed)
        roots, delta = rng_blocks(rng, t), delta_ferret(rng)
        droots = to_dev(roots)
        out = [torch.empty((m, 16), dtype=torch.uint8, device="cuda") for m in (t << h, t * h, t * h, t)]
        st = _noalloc(lib, droots, t, h, delta, *out)
        assert st == 0, lib.cuot_last_error()
        ref = [torch.empty_like(x) for x in out]
        ctx.ferret_pprf_sender(droots, h, delta, *ref)
        torch.cuda.synchronize()
        for got, exp in zip(out, ref):
            assert np.array_equal(to_host(got), to_host(exp))


def test_noalloc_rejects_sizes_beyond_its_scratch(lib):
    small = torch.empty((16, 16), dtype=torch.uint8, device="cuda")
    delta = np.zeros(16, np.uint8)
    # one tree past the limit (2^20 + 2^10 leaves), and twice the limit; the
    # arguments are rejected before anything is launched
    for t, h in [(1025, 10), (2048, 10)]:
        st = _noalloc(lib, small, t, h, delta, small, small, small, small)
        assert st == 1
        assert b"no-alloc limit" in lib.cuot_last_error()
