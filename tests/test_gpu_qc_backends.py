"""The two transforms of the exact QC encode -- the fp64 FFT (four planes
per complex transform, default for n <= 2^20) and the NTT mod 469762049 --
against the oracle and against each other: every supported FFT size, plane
counts that leave a partial transform, the maximum-magnitude inputs (all-ones
`a` and planes: every convolution coefficient equals its bound n), the
rate-1/2 form with odd batches, and the full 128-plane dual LPN at n = 2^20."""
import numpy as np
import pytest

import oracle
from tests.util import rng_blocks, to_dev, to_host

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

NTT, FFT = 1, 2


@pytest.fixture(scope="module", params=[NTT, FFT], ids=["ntt", "fft"])
def bctx(request):
    import cuot_b200
    c = cuot_b200.Context(0)
    c.set_tuning(c.TUNE_QC_BACKEND, request.param)
    yield c
    torch.cuda.synchronize()
    c.close()


def gen_a(ctx, key, n):
    a = torch.empty(n // 64, dtype=torch.int64, device="cuda")
    ctx.qc_gen_a(key, n, a)
    return a


@pytest.mark.parametrize("e,nplanes", [(10, 1), (11, 3), (12, 4), (13, 5), (14, 6), (15, 9), (16, 2),
                                       (17, 3), (18, 4), (19, 5), (20, 7)])
def test_encode_every_size(bctx, e, nplanes):
    n = 1 << e
    rng = np.random.default_rng(500 + e)
    a = gen_a(bctx, rng_blocks(rng, 1)[0], n)
    planes = rng.integers(0, 2**63, (nplanes, n // 64), dtype=np.uint64)
    planes[-1, : n // 128] = np.uint64(0xFFFFFFFFFFFFFFFF)
    d = to_dev(planes.view(np.int64))
    bctx.qc_encode(a, d, n, nplanes)
    exp = oracle.qc_encode(to_host(a).view(np.uint64), planes, n, threads=16)
    assert np.array_equal(to_host(d).view(np.uint64), exp)


@pytest.mark.parametrize("e", [10, 16, 20])
def test_maximum_magnitude_inputs(bctx, e):
    """a = all ones: coefficient k of a*e is the weight of e (the same for
    every k); with e all ones every coefficient equals n, the bound the
    FFT's rounding argument is made for."""
    n = 1 << e
    a = torch.full((n // 64,), -1, dtype=torch.int64, device="cuda")
    rng = np.random.default_rng(e)
    planes = np.full((5, n // 64), np.uint64(0xFFFFFFFFFFFFFFFF), np.uint64)
    planes[1] = rng.integers(0, 2**63, n // 64, dtype=np.uint64)
    planes[3, 1:] = 0                                   # weight 64: all-zero result
    planes[4, 1:] = 0
    planes[4, 0] = np.uint64(0x7FFFFFFFFFFFFFFF)        # weight 63: all-ones result
    d = to_dev(planes.view(np.int64))
    bctx.qc_encode(a, d, n, 5)
    out = to_host(d).view(np.uint64)
    exp = oracle.qc_encode(np.full(n // 64, np.uint64(0xFFFFFFFFFFFFFFFF)), planes, n, threads=16)
    assert np.array_equal(out, exp)
    assert not out[0].any() and not out[2].any() and not out[3].any()
    assert (out[4] == np.uint64(0xFFFFFFFFFFFFFFFF)).all()


@pytest.mark.parametrize("e", [12, 18])
def test_r2_odd_batches(bctx, e):
    n = 1 << e
    rng = np.random.default_rng(700 + e)
    a = gen_a(bctx, rng_blocks(rng, 1)[0], n)
    x = rng_blocks(rng, 2 * n)
    exp = x[:n] ^ oracle.sot_dual_lpn(to_host(a).view(np.uint64), x[n:].copy(), n, threads=16)
    plan = bctx.qc_plan(a, n)
    for batch in (3, 7, 128):
        plan.set_batch(batch)
        out = torch.empty((n, 16), dtype=torch.uint8, device="cuda")
        plan.dual_lpn_r2(to_dev(x), out)
        assert np.array_equal(to_host(out), exp), batch


def test_backends_agree_on_full_dual_lpn():
    """n = 2^20, 128 planes: the FFT and the NTT give the same blocks, and
    the oracle agrees on sampled planes."""
    import cuot_b200
    n = 1 << 20
    rng = np.random.default_rng(2020)
    x = rng_blocks(rng, n)
    outs = []
    for b in (NTT, FFT):
        c = cuot_b200.Context(0)
        c.set_tuning(c.TUNE_QC_BACKEND, b)
        a = gen_a(c, bytes(range(16)), n)
        d = to_dev(x)
        c.sot_dual_lpn(a, d, n)
        outs.append(to_host(d))
        a_np = to_host(a).view(np.uint64)
        c.close()
    assert np.array_equal(outs[0], outs[1])
    planes = oracle.bit_transpose(x, n, 16, 0, 128).view(np.uint64).reshape(128, n // 64)
    outp = oracle.bit_transpose(outs[1], n, 16, 0, 128).view(np.uint64).reshape(128, n // 64)
    for r in (1, 64, 126):
        assert np.array_equal(outp[r], oracle.gf2_cyclic_mul(a_np, planes[r], n))


def test_backend_key_is_checked(ctx):
    import cuot_b200
    with pytest.raises(cuot_b200.CuotError):
        ctx.set_tuning(ctx.TUNE_QC_BACKEND, 3)
