"""The transforms of the exact QC encode -- the fp64 FFT (four planes per
complex transform, default for n <= 2^22; packing base 2^21 + 1 from 2^21;
at 2^22 centred planes against the lighter of `a` and its complement),
GF(2) Karatsuba over it (dual LPN at n = 2^23, 2^24) and the NTT mod
469762049 -- against the oracle and against each other: every supported FFT
size, plane counts that leave a partial transform, the maximum-magnitude
inputs (all-ones `a` and planes: every convolution coefficient equals its
bound n), both sides of the complement at 2^22 (a and ~a, light and heavy
`a`), the rate-1/2 form with odd batches, the full 128-plane dual LPN at
n = 2^20 .. 2^22, the Karatsuba sizes, and the one- and two-stream FFT group
schedules."""
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
                                       (17, 3), (18, 4), (19, 5), (20, 7), (21, 6), (22, 5)])
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


@pytest.mark.parametrize("e", [10, 16, 20, 21, 22])
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


def _ctx(backend):
    import cuot_b200
    c = cuot_b200.Context(0)
    c.set_tuning(c.TUNE_QC_BACKEND, backend)
    return c


@pytest.mark.parametrize("e", [21, 22, 23, 24])
def test_large_sizes_match_ntt_and_oracle(e):
    """n = 2^21 .. 2^24 dual LPN: the default backend (the direct FFT up to
    2^22; GF(2) Karatsuba over 2^22 FFTs, one / two levels, above) gives the
    NTT's blocks, one-shot and through a plan, and sampled planes match the
    oracle's product."""
    n = 1 << e
    rng = np.random.default_rng(900 + e)
    x = rng_blocks(rng, n)
    key = rng_blocks(rng, 1)[0]
    outs = {}
    for name, b in (("ntt", NTT), ("auto", 0)):
        c = _ctx(b)
        a = gen_a(c, key, n)
        d = to_dev(x)
        c.sot_dual_lpn(a, d, n)
        outs[name] = to_host(d)
        if name == "auto":
            plan = c.qc_plan(a, n)
            d2 = to_dev(x)
            plan.dual_lpn(d2)
            outs["plan"] = to_host(d2)
            # plane encodes through the same plan (FFT up to 2^22; above, the
            # NTT A_hat kept beside the Karatsuba leaves)
            pl = oracle.bit_transpose(x, n, 16, 0, 128).view(np.uint64).reshape(128, n // 64)[:2].copy()
            dp = to_dev(pl.view(np.int64))
            plan.encode(dp, 2)
            outs["plan_planes"] = to_host(dp).view(np.uint64)
            del plan
        a_np = to_host(a).view(np.uint64)
        torch.cuda.synchronize()
        c.close()
    assert np.array_equal(outs["auto"], outs["ntt"])
    assert np.array_equal(outs["plan"], outs["ntt"])
    planes = oracle.bit_transpose(x, n, 16, 0, 128).view(np.uint64).reshape(128, n // 64)
    outp = oracle.bit_transpose(outs["auto"], n, 16, 0, 128).view(np.uint64).reshape(128, n // 64)
    for r in (0, 77):
        assert np.array_equal(outp[r], oracle.gf2_cyclic_mul(a_np, planes[r], n))
    for r in (0, 1):
        assert np.array_equal(outs["plan_planes"][r], outp[r])


@pytest.mark.parametrize("e", [21, 22, 23])
def test_rate_half_large(e):
    """Rate-1/2 form at n = 2^21, 2^22 (direct FFT) and 2^23 (Karatsuba):
    out = e0 ^ a*e1, also with out aliasing the first n input blocks."""
    n = 1 << e
    rng = np.random.default_rng(2100 + e)
    x = rng_blocks(rng, 2 * n)
    c = _ctx(0)
    a = gen_a(c, rng_blocks(rng, 1)[0], n)
    out = torch.empty((n, 16), dtype=torch.uint8, device="cuda")
    c.sot_dual_lpn_r2(a, to_dev(x), n, out)
    d = to_dev(x)
    plan = c.qc_plan(a, n)
    plan.dual_lpn_r2(d, d[:n])
    got, got2 = to_host(out), to_host(d)[:n]
    a_np = to_host(a).view(np.uint64)
    del plan
    torch.cuda.synchronize()
    c.close()
    assert np.array_equal(got, got2)
    p0 = oracle.bit_transpose(x[:n].copy(), n, 16, 0, 128).view(np.uint64).reshape(128, n // 64)
    p1 = oracle.bit_transpose(x[n:].copy(), n, 16, 0, 128).view(np.uint64).reshape(128, n // 64)
    po = oracle.bit_transpose(got, n, 16, 0, 128).view(np.uint64).reshape(128, n // 64)
    for r in (3, 100):
        assert np.array_equal(po[r], p0[r] ^ oracle.gf2_cyclic_mul(a_np, p1[r], n))


@pytest.mark.parametrize("e", [17, 20, 21, 22])
def test_one_and_two_stream_encodes_agree(e):
    """CUOT_TUNE_QC_STREAMS = 1 (every group on the caller's stream) and 2
    (groups alternate with the context's second stream) give the oracle's
    blocks; the key accepts only 1 and 2."""
    import cuot_b200
    n = 1 << e
    rng = np.random.default_rng(1700 + e)
    x = rng_blocks(rng, n)
    key = rng_blocks(rng, 1)[0]
    outs = []
    for streams in (1, 2):
        c = _ctx(0)
        c.set_tuning(c.TUNE_QC_STREAMS, streams)
        a = gen_a(c, key, n)
        d = to_dev(x)
        plan = c.qc_plan(a, n)
        plan.dual_lpn(d)
        outs.append(to_host(d))
        a_np = to_host(a).view(np.uint64)
        del plan
        for bad in (0, 3):
            with pytest.raises(cuot_b200.CuotError):
                c.set_tuning(c.TUNE_QC_STREAMS, bad)
        torch.cuda.synchronize()
        c.close()
    assert np.array_equal(outs[0], outs[1])
    planes = oracle.bit_transpose(x, n, 16, 0, 128).view(np.uint64).reshape(128, n // 64)
    outp = oracle.bit_transpose(outs[0], n, 16, 0, 128).view(np.uint64).reshape(128, n // 64)
    for r in (0, 90):
        assert np.array_equal(outp[r], oracle.gf2_cyclic_mul(a_np, planes[r], n))


@pytest.mark.parametrize("kind", ["a", "not_a", "light", "heavy"])
def test_complement_sides_at_2_22(kind):
    """n = 2^22: the FFT packs centred planes against the lighter of `a` and
    ~a.  `a` from the PRG and its complement land on opposite sides of n/2;
    a light (weight ~ n/8) and a heavy (~ 7n/8) `a` exercise each side far
    from the edge.  The full 128-plane dual LPN equals the NTT's, and
    sampled planes equal the oracle's product."""
    e = 22
    n = 1 << e
    rng = np.random.default_rng(2222)
    x = rng_blocks(rng, n)
    c0 = _ctx(0)
    a = gen_a(c0, rng_blocks(rng, 1)[0], n)
    a_np = to_host(a).view(np.uint64)
    if kind == "not_a":
        a_np = ~a_np
    elif kind in ("light", "heavy"):
        r = rng.integers(0, 2**63, (3, n // 64), dtype=np.uint64)
        a_np = r[0] & r[1] & r[2]
        if kind == "heavy":
            a_np = ~a_np
    c0.close()
    outs = []
    for b in (NTT, 0):
        c = _ctx(b)
        d = to_dev(x)
        c.sot_dual_lpn(to_dev(a_np.view(np.int64)), d, n)
        outs.append(to_host(d))
        torch.cuda.synchronize()
        c.close()
    assert np.array_equal(outs[0], outs[1])
    planes = oracle.bit_transpose(x, n, 16, 0, 128).view(np.uint64).reshape(128, n // 64)
    outp = oracle.bit_transpose(outs[1], n, 16, 0, 128).view(np.uint64).reshape(128, n // 64)
    for r in (5, 127):
        assert np.array_equal(outp[r], oracle.gf2_cyclic_mul(a_np, planes[r], n))
