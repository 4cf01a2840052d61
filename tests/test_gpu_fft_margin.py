"""The fp64 FFT QC encode rounds each product coefficient to an integer; it
is exact as long as every computed value lies within 1/2 of that integer.
The analytic bound (Percival, Math. Comp. 72 (2003), Thm. 5.1, with the
packing of qc_fft.cu) is below 0.16 at n = 2^20, 0.32 at 2^21 and 0.24 at
2^22.  These tests switch on the context's margin recorder
(CUOT_TUNE_QC_RECORD_MARGIN), run whole 128-plane dual LPNs, and check that
the largest |v - round(v)| the device actually produced stays below those
bounds, on the inputs that maximise the bound (all-ones planes and `a`; at
2^22, where planes are centred and `a` is replaced by the lighter of a and
~a, an `a` of weight exactly n/2) and on random, heavy and light `a`.
The measured maxima are printed (run with -s to see them).
"""
import numpy as np
import pytest

import cuot_b200

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

BOUND = {20: 0.16, 21: 0.32, 22: 0.24}


def a_bits(n: int, kind: str, rng) -> np.ndarray:
    if kind == "ones":
        bits = np.ones(n, bool)
    elif kind == "half":  # weight exactly n/2
        bits = np.zeros(n, bool)
        bits[rng.permutation(n)[: n // 2]] = True
    else:
        p = {"random": 0.5, "heavy": 0.9, "light": 0.1}[kind]
        bits = rng.random(n) < p
    return np.packbits(bits, bitorder="little").view(np.int64)


def planes(n: int, kind: str, rng) -> np.ndarray:
    if kind == "ones":
        return np.full((n, 16), 0xFF, np.uint8)
    return rng.integers(0, 256, (n, 16), dtype=np.uint8)


CASES = [(20, "ones", "ones"), (20, "random", "random"), (20, "heavy", "random"),
         (21, "ones", "ones"), (21, "random", "random"), (21, "light", "ones"),
         (22, "half", "ones"), (22, "half", "random"), (22, "random", "random"), (22, "heavy", "ones"),
         (22, "light", "random"), (22, "ones", "ones")]


@pytest.mark.parametrize("e,akind,pkind", CASES)
def test_fft_rounding_margin_below_bound(e, akind, pkind):
    n = 1 << e
    rng = np.random.default_rng(1000 * e + len(akind) + 7 * len(pkind))
    ctx = cuot_b200.Context(0)
    try:
        ctx.set_tuning(ctx.TUNE_QC_RECORD_MARGIN, 1)
        a = torch.from_numpy(a_bits(n, akind, rng)).cuda()
        io = torch.from_numpy(planes(n, pkind, rng)).cuda()
        ctx.sot_dual_lpn(a, io, n)
        torch.cuda.synchronize()
        m = ctx.qc_fft_margin()
        print(f"\nn=2^{e} a={akind} planes={pkind}: max |v - round(v)| = {m:.3g} (bound {BOUND[e]})")
        assert 0.0 <= m < BOUND[e]
        # the read reset the record: a second encode (fresh planes of the same
        # kind) starts from zero and stays below the bound too
        io2 = torch.from_numpy(planes(n, pkind, rng)).cuda()
        ctx.sot_dual_lpn(a, io2, n)
        torch.cuda.synchronize()
        assert 0.0 <= ctx.qc_fft_margin() < BOUND[e]
    finally:
        torch.cuda.synchronize()
        ctx.close()


def test_margin_reader_needs_recording(ctx):
    with pytest.raises(cuot_b200.CuotError):
        ctx.qc_fft_margin()
