"""The arithmetic behind the exact fp64 FFT encode (cuot_b200/csrc/qc_fft.cu),
on the CPU: the extraction of two planes' bits from a product coefficient
V = c0 + B c1 with B = 2^21 + 1, the centring shift of the n = 2^22 packing,
the complement identity a*e = w(e) - ~a*e, and the rounding-error bounds
the file quotes (Percival, Math. Comp. 72 (2003), Thm. 5.1).  The kernels
themselves are checked against the oracle by the GPU tests."""
import math
import struct

import numpy as np

MAGIC = 6755399441055744.0  # 1.5 * 2^52
B = (1 << 21) + 1


def round_via_magic(v: float) -> int:
    """round(v) as the kernel gets it: bit pattern of v + 1.5 * 2^52 minus
    that of 1.5 * 2^52 (|v| < 2^51)."""
    bits = struct.unpack("<q", struct.pack("<d", v + MAGIC))[0]
    return bits - struct.unpack("<q", struct.pack("<d", MAGIC))[0]


def plane_bits(v: float, shift: int = 0):
    """(c0 & 1, c1 & 1) by the kernel's rule: hi = V >> 21, lo = V mod 2^21,
    d = hi - lo, c1 = hi - [d > 0] - [d > B], c0 = lo ^ c1 (mod 2)."""
    V = round_via_magic(v) + shift
    lo, hi = V & 0x1FFFFF, V >> 21
    d = hi - lo
    c1 = hi - (d > 0) - (d > B)
    return (lo ^ c1) & 1, c1 & 1


def test_extraction_on_edge_and_random_pairs():
    n = 1 << 21
    rng = np.random.default_rng(21)
    vals = [0, 1, 2, 3, n - 2, n - 1, n] + [int(x) for x in rng.integers(0, n + 1, 60)]
    for c0 in vals:
        for c1 in vals:
            V = c0 + B * c1
            for err in (0.0, 0.31, -0.31):
                assert plane_bits(V + err) == (c0 & 1, c1 & 1), (c0, c1, err)


def test_centred_packing_shift():
    """x = (e0 - 1/2) + B (e1 - 1/2) moves every product coefficient by
    -(1 + B) W / 2 = -(2^20 + 1) W, an integer (B odd); adding it back after
    rounding gives the plain packing's V."""
    W = (1 << 21) - 5
    shift = ((1 << 20) + 1) * W
    assert (1 + B) * W % 2 == 0 and (1 + B) * W // 2 == shift
    rng = np.random.default_rng(22)
    for c0, c1 in rng.integers(0, W + 1, (200, 2)):
        c0, c1 = int(c0), int(c1)
        centred = (c0 - W / 2) + B * (c1 - W / 2)
        for err in (0.0, 0.23, -0.23):
            assert plane_bits(centred + err, shift) == (c0 & 1, c1 & 1)


def cyclic_int(a: np.ndarray, e: np.ndarray) -> np.ndarray:
    n = a.shape[0]
    return np.array([int(np.dot(a, np.roll(e[::-1], k + 1))) for k in range(n)])


def test_complement_identity():
    """Integer cyclic convolution: a*e = w(e) - ~a*e coefficientwise, so the
    GF(2) product is ~a*e XOR parity(w(e))."""
    rng = np.random.default_rng(23)
    n = 64
    for _ in range(20):
        a = rng.integers(0, 2, n)
        e = rng.integers(0, 2, n)
        direct = cyclic_int(a, e)
        assert np.array_equal(direct, e.sum() - cyclic_int(1 - a, e))
        assert np.array_equal(direct & 1, (cyclic_int(1 - a, e) & 1) ^ (e.sum() & 1))


def percival(m: int, norm_xa: float) -> float:
    eps = 2.0 ** -53
    beta = 4 * eps
    f = (math.exp(3 * m * math.log1p(eps) + (3 * m + 1) * math.log1p(eps * math.sqrt(5))
                  + 3 * m * math.log1p(beta)) - 1)
    return norm_xa * f


def test_rounding_bounds_quoted_in_the_kernel():
    # n <= 2^20: B = 2^21, ||x|| ||a|| <= sqrt(2n) (1 + B) sqrt(n)
    n = 1 << 20
    assert percival(20, math.sqrt(2 * n) * (1 + 2**21) * math.sqrt(n)) < 0.16
    # n = 2^21: B = 2^21 + 1
    n = 1 << 21
    assert percival(21, math.sqrt(2 * n) * (1 + B) * math.sqrt(n)) < 0.32
    # ... where B = 2^22 would not do
    assert percival(21, math.sqrt(2 * n) * (1 + 2**22) * math.sqrt(n)) > 0.5
    # n = 2^22: centred planes against the lighter of a, ~a (W <= 2^21)
    n = 1 << 22
    assert percival(22, math.sqrt(2 * n) * (1 + B) / 2 * math.sqrt(1 << 21)) < 0.24
    # without the two changes the bound exceeds 1/2
    assert percival(22, math.sqrt(2 * n) * (1 + n + 1) * math.sqrt(n)) > 1.3
    # and at 2^23 even with both
    n = 1 << 23
    assert percival(23, math.sqrt(2 * n) * (1 + (1 << 22) + 1) / 2 * math.sqrt(1 << 22)) > 0.5
