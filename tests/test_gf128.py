"""GF(2^128) arithmetic of the oracle's consistency-check restatement
(or_gf128_mul, or_ferret_chi_sum) against a pure-Python reference: big-int
carry-less products reduced mod x^128 + x^7 + x^2 + x + 1, natural bit
order (bit i of the little-endian block = coefficient of x^i)."""
import numpy as np

import oracle

POLY = (1 << 128) | 0x87


def to_int(b):
    return int.from_bytes(bytes(np.asarray(b, np.uint8)), "little")


def to_blk(x):
    return np.frombuffer(x.to_bytes(16, "little"), np.uint8)


def py_mul(a, b):
    r = 0
    while b:
        if b & 1:
            r ^= a
        a <<= 1
        b >>= 1
    for i in range(r.bit_length() - 1, 127, -1):
        if (r >> i) & 1:
            r ^= POLY << (i - 128)
    return r


def test_gf128_mul_matches_python():
    rng = np.random.default_rng(128)
    cases = [(0, 0), (1, 1), (1 << 127, 2), (1 << 127, 1 << 127), ((1 << 128) - 1, (1 << 128) - 1)]
    cases += [(int(rng.integers(0, 2**63)) << 65 | int(rng.integers(0, 2**63)),
               int(rng.integers(0, 2**63)) << 64 | int(rng.integers(0, 2**63))) for _ in range(200)]
    for a, b in cases:
        assert to_int(oracle.gf128_mul(to_blk(a), to_blk(b))) == py_mul(a, b)
    # x^128 = x^7 + x^2 + x + 1
    assert to_int(oracle.gf128_mul(to_blk(1 << 127), to_blk(2))) == 0x87


def test_chi_sum_matches_python():
    rng = np.random.default_rng(5)
    t, h = 3, 4
    leaves = rng.integers(0, 256, (t << h, 16), dtype=np.uint8)
    seeds = rng.integers(0, 256, (t, 16), dtype=np.uint8)
    got = oracle.ferret_chi_sum(leaves, h, seeds, threads=2)
    for j in range(t):
        s = to_int(seeds[j])
        chi, acc = s, 0
        for i in range(1 << h):
            acc ^= py_mul(chi, to_int(leaves[j * 16 + i]))
            chi = py_mul(chi, s)
        assert to_int(got[j]) == acc
