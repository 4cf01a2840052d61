"""Per-tree GF(2^128) check values of the malicious consistency check
(cuot_ferret_chi_sum) against the oracle, and the check's own identity at
the ferret_b13 size: V_j ^ W_j = s_j^(alpha_j + 1) * Delta."""
import numpy as np
import pytest

import oracle
from tests.util import delta_ferret, rng_blocks, to_dev, to_host

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def gf_pow(s, e):
    r = np.zeros(16, np.uint8)
    r[0] = 1
    b = s.copy()
    while e:
        if e & 1:
            r = oracle.gf128_mul(r, b)
        b = oracle.gf128_mul(b, b)
        e >>= 1
    return r


@pytest.mark.parametrize("t,h", [(3, 1), (5, 7), (4, 8), (17, 10), (2, 16)])
def test_chi_sum_vs_oracle(ctx, t, h):
    rng = np.random.default_rng(t * 31 + h)
    leaves, seeds = rng_blocks(rng, t << h), rng_blocks(rng, t)
    out = torch.empty((t, 16), dtype=torch.uint8, device="cuda")
    ctx.ferret_chi_sum(to_dev(leaves), h, to_dev(seeds), out)
    assert np.array_equal(to_host(out), oracle.ferret_chi_sum(leaves, h, seeds, threads=8))


def test_chi_sum_check_identity_b13(ctx):
    from cuot_b200.ferret import chi_seeds
    t, h = 1280, 13
    rng = np.random.default_rng(1313)
    roots, delta = rng_blocks(rng, t), delta_ferret(rng)
    choice = rng.integers(0, 2, t * h).astype(np.uint8)
    e = lambda m: torch.empty((m, 16), dtype=torch.uint8, device="cuda")
    v, w, ls, rs, ss, mc = e(t << h), e(t << h), e(t * h), e(t * h), e(t), e(t * h)
    ctx.ferret_pprf_sender(to_dev(roots), h, delta, v, ls, rs, ss)
    dch = to_dev(choice)
    torch.where(dch.view(-1, 1).bool(), rs, ls, out=mc)
    ctx.ferret_pprf_recver(mc, dch, ss, h, w)
    seeds = np.frombuffer(chi_seeds(to_host(ss).tobytes()), np.uint8).reshape(t, 16).copy()
    V, W = e(t), e(t)
    ctx.ferret_chi_sum(v, h, to_dev(seeds), V)
    ctx.ferret_chi_sum(w, h, to_dev(seeds), W)
    Vh, Wh = to_host(V), to_host(W)
    assert np.array_equal(Vh, oracle.ferret_chi_sum(to_host(v), h, seeds, threads=16))
    ch = choice.reshape(t, h)
    for j in range(0, t, 97):
        pos = 0
        for d in range(h):
            pos = pos * 2 + 1 - int(ch[j, d])
        exp = oracle.gf128_mul(gf_pow(seeds[j], pos + 1), delta)
        assert np.array_equal(Vh[j] ^ Wh[j], exp)
