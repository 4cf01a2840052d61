"""CPU tests: the oracle against the golden fixtures (OpenSSL / reference
cryptoTools / pure-Python restatements) and against the protocol's own
guarantees.  No GPU needed."""
import numpy as np
import pytest

import oracle
from tests.util import blocks, hx, rng_blocks, delta_ferret


def test_aes_kat_fips197_and_openssl(golden):
    for case in golden["aes"]:
        key, pt, ct = hx(case["key"]), blocks(case["pt"]), blocks(case["ct"])
        assert oracle.aes_ecb(key, pt).tobytes() == ct.tobytes()
        assert oracle.aes_ecb(key, pt, portable=True).tobytes() == ct.tobytes()


def test_aes_against_reference_cryptotools():
    if oracle.ref_lib() is None:
        pytest.skip("oracle/_ref not built")
    rng = np.random.default_rng(1)
    for n in (1, 7, 64, 1000):
        key = rng_blocks(rng, 1)[0]
        pt = rng_blocks(rng, n)
        assert oracle.ref_aes_ecb(key, pt).tobytes() == oracle.aes_ecb(key, pt).tobytes()


def test_prg_matches_cryptotools_prng(golden):
    for case in golden["prg"]:
        got = oracle.prg(hx(case["seed"]), 40)
        assert got.tobytes().hex() == case["blocks"]
        # offset addressing is consistent with the stream
        assert oracle.prg(hx(case["seed"]), 8, offset=32).tobytes() == got[32:40].tobytes()


def test_ferret_ggm_golden(golden):
    for c in golden["ferret_ggm"]:
        t, h = c["t"], c["h"]
        leaves, lsum, rsum, ss = oracle.ferret_pprf_sender(blocks(c["roots"]), h, hx(c["delta"]))
        assert leaves.tobytes().hex() == c["leaves"]
        assert lsum.tobytes().hex() == c["lsum"]
        assert rsum.tobytes().hex() == c["rsum"]
        assert ss.tobytes().hex() == c["secret_sum"]
        ch = np.array(c["choice"], np.uint8)
        mc = np.where(ch[:, None] == 0, lsum, rsum)
        rl = oracle.ferret_pprf_recver(mc, ch, ss, h)
        assert rl.tobytes().hex() == c["recv_leaves"]


def punctured_ferret(choice: np.ndarray, t: int, h: int) -> np.ndarray:
    """Leaf index of the punctured leaf per tree (spcot_recver.h:33-41)."""
    ch = choice.reshape(t, h)
    pos = np.zeros(t, np.int64)
    for d in range(h):
        pos = pos * 2 + (ch[:, d] == 0)
    return pos


@pytest.mark.parametrize("t,h", [(4, 1), (16, 6), (64, 10)])
def test_ferret_cot_correlation(t, h):
    rng = np.random.default_rng(t * 100 + h)
    roots, delta = rng_blocks(rng, t), delta_ferret(rng)
    leaves, lsum, rsum, ss = oracle.ferret_pprf_sender(roots, h, delta, threads=4)
    ch = rng.integers(0, 2, t * h).astype(np.uint8)
    mc = np.where(ch[:, None] == 0, lsum, rsum)
    rl = oracle.ferret_pprf_recver(mc, ch, ss, h, threads=4)
    pos = punctured_ferret(ch, t, h) + np.arange(t) * (1 << h)
    diff = leaves ^ rl
    assert not diff[np.setdiff1d(np.arange(t << h), pos)].any()
    assert (diff[pos] == delta).all()
    assert ((leaves[:, 0] & 1) == 0).all()


def test_lpn_golden(golden):
    for c in golden["lpn"]:
        out = oracle.lpn_primal(hx(c["seed"]), blocks(c["kk"]), blocks(c["e"]), d=c["d"])
        assert out.tobytes().hex() == c["out"], (c["n"], c["k"], c["d"])


def test_lpn_threads_match_single_range():
    rng = np.random.default_rng(5)
    for n in (101, 4096 + 3):
        kk, e, seed = rng_blocks(rng, 777), rng_blocks(rng, n), rng_blocks(rng, 1)[0]
        assert (oracle.lpn_primal(seed, kk, e, threads=1) == oracle.lpn_primal(seed, kk, e, threads=7)).all()


def test_transpose_golden(golden):
    for c in golden["transpose"]:
        out = oracle.bit_transpose(hx(c["in"]), c["rows"], c["row_bytes"], c["lo"], c["hi"])
        assert out.tobytes().hex() == c["out"]


def test_qc_golden(golden):
    for c in golden["qc"]:
        n = c["n"]
        a = oracle.qc_gen_a(hx(c["key"]), n)
        if "a" in c:
            assert a.tobytes().hex() == c["a"]
            b = hx(c["b"]).view(np.uint64)
            assert oracle.gf2_cyclic_mul(a, b, n).tobytes().hex() == c["ab"]
            assert oracle.qc_encode(a, b, n)[0].tobytes().hex() == c["ab"]
            sp = oracle.qc_encode_sparse(a, np.array(c["pos"], np.uint64), n)
            assert sp.tobytes().hex() == c["sparse"]
        else:
            import hashlib
            out = oracle.sot_dual_lpn(a, blocks(c["dual_in"]), n, threads=4)
            assert hashlib.sha256(out.tobytes()).hexdigest() == c["dual_out_sha"]


def test_qc_karatsuba_vs_schoolbook_bigint():
    rng = np.random.default_rng(9)
    for n in (4096, 1 << 14):
        a = rng.integers(0, 2**63, n // 64, dtype=np.uint64)
        b = rng.integers(0, 2**63, n // 64, dtype=np.uint64)
        ai, bi = int.from_bytes(a.tobytes(), "little"), int.from_bytes(b.tobytes(), "little")
        r, i = 0, 0
        while ai:
            if ai & 1:
                r ^= bi << i
            ai >>= 1
            i += 1
        full = (1 << n) - 1
        exp = (r & full) ^ (r >> n)
        got = int.from_bytes(oracle.gf2_cyclic_mul(a, b, n).tobytes(), "little")
        assert got == exp


def test_sot_pprf_golden_and_correlation(golden):
    for c in golden["sot_pprf"]:
        t, h = c["t"], c["h"]
        leaves, m0, m1 = oracle.sot_pprf_sender(blocks(c["roots"]), h, hx(c["delta"]),
                                                blocks(c["base0"]), blocks(c["base1"]))
        assert leaves.tobytes().hex() == c["leaves"]
        assert m0.tobytes().hex() == c["m0"]
        assert m1.tobytes().hex() == c["m1"]
        ch = np.array(c["choice"], np.uint8)
        rl = oracle.sot_pprf_recver(m0, m1, blocks(c["mc"]), ch, t, h)
        diff = rl ^ leaves
        # punctured leaf of tree ti: path bits 1 - choice[d][ti] (recver.cu:78-87)
        chm = ch.reshape(h, t)
        for ti in range(t):
            pos = 0
            for d in range(h):
                pos = pos * 2 + 1 - int(chm[d, ti])
            idx = ti * (1 << h) + pos
            assert (diff[idx] == hx(c["delta"])).all()
            other = np.delete(diff[ti << h:(ti + 1) << h], pos, axis=0)
            assert not other.any()


def test_planted_mistake_is_caught():
    """A flipped bit in an oracle result must fail the comparison used by
    the parity tests (the mistake is planted on the CPU, in the oracle's
    output)."""
    rng = np.random.default_rng(3)
    kk, e, seed = rng_blocks(rng, 50), rng_blocks(rng, 40), rng_blocks(rng, 1)[0]
    good = oracle.lpn_primal(seed, kk, e)
    bad = good.copy()
    bad[17, 3] ^= 0x10
    assert not np.array_equal(good, bad)
    assert np.array_equal(good, oracle.lpn_primal(seed, kk, e))
