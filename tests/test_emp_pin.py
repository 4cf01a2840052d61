"""CPU tests: the oracle against the reference's OWN emp-ot code.

oracle/_ref/libempref.so is compiled (oracle/build_ref.sh) from the
reference tree's ferret/emp-ot/emp-ot/ferret/{twokeyprp,spcot_sender,
spcot_recver,lpn_f2}.h, unchanged, over the emp-tool shim in oracle/emp_shim.
These tests check that the C oracle the GPU tests compare against computes
what that code computes: the GGM tree and leaf mask, the per-level OT
messages, the secret sum, the receiver's reconstruction and LpnF2::task's
index matrix (including the __compute1 tail).  The shim's AES is itself
pinned to FIPS-197, OpenSSL (the golden file) and the reference's vendored
cryptoTools AES.  No GPU needed.
"""
import numpy as np
import pytest

import oracle
from tests.util import blocks, hx, rng_blocks, delta_ferret

pytestmark = pytest.mark.skipif(oracle.emp_lib() is None,
                                reason="oracle/_ref/libempref.so not built (needs the reference tree)")


def test_shim_aes_is_fips_and_cryptotools(golden):
    for case in golden["aes"]:
        assert oracle.emp_aes_ecb(hx(case["key"]), blocks(case["pt"])).tobytes() == \
            blocks(case["ct"]).tobytes()
    rng = np.random.default_rng(11)
    for n in (1, 5, 333):
        key, pt = rng_blocks(rng, 1)[0], rng_blocks(rng, n)
        got = oracle.emp_aes_ecb(key, pt)
        assert got.tobytes() == oracle.aes_ecb(key, pt).tobytes()
        if oracle.ref_lib() is not None:
            assert got.tobytes() == oracle.ref_aes_ecb(key, pt).tobytes()


def _sender_pair(roots, h, delta):
    ref = oracle.emp_spcot_sender(roots, h, delta)
    ours = oracle.ferret_pprf_sender(roots, h, delta, threads=4)
    return ref, ours


@pytest.mark.parametrize("t,h", [(1, 2), (3, 3), (5, 4), (2, 7), (64, 10), (4, 13), (1, 16)])
def test_spcot_sender_matches_reference(t, h):
    """Leaves (LSB cleared), ot_msg_0 / ot_msg_1 and secret_sum_f2 of
    SPCOT_Sender::compute equal the oracle's sender; (64, 10) is the
    reference's CPU-runnable configuration (t = 64 trees of depth 10)."""
    rng = np.random.default_rng(1000 * t + h)
    roots, delta = rng_blocks(rng, t), delta_ferret(rng)
    (rl, rm0, rm1, rss), (ol, olsum, orsum, oss) = _sender_pair(roots, h, delta)
    assert np.array_equal(rl, ol), "leaves"
    assert np.array_equal(rm0, olsum), "ot_msg_0 (left sums)"
    assert np.array_equal(rm1, orsum), "ot_msg_1 (right sums)"
    assert np.array_equal(rss, oss), "secret_sum_f2"


def test_spcot_sender_golden_trees(golden):
    """The golden GGM fixtures, recomputed by the reference's code."""
    for c in golden["ferret_ggm"]:
        if c["h"] < 2:
            continue
        rl, rm0, rm1, rss = oracle.emp_spcot_sender(blocks(c["roots"]), c["h"], hx(c["delta"]))
        assert rl.tobytes().hex() == c["leaves"]
        assert rm0.tobytes().hex() == c["lsum"]
        assert rm1.tobytes().hex() == c["rsum"]
        assert rss.tobytes().hex() == c["secret_sum"]


@pytest.mark.parametrize("t,h", [(3, 1), (4, 2), (6, 5), (64, 10), (3, 13)])
def test_spcot_recver_matches_reference(t, h):
    """SPCOT_Recver::compute from the OT-chosen messages equals the oracle's
    receiver, and its punctured index is the oracle's (false = right child)."""
    rng = np.random.default_rng(77 * t + h)
    roots, delta = rng_blocks(rng, t), delta_ferret(rng)
    leaves, lsum, rsum, ss = oracle.ferret_pprf_sender(roots, h, delta, threads=4)
    ch = rng.integers(0, 2, t * h).astype(np.uint8)
    mc = np.where(ch[:, None] == 0, lsum, rsum)
    rl, pos = oracle.emp_spcot_recver(mc, ch, ss, h)
    ol = oracle.ferret_pprf_recver(mc, ch, ss, h, threads=4)
    assert np.array_equal(rl, ol)
    chm = ch.reshape(t, h)
    exp = np.zeros(t, np.int64)
    for d in range(h):
        exp = exp * 2 + (chm[:, d] == 0)
    assert np.array_equal(pos, exp)
    # and the pair is a COT: only the punctured leaf differs, by delta
    diff = rl ^ leaves
    idx = exp + np.arange(t) * (1 << h)
    assert (diff[idx] == delta).all()
    assert not np.delete(diff, idx, axis=0).any()


@pytest.mark.parametrize("n", [1, 2, 3, 4, 5, 6, 7, 8, 9, 12, 13, 14, 15, 16, 101, 1024 + 2])
def test_lpn_tail_rows_match_reference(n):
    """LpnF2::task over [0, n): groups of 4 while j < n - 4, then the
    __compute1 tail (makeBlock(i, m) blocks, r % k) for the last <= 4 rows,
    n mod 4 in {0, 1, 2, 3} and n <= 4 (no group at all)."""
    rng = np.random.default_rng(n)
    k = 37 + n
    kk, e, seed = rng_blocks(rng, k), rng_blocks(rng, n), rng_blocks(rng, 1)[0]
    assert np.array_equal(oracle.emp_lpn_task(seed, kk, e), oracle.lpn_primal(seed, kk, e))


@pytest.mark.parametrize("d", [1, 2, 3, 4, 5, 7, 8, 10, 11, 16, 32])
def test_lpn_d_matches_reference(d):
    rng = np.random.default_rng(300 + d)
    n, k = 997, 1 << 9  # k a power of two: the mask is k - 1, nothing subtracted
    for kk_n in (k, 3001):
        kk, e, seed = rng_blocks(rng, kk_n), rng_blocks(rng, n), rng_blocks(rng, 1)[0]
        assert np.array_equal(oracle.emp_lpn_task(seed, kk, e, d=d), oracle.lpn_primal(seed, kk, e, d=d))


def test_lpn_reference_config_c1():
    """The reference's CPU-runnable configuration: n = 65,536 rows,
    k = 8,192, d = 10, e = the sender's GGM leaves of t = 64 trees of depth 10."""
    rng = np.random.default_rng(65536)
    roots, delta = rng_blocks(rng, 64), delta_ferret(rng)
    leaves = oracle.emp_spcot_sender(roots, 10, delta)[0]
    kk, seed = rng_blocks(rng, 8192), rng_blocks(rng, 1)[0]
    assert np.array_equal(oracle.emp_lpn_task(seed, kk, leaves), oracle.lpn_primal(seed, kk, leaves, threads=4))


def test_lpn_golden(golden):
    for c in golden["lpn"]:
        out = oracle.emp_lpn_task(hx(c["seed"]), blocks(c["kk"]), blocks(c["e"]), d=c["d"])
        assert out.tobytes().hex() == c["out"], (c["n"], c["k"], c["d"])


def test_lpn_split_ranges_follow_task_semantics():
    """Two emp-ot tasks [0, m) and [m, n) each send their own last <= 4 rows
    to __compute1, so a split LPN differs from the single range; the oracle
    (and the GPU path) follow one task over [0, n)."""
    rng = np.random.default_rng(8)
    n, k = 64, 100
    kk, e, seed = rng_blocks(rng, k), rng_blocks(rng, n), rng_blocks(rng, 1)[0]
    whole = oracle.emp_lpn_task(seed, kk, e)
    split = oracle.emp_lpn_task(seed, kk, oracle.emp_lpn_task(seed, kk, e, start=0, end=32), start=32, end=64)
    assert np.array_equal(whole, oracle.lpn_primal(seed, kk, e))
    assert not np.array_equal(whole[28:32], split[28:32])
    assert np.array_equal(whole[32:60], split[32:60])
