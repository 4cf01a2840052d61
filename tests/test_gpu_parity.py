"""GPU parity tests: every CUDA entry point, called through the C ABI, is
bit-exact against the CPU oracle on seeded inputs and against the golden
fixtures; full-size configurations are checked through size-independent
properties (COT correlation, sender/receiver agreement, linearity)."""
import hashlib
import zlib

import numpy as np
import pytest

import oracle
from tests.util import blocks, hx, rng_blocks, delta_ferret, to_dev, to_host

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def empty_blocks(n):
    return torch.empty((n, 16), dtype=torch.uint8, device="cuda")


# ---------------------------------------------------------------- AES
@pytest.mark.parametrize("n", [1, 2, 3, 255, 4096, 100003])
def test_aes_ecb(ctx, n):
    rng = np.random.default_rng(n)
    key, pt = rng_blocks(rng, 1)[0], rng_blocks(rng, n)
    d = to_dev(pt)
    ctx.aes128_ecb(key, d)
    assert np.array_equal(to_host(d), oracle.aes_ecb(key, pt))


def test_aes_golden(ctx, golden):
    for c in golden["aes"]:
        d = to_dev(blocks(c["pt"]))
        ctx.aes128_ecb(hx(c["key"]), d)
        assert to_host(d).tobytes().hex() == c["ct"]


# ---------------------------------------------------------------- Ferret GGM
def run_ferret_sender(ctx, roots, h, delta):
    t = roots.shape[0]
    leaves, lsum, rsum, ss = empty_blocks(t << h), empty_blocks(t * h), empty_blocks(t * h), empty_blocks(t)
    ctx.ferret_pprf_sender(to_dev(roots), h, delta, leaves, lsum, rsum, ss)
    return to_host(leaves), to_host(lsum), to_host(rsum), to_host(ss)


def run_ferret_recver(ctx, mc, choice, ss, h):
    t = ss.shape[0]
    leaves = empty_blocks(t << h)
    ctx.ferret_pprf_recver(to_dev(mc), to_dev(choice), to_dev(ss), h, leaves)
    return to_host(leaves)


def test_ferret_ggm_golden(ctx, golden):
    for c in golden["ferret_ggm"]:
        h = c["h"]
        lv, ls, rs, ss = run_ferret_sender(ctx, blocks(c["roots"]), h, hx(c["delta"]))
        assert lv.tobytes().hex() == c["leaves"]
        assert ls.tobytes().hex() == c["lsum"]
        assert rs.tobytes().hex() == c["rsum"]
        assert ss.tobytes().hex() == c["secret_sum"]
        ch = np.array(c["choice"], np.uint8)
        mc = np.where(ch[:, None] == 0, ls, rs)
        assert run_ferret_recver(ctx, mc, ch, ss, h).tobytes().hex() == c["recv_leaves"]


@pytest.mark.parametrize("t,h", [(1, 1), (5, 2), (3, 7), (64, 10), (7, 13), (2, 16), (300, 9)])
def test_ferret_ggm_vs_oracle(ctx, t, h):
    rng = np.random.default_rng(1000 * t + h)
    roots, delta = rng_blocks(rng, t), delta_ferret(rng)
    got = run_ferret_sender(ctx, roots, h, delta)
    exp = oracle.ferret_pprf_sender(roots, h, delta, threads=8)
    for g, e in zip(got, exp):
        assert np.array_equal(g, e)
    ch = rng.integers(0, 2, t * h).astype(np.uint8)
    mc = np.where(ch[:, None] == 0, exp[1], exp[2])
    gr = run_ferret_recver(ctx, mc, ch, exp[3], h)
    er = oracle.ferret_pprf_recver(mc, ch, exp[3], h, threads=8)
    assert np.array_equal(gr, er)


def test_ferret_full_size_b13(ctx):
    """ferret_b13 (constants.h:25): t = 1280 trees of depth 13, bit-exact
    against the multi-threaded oracle, plus the COT correlation."""
    t, h = 1280, 13
    rng = np.random.default_rng(13)
    roots, delta = rng_blocks(rng, t), delta_ferret(rng)
    got = run_ferret_sender(ctx, roots, h, delta)
    exp = oracle.ferret_pprf_sender(roots, h, delta, threads=16)
    for g, e in zip(got, exp):
        assert np.array_equal(g, e)
    ch = rng.integers(0, 2, t * h).astype(np.uint8)
    mc = np.where(ch[:, None] == 0, exp[1], exp[2])
    gr = run_ferret_recver(ctx, mc, ch, exp[3], h)
    diff = gr ^ exp[0]
    rows = np.nonzero(diff.any(axis=1))[0]
    assert rows.shape[0] == t
    assert (diff[rows] == delta).all()


# ---------------------------------------------------------------- LPN
def test_lpn_golden(ctx, golden):
    for c in golden["lpn"]:
        e = to_dev(blocks(c["e"]))
        ctx.lpn_primal(hx(c["seed"]), to_dev(blocks(c["kk"])), e, d=c["d"])
        assert to_host(e).tobytes().hex() == c["out"], (c["n"], c["k"], c["d"])


@pytest.mark.parametrize("n,k,d", [(65536, 8192, 10), (1000, 999, 10), (12345, 4097, 10),
                                   (9999, 511, 3), (777, 65, 16), (6, 2, 10)])
def test_lpn_vs_oracle(ctx, n, k, d):
    rng = np.random.default_rng(n + k + d)
    seed, kk, e = rng_blocks(rng, 1)[0], rng_blocks(rng, k), rng_blocks(rng, n)
    dev = to_dev(e)
    ctx.lpn_primal(seed, to_dev(kk), dev, d=d)
    assert np.array_equal(to_host(dev), oracle.lpn_primal(seed, kk, e, d=d, threads=8))


def test_lpn_full_size_b13(ctx):
    n, k = 10485760, 452000
    rng = np.random.default_rng(452)
    seed, kk, e = rng_blocks(rng, 1)[0], rng_blocks(rng, k), rng_blocks(rng, n)
    dev = to_dev(e)
    ctx.lpn_primal(seed, to_dev(kk), dev)
    assert np.array_equal(to_host(dev), oracle.lpn_primal(seed, kk, e, threads=16))


# ---------------------------------------------------------------- transpose
def test_transpose_golden(ctx, golden):
    for c in golden["transpose"]:
        rows, rb, lo, hi = c["rows"], c["row_bytes"], c["lo"], c["hi"]
        out = torch.empty((hi - lo) * rows // 8, dtype=torch.uint8, device="cuda")
        ctx.bit_transpose(to_dev(hx(c["in"])), rows, rb, lo, hi, out)
        assert to_host(out).tobytes().hex() == c["out"]


@pytest.mark.parametrize("rows,rb,lo,hi", [(1 << 20, 16, 0, 128), (1152, 16, 0, 128), (4096 + 32 * 5, 16, 32, 96),
                                           (128, 1 << 14, 0, 1 << 17), (128, 144, 0, 1152), (128, 512, 0, 2048),
                                           (128, 1024, 0, 4096 + 96), (64, 1024, 0, 8192),
                                           (96, 40, 16, 320), (8, 1, 0, 8)])
@pytest.mark.parametrize("offset", [0, 4])
def test_transpose_vs_oracle(ctx, rows, rb, lo, hi, offset):
    """Every path of the transpose: all 128 planes (partial last tiles at
    1152 rows / columns), plane ranges, fewer than 128 planes, the leading
    columns of wider plane rows (the rate-1/2 form's second transpose), the
    byte-granular shapes; offset 4: input and output 4 bytes past a 16-byte
    boundary, where the 16-byte fast paths give way."""
    rng = np.random.default_rng(rows + rb)
    m = rng.integers(0, 256, rows * rb, dtype=np.uint8)
    nout = (hi - lo) * rows // 8
    src = torch.zeros(rows * rb + 16, dtype=torch.uint8, device="cuda")
    src[offset:offset + rows * rb] = to_dev(m)
    dst = torch.zeros(nout + 16, dtype=torch.uint8, device="cuda")
    ctx.bit_transpose(src[offset:], rows, rb, lo, hi, dst[offset:])
    exp = np.unpackbits(m.reshape(rows, rb), axis=1, bitorder="little")[:, lo:hi].T
    exp = np.packbits(np.ascontiguousarray(exp), axis=1, bitorder="little").reshape(-1)
    got = to_host(dst)
    assert np.array_equal(got[offset:offset + nout], exp)
    assert not got[:offset].any() and not got[offset + nout:].any()  # nothing written outside


def test_transpose_past_2p23_rows(ctx):
    """Rows beyond 2^23 (the reference's transposer indexes wrongly there):
    2^23 + 64 blocks to planes and back, against the oracle's transpose and
    round-tripped."""
    rows = (1 << 23) + 64
    rng = np.random.default_rng(24)
    m = rng.integers(0, 256, (rows, 16), dtype=np.uint8)
    planes = torch.empty(128 * rows // 8, dtype=torch.uint8, device="cuda")
    dm = to_dev(m)
    ctx.bit_transpose(dm, rows, 16, 0, 128, planes)
    exp = oracle.bit_transpose(m, rows, 16, 0, 128)
    assert np.array_equal(to_host(planes), exp.reshape(-1))
    back = torch.empty((rows, 16), dtype=torch.uint8, device="cuda")
    ctx.bit_transpose(planes, 128, rows // 8, 0, rows, back)
    assert torch.equal(back, dm)


# ---------------------------------------------------------------- QC
def test_qc_golden(ctx, golden):
    for c in golden["qc"]:
        n = c["n"]
        a = torch.empty(n // 64, dtype=torch.int64, device="cuda")
        ctx.qc_gen_a(hx(c["key"]), n, a)
        if "a" in c:
            assert to_host(a).tobytes().hex() == c["a"]
            b = to_dev(hx(c["b"]).view(np.int64))
            ctx.qc_encode(a, b, n, 1)
            assert to_host(b).tobytes().hex() == c["ab"]
            out = torch.empty(n // 64, dtype=torch.int64, device="cuda")
            ctx.qc_encode_sparse(a, to_dev(np.array(c["pos"], np.int64)), n, out)
            assert to_host(out).tobytes().hex() == c["sparse"]
        else:
            io = to_dev(blocks(c["dual_in"]))
            ctx.sot_dual_lpn(a, io, n)
            assert hashlib.sha256(to_host(io).tobytes()).hexdigest() == c["dual_out_sha"]


@pytest.mark.parametrize("e,nplanes", [(10, 3), (11, 1), (12, 5), (13, 2), (14, 7), (16, 2), (20, 2)])
def test_qc_encode_vs_oracle(ctx, e, nplanes):
    n = 1 << e
    rng = np.random.default_rng(e)
    key = rng_blocks(rng, 1)[0]
    a = torch.empty(n // 64, dtype=torch.int64, device="cuda")
    ctx.qc_gen_a(key, n, a)
    a_np = oracle.qc_gen_a(key, n)
    assert np.array_equal(to_host(a).view(np.uint64), a_np)
    planes = rng.integers(0, 2**63, (nplanes, n // 64), dtype=np.uint64)
    # include the extreme planes: all-zero and all-ones
    planes[0, :] = 0
    if nplanes > 2:
        planes[2, :] = np.uint64(0xFFFFFFFFFFFFFFFF)
    d = to_dev(planes.view(np.int64))
    ctx.qc_encode(a, d, n, nplanes)
    exp = oracle.qc_encode(a_np, planes, n, threads=8)
    assert np.array_equal(to_host(d).view(np.uint64), exp)


@pytest.mark.parametrize("e", [21, 22, 24, 25])
def test_qc_encode_large_sizes(ctx, e):
    """Plane encodes at n = 2^21 (the FFT's 4096-point row pass, packing base
    2^21 + 1) and the NTT's 2048/4096/8192-point pass kernels (n = 2^22 ..
    2^25, the largest size the row pass fits) against the oracle on two
    planes."""
    n = 1 << e
    rng = np.random.default_rng(e + 1000)
    key = rng_blocks(rng, 1)[0]
    a = torch.empty(n // 64, dtype=torch.int64, device="cuda")
    ctx.qc_gen_a(key, n, a)
    planes = rng.integers(0, 2**63, (2, n // 64), dtype=np.uint64)
    d = to_dev(planes.view(np.int64))
    ctx.qc_encode(a, d, n, 2)
    exp = oracle.qc_encode(to_host(a).view(np.uint64), planes, n, threads=16)
    assert np.array_equal(to_host(d).view(np.uint64), exp)


def test_qc_plan_matches_one_shot(ctx):
    n = 1 << 15
    rng = np.random.default_rng(77)
    a = torch.empty(n // 64, dtype=torch.int64, device="cuda")
    ctx.qc_gen_a(rng_blocks(rng, 1)[0], n, a)
    io = rng_blocks(rng, n)
    d1, d2 = to_dev(io), to_dev(io)
    ctx.sot_dual_lpn(a, d1, n)
    plan = ctx.qc_plan(a, n)
    plan.set_batch(5)
    plan.dual_lpn(d2)
    assert np.array_equal(to_host(d1), to_host(d2))
    exp = oracle.sot_dual_lpn(to_host(a).view(np.uint64), io, n, threads=8)
    assert np.array_equal(to_host(d1), exp)


def test_qc_dual_lpn_full_size_linearity(ctx):
    """n = 2^20, 128 planes: linearity of the encode and a spot check of
    planes against the oracle."""
    n = 1 << 20
    rng = np.random.default_rng(20)
    a = torch.empty(n // 64, dtype=torch.int64, device="cuda")
    ctx.qc_gen_a(rng_blocks(rng, 1)[0], n, a)
    x, y = rng_blocks(rng, n), rng_blocks(rng, n)
    dx, dy, dxy = to_dev(x), to_dev(y), to_dev(x ^ y)
    for d in (dx, dy, dxy):
        ctx.sot_dual_lpn(a, d, n)
    assert np.array_equal(to_host(dx) ^ to_host(dy), to_host(dxy))
    planes = oracle.bit_transpose(x, n, 16, 0, 128).view(np.uint64).reshape(128, n // 64)
    outp = oracle.bit_transpose(to_host(dx), n, 16, 0, 128).view(np.uint64).reshape(128, n // 64)
    a_np = to_host(a).view(np.uint64)
    for r in (0, 63, 127):
        assert np.array_equal(outp[r], oracle.gf2_cyclic_mul(a_np, planes[r], n))


# ---------------------------------------------------------------- SOT
def sot_inputs(rng, t, h):
    return (rng_blocks(rng, t), rng_blocks(rng, 1)[0], rng_blocks(rng, h * t), rng_blocks(rng, h * t),
            rng.integers(0, 2, h * t).astype(np.uint8))


def run_sot(ctx, roots, h, delta, b0, b1, choice):
    t = roots.shape[0]
    leaves, m0, m1 = empty_blocks(t << h), empty_blocks((h + 1) * t), empty_blocks((h + 1) * t)
    ctx.sot_pprf_sender(to_dev(roots), h, delta, to_dev(b0), to_dev(b1), leaves, m0, m1)
    mc = np.where(choice[:, None] == 0, b0, b1)
    rleaves = empty_blocks(t << h)
    ctx.sot_pprf_recver(m0, m1, to_dev(mc), to_dev(choice), t, h, rleaves)
    return to_host(leaves), to_host(m0), to_host(m1), to_host(rleaves), mc


def test_sot_pprf_golden(ctx, golden):
    for c in golden["sot_pprf"]:
        t, h = c["t"], c["h"]
        ch = np.array(c["choice"], np.uint8)
        lv, m0, m1, rl, _ = run_sot(ctx, blocks(c["roots"]), h, hx(c["delta"]), blocks(c["base0"]),
                                    blocks(c["base1"]), ch)
        assert lv.tobytes().hex() == c["leaves"]
        assert m0.tobytes().hex() == c["m0"]
        assert m1.tobytes().hex() == c["m1"]
        assert np.array_equal(rl, oracle.sot_pprf_recver(m0, m1, blocks(c["mc"]), ch, t, h))


@pytest.mark.parametrize("t,h", [(1, 1), (3, 5), (256, 12), (17, 10)])
def test_sot_pprf_vs_oracle(ctx, t, h):
    rng = np.random.default_rng(t * 7 + h)
    roots, delta, b0, b1, ch = sot_inputs(rng, t, h)
    lv, m0, m1, rl, mc = run_sot(ctx, roots, h, delta, b0, b1, ch)
    el, e0, e1 = oracle.sot_pprf_sender(roots, h, delta, b0, b1, threads=8)
    assert np.array_equal(lv, el) and np.array_equal(m0, e0) and np.array_equal(m1, e1)
    assert np.array_equal(rl, oracle.sot_pprf_recver(e0, e1, mc, ch, t, h, threads=8))


def test_sot_end_to_end_cot_n20(ctx):
    """Plain SOT at n = 2^20 (256 trees of depth 12): PPRF -> transpose ->
    exact QC encode -> transpose on both roles; the outputs form a COT:
    w_j = v_j ^ c_j * delta with c = a * e (encode_sparse of the punctured
    positions)."""
    t, h = 256, 12
    n = t << h
    rng = np.random.default_rng(2020)
    roots, delta, b0, b1, ch = sot_inputs(rng, t, h)
    lv, m0, m1, rl, mc = run_sot(ctx, roots, h, delta, b0, b1, ch)
    a = torch.empty(n // 64, dtype=torch.int64, device="cuda")
    ctx.qc_gen_a(rng_blocks(rng, 1)[0], n, a)
    v, w = to_dev(lv), to_dev(rl)
    ctx.sot_dual_lpn(a, v, n)
    ctx.sot_dual_lpn(a, w, n)
    chm = ch.reshape(h, t)
    pos = np.zeros(t, np.int64)
    for d in range(h):
        pos = pos * 2 + 1 - chm[d].astype(np.int64)
    pos += np.arange(t) * (1 << h)
    c = torch.empty(n // 64, dtype=torch.int64, device="cuda")
    ctx.qc_encode_sparse(a, to_dev(pos), n, c)
    cbits = np.unpackbits(to_host(c).view(np.uint8), bitorder="little").astype(bool)
    diff = to_host(v) ^ to_host(w)
    assert not diff[~cbits].any()
    assert (diff[cbits] == delta).all()
    assert 0.4 < cbits.mean() < 0.6


# ---------------------------------------------------------------- SOT rate-1/2 form
@pytest.mark.parametrize("e", [10, 13, 16])
def test_sot_dual_lpn_r2_vs_oracle(ctx, e):
    """out = e0 ^ a * e1 per bit plane over 2n noise blocks; one-shot, plan,
    and in place (out aliasing the first n input blocks)."""
    n = 1 << e
    rng = np.random.default_rng(300 + e)
    a = torch.empty(n // 64, dtype=torch.int64, device="cuda")
    ctx.qc_gen_a(rng_blocks(rng, 1)[0], n, a)
    a_np = to_host(a).view(np.uint64)
    x = rng_blocks(rng, 2 * n)
    exp = x[:n] ^ oracle.sot_dual_lpn(a_np, x[n:].copy(), n, threads=8)
    d, out = to_dev(x), empty_blocks(n)
    ctx.sot_dual_lpn_r2(a, d, n, out)
    assert np.array_equal(to_host(out), exp)
    assert np.array_equal(to_host(d), x)
    plan = ctx.qc_plan(a, n)
    plan.set_batch(3)
    plan.dual_lpn_r2(d, d[:n])
    assert np.array_equal(to_host(d)[:n], exp)
    assert np.array_equal(to_host(d)[n:], x[n:])


def _tree_positions(rng, n, h):
    t = n >> h
    return np.arange(t, dtype=np.int64) * (1 << h) + rng.integers(0, 1 << h, t)


@pytest.mark.parametrize("case", ["tree_h10_n22", "tree_h11_n21", "tree_h14_n20", "tree_h4_n10", "unsorted_wide",
                                  "unsorted_close", "beyond_n", "n_not_pow2", "duplicates"])
def test_qc_encode_sparse_position_orders(ctx, case):
    """The sparse encode (receiver choice bits a * e) against the oracle for
    the position layouts it meets: tree order (one position per GGM tree,
    where a chunk's windows of `a` are staged in shared memory), positions
    spread too wide for the window (the global-memory loop), positions >= n
    (ignored), n not a power of two, repeated positions (they cancel)."""
    rng = np.random.default_rng(zlib.crc32(case.encode()))
    n = {"tree_h10_n22": 1 << 22, "tree_h11_n21": 1 << 21, "tree_h14_n20": 1 << 20, "tree_h4_n10": 1 << 10,
         "n_not_pow2": 64 * 1000}.get(case, 1 << 18)
    if case.startswith("tree"):
        pos = _tree_positions(rng, n, int(case.split("_h")[1].split("_")[0]))
    elif case == "unsorted_wide":
        pos = rng.integers(0, n, 3000)
    elif case == "unsorted_close":
        pos = rng.permutation(np.arange(5000, 5000 + 64 * 300, 64) + rng.integers(0, 64, 300))
    elif case == "beyond_n":
        pos = np.concatenate([rng.integers(0, n, 500), rng.integers(n, 3 * n, 100), [n, n - 1, 0]])
        rng.shuffle(pos)
    elif case == "n_not_pow2":
        pos = np.sort(rng.integers(0, n, 700))
    else:
        base = rng.integers(0, n, 200)
        pos = np.concatenate([base, base[:50], rng.integers(0, n, 30)])
    a_np = rng.integers(0, 2**63, n // 64, dtype=np.uint64) | (rng.integers(0, 2, n // 64, dtype=np.uint64) << np.uint64(63))
    a = to_dev(a_np.view(np.int64))
    out = torch.full((n // 64,), -1, dtype=torch.int64, device="cuda")  # overwritten, not XORed into
    ctx.qc_encode_sparse(a, to_dev(pos.astype(np.int64)), n, out)
    exp = oracle.qc_encode_sparse(a_np, pos.astype(np.uint64), n)
    assert np.array_equal(to_host(out).view(np.uint64), exp)


def test_qc_encode_sparse_r2(ctx):
    n = 1 << 14
    rng = np.random.default_rng(41)
    a = torch.empty(n // 64, dtype=torch.int64, device="cuda")
    ctx.qc_gen_a(rng_blocks(rng, 1)[0], n, a)
    a_np = to_host(a).view(np.uint64)
    pos = np.concatenate([rng.choice(2 * n, 37, replace=False), [0, n - 1, n, 2 * n - 1, 2 * n, 5 * n]])
    out = torch.empty(n // 64, dtype=torch.int64, device="cuda")
    ctx.qc_encode_sparse_r2(a, to_dev(pos.astype(np.int64)), n, out)
    e0 = np.zeros(n, np.uint8)
    for p in pos[pos < n]:
        e0[p] ^= 1
    p1 = pos[(pos >= n) & (pos < 2 * n)] - n
    exp = np.packbits(e0, bitorder="little").view(np.uint64) ^ oracle.qc_encode_sparse(a_np, p1, n)
    assert np.array_equal(to_host(out).view(np.uint64), exp)


def test_sot_end_to_end_cot_n20_r2(ctx):
    """Rate-1/2 SOT with n = 2^20 outputs: 512 trees of depth 12 give 2n
    noise blocks per role; after the rate-1/2 encode w_j = v_j ^ c_j * delta
    with c = e0 ^ a * e1 from the punctured positions."""
    t, h = 512, 12
    n = (t << h) // 2
    rng = np.random.default_rng(2121)
    roots, delta, b0, b1, ch = sot_inputs(rng, t, h)
    lv, m0, m1, rl, mc = run_sot(ctx, roots, h, delta, b0, b1, ch)
    a = torch.empty(n // 64, dtype=torch.int64, device="cuda")
    ctx.qc_gen_a(rng_blocks(rng, 1)[0], n, a)
    v, w = to_dev(lv), to_dev(rl)
    plan = ctx.qc_plan(a, n)
    plan.dual_lpn_r2(v, v[:n])
    plan.dual_lpn_r2(w, w[:n])
    chm = ch.reshape(h, t)
    pos = np.zeros(t, np.int64)
    for d in range(h):
        pos = pos * 2 + 1 - chm[d].astype(np.int64)
    pos += np.arange(t) * (1 << h)
    c = torch.empty(n // 64, dtype=torch.int64, device="cuda")
    ctx.qc_encode_sparse_r2(a, to_dev(pos), n, c)
    cbits = np.unpackbits(to_host(c).view(np.uint8), bitorder="little").astype(bool)
    diff = to_host(v)[:n] ^ to_host(w)[:n]
    assert not diff[~cbits].any()
    assert (diff[cbits] == delta).all()
    assert 0.4 < cbits.mean() < 0.6


# ---------------------------------------------------------------- row-range LPN / sharding
@pytest.mark.parametrize("n,k,cuts", [(4096, 1000, [0, 1024, 2048, 4096]), (1003, 77, [0, 500, 1003]),
                                      (10, 5, [0, 4, 8, 10])])
def test_lpn_row_ranges_equal_unsplit(ctx, n, k, cuts):
    rng = np.random.default_rng(n)
    seed, kk, e = rng_blocks(rng, 1)[0], rng_blocks(rng, k), rng_blocks(rng, n)
    exp = oracle.lpn_primal(seed, kk, e, threads=4)
    dkk = to_dev(kk)
    for lo, hi in zip(cuts[:-1], cuts[1:]):
        part = to_dev(e[lo:hi])
        ctx.lpn_primal_range(seed, dkk, part, lo, hi, n)
        assert np.array_equal(to_host(part), exp[lo:hi])


@pytest.mark.parametrize("side_stream", [False, True])
def test_sharded_ferret_extend_equals_unsplit(ctx, side_stream):
    """The per-rank share computation of cuot_b200.shard, run for each of 3
    ranks in turn on this GPU, concatenates to the unsplit extension, also
    when the caller passes a stream other than the current one (its torch
    ops must then run on that stream too)."""
    from cuot_b200.shard import ShardPlan, ferret_extend_rank
    side = torch.cuda.Stream() if side_stream else None
    t, h, k = 10, 8, 999
    rng = np.random.default_rng(31)
    roots, delta = rng_blocks(rng, t), delta_ferret(rng)
    choice = rng.integers(0, 2, t * h).astype(np.uint8)
    seed, kk_s, kk_r = rng_blocks(rng, 1)[0], rng_blocks(rng, k), rng_blocks(rng, k)
    plan = ShardPlan(t, h, 3)
    vs, ws = [], []
    for r in range(3):
        f, tr = plan.first_tree(r), plan.trees(r)
        v, w = ferret_extend_rank(ctx, plan, r, to_dev(roots[f:f + tr]), delta,
                                  to_dev(choice[f * h:(f + tr) * h]), seed, to_dev(kk_s), to_dev(kk_r),
                                  stream=side)
        if side is not None:
            side.synchronize()
        vs.append(to_host(v))
        ws.append(to_host(w))
    leaves, lsum, rsum, ss = oracle.ferret_pprf_sender(roots, h, delta, threads=4)
    mc = np.where(choice[:, None] == 0, lsum, rsum)
    rleaves = oracle.ferret_pprf_recver(mc, choice, ss, h, threads=4)
    assert np.array_equal(np.concatenate(vs), oracle.lpn_primal(seed, kk_s, leaves))
    assert np.array_equal(np.concatenate(ws), oracle.lpn_primal(seed, kk_r, rleaves))


@pytest.mark.parametrize("side_stream", [False, True])
def test_sharded_sot_dual_lpn_one_rank_nccl(ctx, side_stream):
    """cuot_b200.shard's SOT path (transpose -> all-to-all to plane owners ->
    encode -> reverse all-to-all -> transpose) through a one-rank NCCL group
    on this GPU equals the unsplit dual LPN, on the current stream and on a
    side stream the caller passes.  The multi-rank exchange itself is covered
    by the gloo tests in test_shard.py."""
    import datetime
    import socket
    import torch.distributed as dist
    from cuot_b200.shard import ShardPlan, sot_dual_lpn_rank
    sk = socket.socket()
    sk.bind(("127.0.0.1", 0))
    port = sk.getsockname()[1]
    sk.close()
    dist.init_process_group("nccl", init_method=f"tcp://127.0.0.1:{port}", rank=0, world_size=1,
                            timeout=datetime.timedelta(seconds=60))
    try:
        t, h = 16, 10
        n = t << h
        rng = np.random.default_rng(4242)
        rows = rng_blocks(rng, n)
        a = torch.empty(n // 64, dtype=torch.int64, device="cuda")
        ctx.qc_gen_a(rng_blocks(rng, 1)[0], n, a)
        side = torch.cuda.Stream() if side_stream else None
        out = sot_dual_lpn_rank(ctx, ShardPlan(t, h, 1), 0, a, to_dev(rows), stream=side)
        if side is not None:
            side.synchronize()
        exp = oracle.sot_dual_lpn(to_host(a).view(np.uint64), rows, n, threads=8)
        assert np.array_equal(to_host(out), exp)
    finally:
        dist.destroy_process_group()


def test_pprf_128_threads_per_tree_matches_oracle(ctx):
    """The tuning knob CUOT_TUNE_PPRF_THREADS = 128 changes the CTA size only."""
    ctx.set_tuning(ctx.TUNE_PPRF_THREADS, 128)
    try:
        for t, h in [(3, 7), (20, 11), (1, 1)]:
            rng = np.random.default_rng(t + 100 * h)
            roots, delta = rng_blocks(rng, t), delta_ferret(rng)
            got = run_ferret_sender(ctx, roots, h, delta)
            exp = oracle.ferret_pprf_sender(roots, h, delta, threads=8)
            for g, e in zip(got, exp):
                assert np.array_equal(g, e)
            ch = rng.integers(0, 2, t * h).astype(np.uint8)
            mc = np.where(ch[:, None] == 0, exp[1], exp[2])
            assert np.array_equal(run_ferret_recver(ctx, mc, ch, exp[3], h),
                                  oracle.ferret_pprf_recver(mc, ch, exp[3], h, threads=8))
            r2, d2, b0, b1, ch2 = sot_inputs(rng, t, h)
            lv, m0, m1, rl, mc2 = run_sot(ctx, r2, h, d2, b0, b1, ch2)
            el, e0, e1 = oracle.sot_pprf_sender(r2, h, d2, b0, b1, threads=8)
            assert np.array_equal(lv, el) and np.array_equal(m0, e0)
            assert np.array_equal(rl, oracle.sot_pprf_recver(e0, e1, mc2, ch2, t, h, threads=8))
    finally:
        ctx.set_tuning(ctx.TUNE_PPRF_THREADS, 256)
