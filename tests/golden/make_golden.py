"""Generates the golden fixtures in tests/golden/ (run in the build container).

Independent of the C oracle: AES comes from OpenSSL (python `cryptography`)
and, for the AES/PRG pins, from the reference's own vendored cryptoTools
built from source into oracle/_ref (oracle/build_ref.sh).  The GGM, LPN,
transpose and quasi-cyclic values are computed by the pure-Python
restatements below, each following the reference file:line it cites.

    python tests/golden/make_golden.py
"""
from __future__ import annotations

import hashlib
import json
import os
import sys

import numpy as np
from cryptography.hazmat.primitives.ciphers import Cipher, algorithms, modes

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)


def aes(key: bytes, data: bytes) -> bytes:
    e = Cipher(algorithms.AES(key), modes.ECB()).encryptor()
    return e.update(data) + e.finalize()


def xor(a: bytes, b: bytes) -> bytes:
    return bytes(x ^ y for x, y in zip(a, b))


def make_block(hi: int, lo: int) -> bytes:  # emp-tool makeBlock(hi, lo)
    return lo.to_bytes(8, "little") + hi.to_bytes(8, "little")


K0 = bytes(16)                 # zero_block        (spcot_sender.h:63)
K1 = make_block(0, 1)          # makeBlock(0, 1)


def node(p: bytes):            # TwoKeyPRP (twokeyprp.h:16-23)
    return xor(aes(K0, p), p), xor(aes(K1, p), p)


def mask(b: bytes) -> bytes:   # & makeBlock(~0, ~1)
    return bytes([b[0] & 0xFE]) + b[1:]


def ggm_levels(root: bytes, h: int):
    levels = [[root]]
    for _ in range(h):
        nxt = []
        for p in levels[-1]:
            l, r = node(p)
            nxt += [l, r]
        levels.append(nxt)
    return levels


def xsum(bs):
    acc = bytes(16)
    for b in bs:
        acc = xor(acc, b)
    return acc


def ferret_sender(roots, h, delta):  # spcot_sender.h:47-86
    leaves, lsum, rsum, ss = [], [], [], []
    for root in roots:
        lv = ggm_levels(root, h)
        for d in range(h):
            lsum.append(xsum(lv[d + 1][0::2]))
            rsum.append(xsum(lv[d + 1][1::2]))
        lf = [mask(x) for x in lv[h]]
        leaves += lf
        ss.append(xor(xsum(lf), delta))
    return leaves, lsum, rsum, ss


def ferret_recver(mc, choice, ss, h, t):  # spcot_recver.h:33-95
    leaves = []
    for ti in range(t):
        tree = [bytes(16)]
        pos = 0
        for d in range(h):
            nxt = []
            for p in tree:
                l, r = node(p)
                nxt += [l, r]
            tree = nxt
            f = 2 * pos
            tree[f] = tree[f + 1] = bytes(16)
            b = choice[ti * h + d]
            tree[f + b] = xor(xsum(tree[b::2]), mc[ti * h + d])
            pos = f + 1 - b
        tree[pos] = bytes(16)
        tree = [mask(x) for x in tree]
        tree[pos] = xor(xsum(tree), ss[ti])
        leaves += tree
    return leaves


def lpn(seed: bytes, kk, nn, d=10):  # lpn_f2.h:27-31, 46-79, one task [0, n)
    k, n = len(kk), len(nn)
    msk = 1
    while msk < k:
        msk = (msk << 1) | 1
    out = list(nn)
    j = 0
    while j < n - 4:
        r = aes(seed, b"".join(make_block(j, m) for m in range(d)))
        w = np.frombuffer(r, "<u4")
        for m in range(4):
            for jj in range(d):
                idx = int(w[m * d + jj]) & msk
                idx = idx - k if idx >= k else idx
                out[j + m] = xor(out[j + m], kk[idx])
        j += 4
    nb = d // 4 + (d % 4 != 0)
    while j < n:
        r = aes(seed, b"".join(make_block(j, m) for m in range(nb)))
        w = np.frombuffer(r, "<u4")
        for jj in range(d):
            out[j] = xor(out[j], kk[int(w[jj]) % k])
        j += 1
    return out


def transpose(mat: bytes, rows, row_bytes, lo, hi) -> bytes:  # gpu/gpu_ops.cu:31-70
    bits = np.unpackbits(np.frombuffer(mat, np.uint8).reshape(rows, row_bytes), axis=1, bitorder="little")
    return np.packbits(bits[:, lo:hi].T.copy(), axis=1, bitorder="little").tobytes()


def qc_a(key: bytes, n: int) -> int:  # quasi_cyclic.cu:57-66, gpu_ops.cu:102-109
    nb = n // 128
    pt = b"".join((4 * (i // 10)).to_bytes(8, "little") + (i % 10).to_bytes(8, "little") for i in range(nb))
    return int.from_bytes(aes(key, pt)[: n // 8], "little")


def clmul_cyclic(a: int, b: int, n: int) -> int:  # exact a*b mod (x^n - 1) over GF(2)
    r = 0
    x = b
    i = 0
    while a:
        if a & 1:
            r ^= x << i
        a >>= 1
        i += 1
    full = (1 << n) - 1
    out = 0
    while r:
        out ^= r & full
        r >>= n
    return out


def sot_sender(roots, h, delta, base0, base1, t):  # silent/sender.cu:76-108
    leaves = []
    m0 = [None] * ((h + 1) * t)
    m1 = [None] * ((h + 1) * t)
    for ti, root in enumerate(roots):
        lv = ggm_levels(root, h)
        leaves += lv[h]
        for d in range(h):
            L, R = xsum(lv[d + 1][0::2]), xsum(lv[d + 1][1::2])
            m0[d * t + ti] = xor(base0[d * t + ti], L)
            m1[d * t + ti] = xor(base1[d * t + ti], R)
            if d == h - 1:
                m0[h * t + ti] = xor(xor(base0[d * t + ti], R), delta)
                m1[h * t + ti] = xor(xor(base1[d * t + ti], L), delta)
    return leaves, m0, m1


def sha(b: bytes) -> str:
    return hashlib.sha256(b).hexdigest()


def main():
    import oracle  # only for the reference-built cryptoTools pins
    rng = np.random.default_rng(20241203)
    blk = lambda: rng.bytes(16)
    out = {}

    # ---- AES: FIPS-197 Appendix C.1 + random, OpenSSL == cryptoTools -------
    kat = [{"key": "000102030405060708090a0b0c0d0e0f", "pt": "00112233445566778899aabbccddeeff",
            "ct": "69c4e0d86a7b0430d8cdb78070b4c55a"}]
    assert aes(bytes.fromhex(kat[0]["key"]), bytes.fromhex(kat[0]["pt"])).hex() == kat[0]["ct"]
    for _ in range(8):
        k, p = blk(), rng.bytes(64)
        c = aes(k, p)
        ref = oracle.ref_aes_ecb(k, np.frombuffer(p, np.uint8))
        if ref is None:
            raise SystemExit("oracle/_ref/libctref.so missing: run oracle/build_ref.sh")
        assert ref.tobytes() == c, "cryptoTools AES disagrees with OpenSSL"
        kat.append({"key": k.hex(), "pt": p.hex(), "ct": c.hex()})
    out["aes"] = kat

    # ---- seeded PRG pinned on cryptoTools PRNG (PRNG.cpp:44-56,100-106) ---
    prg = []
    for _ in range(3):
        s = blk()
        prg.append({"seed": s.hex(), "blocks": oracle.ref_prng(s, 40).tobytes().hex()})
    out["prg"] = prg

    # ---- Ferret GGM sender/receiver ---------------------------------------
    ferret = []
    for (t, h) in [(1, 1), (2, 3), (3, 5)]:
        roots = [blk() for _ in range(t)]
        delta = bytearray(blk())
        delta[0] |= 1  # ferret_cot.hpp:29-31
        delta = bytes(delta)
        leaves, lsum, rsum, ss = ferret_sender(roots, h, delta)
        choice = [int(x) for x in rng.integers(0, 2, t * h)]
        mc = [lsum[i] if choice[i] == 0 else rsum[i] for i in range(t * h)]
        rl = ferret_recver(mc, choice, ss, h, t)
        ferret.append({"t": t, "h": h, "roots": b"".join(roots).hex(), "delta": delta.hex(),
                       "leaves": b"".join(leaves).hex(), "lsum": b"".join(lsum).hex(),
                       "rsum": b"".join(rsum).hex(), "secret_sum": b"".join(ss).hex(),
                       "choice": choice, "recv_leaves": b"".join(rl).hex()})
    out["ferret_ggm"] = ferret

    # ---- LPN ----------------------------------------------------------------
    lp = []
    for (n, k, d) in [(1, 5, 10), (4, 3, 10), (5, 7, 10), (8, 16, 10), (37, 19, 10), (64, 100, 10), (41, 33, 7)]:
        seed = blk()
        kk = [blk() for _ in range(k)]
        nn = [blk() for _ in range(n)]
        res = lpn(seed, kk, nn, d)
        lp.append({"n": n, "k": k, "d": d, "seed": seed.hex(), "kk": b"".join(kk).hex(),
                   "e": b"".join(nn).hex(), "out": b"".join(res).hex()})
    out["lpn"] = lp

    # ---- transpose ------------------------------------------------------------
    tr = []
    for (rows, rb, lo, hi) in [(64, 16, 0, 128), (128, 16, 32, 96), (24, 3, 8, 24)]:
        m = rng.bytes(rows * rb)
        tr.append({"rows": rows, "row_bytes": rb, "lo": lo, "hi": hi, "in": m.hex(),
                   "out": transpose(m, rows, rb, lo, hi).hex()})
    out["transpose"] = tr

    # ---- quasi-cyclic -------------------------------------------------------
    qc = []
    for n in [1024, 2048]:
        key = blk()
        a = qc_a(key, n)
        b = int.from_bytes(rng.bytes(n // 8), "little")
        prod = clmul_cyclic(a, b, n)
        pos = [int(x) for x in rng.integers(0, n, 5)]
        sp = 0
        for p_ in pos:
            sp ^= ((a << p_) | (a >> (n - p_))) & ((1 << n) - 1)
        qc.append({"n": n, "key": key.hex(), "a": a.to_bytes(n // 8, "little").hex(),
                   "b": b.to_bytes(n // 8, "little").hex(),
                   "ab": prod.to_bytes(n // 8, "little").hex(), "pos": pos,
                   "sparse": sp.to_bytes(n // 8, "little").hex()})
    # dual LPN on n = 1024 blocks: out block j = XOR_{i: a_i} in[(j - i) mod n]
    n = 1024
    key = blk()
    a = qc_a(key, n)
    blocks = rng.bytes(16 * n)
    planes = transpose(blocks, n, 16, 0, 128)
    enc = b"".join(clmul_cyclic(a, int.from_bytes(planes[r * n // 8:(r + 1) * n // 8], "little"), n)
                   .to_bytes(n // 8, "little") for r in range(128))
    dual = transpose(enc, 128, n // 8, 0, n)
    qc.append({"n": n, "key": key.hex(), "dual_in_sha": sha(blocks), "dual_in_seed_note": "in = blocks",
               "dual_in": blocks.hex(), "dual_out_sha": sha(dual)})
    out["qc"] = qc

    # ---- SOT PPRF sender ----------------------------------------------------
    sot = []
    for (t, h) in [(2, 3), (3, 4)]:
        roots = [blk() for _ in range(t)]
        delta = blk()
        base0 = [blk() for _ in range(h * t)]
        base1 = [blk() for _ in range(h * t)]
        leaves, m0, m1 = sot_sender(roots, h, delta, base0, base1, t)
        choice = [int(x) for x in rng.integers(0, 2, h * t)]
        mc = [base0[i] if choice[i] == 0 else base1[i] for i in range(h * t)]
        sot.append({"t": t, "h": h, "roots": b"".join(roots).hex(), "delta": delta.hex(),
                    "base0": b"".join(base0).hex(), "base1": b"".join(base1).hex(),
                    "leaves": b"".join(leaves).hex(), "m0": b"".join(m0).hex(), "m1": b"".join(m1).hex(),
                    "choice": choice, "mc": b"".join(mc).hex()})
    out["sot_pprf"] = sot

    with open(os.path.join(HERE, "golden.json"), "w") as f:
        json.dump(out, f, indent=0)
    print("wrote", os.path.join(HERE, "golden.json"), os.path.getsize(os.path.join(HERE, "golden.json")), "bytes")


if __name__ == "__main__":
    main()
