"""Generates bitslice_sbox.cuh: the AES S-box as a straight-line circuit of
XOR / AND / NOT gates for the bitsliced AES kernel (aes_bitslice.cu).

Build step, run by hand after editing (python gen_bitslice_sbox.py); the
generated header is committed.  Derivation, from the definitions:

  S(x) = A . x^-1 + 0x63 in GF(2^8) = GF(2)[X] / (X^8 + X^4 + X^3 + X + 1)
  (0^-1 = 0), A the FIPS-197 affine matrix (bit i of S = x_i ^ x_{i+4} ^
  x_{i+5} ^ x_{i+6} ^ x_{i+7} ^ c_i, indices mod 8).

The inversion is computed in an isomorphic tower field
  GF(4)   = GF(2)[w] / (w^2 + w + 1)
  GF(16)  = GF(4)[z] / (z^2 + z + N),  N in GF(4) with trace 1
  GF(256) = GF(16)[y] / (y^2 + y + L), L in GF(16) with trace 1
where (a y + b)^-1 = (a y + (a + b)) / (a^2 L + a b + b^2) and likewise one
level down; GF(4) inversion is squaring.  The isomorphism maps the AES
generator X to a root of X^8 + X^4 + X^3 + X + 1 in the tower field (found by
search), which fixes an 8x8 GF(2) matrix T; the circuit is
  bits -> T -> tower inversion (products by Karatsuba) -> A T^-1 -> ^ 0x63.
Linear layers are emitted with greedy common-subexpression elimination of
XOR pairs (Paar's heuristic).  The program is checked against the S-box
computed from its definition on all 256 inputs before the header is written.
"""
from __future__ import annotations

import itertools
import os

AES_POLY = 0x11B


# ---- reference arithmetic (definitions) ------------------------------------
def gf256_mul(a: int, b: int) -> int:
    r = 0
    while b:
        if b & 1:
            r ^= a
        a <<= 1
        if a & 0x100:
            a ^= AES_POLY
        b >>= 1
    return r


def gf256_inv(a: int) -> int:
    if a == 0:
        return 0
    r, e = 1, 254  # a^254
    while e:
        if e & 1:
            r = gf256_mul(r, a)
        a = gf256_mul(a, a)
        e >>= 1
    return r


def affine(x: int) -> int:
    y = 0
    for i in range(8):
        bit = (x >> i) ^ (x >> ((i + 4) % 8)) ^ (x >> ((i + 5) % 8)) ^ (x >> ((i + 6) % 8)) ^ (x >> ((i + 7) % 8))
        y |= (bit & 1) << i
    return y ^ 0x63


SBOX = [affine(gf256_inv(x)) for x in range(256)]


# ---- tower field on ints -----------------------------------------------------
# GF(4): 2 bits (b1 w + b0); GF(16): 4 bits (hi GF(4) * z + lo); GF(256): 8 bits (hi GF(16) * y + lo).
def g4_mul(a, b):
    a1, a0, b1, b0 = a >> 1, a & 1, b >> 1, b & 1
    hi = (a1 & b1) ^ (a1 & b0) ^ (a0 & b1)
    lo = (a1 & b1) ^ (a0 & b0)
    return (hi << 1) | lo


def g16_mul(a, b, N):
    p1, q1, p2, q2 = a >> 2, a & 3, b >> 2, b & 3
    pp = g4_mul(p1, p2)
    hi = pp ^ g4_mul(p1, q2) ^ g4_mul(q1, p2)
    lo = g4_mul(pp, N) ^ g4_mul(q1, q2)
    return (hi << 2) | lo


def g256_mul(a, b, N, L):
    a1, a0, b1, b0 = a >> 4, a & 15, b >> 4, b & 15
    aa = g16_mul(a1, b1, N)
    hi = aa ^ g16_mul(a1, b0, N) ^ g16_mul(a0, b1, N)
    lo = g16_mul(aa, L, N) ^ g16_mul(a0, b0, N)
    return (hi << 4) | lo


def trace16(x, N):
    t, p = 0, x
    for _ in range(4):
        t ^= p
        p = g16_mul(p, p, N)
    return t  # in GF(2) (0 or 1)


def pick_tower():
    for N in (2, 3):  # w or w + 1 (trace 1 in GF(4))
        if g4_mul(N, N) ^ N == 0:
            continue
        for L in range(1, 16):
            if trace16(L, N) != 1:
                continue
            # X -> beta with beta^8 + beta^4 + beta^3 + beta + 1 = 0
            for beta in range(2, 256):
                pw = [1]
                for _ in range(8):
                    pw.append(g256_mul(pw[-1], beta, N, L))
                if pw[8] ^ pw[4] ^ pw[3] ^ pw[1] ^ pw[0] == 0:
                    return N, L, pw[:8]
    raise RuntimeError("no tower found")


N_, L_, BETA_POWERS = pick_tower()


def to_tower(x: int) -> int:
    r = 0
    for i in range(8):
        if (x >> i) & 1:
            r ^= BETA_POWERS[i]
    return r


TO_TOWER = [to_tower(x) for x in range(256)]
FROM_TOWER = [0] * 256
for _x, _t in enumerate(TO_TOWER):
    FROM_TOWER[_t] = _x
assert sorted(TO_TOWER) == list(range(256))
for _a, _b in itertools.product(range(0, 256, 17), range(0, 256, 13)):  # homomorphism spot check
    assert TO_TOWER[gf256_mul(_a, _b)] == g256_mul(TO_TOWER[_a], TO_TOWER[_b], N_, L_)


# ---- symbolic circuit ------------------------------------------------------------
class Circuit:
    """Straight-line program over GF(2) wires; wires are ints (0..7 inputs)."""

    def __init__(self):
        self.ops = []  # (dst, op, a, b)
        self.n = 8

    def new(self, op, a, b=None):
        w = self.n
        self.n += 1
        self.ops.append((w, op, a, b))
        return w

    def xor(self, a, b):
        if a is None:
            return b
        if b is None:
            return a
        return self.new("^", a, b)

    def and_(self, a, b):
        return self.new("&", a, b)

    def linear(self, rows):
        """rows: list of lists of wires to XOR together (None = constant 0);
        greedy pair elimination across all rows."""
        rows = [list(r) for r in rows]
        while True:
            count = {}
            for r in rows:
                for p in itertools.combinations(sorted(set(r)), 2):
                    count[p] = count.get(p, 0) + 1
            best = max(count.items(), key=lambda kv: kv[1], default=None)
            if not best or best[1] < 2:
                break
            (a, b), _ = best
            w = self.xor(a, b)
            for r in rows:
                if a in r and b in r:
                    r.remove(a)
                    r.remove(b)
                    r.append(w)
        out = []
        for r in rows:
            acc = None
            for v in r:
                acc = self.xor(acc, v)
            out.append(acc)
        return out


def lin_matrix(f, nin, nout):
    """Columns of a GF(2)-linear map f on nin-bit ints -> rows of input bit indices."""
    rows = [[] for _ in range(nout)]
    for i in range(nin):
        y = f(1 << i)
        for j in range(nout):
            if (y >> j) & 1:
                rows[j].append(i)
    return rows


def build():
    C = Circuit()
    x = list(range(8))  # input bits, LSB first
    # into the tower basis
    t = C.linear([[x[i] for i in r] for r in lin_matrix(lambda v: TO_TOWER[v], 8, 8)])

    def lin(fn, ws, nin):  # linear map on a group of wires
        return C.linear([[ws[i] for i in r] for r in lin_matrix(fn, nin, nin)])

    def g4mul(a, b):  # a, b: [lo, hi]; Karatsuba: 3 AND
        a0, a1 = a
        b0, b1 = b
        hh = C.and_(a1, b1)
        ll = C.and_(a0, b0)
        mm = C.and_(C.xor(a0, a1), C.xor(b0, b1))
        return [C.xor(hh, ll), C.xor(mm, ll)]  # lo = a1b1 + a0b0, hi = (a0+a1)(b0+b1) + a0b0

    def g16mul(a, b):  # a, b: 4 wires [q0, q1, p0, p1] (lo GF(4) first)
        q1, p1 = a[:2], a[2:]
        q2, p2 = b[:2], b[2:]
        pp = g4mul(p1, p2)
        qq = g4mul(q1, q2)
        mm = g4mul([C.xor(p1[0], q1[0]), C.xor(p1[1], q1[1])], [C.xor(p2[0], q2[0]), C.xor(p2[1], q2[1])])
        ppn = lin(lambda v: g4_mul(v, N_), pp, 2)
        hi = [C.xor(mm[i], qq[i]) for i in range(2)]  # p1q2 + q1p2 + p1p2 = mm + qq
        lo = [C.xor(ppn[i], qq[i]) for i in range(2)]
        return lo + hi

    def g16inv(u):  # u = p z + q: (p z + (p + q)) * (p^2 N + p q + q^2)^-1
        q, p = u[:2], u[2:]
        e1 = lin(lambda v: g4_mul(g4_mul(v, v), N_), p, 2)
        e2 = g4mul(p, q)
        e3 = lin(lambda v: g4_mul(v, v), q, 2)
        e = [C.xor(C.xor(e1[i], e2[i]), e3[i]) for i in range(2)]
        einv = lin(lambda v: g4_mul(v, v), e, 2)  # GF(4): v^-1 = v^2
        hi = g4mul(p, einv)
        lo = g4mul([C.xor(p[0], q[0]), C.xor(p[1], q[1])], einv)
        return lo + hi

    b, a = t[:4], t[4:]  # x = a y + b
    d1 = lin(lambda v: g16_mul(g16_mul(v, v, N_), L_, N_), a, 4)  # a^2 L
    d2 = g16mul(a, b)
    d3 = lin(lambda v: g16_mul(v, v, N_), b, 4)
    d = [C.xor(C.xor(d1[i], d2[i]), d3[i]) for i in range(4)]
    dinv = g16inv(d)
    hi = g16mul(a, dinv)
    lo = g16mul([C.xor(a[i], b[i]) for i in range(4)], dinv)
    inv = lo + hi  # tower bits of x^-1
    # back from the tower basis, affine matrix (constant applied as NOTs)
    A_of_from = lambda v: affine(FROM_TOWER[v]) ^ 0x63
    out = C.linear([[inv[i] for i in r] for r in lin_matrix(A_of_from, 8, 8)])
    return C, out


def evaluate(C, out, x):
    v = [(x >> i) & 1 for i in range(8)] + [0] * (C.n - 8)
    for dst, op, a, b in C.ops:
        v[dst] = v[a] ^ v[b] if op == "^" else v[a] & v[b]
    y = 0
    for i, w in enumerate(out):
        y |= (v[w] & 1) << i
    return y ^ 0x63


def emit(C, out, path):
    nx = sum(op == "^" for _, op, _, _ in C.ops)
    na = sum(op == "&" for _, op, _, _ in C.ops)
    lines = [
        "// bitslice_sbox.cuh -- GENERATED by gen_bitslice_sbox.py; do not edit.",
        "// The AES S-box as a straight-line GF(2) circuit (tower-field inversion",
        f"// GF(((2^2)^2)^2), N = {N_}, L = {L_}): {na} AND + {nx} XOR gates, NOTs for",
        "// the affine constant 0x63.  Bitsliced: x[i] holds bit i (coefficient of",
        "// X^i) of the byte in each of 32 independent lanes of the word.",
        "#pragma once",
        "#include <stdint.h>",
        "",
        "namespace cuot {",
        "__host__ __device__ __forceinline__ void sbox_bitsliced(uint32_t (&x)[8]) {",
    ]
    for i in range(8):
        lines.append(f"  const uint32_t w{i} = x[{i}];")
    for dst, op, a, b in C.ops:
        lines.append(f"  const uint32_t w{dst} = w{a} {op} w{b};")
    for i, w in enumerate(out):
        lines.append(f"  x[{i}] = {'~' if (0x63 >> i) & 1 else ''}w{w};")
    lines += ["}", "}  // namespace cuot", ""]
    with open(path, "w") as f:
        f.write("\n".join(lines))
    return na, nx


def main():
    C, out = build()
    for x in range(256):
        assert evaluate(C, out, x) == SBOX[x], x
    here = os.path.dirname(os.path.abspath(__file__))
    na, nx = emit(C, out, os.path.join(here, "bitslice_sbox.cuh"))
    print(f"bitslice_sbox.cuh: {na} AND + {nx} XOR, verified on all 256 inputs (N={N_}, L={L_})")


if __name__ == "__main__":
    main()
