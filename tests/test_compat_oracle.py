"""The oracle's restatement of cuOT's own GPU semantics (or_compat_*), used
only to pin how the reference's GPU kernels differ from emp-ot (the GPU side
is tests/test_gpu_ref_kernels.py), checked here against a second, pure-Python
restatement: the key schedule with the round constants one entry early
(gpu/aes_expand.cu:52-65, gpu/utilsBox.h:61), the GGM expansion without the
parent XOR under the keys 3242342 / 8993849 (gpu/aes_op.cu:176-266,
dev_layer.cu:20-59) and the LPN with the swapped index plaintext and % k
(gpu/gpu_ops.cu:102-109, dev_layer.cu:146-186)."""
import numpy as np

import oracle


def _gmul(a, b):
    r = 0
    while b:
        if b & 1:
            r ^= a
        a = ((a << 1) ^ (0x1B if a & 0x80 else 0)) & 0xFF
        b >>= 1
    return r


def _sbox():
    inv = [0] * 256
    for x in range(1, 256):
        for y in range(1, 256):
            if _gmul(x, y) == 1:
                inv[x] = y
                break
    s = []
    for x in range(256):
        b = inv[x]
        v = b
        for k in range(1, 5):
            v ^= ((b << k) | (b >> (8 - k))) & 0xFF
        s.append(v ^ 0x63)
    return s


SBOX = _sbox()


def key_expand(key: bytes, rcons) -> bytes:
    w = [list(key[4 * i:4 * i + 4]) for i in range(4)]
    for i in range(4, 44):
        t = list(w[i - 1])
        if i % 4 == 0:
            t = [SBOX[t[1]] ^ rcons[i // 4 - 1], SBOX[t[2]], SBOX[t[3]], SBOX[t[0]]]
        w.append([a ^ b for a, b in zip(w[i - 4], t)])
    return bytes(b for word in w for b in word)


FIPS_RCON = [0x01, 0x02, 0x04, 0x08, 0x10, 0x20, 0x40, 0x80, 0x1B, 0x36]
GPU_RCON = [0x8D, 0x01, 0x02, 0x04, 0x08, 0x10, 0x20, 0x40, 0x80, 0x1B]


def test_compat_key_schedule_is_fips_with_shifted_round_constants():
    for key in (bytes(16), bytes(range(16)), bytes([0x66, 0x79, 0x31] + [0] * 13)):
        fips = key_expand(key, FIPS_RCON)
        assert fips == oracle.aes_key_expand(key).tobytes()
        compat = key_expand(key, GPU_RCON)
        assert compat == oracle.compat_key_expand(key).tobytes()
        assert compat[:16] == fips[:16] and compat[16:] != fips[16:]


def _word_key(w: int) -> bytes:
    return w.to_bytes(4, "little") + bytes(12)


def test_compat_ferret_sender_small():
    rng = np.random.default_rng(5)
    t, h = 3, 4
    roots = rng.integers(0, 256, (t, 16), dtype=np.uint8)
    delta = rng.integers(0, 256, 16, dtype=np.uint8)
    rk0 = np.frombuffer(key_expand(_word_key(3242342), GPU_RCON), np.uint8)
    rk1 = np.frombuffer(key_expand(_word_key(8993849), GPU_RCON), np.uint8)
    exp_leaves, exp_ss = [], []
    for r in roots:
        level = r.reshape(1, 16)
        for _ in range(h):
            left, right = oracle.aes_ecb_rk(rk0, level), oracle.aes_ecb_rk(rk1, level)
            level = np.stack([left, right], axis=1).reshape(-1, 16)  # children 2j, 2j + 1
        exp_leaves.append(level)
        exp_ss.append(np.bitwise_xor.reduce(level, axis=0) ^ delta)
    leaves, ss = oracle.compat_ferret_sender(roots, h, delta)
    assert np.array_equal(leaves, np.concatenate(exp_leaves))
    assert np.array_equal(ss, np.stack(exp_ss))


def test_compat_lpn_small():
    rng = np.random.default_rng(6)
    n, k, d = 22, 7, 10
    key = rng.integers(0, 256, 16, dtype=np.uint8)
    kk = rng.integers(0, 256, (k, 16), dtype=np.uint8)
    e = rng.integers(0, 256, (n, 16), dtype=np.uint8)
    rk = np.frombuffer(key_expand(key.tobytes(), GPU_RCON), np.uint8)
    nb = (n * d + 3) // 4
    pt = np.zeros((nb, 16), np.uint8)
    for b in range(nb):
        pt[b, :8] = np.frombuffer((4 * (b // 10)).to_bytes(8, "little"), np.uint8)
        pt[b, 8:] = np.frombuffer((b % 10).to_bytes(8, "little"), np.uint8)
    words = oracle.aes_ecb_rk(rk, pt).reshape(-1).view("<u4")
    exp = e.copy()
    for i in range(n):
        for j in range(d):
            exp[i] ^= kk[int(words[i * d + j]) % k]
    assert np.array_equal(oracle.compat_lpn(key, kk, e, d=d), exp)
