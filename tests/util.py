"""Shared helpers for the tests (seeded inputs, conversions)."""
import numpy as np


def hx(s: str) -> np.ndarray:
    return np.frombuffer(bytes.fromhex(s), np.uint8).copy()


def blocks(s: str) -> np.ndarray:
    return hx(s).reshape(-1, 16)


def rng_blocks(rng, n: int) -> np.ndarray:
    return rng.integers(0, 256, (n, 16), dtype=np.uint8)


def delta_ferret(rng) -> np.ndarray:
    d = rng_blocks(rng, 1)[0]
    d[0] |= 1  # ferret_cot.hpp:29-31: LSB of delta is 1
    return d


def to_dev(a: np.ndarray):
    import torch
    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def to_host(t) -> np.ndarray:
    return t.cpu().numpy()
