"""Seeded host-side column generator for the CPU oracle runs (test
infrastructure).  Same distribution as the device generator of the
precision sweep: every one of the p digits uniform 0-9, sign +/- with equal
odds, optionally no zero values."""
from __future__ import annotations

import numpy as np


def compact_digits(rows: int, p: int, nbytes: int, seed: int, signed: bool = True, nonzero: bool = False) -> bytes:
    rng = np.random.default_rng(seed)
    L = (nbytes + 3) // 4
    limbs = np.zeros((rows, L), dtype=np.uint64)
    left = p
    first = True
    while left > 0:
        d = left % 9 if first and left % 9 else 9
        first = False
        left -= d
        chunk = rng.integers(0, 10 ** d, size=rows, dtype=np.uint64)
        if nonzero and left == 0:
            chunk = np.where(np.all(limbs == 0, axis=1) & (chunk == 0), np.uint64(1), chunk)
        carry = chunk
        mul = np.uint64(10 ** d)
        for i in range(L):
            t = limbs[:, i] * mul + carry
            limbs[:, i] = t & np.uint64(0xFFFFFFFF)
            carry = t >> np.uint64(32)
    raw = limbs.astype(np.uint32).view(np.uint8).reshape(rows, 4 * L)[:, :nbytes].copy()
    if signed:
        raw[:, nbytes - 1] |= (rng.integers(0, 2, size=rows, dtype=np.uint8) << 7).astype(np.uint8)
    return raw.tobytes()


def pack_unsigned(values, nbytes: int) -> bytes:
    """Non-negative int64 values as nbytes-wide little-endian compact decimals
    (sign bit clear); nbytes <= 8."""
    v = np.asarray(values, dtype=np.uint64)
    out = np.zeros((v.size, nbytes), dtype=np.uint8)
    for i in range(nbytes):
        out[:, i] = ((v >> np.uint64(8 * i)) & np.uint64(0xFF)).astype(np.uint8)
    return out.tobytes()
