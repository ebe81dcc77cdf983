"""Shared test helpers: seeded data, oracle comparison."""
from __future__ import annotations

import random

from ultraprecise_b200 import abi, codec
from ultraprecise_b200 import expr as E


def rand_digits_value(rng: random.Random, p: int, signed=True, nonzero=False):
    while True:
        mag = int("".join(rng.choice("0123456789") for _ in range(p)))
        if mag or not nonzero:
            break
    sign = rng.randint(0, 1) if signed else 0
    return (sign, mag)


def column_bytes(values, p: int) -> bytes:
    return codec.encode(values, p)


def edge_values(p: int, rng: random.Random, n: int):
    """Zeros of both signs, ones, the largest p-digit value, powers of two
    around limb boundaries, and random values."""
    top = 10 ** p - 1
    base = [(0, 0), (1, 0), (0, 1), (1, 1), (0, top), (1, top), (0, top // 2), (1, 10 ** (p - 1))]
    for k in (31, 32, 33, 63, 64, 65, 95, 96, 127, 128):
        v = (1 << k) - 1
        if v <= top:
            base += [(0, v), (1, v + 1 if v + 1 <= top else v)]
    out = list(base)
    while len(out) < n:
        out.append(rand_digits_value(rng, rng.randint(1, p), signed=True))
    rng.shuffle(out)
    return out[:n] if n >= len(base) else out
