"""Host-side codec of the compact decimal layout.

Compact value of precision p: B(p) bytes holding the little-endian binary
magnitude of the unscaled integer, with the sign in bit 7 of the last byte
(the reference's CompactDecimal + SET_SIGN_BIT / GET_SIGN_FROM_BIT,
src/datatypes/decimal.hxx:91-92,126-128).  Scale and precision are column
metadata and are not stored.
"""
from __future__ import annotations

from typing import Iterable, Sequence

import numpy as np

from . import abi


def compact_bytes(p: int) -> int:
    b = abi.load().up_compact_bytes(p)
    if b < 1:
        raise ValueError(f"precision {p} out of range")
    return b


def encode(values: Iterable[tuple[int, int]], p: int) -> bytes:
    """values: (sign, magnitude) pairs.  Magnitudes must fit 8*B-1 bits."""
    b = compact_bytes(p)
    out = bytearray()
    for sign, mag in values:
        if mag < 0 or mag.bit_length() > 8 * b - 1:
            raise ValueError(f"magnitude does not fit {b} compact bytes")
        raw = bytearray(mag.to_bytes(b, "little"))
        raw[-1] |= (1 if sign else 0) << 7
        out += raw
    return bytes(out)


def encode_ints(values: Iterable[int], p: int) -> bytes:
    return encode(((1 if v < 0 else 0, abs(v)) for v in values), p)


def decode(buf: bytes | bytearray | memoryview | np.ndarray, nbytes: int) -> list[tuple[int, int]]:
    """Decode a run of nbytes-wide compact values into (sign, magnitude)."""
    data = bytes(buf) if not isinstance(buf, (bytes, bytearray)) else buf
    out = []
    for i in range(0, len(data), nbytes):
        raw = bytearray(data[i:i + nbytes])
        sign = raw[-1] >> 7
        raw[-1] &= 0x7F
        out.append((sign, int.from_bytes(raw, "little")))
    return out


def to_str(sign: int, mag: int, scale: int) -> str:
    s = str(mag).rjust(scale + 1, "0")
    txt = s if scale == 0 else s[:-scale] + "." + s[-scale:]
    return ("-" if sign else "") + txt


def parse(text: str, scale: int) -> tuple[int, int]:
    t = text.strip()
    sign = 1 if t.startswith("-") else 0
    t = t.lstrip("+-")
    ip, _, fp = t.partition(".")
    if len(fp) > scale:
        raise ValueError("more fraction digits than the scale")
    return sign, int((ip or "0") + fp.ljust(scale, "0"))


AGG_BYTES = abi.UP_AGG_DECIMAL_BYTES


def decode_agg(buf: bytes, n: int) -> list[dict]:
    """Decode n 133-byte SUM/AVG images (flag, sign, prec, frac, error, v[32])."""
    out = []
    for g in range(n):
        img = buf[g * AGG_BYTES:(g + 1) * AGG_BYTES]
        out.append({"flag": img[0], "sign": img[1], "prec": img[2], "frac": img[3], "error": img[4],
                    "mag": int.from_bytes(img[5:133], "little")})
    return out


def np_compact_from_int64(values: np.ndarray, p: int) -> np.ndarray:
    """Vectorised encode of int64 unscaled values (|v| < 2^63) to an
    (n, B) uint8 array."""
    b = compact_bytes(p)
    v = np.asarray(values, dtype=np.int64)
    mag = np.abs(v).astype(np.uint64)
    raw = mag.view(np.uint8).reshape(-1, 8)
    out = np.zeros((len(v), b), dtype=np.uint8)
    k = min(8, b)
    out[:, :k] = raw[:, :k]
    if b < 8 and np.any(raw[:, b:]):
        raise ValueError("values do not fit the compact width")
    out[:, b - 1] |= (v < 0).astype(np.uint8) << 7
    return out


def pack_rows(rows: Sequence[bytes]) -> bytes:
    return b"".join(rows)
