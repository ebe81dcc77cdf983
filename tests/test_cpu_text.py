"""Decimal text in and out: the Python restatement of the reference's parse
(StringToDecimal + cast + ToCompactDecimal) and output image (GetDecimal),
on hand-checked cases, and the round trip of the decimal string."""
import random

from oracle import pyref
from ultraprecise_b200 import codec


def _val(raw, scale):
    sign, mag, _ = pyref.decode(raw, scale)
    return sign, mag


def test_parse_cases():
    B = codec.compact_bytes(15)
    assert _val(pyref.parse_decimal(b"123.45", B, 2)[0], 2) == (0, 12345)
    assert _val(pyref.parse_decimal(b"-123.4", B, 2)[0], 2) == (1, 12340)       # padded
    assert _val(pyref.parse_decimal(b"123.456789", B, 2)[0], 2) == (0, 12345)   # cut, not rounded
    assert _val(pyref.parse_decimal(b"-0.00", B, 2)[0], 2) == (1, 0)            # sign kept
    assert _val(pyref.parse_decimal(b"", B, 2)[0], 2) == (0, 0)
    assert _val(pyref.parse_decimal(b"7", B, 0)[0], 0) == (0, 7)
    assert _val(pyref.parse_decimal(b"12.", B, 1)[0], 1) == (0, 120)
    assert pyref.parse_decimal(b"1.2.3", B, 2)[1] == pyref.UP_ROWERR_DOMAIN
    assert pyref.parse_decimal(b"+5", B, 2)[1] == pyref.UP_ROWERR_DOMAIN
    big = b"9" * 20
    raw, err = pyref.parse_decimal(big, B, 0)                                  # 20 digits in 7 bytes
    assert err == pyref.UP_ROWERR_OVERFLOW


def test_format_cases():
    B = codec.compact_bytes(15)
    raw = codec.encode([(1, 12345)], 15)
    assert pyref.format_decimal(raw, 2) == "-123.45"
    assert pyref.format_decimal(codec.encode([(0, 5)], 15), 3) == "0.005"
    assert pyref.format_decimal(codec.encode([(0, 0)], 15), 0) == "0"
    assert pyref.format_decimal(codec.encode([(0, 0x1_0000_0002)], 15), 4, True) == "+0000000100000002(004)"
    assert pyref.format_decimal(codec.encode([(1, 0)], 15), 2, True) == "-(002)"


def test_round_trip():
    rng = random.Random(3)
    for p in (1, 9, 15, 38, 76, 300, 1000):
        B = codec.compact_bytes(p)
        for _ in range(200):
            s = rng.randint(0, p)
            v = (rng.randint(0, 1), rng.randint(0, 10 ** rng.randint(0, p) - 1))
            raw = codec.encode([v], p)
            text = pyref.format_decimal(raw, s).encode()
            back, err = pyref.parse_decimal(text, B, s)
            assert err == 0 and back == raw, (p, s, v, text)
