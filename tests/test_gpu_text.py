"""GPU parity of decimal text in and out (up_parse_decimal, up_format_decimal)
against the Python restatement of the reference's parse and output image,
and the round trip of the decimal string at full size."""
import random

import pytest

torch = pytest.importorskip("torch")

from oracle import pyref
from ultraprecise_b200 import codec, runtime

pytestmark = pytest.mark.gpu

EDGE = [b"", b"-", b"0", b"-0.00", b"12.", b".5", b"1.2.3", b"+5", b"abc", b"1e5", b" 1", b"9" * 40,
        b"-" + b"9" * 1500, b"1" * 1501, b"00000123.4500000"]


def _fields(p, s, n, rng):
    out = list(EDGE)
    while len(out) < n:
        ip = str(rng.randint(0, 10 ** rng.randint(0, max(0, p - s)) - 1)) if rng.random() < 0.9 else ""
        fd = rng.randint(0, s + 3)
        fp = "".join(rng.choice("0123456789") for _ in range(fd))
        txt = ("-" if rng.random() < 0.5 else "") + ip + ("." + fp if fd or rng.random() < 0.2 else "")
        out.append(txt.encode())
    rng.shuffle(out)
    return out


@pytest.mark.parametrize("p,s", [(15, 2), (38, 9), (150, 37), (1000, 998)])
def test_parse_matches_restatement(p, s):
    rng = random.Random(p)
    fields = _fields(p, s, 3000, rng)
    got, err = runtime.parse_decimal(fields, p, s)
    B = codec.compact_bytes(p)
    exp, exp_err = bytearray(), 0
    for f in fields:
        raw, e = pyref.parse_decimal(f, B, s)
        exp += raw
        exp_err |= e
    assert bytes(got.cpu().numpy().tobytes()) == bytes(exp)
    assert err == exp_err


@pytest.mark.parametrize("p,s", [(15, 2), (38, 0), (150, 37), (1000, 998)])
@pytest.mark.parametrize("hex_image", [False, True])
def test_format_matches_restatement(p, s, hex_image):
    rows = 2000
    col = runtime.gen_digits(rows, p, 40 + p)
    got = runtime.format_strings(col, rows, p, s, hex_image)
    B = codec.compact_bytes(p)
    raw = bytes(col.cpu().numpy().tobytes())
    for r in (0, 1, rows // 2, rows - 1):
        assert got[r] == pyref.format_decimal(raw[r * B:(r + 1) * B], s, hex_image)
    assert got == [pyref.format_decimal(raw[r * B:(r + 1) * B], s, hex_image) for r in range(rows)]


@pytest.mark.parametrize("p,s,rows", [(38, 9, 4 << 20), (300, 75, 100_000)])
def test_round_trip_on_device(p, s, rows):
    """format -> compact the slots on the GPU -> parse gives back every byte."""
    col = runtime.gen_digits(rows, p, 77)
    text, lens = runtime.format_decimal(col, rows, p, s)
    assert int(lens.min()) > 0
    width = text.shape[1]
    mask = torch.arange(width, device="cuda")[None, :] < lens[:, None].to(torch.int64)
    flat = text[mask].contiguous()
    offsets = torch.zeros(rows + 1, dtype=torch.int64, device="cuda")
    offsets[1:] = torch.cumsum(lens.to(torch.int64), 0)
    back, err = runtime.parse_decimal(None, p, s, text=flat, offsets=offsets)
    assert err == 0
    assert torch.equal(back, col)
