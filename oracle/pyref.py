"""Independent Python-int restatement of the decimal semantics.

TEST INFRASTRUCTURE ONLY.  A second, independently written arbiter for the
C oracle (up_oracle.c): CPython's arbitrary-precision int stands in for the
"independent host arbitrary-precision library".  Values are (sign, mag,
frac) triples; the rules follow src/datatypes/AriesDecimal.hxx with an
unbounded limb count (file:line cited per function).
"""
from __future__ import annotations

M64 = (1 << 64) - 1
M32 = (1 << 32) - 1


def decode(raw: bytes, frac: int):
    """AriesDecimal(const CompactDecimal*, p, s), AriesDecimal.hxx:105-114."""
    b = bytearray(raw)
    sign = b[-1] >> 7
    b[-1] &= 0x7F
    return (sign, int.from_bytes(b, "little"), frac)


def encode(v, nbytes: int):
    """ToCompactDecimal + SET_SIGN_BIT, AriesDecimal.hxx:308-313, decimal.hxx:91."""
    sign, mag, _ = v
    raw = bytearray((mag & ((1 << (8 * nbytes)) - 1)).to_bytes(nbytes, "little"))
    raw[-1] |= sign << 7
    overflow = mag.bit_length() > 8 * nbytes - 1
    return bytes(raw), overflow


def _align(a, b):
    (sa, ma, fa), (sb, mb, fb) = a, b
    if fa < fb:
        ma *= 10 ** (fb - fa)
        fa = fb
    elif fb < fa:
        mb *= 10 ** (fa - fb)
        fb = fa
    return (sa, ma, fa), (sb, mb, fb)


def add(a, b):
    """operator+=, AriesDecimal.hxx:171-223."""
    (sa, ma, f), (sb, mb, _) = _align(a, b)
    if sa == sb:
        return (sa, ma + mb, f)
    if ma >= mb:
        r = ma - mb
    else:
        r = mb - ma
    sign = 1 if ((ma > mb and not sb) or (ma < mb and sb)) else 0
    return (sign, r, f)


def sub(a, b):
    """operator-=, AriesDecimal.hxx:234-289."""
    (sa, ma, f), (sb, mb, _) = _align(a, b)
    if sa != sb:
        return (sa, ma + mb, f)
    r = abs(ma - mb)
    sign = 1 if ((ma > mb and sb) or (ma < mb and not sb)) else 0
    return (sign, r, f)


def mul(a, b):
    """operator*=, AriesDecimal.hxx:316-404."""
    return (a[0] ^ b[0], a[1] * b[1], a[2] + b[2])


def _shift_bits(shift: int) -> int:
    return (shift // 3) * 10 + {0: 0, 1: 4, 2: 7}[shift % 3]


def div(a, b):
    """DivOrMod(d, false), AriesDecimal.hxx:748-878; returns (value, div0)."""
    (sa, ma, fa), (sb, mb, fb) = a, b
    sign = sa ^ sb
    frac = fa + 4
    if ma == 0:
        return (0, 0, frac), False
    if mb == 0:
        return (sign, ma, frac), True
    shift = fb + 4
    if ma.bit_length() + _shift_bits(shift) - 1 <= 64 and mb.bit_length() <= 64:
        dvs = (ma * 10 ** shift) & M64          # DivByInt64, :581-596
        q = dvs // mb
        rem = dvs % mb
        q += 1 if ((rem << 1) & M64) >= mb else 0
        return (sign, q, frac), False
    x = ma * 10 ** shift
    q, rem = divmod(x, mb)
    if mb.bit_length() <= 32:                   # DivByInt, :598-626
        up = ((rem * 2) & M32) >= mb
    else:                                       # long division, :791-873
        up = 2 * rem >= mb
    return (sign, q + (1 if up else 0), frac), False


def mod(a, b):
    """ModCalc, AriesDecimal.hxx:953-1012 (raw magnitudes, scale 0)."""
    (sa, ma, _), (sb, mb, _) = a, b
    if ma == 0:
        return (0, 0, 0), False
    if mb == 0:
        return (sa ^ sb, 0, 0), True
    return (sa ^ sb, ma % mb, 0), False


def rescale(a, scale: int):
    s, m, f = a
    if scale >= f:
        return (s, m * 10 ** (scale - f), scale)
    return (s, m // 10 ** (f - scale), scale)


def compare(op: int, a, b) -> int:
    """AriesDecimal.hxx:458-570, 1023-1061; op = UP_NODE_LT..NE - 10."""
    if a[0] != b[0]:
        lt, gt, eq = a[0] == 1, a[0] == 0, False
    else:
        (s, ma, _), (_, mb, _) = _align(a, b)
        eq = ma == mb
        lt = (ma < mb) if s == 0 else (ma > mb)
        gt = (ma > mb) if s == 0 else (ma < mb)
    return int([lt, not gt, gt, not lt, eq, not eq][op])


def neg(a):
    return (a[0] ^ 1, a[1], a[2])


def eval_nodes(nodes, root: int, col_types, row_values):
    """Evaluate a node array (abi.UpExprNode) for one row.  row_values[c]
    is the compact bytes of column c.  Returns (value or 0/1, div0 flag)."""
    memo = {}
    flags = {"div0": False}

    def ev(k):
        if k in memo:
            return memo[k]
        nd = nodes[k]
        kind = nd.kind
        if kind == 0:
            v = decode(row_values[nd.column], col_types[nd.column].scale)
        elif kind == 1:
            mag = 0
            for i in range(nd.const_nlimbs):
                mag |= nd.const_limbs[i] << (32 * i)
            v = (1 if nd.const_sign else 0, mag, nd.scale)
        elif kind == 2:
            v = (1 if nd.int_value < 0 else 0, abs(nd.int_value), 0)
        elif kind in (3, 4, 5, 6, 7):
            a, b = ev(nd.left), ev(nd.right)
            if kind == 3:
                v = add(a, b)
            elif kind == 4:
                v = sub(a, b)
            elif kind == 5:
                v = mul(a, b)
            elif kind == 6:
                v, z = div(a, b)
                flags["div0"] |= z
            else:
                v, z = mod(a, b)
                flags["div0"] |= z
        elif kind == 20:
            v = rescale(ev(nd.left), nd.scale)
        elif 10 <= kind <= 15:
            v = compare(kind - 10, ev(nd.left), ev(nd.right))
            memo[k] = v
            return v
        elif kind in (16, 17):
            # AND / OR of boolean children (AEExprAndOrNode, AriesExprCalcNode.cpp:667-760)
            lv, rv = ev(nd.left), ev(nd.right)
            v = int(bool(lv) and bool(rv)) if kind == 16 else int(bool(lv) or bool(rv))
            memo[k] = v
            return v
        else:
            raise ValueError(kind)
        if nd.reverse:
            v = neg(v)
        memo[k] = v
        return v

    return ev(root), flags["div0"]


# ------------------------------------------------------------ decimal text
UP_ROWERR_OVERFLOW, UP_ROWERR_DOMAIN = 1, 4
TEXT_MAX_DIGITS = 1500


def parse_decimal(text: bytes, nbytes: int, scale: int):
    """Text -> compact bytes of a column of scale `scale` (nbytes per value)
    and its row-error bits.  StringToDecimal (decimal.cu:2980-3025): optional
    '-', the magnitude is every digit, the scale is the digit count after '.';
    then Decimal::cast (decimal.cu:471-533): pad with zeros or cut digits off
    (truncation); ToCompactDecimal (decimal.cu:337-341): low bytes, sign bit.
    Text the reference would misread (another character, a second '.') is a
    domain error here and stores zeros."""
    sign, i = 0, 0
    if text[:1] == b"-":
        sign, i = 1, 1
    mag, frac, dot, digits = 0, 0, False, 0
    for c in text[i:]:
        if c == ord(".") and not dot:
            dot = True
            continue
        if not (ord("0") <= c <= ord("9")) or digits >= TEXT_MAX_DIGITS:
            return bytes(nbytes), UP_ROWERR_DOMAIN
        mag = mag * 10 + (c - ord("0"))
        digits += 1
        frac += 1 if dot else 0
    if scale >= frac:
        mag *= 10 ** (scale - frac)
    else:
        mag //= 10 ** (frac - scale)
    err = UP_ROWERR_OVERFLOW if mag >> (8 * nbytes - 1) else 0
    low = mag & ((1 << (8 * nbytes)) - 1)
    b = bytearray(low.to_bytes(nbytes, "little"))
    b[-1] |= sign << 7
    return bytes(b), err


def format_decimal(raw: bytes, scale: int, hex_image: bool = False) -> str:
    """Compact bytes -> text.  hex_image: Decimal::GetDecimal
    (decimal.cu:362-398), sign, 8 upper-case hex digits per 32-bit limb from
    the highest nonzero one, "(fff)"; else the decimal string with a '.'
    before the last `scale` digits and '-' when the sign bit is set."""
    sign, mag, _ = decode(raw, scale)
    if hex_image:
        limbs = []
        while mag:
            limbs.append(mag & M32)
            mag >>= 32
        body = "".join("%08X" % w for w in reversed(limbs))
        return ("-" if sign else "+") + body + "(%03d)" % scale
    digits = str(mag).rjust(scale + 1, "0")
    body = digits[:-scale] + "." + digits[-scale:] if scale > 0 else digits
    return ("-" if sign else "") + body
