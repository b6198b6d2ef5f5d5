"""CPU: the generator text format of Tessellation::read_generators /
import_generators (tessellation.rs:126-171), read by the library's native
parser (vd_parse_generators, host only): lines at '\\n', tokens at Unicode
White_Space, the id ignored, each coordinate read with Rust's
`str::parse::<f64>` grammar and 0.0 when missing or unparsable, UTF-8 only."""
import math
import struct

import numpy as np
import pytest

from common import golden


def parse(text):
    import vorothree_b200 as v
    return v.parse_generators(text)


def first(token):
    return parse("0 " + token)[0, 0]


def bits(x):
    return struct.pack("<d", x)


# tokens Rust's f64 FromStr accepts, with the value it gives
ACCEPTED = [
    ("1", 1.0), ("+1", 1.0), ("-1", -1.0), ("1.", 1.0), (".5", 0.5), ("+.5", 0.5), ("-.5", -0.5),
    ("1.5e3", 1500.0), ("1.5E3", 1500.0), ("1e+3", 1000.0), ("1e-3", 1e-3), ("1.e3", 1000.0),
    ("00012", 12.0), ("0", 0.0), ("-0", -0.0), ("-0.0e5", -0.0),
    ("inf", math.inf), ("-inf", -math.inf), ("+inf", math.inf), ("INF", math.inf),
    ("Infinity", math.inf), ("-infinity", -math.inf),
    ("1e400", math.inf), ("-1e400", -math.inf), ("1e-400", 0.0), ("-1e-400", -0.0),
    ("1e99999999999999999999", math.inf), ("1e-99999999999999999999", 0.0),
    ("0e99999999999999999999", 0.0), ("0.000e-99999999999999999999", 0.0),
    ("1e-320", 1e-320), ("4.9e-324", 5e-324), ("2.4e-324", 0.0), ("2.5e-324", 5e-324),
    ("2.4703282292062327e-324", 0.0), ("2.4703282292062328e-324", 5e-324),   # either side of half the least subnormal
    ("2.2250738585072014e-308", 2.2250738585072014e-308),
    ("1.7976931348623157e308", 1.7976931348623157e308), ("1.7976931348623159e308", math.inf),
    ("0.1000000000000000055511151231257827021181583404541015625", 0.1),
    ("9007199254740993", 9007199254740992.0),   # tie, to even
    ("9007199254740995", 9007199254740996.0),   # tie, to even
    ("3.14159265358979323846264338327950288419716939937510", math.pi),
]

# tokens it rejects (read as 0.0)
REJECTED = [".", "e5", "1e", "1e+", "+", "-", "1.5.2", "1_000", "0x10", "0x1p3", "nan(1)", "infinit",
            "inff", "infinityy", "1,5", "1e5.0", "++1", "--1", "+-1", "in", "i", "n", "na", "1d5", "1f",
            "\u0661", "\uff11", "1e\u0661", "\u200b1"]


@pytest.mark.parametrize("token,value", ACCEPTED)
def test_accepted_tokens(token, value):
    got = first(token)
    assert bits(got) == bits(value), (token, got, value)
    assert bits(got) == bits(float(token))   # Python's float() rounds correctly too


@pytest.mark.parametrize("token", REJECTED)
def test_rejected_tokens(token):
    got = parse("0 " + token + " 2 3")
    assert bits(got[0, 0]) == bits(0.0)
    assert got[0, 1] == 2.0 and got[0, 2] == 3.0


@pytest.mark.parametrize("token,negative", [("nan", False), ("NaN", False), ("+nan", False), ("-nan", True),
                                            ("-NAN", True)])
def test_nan_tokens(token, negative):
    got = first(token)
    assert math.isnan(got) and bool(np.signbit(got)) == negative


def test_lines_and_tokens():
    # blank and whitespace-only lines are skipped; an id alone gives (0, 0, 0);
    # extra tokens are ignored; a line without '\n' at the end still counts
    text = "\n  \n\t\n7\n1 2 3 4 5\r\n\r\n2 9 8\n3 1 2 3"
    got = parse(text)
    assert got.tolist() == [[0, 0, 0], [2, 3, 4], [9, 8, 0], [1, 2, 3]]
    assert parse("").shape == (0, 3)
    assert parse("\n\n\n").shape == (0, 3)


def test_unicode_whitespace():
    # Rust's char::is_whitespace (Unicode White_Space) separates tokens
    seps = ["\t", "\x0b", "\x0c", "\r", " ", "\u0085", "\u00a0", "\u1680", "\u2000", "\u200a", "\u2028",
            "\u2029", "\u202f", "\u205f", "\u3000"]
    for s in seps:
        got = parse(s.join(["id", "1", "2", "3"]) + s)
        assert got.tolist() == [[1, 2, 3]], repr(s)
    # whitespace only: skipped
    assert parse("\u3000\u2028\n\u00a0").shape == (0, 3)
    # not White_Space (although Python's str.split() splits at \x1c-\x1f):
    # the character is part of a token
    assert parse("\x1c 1 2 3").tolist() == [[1, 2, 3]]
    assert parse("id 1\x1f2 3 4").tolist() == [[0, 3, 4]]
    # zero-width space and BOM are not White_Space either
    assert parse("\ufeffid 1 2 3").tolist() == [[1, 2, 3]]
    assert parse("id 1\u200b 2 3").tolist() == [[0, 2, 3]]
    # a 4-byte character as the id
    assert parse("\U0001f600 4 5 6").tolist() == [[4, 5, 6]]


@pytest.mark.parametrize("data", [b"1 2 3\xff\n", b"\xc0\x80 1 2 3", b"1 \xed\xa0\x80 2 3", b"1 2 3 \xe2\x82",
                                  b"\xf4\x90\x80\x80 1 2 3", b"\xe0\x80\x80", b"1 2 3\n\x80"])
def test_invalid_utf8(data):
    # a Rust &str is always UTF-8 and BufRead::lines fails on a file that is not
    import vorothree_b200 as v
    with pytest.raises(v.VoronoidError) as e:
        parse(data)
    assert "UTF-8" in str(e.value)


def test_bytes_and_str_agree():
    text = "0 0.25 0.5 0.75\n1 1e-3 2E2 -3.5\n"
    assert np.array_equal(parse(text), parse(text.encode()))


def test_round_trip_golden_generators():
    # the reference's own generator files, as the golden fixtures hold them,
    # written with shortest round-trip decimals and read back bit for bit
    for name in ("voro_face_counts.json", "voro_vertex_positions.json"):
        rows = golden(name)["generators"]   # [id, x, y, z]
        text = "".join(f"{int(i)} {float(x)!r} {float(y)!r} {float(z)!r}\n" for i, x, y, z in rows)
        assert np.array_equal(parse(text), np.asarray(rows, np.float64)[:, 1:])


def test_random_round_trip():
    rng = np.random.Generator(np.random.PCG64(5))
    g = np.concatenate([rng.uniform(-1e3, 1e3, (300, 3)), rng.normal(0, 1e-200, (100, 3)),
                        rng.normal(0, 1e200, (100, 3))]).tolist()
    for fmt in ("{!r}", "{:.17g}", "{:.17e}", "{:.40f}"):
        text = "\n".join("x " + " ".join(fmt.format(c) for c in p) for p in g)
        got = parse(text)
        want = np.array([[float(fmt.format(c)) for c in p] for p in g])
        assert np.array_equal(got, want), fmt


def test_random_tokens_against_grammar():
    """20,000 random tokens over the characters the grammar uses, each read as
    a model of Rust's f64 FromStr reads it: the token must match the grammar
    (case-insensitive), and then its value is the correctly rounded one
    (Python's float, which accepts every such token, rounds the same way)."""
    import re
    rust = re.compile(r"[+-]?(inf|infinity|nan|(\d+\.?\d*|\.\d+)(e[+-]?\d+)?)", re.I)
    rng = np.random.Generator(np.random.PCG64(77))
    alphabet = list("0123456789012345678901234567890123456789..eE+-+-infatyINFATY_x,")
    toks = []
    for _ in range(20000):
        n = int(rng.integers(1, 14))
        toks.append("".join(alphabet[i] for i in rng.integers(0, len(alphabet), n)))
    text = "".join(f"{k} {toks[3 * k]} {toks[3 * k + 1]} {toks[3 * k + 2]}\n" for k in range(len(toks) // 3))
    got = parse(text).reshape(-1)
    valid = 0
    for tok, g in zip(toks, got):
        want = float(tok) if rust.fullmatch(tok) else 0.0
        valid += rust.fullmatch(tok) is not None
        if math.isnan(want):
            assert math.isnan(g) and bool(np.signbit(g)) == tok.startswith("-"), tok
        else:
            assert bits(g) == bits(want), (tok, g, want)
    assert valid > 2000
