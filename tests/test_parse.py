"""MULTICUT text parsed on the device (rama_parse_multicut): the reference's
read_file semantics (src/multicut_text_parser.cpp:6-31) and costs rounded to
nearest like strtof, hard cases included."""
import ctypes as C
import random
from fractions import Fraction

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

_libc = C.CDLL(None)
_libc.strtof.restype = C.c_float
_libc.strtof.argtypes = [C.c_char_p, C.c_void_p]


def strtof(s: str) -> np.float32:
    return np.float32(_libc.strtof(s.encode(), None))


def _parse(solver, text: bytes):
    i, j, c = solver.parse_multicut(text)
    return i.cpu().numpy(), j.cpu().numpy(), c.cpu().numpy()


def _dec(fr: Fraction) -> str:
    """Exact decimal expansion of a dyadic rational."""
    sign = "-" if fr < 0 else ""
    fr = abs(fr)
    ip = fr.numerator // fr.denominator
    rem = fr - ip
    digits = []
    while rem:
        rem *= 10
        d = rem.numerator // rem.denominator
        digits.append(str(d))
        rem -= d
    return sign + str(ip) + ("." + "".join(digits) if digits else "")


def hard_costs(seed=7):
    rng = random.Random(seed)
    out = ["0", "-0", "+1.5", ".5", "5.", "1e0", "1E+2", "-2.5e-3", "123456789012345678901234567890",
           "0.000000000000000000000000000000000000000000001", "1e-45", "7e-46", "1e-46", "1.4e-45",
           "1.17549435e-38", "1.1754942e-38", "3.40282347e38", "3.4028235e38", "3.402823567e38",
           "0.1", "0.2", "0.3", "16777217", "16777219", "33554435", "9007199254740993",
           "1.00000005960464477539062500", "1.000000059604644775390625000000001", "1.0000000596046447753906249999"]
    for _ in range(300):
        e = rng.randint(-140, 120)
        m = rng.randint(1 << 23, (1 << 24) - 1)
        f = Fraction(m) * Fraction(2) ** e
        if f > Fraction(3.4e38):
            continue
        mid = f + Fraction(2) ** e / 2  # midpoint between m and m + 1 (times 2^e)
        s = _dec(mid)
        out.append(s)
        out.append(s + ("" if "." in s else ".") + "0000000001")  # just above the midpoint
        # just below: subtract a tiny amount
        out.append(_dec(mid - Fraction(1, 10 ** 60)) if mid > Fraction(1, 10 ** 30) else s)
        out.append(("%.9e" % float(f)))
        out.append(("%.17g" % float(f)))
    return out


def test_costs_round_like_strtof(solver):
    costs = hard_costs()
    lines = ["MULTICUT"] + [f"{k} {k + 1} {c}" for k, c in enumerate(costs)]
    i, j, c = _parse(solver, ("\n".join(lines) + "\n").encode())
    assert len(c) == len(costs)
    assert np.array_equal(i, np.arange(len(costs))) and np.array_equal(j, np.arange(len(costs)) + 1)
    want = np.array([strtof(x) for x in costs], np.float32)
    bad = [(costs[k], c[k], want[k]) for k in range(len(costs)) if c[k].view(np.uint32) != want[k].view(np.uint32)]
    assert not bad, bad[:5]


def test_random_file_matches_host_parse(solver):
    rng = np.random.default_rng(3)
    n = 200_000
    i = rng.integers(0, 10 ** 6, n)
    j = rng.integers(0, 10 ** 6, n)
    vals = rng.normal(size=n) * 10.0 ** rng.integers(-8, 8, n)
    fmts = ["%.3f", "%.9g", "%.6e", "%r", "%.12f"]
    toks = [fmts[k % len(fmts)] % v if fmts[k % len(fmts)] != "%r" else repr(float(v)) for k, v in enumerate(vals)]
    seps = [" ", "\t", "  ", " \r\n"]
    body = "".join(f"{a}{seps[k % 4]}{b} {t}\n" for k, (a, b, t) in enumerate(zip(i, j, toks)))
    gi, gj, gc = _parse(solver, ("MULTICUT\r\n" + body).encode())
    assert np.array_equal(gi, i) and np.array_equal(gj, j)
    want = np.array([strtof(t) for t in toks], np.float32)
    assert np.array_equal(gc.view(np.uint32), want.view(np.uint32))


@pytest.mark.parametrize("third", ["2 3 abc", "2 3 1.2.3", "2 3 1e", "2 3 4e38", "99999999999 3 1.0", "2 3 nan",
                                   "2 - 1.0", "2 3.5 1.0"])
def test_input_ends_at_first_bad_token(solver, third):
    """The third triple holds a token that does not read as its kind: the
    input ends before it, as the reference's stream extraction does."""
    text = f"MULTICUT\n0 1 1.0\n1 2 -2\n{third}\n3 4 5\n"
    i, j, c = _parse(solver, text.encode())
    assert i.tolist() == [0, 1] and j.tolist() == [1, 2] and c.tolist() == [1.0, -2.0]


def test_trailing_incomplete_triple_is_dropped(solver):
    i, j, c = _parse(solver, b"MULTICUT\n0 1 1.5\n1 2")
    assert i.tolist() == [0] and j.tolist() == [1] and c.tolist() == [1.5]


def test_first_line_must_be_multicut(solver):
    from rama_b200._lib import RamaError

    with pytest.raises(RamaError, match="first line must be 'MULTICUT'"):
        _parse(solver, b"GRAPH\n0 1 1\n")
    i, j, c = _parse(solver, b"MULTICUT")
    assert len(c) == 0
