"""The GLV constants of the blinding kernel (nkr-zkp_b200/csrc/blind.cu), derived
again from the curve in pure Python: beta and lambda are cube roots of unity
that agree on G1, (a1, b1), (a2, b2) is a basis of the lattice
{(a, b) : a + b lambda = 0 mod r} with determinant r, g1 and g2 are the rounded
2^256-scaled quotients, and the split done the kernel's way (floor products,
128-bit two's complement) gives k = k1 + k2 lambda with |k1|, |k2| < 2^127 on
edge-case and random scalars."""
import os
import random
import re

import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = open(os.path.join(ROOT, "nkr-zkp_b200", "csrc", "blind.cu")).read()
R, P = O.R, O.P


def _words(name):
    m = re.search(r"constexpr uint64_t %s(?:\[\d\])? = \{?([^;}]*)\}?;" % name, SRC)
    assert m, name
    vals = [int(v.strip().rstrip("ull"), 0) for v in m.group(1).split(",")]
    return sum(v << (64 * i) for i, v in enumerate(vals))


def _beta_r260():
    m = re.search(r"Fq52 glv_beta\(\)\s*\{\s*return \{\{([^}]*)\}\};", SRC)
    limbs = [int(v.strip().rstrip("ull"), 0) for v in m.group(1).split(",")]
    return sum(v << (52 * i) for i, v in enumerate(limbs)) * pow(2, -260, P) % P


LAM = _words("kLambda")
A1 = _words("kGlvA1")
A2 = _words("kGlvA2")
B1 = -_words("kGlvB1Abs")
B2 = A1
G1C = _words("kGlvG1")
G2C = _words("kGlvG2")
BETA = _beta_r260()


def _add(p, q):
    if p is None:
        return q
    if q is None:
        return p
    (x1, y1), (x2, y2) = p, q
    if x1 == x2:
        if (y1 + y2) % P == 0:
            return None
        m = 3 * x1 * x1 * pow(2 * y1, -1, P) % P
    else:
        m = (y2 - y1) * pow(x2 - x1, -1, P) % P
    x3 = (m * m - x1 - x2) % P
    return x3, (m * (x1 - x3) - y1) % P


def _mul(k, p):
    acc = None
    for bit in bin(k)[2:]:
        acc = _add(acc, acc)
        if bit == "1":
            acc = _add(acc, p)
    return acc


def test_cube_roots_agree_on_g1():
    assert pow(BETA, 3, P) == 1 and BETA != 1
    assert (LAM * LAM + LAM + 1) % R == 0
    g = (1, 2)
    assert _mul(LAM, g) == (BETA * g[0] % P, g[1])
    q = _mul(0x1234567890abcdef, g)
    assert _mul(LAM, q) == (BETA * q[0] % P, q[1])


def test_lattice_basis_and_quotients():
    assert (A1 + B1 * LAM) % R == 0 and (A2 + B2 * LAM) % R == 0
    assert A1 * B2 - A2 * B1 == R
    assert G1C == (2 * (B2 << 256) + R) // (2 * R)
    assert G2C == (2 * (-B1 << 256) + R) // (2 * R)


def _split(k):
    m = 1 << 128
    c1, c2 = (k * G1C) >> 256, (k * G2C) >> 256
    k1 = (k - c1 * A1 - c2 * A2) % m
    k2 = (c1 * -B1 - c2 * B2) % m
    k1 = k1 - m if k1 >> 127 else k1
    k2 = k2 - m if k2 >> 127 else k2
    return k1, k2


def test_split_identity_and_bounds():
    rng = random.Random(11)
    cases = [0, 1, 2, R - 1, R - 2, LAM, R - LAM, 2**127, 2**253, A2, R // 2]
    cases += [rng.randrange(R) for _ in range(20000)]
    for k in cases:
        k1, k2 = _split(k)
        assert (k1 + k2 * LAM - k) % R == 0
        assert abs(k1) < 2**127 and abs(k2) < 2**127
