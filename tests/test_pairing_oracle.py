"""The pairing oracle (oracle/pairing.py) pinned against the reference's own
libff reduced pairing (compiled from its sources, oracle/_ref), and the constants
of the device pairing (nkr-zkp_b200/csrc/pairing.cuh) derived again from the
curve: the ate loop 6z + 2, z, the twist Frobenius coefficients xi^((q-1)/3),
xi^((q-1)/2), xi^((q^2-1)/3) and the Fq12 Frobenius table xi^(m (q^k - 1)/6); the
final exponentiation's addition chain (libff's) is checked against the plain
exponent (q^2 + 1) k (q^4 - q^2 + 1)/r, k = 2z(6z^2 + 3z + 1), and libff."""
import os
import re

import numpy as np

import oracle as O
import pairing as OP

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = open(os.path.join(ROOT, "nkr-zkp_b200", "csrc", "pairing.cuh")).read()
Q, R = O.P, O.R
Z = 4965661367192848881


def _fq2_pow(a, e):
    res = (1, 0)
    while e:
        if e & 1:
            res = ((res[0] * a[0] - res[1] * a[1]) % Q, (res[0] * a[1] + res[1] * a[0]) % Q)
        a = ((a[0] * a[0] - a[1] * a[1]) % Q, (2 * a[0] * a[1]) % Q)
        e >>= 1
    return res


def _fq_mont_int(words):
    return sum(w << (64 * i) for i, w in enumerate(words)) * pow(2, -256, Q) % Q


def _fq_literal(body):
    """the four 64-bit words of an fq_from_u64(...) call"""
    return [int(w.strip().rstrip("ull"), 0) for w in body.split(",")]


def test_oracle_pairing_matches_reference_libff(ref):
    rng = np.random.default_rng(21)
    for a, b in O.random_fr(4, rng).reshape(2, 2, 4):
        p, q = ref.mul_gen(1, a), ref.mul_gen(2, b)
        assert np.array_equal(OP.reduced_pairing_limbs(p, q), ref.reduced_pairing(p, q))


def test_final_exponent_chain_matches_reference_libff(ref):
    """libff's addition chain (the device's final exponentiation) equals both the
    plain exponentiation by (q^2 + 1) k (q^4 - q^2 + 1)/r and libff's own value."""
    rng = np.random.default_rng(22)
    a, b = O.random_fr(2, rng)
    p, q = ref.mul_gen(1, a), ref.mul_gen(2, b)
    P = (O.fq_int(p[0:4]), O.fq_int(p[4:8]))
    Qa = ((O.fq_int(q[0:4]), O.fq_int(q[4:8])), (O.fq_int(q[8:12]), O.fq_int(q[12:16])))
    f = OP.miller(P, Qa)
    chain = OP.gt_limbs(OP.final_exp_chain(f))
    assert np.array_equal(chain, OP.gt_limbs(OP.final_exp(f)))
    assert np.array_equal(chain, ref.reduced_pairing(p, q))


def test_device_pairing_constants():
    lo = int(re.search(r"kAteLoopLo = (0x[0-9a-f]+)ull", SRC).group(1), 16)
    top = int(re.search(r"kAteTopBit = (\d+);", SRC).group(1))
    assert lo | (1 << top) == 6 * Z + 2
    adds = int(re.search(r"kAteLines = 64 \+ (\d+) \+ 2;", SRC).group(1))
    assert adds == bin(lo).count("1") and top == 64
    assert int(re.search(r"kZ = (0x[0-9a-f]+)ull", SRC).group(1), 16) == Z
    table = SRC[SRC.index("kFrobGamma[15][2][4] = {"):]
    rows = re.findall(r"\{\{([^}]*)\}, \{([^}]*)\}\}, // k = (\d), m = (\d)", table)
    assert len(rows) == 15
    for c0, c1, k, m in rows:
        k, m = int(k), int(m)
        got = (_fq_mont_int(_fq_literal(c0)), _fq_mont_int(_fq_literal(c1)))
        assert got == _fq2_pow((9, 1), m * (Q**k - 1) // 6), (k, m)
    xi = (9, 1)
    calls = re.findall(r"fq_from_u64\(([^)]*)\)", SRC[SRC.index("frob_gx1()"):])
    gx1 = tuple(_fq_mont_int(_fq_literal(c)) for c in calls[0:2])
    gy1 = tuple(_fq_mont_int(_fq_literal(c)) for c in calls[2:4])
    gx2 = _fq_mont_int(_fq_literal(calls[4]))
    assert gx1 == _fq2_pow(xi, (Q - 1) // 3)
    assert gy1 == _fq2_pow(xi, (Q - 1) // 2)
    assert (gx2, 0) == _fq2_pow(xi, (Q * Q - 1) // 3)
    assert _fq2_pow(xi, (Q * Q - 1) // 2) == (Q - 1, 0)   # gy2 = -1
