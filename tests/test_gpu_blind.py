"""Blinding (nkr_b200_blind, replacing blind_proof of common/src/protocol.cpp:85-94)
bit-exact against the oracle's double-and-add blinding over edge-case and random
scalars, raw proofs given in unnormalised Jacobian form, and raw points at
infinity.  The B200 path uses fixed-base tables for the proving-key multiples
and the GLV split for s ar and r bs1, so scalars at the ends of the range and
at the split's sign changes are the cases to cover."""
import ctypes
import json
import os

import numpy as np
import pytest

import nkr_b200 as nk
import oracle as O
from conftest import GOLDEN

pytestmark = pytest.mark.gpu

R = O.R
P = O.P
# the cube root of unity in Fr that acts on G1 as (x, y) -> (beta x, y)
LAMBDA = 0xb3c4d79d41a917585bfc41088d8daaa78b17ea66b99c90dd


@pytest.fixture(scope="module")
def keyed(ctx):
    g = json.load(open(os.path.join(GOLDEN, "matmul4.json")))
    r1 = nk.generate(g["kind"], g["param"], g["density"], seed=g["seed"])
    pk = O.read_proving_key(os.path.join(GOLDEN, "matmul4.pk.bin"))
    be = nk.Backend(ctx)
    be.prepare(r1, pk)
    raw = be.prove(r1.witness)
    yield be, pk, raw
    be.free()


def _affine(raw):
    g1, g2 = nk.raw_to_arrays(raw)
    return np.stack([x[:8] for x in g1]), g2[:16]


def _check(be, orc, pk, raw, r, s, g1=None, g2=None):
    proof = be.blind(raw, r, s)
    if g1 is None:
        g1, g2 = _affine(raw)
    a, b, c = orc.blind(O.pk_affine(pk, orc), g1, g2, r, s)
    assert np.array_equal(np.frombuffer(bytes(proof.a), np.uint64), O.affine_to_jac(1, a)[0])
    assert np.array_equal(np.frombuffer(bytes(proof.b), np.uint64), O.affine_to_jac(2, b)[0])
    assert np.array_equal(np.frombuffer(bytes(proof.c), np.uint64), O.affine_to_jac(1, c)[0])
    return proof


EDGE = [(0, 0), (1, 1), (R - 1, R - 1), (0, 5), (7, 0), (2, R - 2),
        (2**127, 2**127 - 1), (2**253, R - 2**200), (LAMBDA, R - LAMBDA),
        (LAMBDA * LAMBDA % R, 1 + LAMBDA), (0x89d3256894d213e3, 0x6f4d8248eeb859fd0be4e1541221250b)]


@pytest.mark.parametrize("r,s", EDGE)
def test_blind_edge_scalars(keyed, orc, r, s):
    be, pk, raw = keyed
    _check(be, orc, pk, raw, O.fr_mont(r), O.fr_mont(s))


def test_blind_random_scalars(keyed, orc):
    be, pk, raw = keyed
    rng = np.random.default_rng(2024)
    for r, s in O.random_fr(48, rng).reshape(24, 2, 4):
        _check(be, orc, pk, raw, r, s)


def _jacobian_scaled(limbs, z, fq2):
    """libff (X, Y, Z = 1) -> (X z^2, Y z^3, z) for a random z (Fq or Fq2 coordinates)."""
    if not fq2:
        x, y = (O.fq_int(limbs[4 * i:4 * i + 4]) for i in range(2))
        z2 = z * z % P
        return np.concatenate([O.fq_mont(x * z2), O.fq_mont(y * z2 * z), O.fq_mont(z)])

    def get(i):
        return (O.fq_int(limbs[8 * i:8 * i + 4]), O.fq_int(limbs[8 * i + 4:8 * i + 8]))

    def mul(u, v):  # Fq2 with u^2 = -1
        return ((u[0] * v[0] - u[1] * v[1]) % P, (u[0] * v[1] + u[1] * v[0]) % P)

    zz = (z, 3 * z % P)
    x, y = get(0), get(1)
    z2 = mul(zz, zz)
    z3 = mul(z2, zz)
    xs, ys = mul(x, z2), mul(y, z3)
    return np.concatenate([O.fq_mont(xs[0]), O.fq_mont(xs[1]), O.fq_mont(ys[0]), O.fq_mont(ys[1]),
                           O.fq_mont(zz[0]), O.fq_mont(zz[1])])


def test_blind_accepts_unnormalised_raw(keyed, orc):
    """A raw proof in Jacobian form with Z != 1 blinds to the same proof."""
    be, pk, raw = keyed
    r, s = O.random_fr(2, np.random.default_rng(77))
    want = be.blind(raw, r, s)
    g1, g2 = nk.raw_to_arrays(raw)
    jac = nk.RawProofC()
    for k, f in enumerate(("ar", "bs1", "zk", "qz")):
        v = _jacobian_scaled(g1[k], 1234567 + 1000 * k, False)
        ctypes.memmove(getattr(jac, f), v.tobytes(), 96)
    ctypes.memmove(jac.bs2, _jacobian_scaled(g2, 987654321, True).tobytes(), 192)
    got = be.blind(jac, r, s)
    assert bytes(got) == bytes(want)


def test_blind_raw_points_at_infinity(keyed, orc):
    """ar, bs1, zk and qz at infinity (libff (0, 1, 0)) blind like the oracle."""
    be, pk, raw = keyed
    inf = np.concatenate([O.fq_mont(0), O.fq_mont(1), O.fq_mont(0)])
    zero = nk.RawProofC.from_buffer_copy(bytes(raw))
    for f in ("ar", "bs1", "zk", "qz"):
        ctypes.memmove(getattr(zero, f), inf.tobytes(), 96)
    g1, g2 = _affine(raw)
    g1 = np.stack([np.concatenate([O.fq_mont(0), O.fq_mont(1)])] * 4)
    r, s = O.random_fr(2, np.random.default_rng(78))
    _check(be, orc, pk, zero, r, s, g1, g2)


def test_blind_is_repeatable(keyed):
    be, pk, raw = keyed
    r, s = O.random_fr(2, np.random.default_rng(79))
    assert bytes(be.blind(raw, r, s)) == bytes(be.blind(raw, r, s))


def test_blind_of_a_raw_proof_the_slot_did_not_make(keyed, orc):
    """A raw proof whose ar is not the slot's last prove's (here 2 ar, a valid
    point) takes the chain path for s ar and the tables for r bs1; both agree
    with the oracle, and the slot's own proof still blinds through the tables."""
    be, pk, raw = keyed
    g1, g2 = _affine(raw)
    ar2 = orc.add_affine(1, g1[0], g1[0])
    other = nk.RawProofC.from_buffer_copy(bytes(raw))
    ctypes.memmove(other.ar, np.concatenate([ar2, O.fq_mont(1)]).tobytes(), 96)
    g1o = g1.copy()
    g1o[0] = ar2
    for seed in (81, 82):
        r, s = O.random_fr(2, np.random.default_rng(seed))
        _check(be, orc, pk, other, r, s, g1o, g2)
        _check(be, orc, pk, raw, r, s)
