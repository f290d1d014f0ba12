"""Field and group primitives on the B200 against big-integer arithmetic and
the oracle (bit-exact)."""
import numpy as np
import pytest

import oracle as O

pytestmark = pytest.mark.gpu


def _edge_and_random(mod, rng, n=200):
    vals = [0, 1, 2, mod - 1, mod - 2, 2**255 % mod, 2**254 % mod, (mod - 1) // 2]
    vals += [int.from_bytes(rng.bytes(32), "little") % mod for _ in range(n)]
    return vals


@pytest.mark.parametrize("field,mod", [(0, O.R), (1, O.P)])
def test_field_ops_exact(ctx, rng, field, mod):
    conv = O.fr_mont if field == 0 else O.fq_mont
    back = O.fr_int if field == 0 else O.fq_int
    a_int = _edge_and_random(mod, rng)
    b_int = list(reversed(a_int))
    a = np.stack([conv(x) for x in a_int])
    b = np.stack([conv(x) for x in b_int])
    mul = ctx.field_op(field, 0, a, b)
    add = ctx.field_op(field, 1, a, b)
    sub = ctx.field_op(field, 2, a, b)
    sq = ctx.field_op(field, 3, a)
    inv = ctx.field_op(field, 4, a)
    for i, (x, y) in enumerate(zip(a_int, b_int)):
        assert back(mul[i]) == x * y % mod
        assert back(add[i]) == (x + y) % mod
        assert back(sub[i]) == (x - y) % mod
        assert back(sq[i]) == x * x % mod
        assert back(inv[i]) == (pow(x, -1, mod) if x else 0)
    # Montgomery conversions: canonical limbs in, Montgomery out and back
    canon = np.stack([O.int_to_limbs(x) for x in a_int])
    m = ctx.field_op(field, 5, canon)
    assert all(back(m[i]) == a_int[i] for i in range(len(a_int)))
    assert np.array_equal(ctx.field_op(field, 6, m), canon)


def test_fp64_limb_arithmetic_matches_integer_arithmetic(ctx, rng):
    """The MSM's FP64-limb Fq (five 52-bit limbs, R = 2^260; fields 3 and 4) gives
    exactly the integer library's results (fields 1 and 2) on edge and random values."""
    a_int = _edge_and_random(O.P, rng, n=2000)
    b_int = list(reversed(a_int))
    a = np.stack([O.fq_mont(x) for x in a_int])
    b = np.stack([O.fq_mont(x) for x in b_int])
    for op in range(4):
        assert np.array_equal(ctx.field_op(3, op, a, b), ctx.field_op(1, op, a, b)), f"op {op}"
    neg = ctx.field_op(3, 4, a)
    assert all(O.fq_int(neg[i]) == (-x) % O.P for i, x in enumerate(a_int))
    a2 = np.concatenate([a, b], axis=1)
    b2 = np.concatenate([b[::-1], a[::-1]], axis=1)
    P = O.P
    for field, op in [(f, o) for o in range(4) for f in (2, 4)]:
        got = ctx.field_op(field, op, a2, b2)
        bad = []
        for i in range(len(a_int)):
            x0, x1, y0, y1 = a_int[i], b_int[i], b_int[::-1][i], a_int[::-1][i]
            want = {0: ((x0 * y0 - x1 * y1) % P, (x0 * y1 + x1 * y0) % P),
                    1: ((x0 + y0) % P, (x1 + y1) % P), 2: ((x0 - y0) % P, (x1 - y1) % P),
                    3: ((x0 * x0 - x1 * x1) % P, 2 * x0 * x1 % P)}[op]
            if (O.fq_int(got[i][:4]), O.fq_int(got[i][4:])) != want:
                bad.append((i, hex(x0), hex(x1), hex(y0), hex(y1)))
        assert not bad, f"field {field} op {op}: {len(bad)} wrong, first {bad[:3]}"


def test_fq2_ops_exact(ctx, rng):
    n = 64
    ai = [(int.from_bytes(rng.bytes(32), "little") % O.P, int.from_bytes(rng.bytes(32), "little") % O.P)
          for _ in range(n)]
    bi = [(int.from_bytes(rng.bytes(32), "little") % O.P, int.from_bytes(rng.bytes(32), "little") % O.P)
          for _ in range(n)]
    ai[0] = (0, 0)
    ai[1] = (1, 0)
    enc = lambda v: np.concatenate([O.fq_mont(v[0]), O.fq_mont(v[1])])
    a = np.stack([enc(v) for v in ai])
    b = np.stack([enc(v) for v in bi])
    mul = ctx.field_op(2, 0, a, b)
    sq = ctx.field_op(2, 3, a)
    inv = ctx.field_op(2, 4, a)
    for i in range(n):
        (a0, a1), (b0, b1) = ai[i], bi[i]
        assert (O.fq_int(mul[i][:4]), O.fq_int(mul[i][4:])) == ((a0 * b0 - a1 * b1) % O.P, (a0 * b1 + a1 * b0) % O.P)
        assert (O.fq_int(sq[i][:4]), O.fq_int(sq[i][4:])) == ((a0 * a0 - a1 * a1) % O.P, 2 * a0 * a1 % O.P)
        if a0 or a1:
            d = pow(a0 * a0 + a1 * a1, -1, O.P)
            assert (O.fq_int(inv[i][:4]), O.fq_int(inv[i][4:])) == (a0 * d % O.P, -a1 * d % O.P)


@pytest.mark.parametrize("group", [1, 2])
def test_group_ops_match_oracle(ctx, orc, rng, group):
    n = 24
    gen = orc.g1_generator() if group == 1 else orc.g2_generator()
    ks = O.random_fr(n, rng)
    pts = np.stack([orc.mul_affine(group, gen, k) for k in ks])
    other = np.roll(pts, 1, axis=0)
    other[0] = pts[0]                              # P + P (doubling branch)
    neg = pts[1].copy()
    w = 4 * group
    for j in range(group):                         # -P: negate each y coordinate limb group
        yj = O.fq_int(neg[w + 4 * j:w + 4 * j + 4])
        neg[w + 4 * j:w + 4 * j + 4] = O.fq_mont(-yj)
    other[1] = neg                                 # P + (-P) = infinity
    other[2] = 0
    other[2, w:w + 4] = O.fq_mont(1)               # P + infinity
    ja, jb = O.affine_to_jac(group, pts), O.affine_to_jac(group, other)
    got = ctx.group_op(group, 0, ja, jb)
    for i in range(n):
        want = orc.add_affine(group, pts[i], other[i])
        assert np.array_equal(O.affine_to_jac(group, want)[0], got[i]), i
    dbl = ctx.group_op(group, 1, ja)
    for i in range(4):
        assert np.array_equal(dbl[i], O.affine_to_jac(group, orc.add_affine(group, pts[i], pts[i]))[0])
    sc = O.random_fr(n, rng)
    sc[0] = 0
    sc[1] = O.fr_mont(O.R - 1)
    mul = ctx.group_op(group, 2, ja, sc)
    for i in range(6):
        assert np.array_equal(mul[i], O.affine_to_jac(group, orc.mul_affine(group, pts[i], sc[i]))[0])


def test_mul_throughput_positive(ctx):
    for field in (0, 1):
        rate, ms = ctx.bench_mul(field)
        assert rate > 1e9 and ms > 0
    # the FP64 forms check themselves against the library product before timing
    # (the lazily reduced one also with an input in [p, 2p))
    for variant in (3, 4):
        rate, ms = ctx.bench_mul(1 | (variant << 8))
        assert rate > 1e9 and ms > 0
