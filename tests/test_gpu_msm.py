"""Pippenger MSM on the B200 (G1 and G2, plain and resident-folded bases)
against the oracle and the reference's BDLO12 golden results: bit-exact after
affine normalisation, including zero scalars, repeated points (doubling inside
a bucket), P and -P, infinity bases, r - 1, and skewed scalar distributions."""
import json
import os

import numpy as np
import pytest

import nkr_b200 as nk
import oracle as O
from conftest import GOLDEN

pytestmark = pytest.mark.gpu


def _points(orc, group, n, rng, distinct=None):
    gen = orc.g1_generator() if group == 1 else orc.g2_generator()
    m = n if distinct is None else distinct
    ks = O.random_fr(m, rng)
    pts = np.stack([orc.mul_affine(group, gen, k) for k in ks])
    if m < n:
        pts = pts[rng.integers(0, m, n)]
    return pts


def _check(ctx, orc, group, aff, sc, folded):
    jac = O.affine_to_jac(group, aff)
    want = O.affine_to_jac(group, orc.msm(group, aff, sc))[0]
    if folded:
        b = nk.MsmBases(ctx, group, jac)
        got, _ = b.run(sc)
        got2, _ = b.run(sc)           # reruns reuse the resident bases and scratch
        assert np.array_equal(got, got2)
        b.free()
    else:
        got = ctx.msm(group, jac, sc)
    assert np.array_equal(got, want)


@pytest.mark.parametrize("folded", [False, True])
@pytest.mark.parametrize("group", [1, 2])
@pytest.mark.parametrize("n", [1, 2, 7, 100, 1000])
def test_msm_uniform(ctx, orc, rng, group, n, folded):
    aff = _points(orc, group, n, rng)
    sc = O.random_fr(n, rng)
    _check(ctx, orc, group, aff, sc, folded)


@pytest.mark.parametrize("folded", [False, True])
@pytest.mark.parametrize("group", [1, 2])
def test_msm_edge_cases(ctx, orc, rng, group, folded):
    n = 300
    aff = _points(orc, group, n, rng, distinct=40)    # many repeated bases
    sc = O.random_fr(n, rng)
    sc[:50] = 0
    sc[50:80] = O.fr_mont(1)
    sc[80:90] = O.fr_mont(O.R - 1)
    sc[90:150] = sc[90]                               # one scalar repeated on repeated bases
    w = 4 * group
    aff[150:160] = 0
    aff[150:160, w:w + 4] = O.fq_mont(1)              # infinity bases
    neg = aff[160].copy()
    for j in range(group):
        neg[w + 4 * j:w + 4 * j + 4] = O.fq_mont(-O.fq_int(neg[w + 4 * j:w + 4 * j + 4]))
    aff[161] = neg
    sc[161] = sc[160]                                 # P and -P with the same scalar cancel
    _check(ctx, orc, group, aff, sc, folded)


@pytest.mark.parametrize("group", [1, 2])
def test_msm_mostly_and_all_infinity_bases(ctx, orc, rng, group):
    """Resident bases keep only their finite points (a B query is ~70% infinity)
    and gather the scalars through the kept indices; all-infinity bases give 0."""
    n = 2000
    aff = _points(orc, group, n, rng, distinct=200)
    w = 4 * group
    inf = np.nonzero(rng.random(n) < 0.7)[0]
    aff[inf] = 0
    aff[inf, w:w + 4] = O.fq_mont(1)
    sc = O.random_fr(n, rng)
    _check(ctx, orc, group, aff, sc, folded=True)
    aff[:] = 0
    aff[:, w:w + 4] = O.fq_mont(1)
    _check(ctx, orc, group, aff, sc, folded=True)


def test_autotuned_window_matches_model_window(ctx, orc, rng):
    """The tuner picks a window per size class on this GPU; any window gives the
    same canonical result, so tuned and cost-model MSMs agree with the oracle."""
    n = 1 << 14
    c, ms = ctx.tune_msm(n)
    assert 6 <= c <= 22 and ms > 0
    assert ctx.tune_msm(n - 1000) == (c, ms)  # same size class, measured once
    model = nk.Context(0)
    model.set_autotune(False)
    aff = _points(orc, 1, n, rng, distinct=512)
    sc = O.random_fr(n, rng)
    jac = O.affine_to_jac(1, aff)
    want = O.affine_to_jac(1, orc.msm(1, aff, sc))[0]
    for cx in (ctx, model):
        b = nk.MsmBases(cx, 1, jac)
        got, _ = b.run(sc)
        assert np.array_equal(got, want)
        b.free()
    model.close()


@pytest.mark.parametrize("folded", [False, True])
def test_msm_all_zero_scalars_is_infinity(ctx, orc, rng, folded):
    aff = _points(orc, 1, 50, rng)
    sc = np.zeros((50, 4), np.uint64)
    _check(ctx, orc, 1, aff, sc, folded)


@pytest.mark.parametrize("folded", [False, True])
def test_msm_sparse_witness_mix(ctx, orc, rng, folded):
    """10% uniform, 30% zero, 60% in {0, 1, small < 2^16} (the sparse-scalar config)."""
    n = 1 << 13
    aff = _points(orc, 1, n, rng, distinct=512)
    sc = O.random_fr(n, rng)
    u = rng.random(n)
    sc[(u >= 0.1) & (u < 0.4)] = 0
    cat = rng.integers(0, 3, n)
    sel = u >= 0.4
    sc[sel & (cat == 0)] = 0
    sc[sel & (cat == 1)] = O.fr_mont(1)
    small = np.nonzero(sel & (cat == 2))[0]
    for i in small:
        sc[i] = O.fr_mont(int(rng.integers(0, 1 << 16)))
    _check(ctx, orc, 1, aff, sc, folded)


@pytest.mark.parametrize("group", [1, 2])
def test_msm_golden(ctx, orc, group):
    g = json.load(open(os.path.join(GOLDEN, "msm.json")))[f"g{group}"]
    r = np.random.default_rng(g["seed"])
    ks = O.random_fr(g["n"], r)
    sc = O.random_fr(g["n"], r)
    sc[0] = 0
    sc[1] = O.fr_mont(1)
    sc[2] = O.fr_mont(O.R - 1)
    sc[3] = sc[4]
    ks[3] = ks[4]
    sc[5] = O.fr_mont(2**16 - 1)
    gen = orc.g1_generator() if group == 1 else orc.g2_generator()
    aff = np.stack([orc.mul_affine(group, gen, k) for k in ks])
    aff[6] = 0
    aff[6, 4 * group:4 * group + 4] = O.fq_mont(1)
    jac = O.affine_to_jac(group, aff)
    assert O.sha256_arr(jac) == g["bases_sha256"]
    got = ctx.msm(group, jac, sc)
    assert got[:8 * group].tobytes().hex() == g["result_affine"]


def test_msm_2_16_matches_oracle(ctx, orc, rng):
    n = 1 << 16
    aff = _points(orc, 1, n, rng, distinct=4096)
    sc = O.random_fr(n, rng)
    _check(ctx, orc, 1, aff, sc, folded=True)


def test_msm_linearity_at_2_20(ctx, orc, rng):
    """Size-independent check at the benchmark size: MSM(P, a) + MSM(P, b) = MSM(P, a + b)
    and MSM over the whole = MSM of the halves added."""
    n = 1 << 20
    aff = _points(orc, 1, n, rng, distinct=2048)
    jac = O.affine_to_jac(1, aff)
    b = nk.MsmBases(ctx, 1, jac)
    a_s = O.random_fr(n, rng)
    b_s = O.random_fr(n, rng)
    ai = np.frombuffer(a_s.tobytes(), dtype=np.uint8).reshape(n, 32)
    # a + b mod r via python ints on the limb images (Montgomery form is linear)
    s = np.empty_like(a_s)
    for i in range(n):
        v = (int.from_bytes(a_s[i].tobytes(), "little") + int.from_bytes(b_s[i].tobytes(), "little")) % O.R
        s[i] = np.frombuffer(v.to_bytes(32, "little"), np.uint64)
    ra, _ = b.run(a_s)
    rb, _ = b.run(b_s)
    rs, _ = b.run(s)
    want = orc.add_affine(1, ra[:8], rb[:8])
    assert np.array_equal(rs[:8], want)
    b.free()
    del ai


def _sparse_witness_scalars(n, rng):
    """10% uniform, 30% zero, 60% uniformly one of {zero, one, small < 2^16}."""
    small = np.stack([O.fr_mont(v) for v in range(1 << 16)])
    out = np.zeros((n, 4), np.uint64)
    n_uni, n_zero = n // 10, (3 * n) // 10
    out[:n_uni] = O.random_fr(n_uni, rng)
    rest = n - n_uni - n_zero
    cat = rng.integers(0, 3, rest)
    vals = np.where(cat == 0, 0, np.where(cat == 1, 1, rng.integers(0, 1 << 16, rest)))
    out[n_uni + n_zero:] = small[vals]
    return out[rng.permutation(n)]


@pytest.mark.parametrize("group,logn,mix", [(1, 22, "uniform"), (1, 22, "sparse"), (1, 20, "sparse"),
                                            (2, 18, "uniform"), (2, 18, "sparse")])
def test_msm_full_size_equals_scalar_sum(ctx, orc, rng, group, logn, mix):
    """The operator-bench sizes with distinct bases P_i = k_i G: the MSM must equal
    (sum_i s_i k_i) G, computed by the oracle (one scalar multiplication)."""
    n = 1 << logn
    gen = orc.g1_generator() if group == 1 else orc.g2_generator()
    gen_jac = O.affine_to_jac(group, gen[None])[0]
    ks = O.random_fr(n, rng)
    bases = ctx.group_op(group, 2, np.tile(gen_jac, (n, 1)), ks)
    for j in rng.integers(0, n, 3):   # spot-check the bases themselves
        assert np.array_equal(bases[j], O.affine_to_jac(group, orc.mul_affine(group, gen, ks[j])[None])[0])
    sc = O.random_fr(n, rng) if mix == "uniform" else _sparse_witness_scalars(n, rng)
    ints = lambda a: [int.from_bytes(row.tobytes(), "little") for row in a]  # noqa: E731
    t = sum(a * b for a, b in zip(ints(sc), ints(ks))) * pow(2, -512, O.R) % O.R
    want = O.affine_to_jac(group, orc.mul_affine(group, gen, O.fr_mont(t))[None])[0]
    b = nk.MsmBases(ctx, group, bases)
    del bases
    got, _ = b.run(sc)
    b.free()
    assert np.array_equal(got, want)
