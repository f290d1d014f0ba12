"""The benchmark's own input helpers (CPU): its generator constants equal the
oracle's generators, and its seeded scalar mixes have the stated shape."""
import os
import sys

import numpy as np

import oracle as O

sys.path.insert(0, os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
import bench  # noqa: E402


def test_generators_match_oracle(orc):
    assert np.array_equal(bench._generator_jac(1), O.affine_to_jac(1, orc.g1_generator()[None])[0])
    assert np.array_equal(bench._generator_jac(2), O.affine_to_jac(2, orc.g2_generator()[None])[0])


def test_uniform_fr_below_modulus():
    a = bench._uniform_fr(5000, np.random.default_rng(2))
    assert all(O.limbs_to_int(r) < O.R for r in a)
    assert len({r.tobytes() for r in a}) == 5000


def test_sparse_witness_mix_shape():
    n = 20000
    s = bench._sparse_witness_scalars(n, np.random.default_rng(3))
    vals = [O.fr_int(r) for r in s]
    zero = sum(v == 0 for v in vals) / n
    one = sum(v == 1 for v in vals) / n
    big = sum(v >= 1 << 16 for v in vals) / n
    assert 0.47 < zero < 0.53          # 30% + a third of 60%
    assert 0.18 < one < 0.22           # a third of 60%
    assert 0.09 < big < 0.11           # the uniform 10%


def test_verify_mode_scalars_are_uniform_fr():
    """bench.py's verify mode draws r, s as Fr Montgomery limbs below r, deterministically."""
    import numpy as np
    import bench
    a = bench._uniform_fr_rows(np.random.default_rng(12), 64)
    b = bench._uniform_fr_rows(np.random.default_rng(12), 64)
    assert np.array_equal(a, b) and a.shape == (64, 4)
    r = 21888242871839275222246405745257275088548364400416034343698204186575808495617
    vals = [sum(int(w) << (64 * i) for i, w in enumerate(row)) for row in a]
    assert all(v < r for v in vals) and len(set(vals)) == 64
