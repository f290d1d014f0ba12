"""The seeded circuit generator (nkr-zkp_b200/host/circuits.cpp) against the
reference: Poseidon parameters from its constants file, its known answer, and
entry-for-entry equality with circuits the reference's own R1CSManager and
gadgets build from the same inputs (where oracle/_ref is built)."""
import json
import os

import numpy as np
import pytest

import nkr_b200 as nk
import oracle as O
from conftest import GOLDEN


def test_poseidon_parameters_match_reference_constants():
    g = json.load(open(os.path.join(GOLDEN, "poseidon_constants.json")))
    rc, mds = nk.poseidon_parameters()
    assert [O.fr_int(x) for x in rc] == [int(x, 16) for x in g["round_constants"]]
    assert [O.fr_int(x) for x in mds] == [int(x, 16) for x in g["mds"]]


def test_poseidon_known_answer():
    d = nk.poseidon_hash2(O.fr_mont(1), O.fr_mont(2))
    assert O.fr_int(d) == 7853200120776062878684798364095072458815029376092732009249414926327459813530


def test_poseidon_counts_match_reference_test():
    # protocols/groth16/tests/poseidon_test.cpp:40-48: 439 constraints, 442 variables, 512x512
    r = nk.generate("poseidon", 1, 0, seed=1)
    assert (r.constraints, r.variables, r.rows, r.cols, r.public_inputs) == (439, 442, 512, 512, 1)


def test_sql_counts_match_reference():
    # sql_aggregate_test.cpp:43-54 and README: 947 N - 404 constraints
    for n in (2, 4, 8):
        r = nk.generate("sql-aggregate", n, 0, seed=2)
        assert r.constraints == 947 * n - 404


def test_matmul_counts_and_sizes():
    for s in (2, 3, 32):
        r = nk.generate("matmul", s, 0, seed=1)
        assert r.constraints == s**3 + s**2
        assert r.variables == 1 + 3 * s * s + s**3
    r = nk.generate("matmul", 32, 0, seed=1)
    assert (r.rows, r.cols) == (2**16, 2**16)


def test_density_nonzero_counts():
    # density.hpp:155-163: full, hybrid count - count/2, sparse ceil(count/10)
    s = 10
    for dens, nz in ((0, 100), (1, 50), (2, 10)):
        r = nk.generate("matmul", s, dens, seed=4)
        a = r.witness[1:1 + s * s]
        assert int(np.count_nonzero(np.any(a != 0, axis=1))) == nz


def test_generator_is_seeded():
    a = nk.generate("poseidon", 3, 1, seed=5)
    b = nk.generate("poseidon", 3, 1, seed=5)
    c = nk.generate("poseidon", 3, 1, seed=6)
    assert np.array_equal(a.witness, b.witness)
    assert not np.array_equal(a.witness, c.witness)


def test_witness_satisfies_r1cs(orc):
    for kind, p, d in (("matmul", 3, 1), ("poseidon", 2, 2), ("sql-aggregate", 2, 0), ("fibonacci", 9, 0)):
        r = nk.generate(kind, p, d, seed=3)
        az = orc.spmv(r.rows, r.row_ptr[0], r.col_idx[0], r.values[0], r.witness)
        bz = orc.spmv(r.rows, r.row_ptr[1], r.col_idx[1], r.values[1], r.witness)
        cz = orc.spmv(r.rows, r.row_ptr[2], r.col_idx[2], r.values[2], r.witness)
        for i in range(r.rows):
            assert O.fr_int(az[i]) * O.fr_int(bz[i]) % O.R == O.fr_int(cz[i]), (kind, i)


def _same(mine, theirs):
    assert (mine.rows, mine.cols, mine.public_inputs) == (theirs["rows"], theirs["cols"],
                                                         theirs["public_inputs"])
    for k in range(3):
        assert np.array_equal(mine.row_ptr[k], theirs["row_ptr"][k])
        assert np.array_equal(mine.col_idx[k], theirs["col_idx"][k])
        assert np.array_equal(mine.values[k], theirs["values"][k])
    assert np.array_equal(mine.witness, theirs["witness"])


@pytest.mark.parametrize("s,dens", [(2, 0), (4, 1), (5, 2)])
def test_matmul_equals_reference_builder(ref, s, dens):
    m = nk.generate("matmul", s, dens, seed=7)
    _same(m, ref.matmul_circuit(s, m.witness[1:1 + s * s], m.witness[1 + s * s:1 + 2 * s * s]))


@pytest.mark.parametrize("count,dens", [(1, 0), (3, 2)])
def test_poseidon_equals_reference_gadget(ref, count, dens):
    m = nk.generate("poseidon", count, dens, seed=3)
    per = (m.variables - 1 - m.public_inputs) // count
    lr = []
    for i in range(count):
        base = 1 + m.public_inputs + i * per
        lr += [m.witness[base], m.witness[base + 1]]
    _same(m, ref.poseidon_circuit_n(np.array(lr)))


@pytest.mark.parametrize("n,dens", [(2, 0), (4, 2)])
def test_sql_equals_reference_gadget(ref, n, dens):
    m = nk.generate("sql-aggregate", n, dens, seed=5)
    base = 1 + m.public_inputs + 32
    per_row = 2 + 64 + 1 + (3 * (8 * 3 + 57) + 3 * 65)
    cats = [m.witness[base + i * per_row] for i in range(n)]
    amts = [m.witness[base + i * per_row + 1] for i in range(n)]
    _same(m, ref.sql_circuit(np.array(cats), np.array(amts)))


def test_reference_accepts_generated_witness(ref):
    for kind, p, d in (("matmul", 4, 1), ("poseidon", 2, 0), ("fibonacci", 20, 0)):
        r = nk.generate(kind, p, d, seed=8)
        assert ref.check_witness(r, r.witness)
        bad = r.witness.copy()
        bad[1] = O.fr_mont(O.fr_int(bad[1]) + 1)
        assert not ref.check_witness(r, bad)


def test_benchmark_witness_repeats_values():
    """The 2^20-constraint benchmark witness (poseidon count 2048, sparse) repeats
    values: 899,483 nonzero of 1,048,576 variables take 169,390 distinct values
    (one of them zero), 829 of which cover 880,015 variables.  The witness MSMs'
    class path sums the bases of each repeated value once, so the prove time of the
    benchmark depends on this (bench.py also reports a prove over distinct values)."""
    r1 = nk.generate("poseidon", 2048, 2, seed=1)
    w = np.ascontiguousarray(np.asarray(r1.witness)).view(np.uint8).reshape(-1, 32)
    vals, counts = np.unique(w, axis=0, return_counts=True)
    assert w.shape[0] == 1 << 20
    assert int(w.any(axis=1).sum()) == 899483
    assert vals.shape[0] == 169390
    assert int((counts >= 2).sum()) == 829 and int(counts[counts >= 2].sum()) == 880015
