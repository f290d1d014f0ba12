"""R1CS SpMV on the B200 against the oracle (backend.cpp:25-35 semantics),
bit-exact: empty rows, unit / zero / general coefficients, long rows, and the
generated benchmark circuits."""
import numpy as np
import pytest

import nkr_b200 as nk
import oracle as O

pytestmark = pytest.mark.gpu


def _random_csr(rng, rows, cols, max_len):
    lens = rng.integers(0, max_len + 1, rows)
    lens[: rows // 8] = 0                      # empty rows
    row_ptr = np.concatenate([[0], np.cumsum(lens)]).astype(np.uint32)
    nnz = int(row_ptr[-1])
    col = rng.integers(0, cols, nnz).astype(np.uint32)
    vals = O.random_fr(nnz, rng)
    kind = rng.integers(0, 4, nnz)
    vals[kind == 0] = O.fr_mont(1)             # unit coefficients (tagged path)
    vals[kind == 1] = 0                        # explicit zeros (skipped path)
    return row_ptr, col, vals


@pytest.mark.parametrize("rows,cols,max_len", [(1, 1, 1), (64, 16, 3), (1000, 700, 9), (4096, 5000, 70)])
def test_spmv_matches_oracle(ctx, orc, rng, rows, cols, max_len):
    rp, ci, vals = _random_csr(rng, rows, cols, max_len)
    z = O.random_fr(cols, rng)
    z[0] = O.fr_mont(1)
    got = ctx.spmv(rows, cols, rp, ci, vals, z)
    assert np.array_equal(got, orc.spmv(rows, rp, ci, vals, z))


@pytest.mark.parametrize("kind,param,dens", [("matmul", 8, 0), ("poseidon", 4, 2), ("sql-aggregate", 4, 1)])
def test_spmv_on_circuits(ctx, orc, kind, param, dens):
    r = nk.generate(kind, param, dens, seed=21)
    for k in range(3):
        got = ctx.spmv(r.rows, r.cols, r.row_ptr[k], r.col_idx[k], r.values[k], r.witness)
        want = orc.spmv(r.rows, r.row_ptr[k], r.col_idx[k], r.values[k], r.witness)
        assert np.array_equal(got, want), (kind, k)


def test_spmv_rejects_out_of_range_column(ctx):
    with pytest.raises(nk.B200Error):
        ctx.spmv(2, 3, np.array([0, 1, 2], np.uint32), np.array([0, 3], np.uint32),
                 np.zeros((2, 4), np.uint64), np.zeros((3, 4), np.uint64))


@pytest.mark.parametrize("fill", ["all_unit", "all_zero", "all_general"])
def test_spmv_single_coefficient_class(ctx, orc, rng, fill):
    """Matrices whose terms all take one path: no non-unit terms (the product
    launch is skipped), only skipped zero terms, or only general products."""
    rows, cols = 700, 300
    rp, ci, vals = _random_csr(rng, rows, cols, 6)
    if fill == "all_unit":
        vals[:] = O.fr_mont(1)
    elif fill == "all_zero":
        vals[:] = 0
    else:
        vals[:] = O.random_fr(len(vals), rng)
    z = O.random_fr(cols, rng)
    got = ctx.spmv(rows, cols, rp, ci, vals, z)
    assert np.array_equal(got, orc.spmv(rows, rp, ci, vals, z))
