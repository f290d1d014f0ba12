"""GPU setup with seeded toxic waste against the oracle's restatement of the
reference setup scalars, and full-size (2^20 constraints) prove checks: SpMV
vectors and H bit-exact against the oracle, and the reference verifier accepts
the blinded proof."""
import os

import numpy as np
import pytest

import nkr_b200 as nk
import oracle as O

pytestmark = pytest.mark.gpu


def _toxic(seed):
    return list(O.random_fr(5, np.random.default_rng(seed)))


def test_setup_matches_oracle_scalars(ctx, orc):
    r1 = nk.generate("matmul", 4, 1, seed=3)
    tox = _toxic(1)
    pk, vk = nk.setup(ctx, r1, tox)
    at, bt, lt, ic, ht = orc.setup_scalars(r1, tox)
    g1, g2 = orc.g1_generator(), orc.g2_generator()

    def check(group, pts, scalars):
        for i in range(scalars.shape[0]):
            want = O.affine_to_jac(group, orc.mul_affine(group, g1 if group == 1 else g2, scalars[i]))[0]
            assert np.array_equal(pts[i], want), i

    check(1, pk["a_query"], at)
    check(1, pk["b_g1_query"], bt)
    check(2, pk["b_g2_query"], bt)
    check(1, pk["l_query"], lt)
    check(1, pk["h_query"], ht)
    check(1, vk["ic"], ic)
    for name, k, grp in (("alpha_g1", tox[1], 1), ("beta_g1", tox[2], 1), ("delta_g1", tox[4], 1),
                         ("beta_g2", tox[2], 2), ("delta_g2", tox[4], 2)):
        want = O.affine_to_jac(grp, orc.mul_affine(grp, g1 if grp == 1 else g2, k))[0]
        assert np.array_equal(pk[name], want), name


def _prove_and_verify(ctx, ref, r1, tox, tmp_path):
    pk, vk = nk.setup(ctx, r1, tox)
    vk_path = tmp_path / "vk.bin"
    ref.write_vk(vk, vk_path)
    be = nk.Backend(ctx)
    be.prepare(r1, pk)
    raw = be.prove(r1.witness)
    r, s = O.random_fr(2, np.random.default_rng(3))
    proof = be.blind(raw, r, s)
    path = tmp_path / "proof.bin"
    O.write_proof(path, np.frombuffer(bytes(proof.a), np.uint64), np.frombuffer(bytes(proof.b), np.uint64),
                  np.frombuffer(bytes(proof.c), np.uint64))
    ok = ref.verify(vk_path, r1.witness[1:1 + r1.public_inputs], path)
    return be, ok


def test_gpu_setup_proof_verifies(ctx, ref, tmp_path):
    r1 = nk.generate("poseidon", 4, 1, seed=13)
    be, ok = _prove_and_verify(ctx, ref, r1, _toxic(2), tmp_path)
    assert ok
    be.free()


@pytest.mark.parametrize("count,logn", [(2048, 20), (4096, 21)])
def test_full_size_prove(ctx, orc, ref, tmp_path, count, logn):
    """poseidon at sparse density, count 2048 (2^20 constraints and columns, the
    headline size) and count 4096 (2^21, the full-prove config)."""
    r1 = nk.generate("poseidon", count, 2, seed=1)
    assert r1.rows == 1 << logn
    be, ok = _prove_and_verify(ctx, ref, r1, _toxic(4), tmp_path)
    assert ok
    az, bz, cz, h = be.intermediates()
    for k, got in enumerate((az, bz, cz)):
        want = orc.spmv(r1.rows, r1.row_ptr[k], r1.col_idx[k], r1.values[k], r1.witness)
        assert np.array_equal(got, want)
    assert np.array_equal(h, orc.quotient(az, bz, cz))
    be.free()
