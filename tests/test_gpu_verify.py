"""Groth16 verification and the reduced pairing on the B200.

nkr_b200_reduced_pairing must return libff's GT values bit for bit (the
reference's verify, common/src/protocol.cpp:96-108, compares pairings against
the key's libff-computed e(alpha, beta)); nkr_b200_verify_batch must give the
reference verifier's verdict for every proof: valid proofs (the golden matmul-4
circuit and keys, blinded with many r, s), tampered ones (C moved, A and C
swapped, a public input changed, points at infinity) and a public-input count
that does not match the key."""
import ctypes
import json
import os

import numpy as np
import pytest

import nkr_b200 as nk
import oracle as O
from conftest import GOLDEN

pytestmark = pytest.mark.gpu


def test_reduced_pairing_matches_libff(ctx, ref):
    rng = np.random.default_rng(41)
    ps, qs = [], []
    for a, b in O.random_fr(12, rng).reshape(6, 2, 4):
        ps.append(ref.mul_gen(1, a))
        qs.append(ref.mul_gen(2, b))
    got = nk.reduced_pairing(ctx, np.stack(ps), np.stack(qs))
    for i in range(len(ps)):
        assert np.array_equal(got[i], ref.reduced_pairing(ps[i], qs[i])), i


def test_reduced_pairing_bilinear_and_at_infinity(ctx, ref):
    g1 = ref.mul_gen(1, O.fr_mont(1))
    g2 = ref.mul_gen(2, O.fr_mont(1))
    a, b = 123456789, 987654321
    pa, qb = ref.mul_gen(1, O.fr_mont(a)), ref.mul_gen(2, O.fr_mont(b))
    pab = ref.mul_gen(1, O.fr_mont(a * b))
    e1, e2 = nk.reduced_pairing(ctx, np.stack([pa, pab]), np.stack([qb, g2]))
    assert np.array_equal(e1, e2)                       # e(aG, bH) = e(abG, H)
    inf1 = np.concatenate([O.fq_mont(0), O.fq_mont(1), O.fq_mont(0)])
    inf2 = np.concatenate([O.fq_mont(0), O.fq_mont(0), O.fq_mont(1), O.fq_mont(0),
                           O.fq_mont(0), O.fq_mont(0)])
    one = np.zeros(48, np.uint64)
    one[0:4] = O.fq_mont(1)
    e = nk.reduced_pairing(ctx, np.stack([inf1, g1]), np.stack([g2, inf2]))
    assert np.array_equal(e[0], one) and np.array_equal(e[1], one)


@pytest.fixture(scope="module")
def golden(ctx):
    g = json.load(open(os.path.join(GOLDEN, "matmul4.json")))
    r1 = nk.generate(g["kind"], g["param"], g["density"], seed=g["seed"])
    pk = O.read_proving_key(os.path.join(GOLDEN, "matmul4.pk.bin"))
    vkp = O.read_verification_key(os.path.join(GOLDEN, "matmul4.vk.bin"))
    be = nk.Backend(ctx)
    be.prepare(r1, pk)
    raw = be.prove(r1.witness)
    vk = nk.VerifyingKey(ctx, vkp["alpha_g1_beta_g2"], vkp["gamma_g2"], vkp["delta_g2"], vkp["ic"])
    pub = np.ascontiguousarray(r1.witness[1:1 + r1.public_inputs])
    yield be, raw, vk, pub, r1
    vk.free()
    be.free()


def _proof_array(proof):
    return np.frombuffer(bytes(proof), np.uint64).copy()


def _ref_verdict(ref, tmp_path, pub, pr, name):
    path = tmp_path / f"{name}.proof.bin"
    O.write_proof(path, pr[0:12], pr[12:36], pr[36:48])
    return ref.verify(os.path.join(GOLDEN, "matmul4.vk.bin"), pub, path)


def test_verify_matches_reference_verdicts(golden, ref, orc, tmp_path):
    be, raw, vk, pub, r1 = golden
    r, s = O.random_fr(2, np.random.default_rng(43))
    good = _proof_array(be.blind(raw, r, s))
    a, b, c = good[0:12], good[12:36], good[36:48]
    g1 = ref.mul_gen(1, O.fr_mont(1))
    c_moved = np.concatenate([orc.add_affine(1, c[:8], g1[:8]), O.fq_mont(1)])
    inf1 = np.concatenate([O.fq_mont(0), O.fq_mont(1), O.fq_mont(0)])
    cases = {
        "valid": good,
        "c_moved": np.concatenate([a, b, c_moved]),
        "a_c_swapped": np.concatenate([c, b, a]),
        "a_at_infinity": np.concatenate([inf1, b, c]),
        "c_at_infinity": np.concatenate([a, b, inf1]),
    }
    pub_bad = pub.copy()
    pub_bad[0] = O.fr_mont(O.fr_int(pub[0]) + 1)
    names = list(cases)
    proofs = np.stack([cases[n] for n in names] + [good])
    publics = np.stack([pub] * len(names) + [pub_bad])
    got = vk.verify_batch(publics, proofs)
    want = [_ref_verdict(ref, tmp_path, pub, cases[n], n) for n in names]
    want.append(_ref_verdict(ref, tmp_path, pub_bad, good, "public_changed"))
    assert list(got) == want
    assert want[0] and not any(want[1:])


def test_verify_batch_of_many_proofs(golden, orc):
    """512 proofs (one raw proof blinded with 512 r, s pairs); every fourth one has
    C replaced by 2C.  All untouched proofs verify, all tampered ones do not."""
    be, raw, vk, pub, r1 = golden
    rng = np.random.default_rng(44)
    n = 512
    rs = O.random_fr(2 * n, rng).reshape(n, 2, 4)
    proofs = np.stack([_proof_array(be.blind(raw, r, s)) for r, s in rs])
    bad = np.arange(n) % 4 == 3
    for i in np.nonzero(bad)[0]:
        c = proofs[i, 36:48]
        proofs[i, 36:48] = np.concatenate([orc.add_affine(1, c[:8], c[:8]), O.fq_mont(1)])
    got = vk.verify_batch(np.stack([pub] * n), proofs)
    assert np.array_equal(got, ~bad)


def test_verify_public_input_count_mismatch_rejects(golden):
    be, raw, vk, pub, r1 = golden
    r, s = O.random_fr(2, np.random.default_rng(45))
    good = _proof_array(be.blind(raw, r, s))
    got = vk.verify_batch(np.stack([np.concatenate([pub, pub[:1]])] * 2), np.stack([good, good]))
    assert not got.any()
    assert vk.verify_batch(np.zeros((0, 4 * len(pub)), np.uint64), np.zeros((0, 48), np.uint64)).size == 0


def test_gpu_setup_key_verifies_its_proofs(ctx, ref):
    """Setup, prove, blind and verify all on the device: the setup's e(alpha, beta)
    equals libff's, and its key accepts the blinded proofs of its circuit."""
    r1 = nk.generate("poseidon", 3, 2, seed=8)
    pk, vkp = nk.setup(ctx, r1, O.random_fr(5, np.random.default_rng(46)))
    assert np.array_equal(vkp["alpha_g1_beta_g2"], ref.reduced_pairing(vkp["alpha_g1"], vkp["beta_g2"]))
    be = nk.Backend(ctx)
    be.prepare(r1, pk)
    raw = be.prove(r1.witness)
    rs = O.random_fr(8, np.random.default_rng(47)).reshape(4, 2, 4)
    proofs = np.stack([_proof_array(be.blind(raw, r, s)) for r, s in rs])
    vk = nk.VerifyingKey(ctx, vkp["alpha_g1_beta_g2"], vkp["gamma_g2"], vkp["delta_g2"], vkp["ic"])
    pub = np.ascontiguousarray(r1.witness[1:1 + r1.public_inputs])
    assert vk.verify_batch(np.stack([pub] * 4), proofs).all()
    vk.free()
    be.free()
