"""End-to-end Groth16 prove on the B200 through the C ABI, bit-exact against
the reference CPU backend (golden raw proof from its own prover, and live via
oracle/_ref when built) and the oracle: SpMV vectors, H, each MSM result and the
blinded proof with seeded r, s; the reference verifier accepts the proof."""
import json
import os

import numpy as np
import pytest

import nkr_b200 as nk
import oracle as O
from conftest import GOLDEN

pytestmark = pytest.mark.gpu


def _golden_matmul4():
    g = json.load(open(os.path.join(GOLDEN, "matmul4.json")))
    r1 = nk.generate(g["kind"], g["param"], g["density"], seed=g["seed"])
    pk = O.read_proving_key(os.path.join(GOLDEN, "matmul4.pk.bin"))
    return g, r1, pk


def _raw_affine(raw):
    g1, g2 = nk.raw_to_arrays(raw)
    return np.stack([x[:8] for x in g1]), g2[:16]


def test_prove_matches_reference_golden(ctx):
    g, r1, pk = _golden_matmul4()
    be = nk.Backend(ctx)
    be.prepare(r1, pk)
    raw = be.prove(r1.witness)
    g1, g2 = _raw_affine(raw)
    assert [g1[i].tobytes().hex() for i in range(4)] == g["raw_g1_affine"]
    assert g2.tobytes().hex() == g["raw_g2_affine"]
    # the Z coordinate is libff's affine one
    assert np.array_equal(nk.raw_to_arrays(raw)[0][0][8:], O.fq_mont(1))
    be.free()


def test_intermediates_match_oracle(ctx, orc):
    g, r1, pk = _golden_matmul4()
    be = nk.Backend(ctx)
    be.prepare(r1, pk)
    be.prove(r1.witness)
    az, bz, cz, h = be.intermediates()
    for k, got in enumerate((az, bz, cz)):
        want = orc.spmv(r1.rows, r1.row_ptr[k], r1.col_idx[k], r1.values[k], r1.witness)
        assert np.array_equal(got, want)
    assert np.array_equal(h, orc.quotient(az, bz, cz))
    be.free()


def test_blind_matches_oracle_and_verifies(ctx, orc, ref, tmp_path):
    g, r1, pk = _golden_matmul4()
    be = nk.Backend(ctx)
    be.prepare(r1, pk)
    raw = be.prove(r1.witness)
    r, s = O.random_fr(2, np.random.default_rng(5))
    proof = be.blind(raw, r, s)
    pka = O.pk_affine(pk, orc)
    g1, g2 = _raw_affine(raw)
    a, b, c = orc.blind(pka, g1, g2, r, s)
    pa = np.frombuffer(bytes(proof.a), np.uint64)
    pb = np.frombuffer(bytes(proof.b), np.uint64)
    pc = np.frombuffer(bytes(proof.c), np.uint64)
    assert np.array_equal(pa, O.affine_to_jac(1, a)[0])
    assert np.array_equal(pb, O.affine_to_jac(2, b)[0])
    assert np.array_equal(pc, O.affine_to_jac(1, c)[0])
    path = tmp_path / "proof.bin"
    O.write_proof(path, pa, pb, pc)
    assert ref.verify(os.path.join(GOLDEN, "matmul4.vk.bin"), r1.witness[1:1 + r1.public_inputs], path)
    be.free()


@pytest.mark.parametrize("kind,param,dens", [("poseidon", 3, 2), ("sql-aggregate", 2, 1),
                                            ("matmul", 6, 1), ("fibonacci", 100, 0),
                                            ("matmul", 32, 0)])   # the matmul-32 config: 2^16, full density
def test_prove_matches_reference_live(ctx, ref, tmp_path, kind, param, dens):
    r1 = nk.generate(kind, param, dens, seed=31)
    pk_path, vk_path = tmp_path / "c.pk.bin", tmp_path / "c.vk.bin"
    ref.cpu_setup(r1, pk_path, vk_path)      # unnormalised Jacobian PK (hazard H2)
    pk = O.read_proving_key(pk_path)
    be = nk.Backend(ctx)
    be.prepare(r1, pk)
    raw = be.prove(r1.witness)
    g1, g2 = _raw_affine(raw)
    rg1, rg2 = ref.cpu_prove(r1, pk_path, r1.witness)
    assert np.array_equal(g1, rg1) and np.array_equal(g2, rg2)
    r, s = O.random_fr(2, np.random.default_rng(9))
    proof = be.blind(raw, r, s)
    path = tmp_path / "proof.bin"
    O.write_proof(path, np.frombuffer(bytes(proof.a), np.uint64),
                  np.frombuffer(bytes(proof.b), np.uint64), np.frombuffer(bytes(proof.c), np.uint64))
    assert ref.verify(vk_path, r1.witness[1:1 + r1.public_inputs], path)
    be.free()


def test_repeated_proves_and_batch_agree(ctx):
    g, r1, pk = _golden_matmul4()
    be = nk.Backend(ctx)
    be.prepare(r1, pk)
    first = bytes(be.prove(r1.witness))
    second = bytes(be.prove(r1.witness))
    assert first == second
    # a second witness for the same circuit (different A, B)
    r2 = nk.generate("matmul", 4, 0, seed=12)
    be2 = nk.Backend(ctx)
    be2.prepare(r2, pk)
    single2 = bytes(be2.prove(r2.witness))
    out = nk.prove_batch([be, be2, be], [r1.witness, r2.witness, r1.witness])
    assert bytes(out[0]) == first and bytes(out[1]) == single2 and bytes(out[2]) == first
    be.free()
    be2.free()


def test_batch_mix_equals_single_proves(ctx):
    """A batch of 18 proofs over 4 keys of different kinds and sizes (up to 6 proofs
    of one key, more than its 4 slots, with distinct witnesses) returns exactly the
    raw proof each witness gives alone through the plain path."""
    specs = [("poseidon", 4, 1, 6), ("sql-aggregate", 8, 2, 5), ("matmul", 5, 0, 3),
             ("poseidon", 16, 2, 4)]
    backends, wits = [], []
    for j, (kind, param, dens, nwit) in enumerate(specs):
        r1 = nk.generate(kind, param, dens, seed=100 + j)
        toxic = O.random_fr(5, np.random.default_rng(200 + j))
        pk, _ = nk.setup(ctx, r1, toxic)
        be = nk.Backend(ctx)
        be.prepare(r1, pk)
        backends.append(be)
        # poseidon / sql circuits do not depend on the seed, only their witnesses do
        ws = [nk.generate(kind, param, dens, seed=300 + 10 * j + i).witness for i in range(nwit)]
        wits.append(ws)
    single = [[bytes(be.prove(w)) for w in ws] for be, ws in zip(backends, wits)]
    order = []
    for i in range(max(len(w) for w in wits)):
        for j in range(len(specs)):
            if i < len(wits[j]):
                order.append((j, i))
    out = nk.prove_batch([backends[j] for j, _ in order], [wits[j][i] for j, i in order])
    for (j, i), raw in zip(order, out):
        assert bytes(raw) == single[j][i], f"key {j} witness {i}"
    # a second batch reuses the captured graphs and slots
    out2 = nk.prove_batch([backends[j] for j, _ in order], [wits[j][i] for j, i in order])
    assert [bytes(r) for r in out2] == [bytes(r) for r in out]
    # cross-proof launches (work lists over the proofs of a wave; 6 proofs of one
    # key over its 4 slots make two waves): the same raw proofs
    out3 = nk.prove_batch([backends[j] for j, _ in order], [wits[j][i] for j, i in order],
                          lists=True)
    for (j, i), raw in zip(order, out3):
        assert bytes(raw) == single[j][i], f"lists: key {j} witness {i}"
    # and in a different order, the first proofs of each key in the last wave
    rev = order[::-1]
    out4 = nk.prove_batch([backends[j] for j, _ in rev], [wits[j][i] for j, i in rev], lists=True)
    for (j, i), raw in zip(rev, out4):
        assert bytes(raw) == single[j][i], f"lists, reversed: key {j} witness {i}"
    for be in backends:
        be.free()


def test_prepare_rejects_bad_shapes(ctx):
    g, r1, pk = _golden_matmul4()
    be = nk.Backend(ctx)
    bad = nk.R1CS(r1.rows - 1, r1.cols, r1.public_inputs, [x[:-1] for x in r1.row_ptr], r1.col_idx,
                  r1.values, r1.witness)
    with pytest.raises(nk.B200Error):
        be.prepare(bad, pk)
    be.prepare(r1, pk)
    with pytest.raises(nk.B200Error):
        be.prove(r1.witness[:-1])
    be.free()


def test_prove_repeated_witness_values(ctx, ref, tmp_path):
    """Repeated witness values go through the class path of the G1 witness MSMs:
    variables of equal value form a class whose bases are summed once, and a small
    MSM over the class values adds v_c S_c.  A crafted witness with more
    minimum-size classes (4 members) than one prove takes (4,096; the others stay
    singletons), groups below the minimum, large classes (fix-up levels), values
    beside their negations and zeros gives the reference CPU prover's raw proof,
    before and after a prove of the circuit's own witness on the same slot."""
    r1 = nk.generate("matmul", 32, 0, seed=31)
    pk_path, vk_path = tmp_path / "c.pk.bin", tmp_path / "c.vk.bin"
    ref.cpu_setup(r1, pk_path, vk_path)
    pk = O.read_proving_key(pk_path)
    rng = np.random.default_rng(77)
    n = r1.cols
    w = O.random_fr(n, rng)
    w[0] = O.fr_mont(1)
    vals = O.random_fr(4400, rng)
    pos = rng.permutation(np.arange(1, n))
    k = 0

    def put(v, m):
        nonlocal k
        w[pos[k:k + m]] = v
        k += m

    for j in range(4200):
        put(vals[j], 4)
    for j in range(4200, 4300):
        put(vals[j], 3)
    for j in range(4300, 4310):
        put(vals[j], 500)
    for j in range(4310, 4320):
        put(vals[j], 8)
        put(O.int_to_limbs((O.R - O.limbs_to_int(vals[j])) % O.R), 8)
    w[pos[k:k + 2000]] = 0
    be = nk.Backend(ctx)
    be.prepare(r1, pk)
    raw = be.prove(w)
    g1, g2 = _raw_affine(raw)
    rg1, rg2 = ref.cpu_prove(r1, pk_path, w)
    assert np.array_equal(g1, rg1) and np.array_equal(g2, rg2)
    be.prove(r1.witness)
    assert bytes(be.prove(w)) == bytes(raw)
    be.free()
