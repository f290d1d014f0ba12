"""Regenerates the golden fixtures in tests/golden/ from the reference itself.

Run in a checkout where the reference source tree is present and
oracle/_ref/libnkr_ref.so has been built from it (`make -C oracle ref`):

    python tests/golden/make_golden.py <reference source tree>   (or NKR_REFERENCE_SRC)

Everything here is computed by the reference's own code (libff, libfqfft, the
groth16 CPU backend and setup, its Poseidon helper) through oracle/_ref, except
the input draws, which come from seeded numpy generators so the tests can
rebuild the same inputs.  Outputs:
  poseidon_constants.json  round constants + MDS parsed from the reference's
                           crypto/poseidon_constants.inc, and the known-answer
                           hash2(1, 2) of protocols/groth16/tests/poseidon_test.cpp:21-24
  domain_ops.json          sha256 of libfqfft FFT / iFFT / cosetFFT / icosetFFT /
                           divide_by_Z_on_coset outputs at n = 2^10 (seed 101)
  msm.json                 libff BDLO12 results for G1 (n = 200) and G2 (n = 64)
  matmul4.*                a matmul-4 circuit (generator seed 11), the reference
                           CPU setup's proving / verification keys, and the raw
                           proof of the reference CPU prover
"""
import json
import os
import re
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
sys.path.insert(0, os.path.join(ROOT, "nkr-zkp_b200"))
import oracle as O  # noqa: E402

GOLD = os.path.dirname(os.path.abspath(__file__))
REF_SRC = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("NKR_REFERENCE_SRC")
if not REF_SRC:
    sys.exit("usage: make_golden.py <reference source tree> (or set NKR_REFERENCE_SRC)")


def hexs(a):
    return np.ascontiguousarray(a, np.uint64).tobytes().hex()


def msm_inputs(group, n, seed):
    """bases k_i * G (Jacobian, Z = 1), scalars with edge cases mixed in"""
    rng = np.random.default_rng(seed)
    ks = O.random_fr(n, rng)
    sc = O.random_fr(n, rng)
    one = O.fr_mont(1)
    sc[0] = 0                 # zero scalar
    sc[1] = one               # one
    sc[2] = O.fr_mont(O.R - 1)  # r - 1
    sc[3] = sc[4]             # equal scalars ...
    ks[3] = ks[4]             # ... on equal bases (forces doubling in a bucket)
    sc[5] = O.fr_mont(2**16 - 1)
    return ks, sc


def main():
    ref = O.Ref()
    # Poseidon constants and known answer
    txt = open(os.path.join(REF_SRC, "common/include/crypto/poseidon_constants.inc")).read()
    rcs = re.findall(r"POSEIDON_RC\((0x[0-9a-f]+)\)", txt)
    mds = re.findall(r"0x[0-9a-f]{60,}", txt.split("POSEIDON_MDS_ROW", 1)[1])
    kat = O.fr_int(ref.poseidon_hash2(O.fr_mont(1), O.fr_mont(2)))
    assert kat == 7853200120776062878684798364095072458815029376092732009249414926327459813530
    json.dump({"round_constants": rcs, "mds": mds, "hash2_1_2": str(kat)},
              open(os.path.join(GOLD, "poseidon_constants.json"), "w"), indent=1)

    # libfqfft domain ops
    rng = np.random.default_rng(101)
    x = O.random_fr(1024, rng)
    dom = {"n": 1024, "seed": 101, "input_sha256": O.sha256_arr(x), "ops": {}}
    for op in range(5):
        dom["ops"][str(op)] = O.sha256_arr(ref.domain_op(op, x))
    json.dump(dom, open(os.path.join(GOLD, "domain_ops.json"), "w"), indent=1)

    # BDLO12 multi-exponentiation
    out = {}
    for group, n, seed in ((1, 200, 202), (2, 64, 203)):
        ks, sc = msm_inputs(group, n, seed)
        bases = np.stack([ref.mul_gen(group, k) for k in ks])
        bases[6] = 0                       # an infinity base: (0, 1, 0) in libff layout
        bases[6, 4 * group:4 * group + 4] = O.fq_mont(1)
        res = ref.multiexp(group, bases, sc)
        out[f"g{group}"] = {"n": n, "seed": seed, "bases_sha256": O.sha256_arr(bases),
                            "result_affine": hexs(res[:8 * group])}
    json.dump(out, open(os.path.join(GOLD, "msm.json"), "w"), indent=1)

    # matmul-4: circuit, reference setup, reference raw proof
    import nkr_b200 as nk
    r1 = nk.generate("matmul", 4, 0, seed=11)
    pk_path = os.path.join(GOLD, "matmul4.pk.bin")
    vk_path = os.path.join(GOLD, "matmul4.vk.bin")
    ref.cpu_setup(r1, pk_path, vk_path)
    g1, g2 = ref.cpu_prove(r1, pk_path, r1.witness)
    json.dump({"kind": "matmul", "param": 4, "density": 0, "seed": 11,
               "circuit_sha256": O.sha256_arr(np.concatenate(
                   [np.concatenate([r1.row_ptr[k].view(np.uint8), r1.col_idx[k].view(np.uint8),
                                    r1.values[k].view(np.uint8).reshape(-1)]) for k in range(3)])),
               "witness_sha256": O.sha256_arr(r1.witness),
               "raw_g1_affine": [hexs(g1[i]) for i in range(4)],
               "raw_g2_affine": hexs(g2)},
              open(os.path.join(GOLD, "matmul4.json"), "w"), indent=1)
    print("golden fixtures written to", GOLD)


if __name__ == "__main__":
    main()
