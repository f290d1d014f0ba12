"""Writes tests/golden/prove_poseidon2048.json: digests of a full 2^20-constraint
Groth16 prove computed by the reference's own CPU code, for the GPU test
tests/test_gpu_prove_2_20.py to compare against byte for byte.

Run where oracle/_ref/libnkr_ref.so has been built from the reference sources
(`make -C oracle ref`); takes a few minutes on 8 cores:

    python tests/golden/make_golden_prove_2_20.py

Inputs, all seeded so the GPU side can rebuild them without the reference:
  circuit   generate("poseidon", 2048, density=2 (sparse), seed=1), built here by
            the reference's own Poseidon gadget and R1CSManager from the seeded
            preimages (899,072 constraints padded to 2^20 rows and columns);
  key       toxic waste (t, alpha, beta, gamma, delta) = 5 uniform Fr from
            numpy default_rng(TOXIC_SEED); the query scalars come from the
            oracle's restatement of the CPU setup (backend.cpp:41-107) and the
            points k G from the oracle's fixed-base multiplication, written as a
            reference proving-key artifact;
  r, s      2 uniform Fr from default_rng(RS_SEED).
Computed by the reference (oracle/_ref):
  az, bz, cz, H   the CPU backend's SpMV and quotient chain (backend.cpp:163-179);
  raw proof       CpuBackend::prove on the key file (backend.cpp:156-201):
                  ar, bs1, zk, qz (G1) and bs2 (G2), affine-normalised;
  verdict         the reference verifier (protocol.cpp:96-108) on the blinded proof.
Computed by the oracle: the blinded proof with the given r, s (protocol.cpp:85-94;
the reference draws r, s itself, so blind_proof is restated with given values).
Every digest is sha256 over the little-endian u64 limbs (Montgomery form), points
as affine X || Y (infinity = (0, 1)).
"""
import json
import os
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import oracle as O  # noqa: E402

GOLD = os.path.dirname(os.path.abspath(__file__))
COUNT, DENSITY, SEED = 2048, 2, 1
TOXIC_SEED, RS_SEED = 2020, 2021


def main():
    t0 = time.time()
    ref, orc = O.Ref(), O.Oracle()
    c = ref.poseidon_circuit_seeded(COUNT, DENSITY, SEED)
    assert c.rows == 1 << 20 and c.cols == 1 << 20
    print(f"circuit {time.time() - t0:.1f}s", flush=True)

    toxic = list(O.random_fr(5, np.random.default_rng(TOXIC_SEED)))
    at, bt, lt, ic, ht = orc.setup_scalars(c, toxic)
    g1, g2 = orc.g1_generator(), orc.g2_generator()
    key = {
        "a_query": orc.fixed_base(1, g1, at),
        "b_g1_query": orc.fixed_base(1, g1, bt),
        "b_g2_query": orc.fixed_base(2, g2, bt),
        "l_query": orc.fixed_base(1, g1, lt),
        "h_query": orc.fixed_base(1, g1, ht),
        "alpha_g1": orc.mul_affine(1, g1, toxic[1]),
        "beta_g1": orc.mul_affine(1, g1, toxic[2]),
        "delta_g1": orc.mul_affine(1, g1, toxic[4]),
        "beta_g2": orc.mul_affine(2, g2, toxic[2]),
        "delta_g2": orc.mul_affine(2, g2, toxic[4]),
    }
    ic_pts = orc.fixed_base(1, g1, ic)
    gamma_g2 = orc.mul_affine(2, g2, toxic[3])
    print(f"key {time.time() - t0:.1f}s", flush=True)

    d = tempfile.mkdtemp()
    pk_path, vk_path, proof_path = (os.path.join(d, n) for n in ("pk", "vk", "proof"))
    O.write_proving_key(pk_path, {k: O.affine_to_jac(2 if "g2" in k else 1, v).reshape(
        (-1,) if v.ndim == 1 else (v.shape[0], -1)) for k, v in key.items()})
    ref.write_vk({"alpha_g1": O.affine_to_jac(1, key["alpha_g1"])[0],
                  "beta_g2": O.affine_to_jac(2, key["beta_g2"])[0],
                  "gamma_g2": O.affine_to_jac(2, gamma_g2)[0],
                  "delta_g2": O.affine_to_jac(2, key["delta_g2"])[0],
                  "ic": O.affine_to_jac(1, ic_pts)}, vk_path)

    az, bz, cz, h = ref.quotient_vectors(c, c.witness)
    print(f"quotient {time.time() - t0:.1f}s", flush=True)
    raw_g1, raw_g2 = ref.cpu_prove(c, pk_path, c.witness)
    print(f"reference prove {time.time() - t0:.1f}s", flush=True)

    r, s = O.random_fr(2, np.random.default_rng(RS_SEED))
    a, b, cc = orc.blind(key, raw_g1.reshape(-1), raw_g2, r, s)
    O.write_proof(proof_path, O.affine_to_jac(1, a)[0], O.affine_to_jac(2, b)[0],
                  O.affine_to_jac(1, cc)[0])
    ok = ref.verify(vk_path, c.witness[1:1 + c.public_inputs], proof_path)
    assert ok, "the reference verifier rejected the golden proof"

    sha = O.sha256_arr
    out = {
        "circuit": {"kind": "poseidon", "count": COUNT, "density": DENSITY, "seed": SEED,
                    "rows": c.rows, "cols": c.cols, "public_inputs": c.public_inputs,
                    "witness": sha(c.witness)},
        "toxic_seed": TOXIC_SEED, "rs_seed": RS_SEED,
        "key": {k: sha(v) for k, v in key.items()},
        "vectors": {"az": sha(az), "bz": sha(bz), "cz": sha(cz), "h": sha(h)},
        "raw": {"ar": sha(raw_g1[0]), "bs1": sha(raw_g1[1]), "zk": sha(raw_g1[2]),
                "qz": sha(raw_g1[3]), "bs2": sha(raw_g2)},
        "raw_hex": {"ar": raw_g1[0].tobytes().hex(), "bs1": raw_g1[1].tobytes().hex(),
                    "zk": raw_g1[2].tobytes().hex(), "qz": raw_g1[3].tobytes().hex(),
                    "bs2": raw_g2.tobytes().hex()},
        "proof": {"a": sha(a), "b": sha(b), "c": sha(cc)},
        "reference_verifier_accepts": ok,
    }
    with open(os.path.join(GOLD, "prove_poseidon2048.json"), "w") as f:
        json.dump(out, f, indent=1)
    print(f"done {time.time() - t0:.1f}s", flush=True)


if __name__ == "__main__":
    main()
