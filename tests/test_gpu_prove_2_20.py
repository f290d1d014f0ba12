"""The headline prove (poseidon count 2048, sparse, seed 1: 2^20 constraints and
columns) byte for byte against the reference's own CPU code.

tests/golden/prove_poseidon2048.json (written by make_golden_prove_2_20.py from
oracle/_ref) holds sha256 digests of the reference CPU backend's az, bz, cz and H
(backends/cpu/src/backend.cpp:163-179), of its five MSM results ar, bs1, zk, qz,
bs2 (backend.cpp:181-200) proved with a key from seeded toxic waste, and of the
proof blinded with seeded r, s (protocol.cpp:85-94), which the reference verifier
accepted.  Here the same circuit is generated, the key comes from the GPU setup
with the same toxic waste, and the GPU prove and blinding must reproduce every
digest."""
import json
import os

import numpy as np
import pytest

import nkr_b200 as nk
import oracle as O
from conftest import GOLDEN

pytestmark = pytest.mark.gpu


def _gold():
    return json.load(open(os.path.join(GOLDEN, "prove_poseidon2048.json")))


def _affine_bytes(jac, group):
    """X || Y of libff-layout points that are affine-normalised (Z = 1, or the
    (0, 1, 0) encoding of infinity)."""
    a = np.ascontiguousarray(jac, np.uint64).reshape(-1, 12 * group)[:, :8 * group]
    return np.ascontiguousarray(a)


def test_prove_2_20_bit_exact_against_reference_cpu_backend(ctx):
    g = _gold()
    c = g["circuit"]
    r1 = nk.generate(c["kind"], c["count"], c["density"], seed=c["seed"])
    assert (r1.rows, r1.cols, r1.public_inputs) == (c["rows"], c["cols"], c["public_inputs"])
    assert O.sha256_arr(r1.witness) == c["witness"]

    toxic = list(O.random_fr(5, np.random.default_rng(g["toxic_seed"])))
    pk, _vk = nk.setup(ctx, r1, toxic)
    for name, want in g["key"].items():
        group = 2 if "g2" in name else 1
        assert O.sha256_arr(_affine_bytes(pk[name], group)) == want, name

    be = nk.Backend(ctx)
    be.prepare(r1, pk)
    del pk
    raw = be.prove(r1.witness)
    az, bz, cz, h = be.intermediates()
    for name, v in (("az", az), ("bz", bz), ("cz", cz), ("h", h)):
        assert O.sha256_arr(v) == g["vectors"][name], name

    g1, g2 = nk.raw_to_arrays(raw)
    for name, p in zip(("ar", "bs1", "zk", "qz"), g1):
        assert O.sha256_arr(p[:8]) == g["raw"][name], name
        assert p[:8].tobytes().hex() == g["raw_hex"][name], name
    assert O.sha256_arr(g2[:16]) == g["raw"]["bs2"]

    r, s = O.random_fr(2, np.random.default_rng(g["rs_seed"]))
    proof = be.blind(raw, r, s)
    assert O.sha256_arr(_affine_bytes(np.frombuffer(bytes(proof.a), np.uint64), 1)) == g["proof"]["a"]
    assert O.sha256_arr(_affine_bytes(np.frombuffer(bytes(proof.b), np.uint64), 2)) == g["proof"]["b"]
    assert O.sha256_arr(_affine_bytes(np.frombuffer(bytes(proof.c), np.uint64), 1)) == g["proof"]["c"]
    be.free()
