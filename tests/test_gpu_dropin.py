"""The drop-in: the reference's own Groth16 code (validate, Backend::prepare /
prove, blind_proof, verify; protocols/groth16/app/prove.cpp:70-88) driving the
B200 backend through nkr::groth16::Backend via the adapter in
nkr-zkp_b200/integration/b200_backend.cpp.  The raw proof must equal the
reference CPU backend's (libff equality) and the blinded proof must verify."""
import numpy as np
import pytest

import nkr_b200 as nk
import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def dropin():
    if not O.dropin_available():
        pytest.skip("oracle/_ref/libnkr_ref_b200.so (reference + adapter) is not built here")
    return O.RefDropIn()


@pytest.mark.parametrize("kind,param,dens", [("matmul", 5, 0), ("poseidon", 3, 2), ("sql-aggregate", 2, 1)])
def test_reference_drives_b200_with_cpu_setup_keys(ctx, ref, dropin, tmp_path, kind, param, dens):
    r1 = nk.generate(kind, param, dens, seed=41)
    pk, vk = tmp_path / "k.pk.bin", tmp_path / "k.vk.bin"
    ref.cpu_setup(r1, pk, vk)
    verified, raw_equal, name = dropin.prove_verify(r1, pk, vk, r1.witness)
    assert name == "b200"
    assert raw_equal, "B200 raw proof differs from the reference CPU backend's"
    assert verified, "reference verifier rejected the B200 proof"


def test_reference_drives_b200_setup_and_prove(ctx, dropin, tmp_path):
    r1 = nk.generate("poseidon", 2, 1, seed=43)
    verified, raw_equal, _ = dropin.prove_verify(r1, "", "", r1.witness, gpu_setup=True)
    assert raw_equal and verified
