"""Proving-key artifacts (BinaryArchive "LKZ1" v1, protocols/groth16/common/src/
io.cpp:54-61) read and written by this library without the reference reader's
1 GiB per-vector limit.  CPU tests pin the writer byte for byte against a file
the reference's own io.cpp wrote (tests/golden/matmul4.pk.bin) and check the
reader's structure checks; the GPU test proves from files."""
import ctypes
import json
import os

import numpy as np
import pytest

import nkr_b200 as nk
import oracle as O
from conftest import GOLDEN

REF_PK = os.path.join(GOLDEN, "matmul4.pk.bin")


def test_file_info_of_a_reference_written_key():
    assert nk.pk_file_info(REF_PK) == (128, 128)


def test_writer_reproduces_the_reference_file(tmp_path):
    pk = O.read_proving_key(REF_PK)
    out = tmp_path / "k.pk.bin"
    nk.write_proving_key(out, pk, rows=128, cols=128)
    assert out.read_bytes() == open(REF_PK, "rb").read()


@pytest.mark.parametrize("cut", [3, 8, 100, 128 * 96 + 16, -1])
def test_truncated_files_are_rejected(tmp_path, cut):
    data = open(REF_PK, "rb").read()
    p = tmp_path / "t.pk.bin"
    p.write_bytes(data[:cut] if cut > 0 else data[:len(data) - 10])
    with pytest.raises(nk.B200Error, match="truncated|magic"):
        nk.pk_file_info(p)


def test_bad_magic_version_and_lengths_are_rejected(tmp_path):
    data = bytearray(open(REF_PK, "rb").read())
    bad = tmp_path / "b.pk.bin"
    bad.write_bytes(b"XKZ1" + bytes(data[4:]))
    with pytest.raises(nk.B200Error, match="magic"):
        nk.pk_file_info(bad)
    bad.write_bytes(bytes(data[:4]) + (2).to_bytes(4, "little") + bytes(data[8:]))
    with pytest.raises(nk.B200Error, match="version"):
        nk.pk_file_info(bad)
    wrong = bytearray(data)
    wrong[8:16] = (128 * 96 + 5).to_bytes(8, "little")   # not a whole number of points
    bad.write_bytes(bytes(wrong))
    with pytest.raises(nk.B200Error, match="whole number"):
        nk.pk_file_info(bad)


def test_prepare_file_checks_the_file_before_any_device_work(tmp_path):
    """A key that does not fit the circuit is refused before the context is used."""
    g = json.load(open(os.path.join(GOLDEN, "matmul4.json")))
    r1 = nk.generate(g["kind"], g["param"], g["density"], seed=g["seed"])
    small = nk.generate("matmul", 2, 0, seed=1)
    h = ctypes.c_void_p()
    c = small.c_circuit()
    rc = nk.lib().nkr_b200_prepare_file(None, ctypes.byref(c), REF_PK.encode(), ctypes.byref(h))
    assert rc == nk.EINVAL and b"needs" in nk.lib().nkr_b200_last_error()
    assert r1.rows == 128


@pytest.mark.gpu
def test_prove_from_files_equals_prove_from_memory(ctx, tmp_path):
    # the reference CPU setup's key, as the reference wrote it
    g = json.load(open(os.path.join(GOLDEN, "matmul4.json")))
    r1 = nk.generate(g["kind"], g["param"], g["density"], seed=g["seed"])
    be = nk.Backend(ctx)
    be.prepare_file(r1, REF_PK)
    g1, g2 = nk.raw_to_arrays(be.prove(r1.witness))
    assert [x[:8].tobytes().hex() for x in g1] == g["raw_g1_affine"]
    assert g2[:16].tobytes().hex() == g["raw_g2_affine"]
    be.free()
    # a GPU-setup key written by this library
    r2 = nk.generate("poseidon", 8, 2, seed=4)
    pk, _ = nk.setup(ctx, r2, O.random_fr(5, np.random.default_rng(8)))
    path = tmp_path / "p.pk.bin"
    nk.write_proving_key(path, pk, r2.rows, r2.cols)
    a, b = nk.Backend(ctx), nk.Backend(ctx)
    a.prepare(r2, pk)
    b.prepare_file(r2, path)
    assert bytes(a.prove(r2.witness)) == bytes(b.prove(r2.witness))
    a.free()
    b.free()
