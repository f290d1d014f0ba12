"""The reference-shaped operator API (include/nkr_b200_operators.hpp: NTTContext,
BucketContext and MSMContext of operators/cuda/include over the C ABI).

tests/operator_api_driver.cpp uses the header the way the reference's CUDA
backend uses its contexts in a prove (backends/cuda/src/groth16_backend.cu:
242-279); it is compiled here with g++ against libnkr_b200.so.  On the CPU the
test checks that the header compiles and links; on the GPU the driver's quotient
H and its G1, G2 and quotient MSM results must equal the oracle's."""
import os
import subprocess

import numpy as np
import pytest

import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "nkr-zkp_b200")
CUDA = os.environ.get("CUDA_HOME", "/usr/local/cuda")


def _build(tmp_path):
    exe = str(tmp_path / "operator_api_driver")
    cmd = ["g++", "-std=c++17", "-O1", "-Wall", "-I", os.path.join(ROOT, "include"),
           "-I", os.path.join(CUDA, "include"), os.path.join(ROOT, "tests", "operator_api_driver.cpp"),
           "-o", exe, "-L", PKG, "-lnkr_b200", "-L", os.path.join(CUDA, "lib64"), "-lcudart",
           f"-Wl,-rpath,{PKG}", f"-Wl,-rpath,{os.path.join(CUDA, 'lib64')}"]
    p = subprocess.run(cmd, capture_output=True, text=True)
    assert p.returncode == 0, p.stdout + p.stderr
    return exe


def test_operator_header_compiles_and_links(tmp_path):
    _build(tmp_path)


def _bases(orc, group, ks):
    gen = orc.g1_generator() if group == 1 else orc.g2_generator()
    aff = orc.fixed_base(group, gen, ks)
    return aff, O.affine_to_jac(group, aff)


@pytest.mark.gpu
def test_operator_api_prove_sequence_matches_oracle(tmp_path, orc):
    exe = _build(tmp_path)
    rng = np.random.default_rng(404)
    logn, cols = 12, 3000
    rows = 1 << logn
    a, b, c = (O.random_fr(rows, rng) for _ in range(3))
    z = O.random_fr(cols, rng)
    z[:100] = 0
    z[100:200] = O.fr_mont(1)
    ks1, ks2, ksh = O.random_fr(cols, rng), O.random_fr(cols, rng), O.random_fr(rows, rng)
    ks1[5:9] = 0          # bases at infinity
    ks1[20] = ks1[21]     # a repeated base
    g1_aff, g1_jac = _bases(orc, 1, ks1)
    g2_aff, g2_jac = _bases(orc, 2, ks2)
    hb_aff, hb_jac = _bases(orc, 1, ksh)
    root = O.fr_int(orc.fr_constant(2))  # the 2^28-th root of unity libfqfft uses
    omega = O.fr_mont(pow(root, 1 << (28 - logn), O.R))
    d = str(tmp_path)
    files = {"shape": np.array([rows, cols], np.uint64), "omega": omega, "coset": orc.fr_constant(1),
             "a": a, "b": b, "c": c, "z": z, "g1": g1_jac, "g2": g2_jac, "hb": hb_jac}
    for name, arr in files.items():
        np.ascontiguousarray(arr, np.uint64).tofile(os.path.join(d, name + ".bin"))
    p = subprocess.run([exe, d], capture_output=True, text=True, timeout=600)
    assert p.returncode == 0, p.stdout + p.stderr

    def read(name, width):
        return np.fromfile(os.path.join(d, name + ".bin"), np.uint64).reshape(-1, width)

    h_want = orc.quotient(a, b, c)
    assert np.array_equal(read("h", 4), h_want)
    assert np.array_equal(read("msm_g1", 12)[0, :8], orc.msm(1, g1_aff, z))
    assert np.array_equal(read("msm_g2", 24)[0, :16], orc.msm(2, g2_aff, z))
    assert np.array_equal(read("msm_h", 12)[0, :8], orc.msm(1, hb_aff, h_want))
