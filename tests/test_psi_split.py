"""The split of G2 class values used by the witness MSMs' class path (msm.cu,
k_cls_split_psi / k_cls_psi): the twist Frobenius psi(x, y) = (conj(x) gx1,
conj(y) gy1) acts on G2 as multiplication by lambda = p mod r = 6 u^2, so
v Q = k0 Q + k1 psi(Q) with k0 = v mod lambda, k1 = v div lambda.  Checked on the
CPU against the oracle's G2 scalar multiplication, with lambda and the Frobenius
constants read from the CUDA sources."""
import os
import re

import numpy as np

import oracle as O

CSRC = os.path.join(os.path.dirname(__file__), "..", "nkr-zkp_b200", "csrc")
U = 4965661367192848881  # the BN254 curve parameter


def _src(name):
    return open(os.path.join(CSRC, name)).read()


def _lambda_from_source():
    s = _src("msm.cu")
    lo = int(re.search(r"kPsiLambdaLo = (0x[0-9a-f]+)ull", s).group(1), 16)
    hi = int(re.search(r"kPsiLambdaHi = (0x[0-9a-f]+)ull", s).group(1), 16)
    return hi << 64 | lo


def _fq2_const(fn):
    """an Fq2 constant of pairing.cuh (Montgomery limbs, low word first) as integers"""
    s = _src("pairing.cuh")
    body = s[s.index(f"Fq2 {fn}()"):]
    body = body[:body.index("}\n")]
    words = [int(w, 16) for w in re.findall(r"0x([0-9a-f]+)ull", body)]
    rinv = pow(2, -256, O.P)
    c0 = sum(w << (64 * i) for i, w in enumerate(words[:4])) * rinv % O.P
    c1 = sum(w << (64 * i) for i, w in enumerate(words[4:8])) * rinv % O.P
    return c0, c1


def _m2(a, b):
    p = O.P
    return ((a[0] * b[0] - a[1] * b[1]) % p, (a[0] * b[1] + a[1] * b[0]) % p)


def _fq2_of(limbs, off):
    return O.fq_int(limbs[off:off + 4]), O.fq_int(limbs[off + 4:off + 8])


def test_lambda_is_the_frobenius_eigenvalue():
    lam = _lambda_from_source()
    assert lam == 6 * U * U == O.P - O.R
    assert lam.bit_length() == 127
    # every value below r splits into two halves below 2^128 (the 13 windows of
    # 10 bits of the G2 class MSM cover 130 bits with no carry out)
    assert (O.R - 1) // lam < 2**128


def test_psi_split_matches_oracle_scalar_multiplication():
    lam = _lambda_from_source()
    gx1, gy1 = _fq2_const("frob_gx1"), _fq2_const("frob_gy1")
    orc = O.Oracle()
    rng = np.random.default_rng(4)
    g2 = np.asarray(orc.g2_generator()).reshape(-1)
    for t in range(3):
        q = np.asarray(orc.mul_affine(2, g2, O.random_fr(1, rng)[0])).reshape(-1)
        x, y = _fq2_of(q, 0), _fq2_of(q, 8)
        conj = lambda a: (a[0], (-a[1]) % O.P)  # noqa: E731
        psi = np.concatenate([O.fq_mont(v) for v in (*_m2(conj(x), gx1), *_m2(conj(y), gy1))])
        # psi(Q) = lambda Q
        lq = np.asarray(orc.mul_affine(2, q, O.fr_mont(lam))).reshape(-1)
        assert np.array_equal(psi, lq[:16])
        for v in (O.R - 1, lam, lam - 1, int(rng.integers(1, 2**62)) * 2**190 + 12345):
            k1, k0 = divmod(v, lam)
            assert k0 < lam and k1 < 2**128
            want = np.asarray(orc.mul_affine(2, q, O.fr_mont(v))).reshape(-1)
            a = np.asarray(orc.mul_affine(2, q, O.fr_mont(k0))).reshape(-1)
            b = np.asarray(orc.mul_affine(2, psi, O.fr_mont(k1))).reshape(-1)
            got = np.asarray(orc.add_affine(2, a, b)).reshape(-1)
            assert np.array_equal(got[:16], want[:16])
