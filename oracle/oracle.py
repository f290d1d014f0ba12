"""Python access to the CPU oracle (test infrastructure only).

Two checkers live here, both used only by tests/, __graft_entry__.smoke() and
the CPU-baseline leg of bench.py:
  * liboracle_bn254.so -- this repo's C restatement of the reference's CPU
    prove path (bn254_oracle.c), always available;
  * _ref/libnkr_ref.so -- the reference's own CPU path (libff, libfqfft, the
    groth16 CPU backend, its verifier) compiled from the reference sources by
    oracle/Makefile; available where it was built (it travels with the repo
    snapshot as a built file).
Plus readers/writers of the reference's BinaryArchive artifact format
(common/include/binary_archive.hpp:17-98; groth16 io.cpp:16-96).
All buffers are numpy uint64 arrays in libff's layout (Fr = 4 limbs Montgomery).
"""
import ctypes
import hashlib
import os
import struct
from types import SimpleNamespace

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORC_PATH = os.path.join(HERE, "liboracle_bn254.so")
REF_PATH = os.path.join(HERE, "_ref", "libnkr_ref.so")

R = 21888242871839275222246405745257275088548364400416034343698204186575808495617
P = 21888242871839275222246405745257275088696311157297823662689037894645226208583
_R_LIMBS = np.array([(R >> (64 * i)) & (2**64 - 1) for i in range(4)], dtype=np.uint64)
_VP = ctypes.c_void_p
_U64 = ctypes.c_uint64


def _p(a):
    return None if a is None else a.ctypes.data_as(_VP)


def _arr(a):
    return np.ascontiguousarray(a, dtype=np.uint64)


# ---------------------------------------------------------------------------
# numbers <-> limbs
# ---------------------------------------------------------------------------

def limbs_to_int(a):
    a = np.asarray(a, dtype=np.uint64).reshape(-1)
    return sum(int(a[i]) << (64 * i) for i in range(a.size))


def int_to_limbs(x, n=4):
    return np.array([(x >> (64 * i)) & (2**64 - 1) for i in range(n)], dtype=np.uint64)


def fr_mont(x):
    """canonical int -> Fr Montgomery limbs"""
    return int_to_limbs((x % R) * pow(2, 256, R) % R)


def fr_int(m):
    """Fr Montgomery limbs -> canonical int"""
    return limbs_to_int(m) * pow(2, -256, R) % R


def fq_mont(x):
    return int_to_limbs((x % P) * pow(2, 256, P) % P)


def fq_int(m):
    return limbs_to_int(m) * pow(2, -256, P) % P


def random_fr(n, rng):
    """n uniform Fr elements (4 x u64, taken as the Montgomery representation),
    drawn like libff random_element: 254-bit limbs, rejection of values >= r."""
    out = np.empty((n, 4), np.uint64)
    filled = 0
    while filled < n:
        k = n - filled
        cand = rng.integers(0, 2**64, size=(k, 4), dtype=np.uint64, endpoint=False)
        cand[:, 3] &= np.uint64((1 << 62) - 1)
        less = np.zeros(k, bool)
        equal = np.ones(k, bool)
        for i in range(3, -1, -1):  # lexicographic compare from the top limb
            less |= equal & (cand[:, i] < _R_LIMBS[i])
            equal &= cand[:, i] == _R_LIMBS[i]
        good = cand[less]
        out[filled:filled + good.shape[0]] = good
        filled += good.shape[0]
    return out


# ---------------------------------------------------------------------------
# the C restatement
# ---------------------------------------------------------------------------

class Oracle:
    def __init__(self):
        if not os.path.exists(ORC_PATH):
            raise FileNotFoundError(f"{ORC_PATH} missing; run `make -C oracle oracle`")
        self.lib = ctypes.CDLL(ORC_PATH)

    def fe(self, name, which, a, b=None):
        a = _arr(a)
        out = np.zeros(4, np.uint64)
        f = getattr(self.lib, "orc_fe_" + name)
        if b is None:
            f(ctypes.c_int(which), _p(a), _p(out))
        else:
            f(ctypes.c_int(which), _p(a), _p(_arr(b)), _p(out))
        return out

    def fr_constant(self, which):
        out = np.zeros(4, np.uint64)
        self.lib.orc_fr_constant(ctypes.c_int(which), _p(out))
        return out

    def domain_op(self, op, data):
        d = _arr(data).copy()
        rc = self.lib.orc_domain_op(ctypes.c_int(op), _p(d), _U64(d.size // 4))
        assert rc == 0
        return d.reshape(-1, 4)

    def spmv(self, rows, row_ptr, col_idx, values, z):
        y = np.zeros((rows, 4), np.uint64)
        rp = np.ascontiguousarray(row_ptr, np.uint32)
        ci = np.ascontiguousarray(col_idx, np.uint32)
        self.lib.orc_spmv(_U64(rows), _p(rp), _p(ci), _p(_arr(values)), _p(_arr(z)), _p(y))
        return y

    def g1_generator(self):
        out = np.zeros(8, np.uint64)
        self.lib.orc_g1_generator(_p(out))
        return out

    def g2_generator(self):
        out = np.zeros(16, np.uint64)
        self.lib.orc_g2_generator(_p(out))
        return out

    def mul_affine(self, group, point, k):
        out = np.zeros(8 * group, np.uint64)
        f = self.lib.orc_g1_mul_affine if group == 1 else self.lib.orc_g2_mul_affine
        f(_p(_arr(point)), _p(_arr(k)), _p(out))
        return out

    def add_affine(self, group, a, b):
        out = np.zeros(8 * group, np.uint64)
        f = self.lib.orc_g1_add_affine if group == 1 else self.lib.orc_g2_add_affine
        f(_p(_arr(a)), _p(_arr(b)), _p(out))
        return out

    def to_affine(self, group, jac):
        jac = _arr(jac).reshape(-1, 12 * group)
        out = np.zeros((jac.shape[0], 8 * group), np.uint64)
        f = self.lib.orc_g1_to_affine if group == 1 else self.lib.orc_g2_to_affine
        for i in range(jac.shape[0]):
            f(_p(jac[i]), _p(out[i]))
        return out

    def on_curve(self, group, aff):
        f = self.lib.orc_g1_on_curve if group == 1 else self.lib.orc_g2_on_curve
        return bool(f(_p(_arr(aff))))

    def msm(self, group, bases_aff, scalars, threads=0):
        out = np.zeros(8 * group, np.uint64)
        s = _arr(scalars)
        f = self.lib.orc_msm_g1 if group == 1 else self.lib.orc_msm_g2
        f(_p(_arr(bases_aff)), _p(s), _U64(s.size // 4), ctypes.c_int(threads), _p(out))
        return out

    def fixed_base(self, group, base_aff, scalars, threads=0):
        """k_i * P for every scalar k_i (Fr Montgomery), affine (8 / 16 u64 per point)."""
        s = _arr(scalars)
        n = s.size // 4
        out = np.zeros((n, 8 * group), np.uint64)
        self.lib.orc_fixed_base(ctypes.c_int(group), _p(_arr(base_aff)), _p(s), _U64(n),
                                ctypes.c_int(threads), _p(out))
        return out

    def quotient(self, az, bz, cz):
        n = _arr(az).size // 4
        a, b, c = _arr(az).copy(), _arr(bz).copy(), _arr(cz).copy()
        h = np.zeros((n, 4), np.uint64)
        assert self.lib.orc_quotient(_U64(n), _p(a), _p(b), _p(c), _p(h)) == 0
        return h

    def _circuit(self, r1cs):
        class C(ctypes.Structure):
            _fields_ = [("rows", _U64), ("cols", _U64), ("pub", _U64), ("rp", _VP * 3),
                        ("ci", _VP * 3), ("vals", _VP * 3)]
        c = C()
        c.rows, c.cols, c.pub = r1cs.rows, r1cs.cols, r1cs.public_inputs
        for k in range(3):
            c.rp[k] = r1cs.row_ptr[k].ctypes.data
            c.ci[k] = r1cs.col_idx[k].ctypes.data if r1cs.col_idx[k].size else None
            c.vals[k] = r1cs.values[k].ctypes.data if r1cs.values[k].size else None
        return c

    def _pk(self, pk_aff):
        class K(ctypes.Structure):
            _fields_ = [(n, _VP) for n in ("a", "b1", "b2", "l", "h", "alpha1", "beta1", "beta2",
                                           "delta1", "delta2")]
        keep = {k: _arr(v) for k, v in pk_aff.items()}
        k = K()
        for f, name in zip(("a", "b1", "b2", "l", "h", "alpha1", "beta1", "beta2", "delta1", "delta2"),
                           ("a_query", "b_g1_query", "b_g2_query", "l_query", "h_query",
                            "alpha_g1", "beta_g1", "beta_g2", "delta_g1", "delta_g2")):
            setattr(k, f, keep[name].ctypes.data)
        return k, keep

    def prove(self, r1cs, pk_aff, witness, threads=0):
        """pk_aff: dict of AFFINE arrays (8 / 16 u64 per point)."""
        c = self._circuit(r1cs)
        k, keep = self._pk(pk_aff)
        g1 = np.zeros((4, 8), np.uint64)
        g2 = np.zeros(16, np.uint64)
        assert self.lib.orc_prove(ctypes.byref(c), ctypes.byref(k), _p(_arr(witness)),
                                  ctypes.c_int(threads), _p(g1), _p(g2)) == 0
        return g1, g2

    def blind(self, pk_aff, raw_g1, raw_g2, r, s):
        k, keep = self._pk(pk_aff)
        a, b, c = np.zeros(8, np.uint64), np.zeros(16, np.uint64), np.zeros(8, np.uint64)
        self.lib.orc_blind(ctypes.byref(k), _p(_arr(raw_g1)), _p(_arr(raw_g2)), _p(_arr(r)),
                           _p(_arr(s)), _p(a), _p(b), _p(c))
        return a, b, c

    def setup_scalars(self, r1cs, toxic):
        c = self._circuit(r1cs)
        tox = _arr(np.stack(toxic))
        at, bt, lt = (np.zeros((r1cs.cols, 4), np.uint64) for _ in range(3))
        ic = np.zeros((r1cs.public_inputs + 1, 4), np.uint64)
        ht = np.zeros((r1cs.rows, 4), np.uint64)
        assert self.lib.orc_setup_scalars(ctypes.byref(c), _p(tox), _p(at), _p(bt), _p(lt), _p(ic),
                                          _p(ht)) == 0
        return at, bt, lt, ic, ht

    def poseidon_hash2(self, rc, mds, left, right):
        out = np.zeros(4, np.uint64)
        self.lib.orc_poseidon_hash2(_p(_arr(rc)), _p(_arr(mds)), _p(_arr(left)), _p(_arr(right)),
                                    _p(out))
        return out


# ---------------------------------------------------------------------------
# the reference's own CPU path (compiled from its sources)
# ---------------------------------------------------------------------------

class Ref:
    def __init__(self):
        if not os.path.exists(REF_PATH):
            raise FileNotFoundError(f"{REF_PATH} missing; run `make -C oracle ref`")
        self.lib = ctypes.CDLL(REF_PATH)
        self.lib.ref_last_error.restype = ctypes.c_char_p
        self.lib.ref_prover_open.restype = _VP
        self.lib.ref_prover_open.argtypes = [_VP, ctypes.c_char_p]
        self.lib.ref_prover_prove.argtypes = [_VP, _VP, _VP, _VP]
        self.lib.ref_prover_prove_blind.argtypes = [_VP, _VP, _VP, _VP, _VP]
        self.lib.ref_prover_close.argtypes = [_VP]
        assert self.lib.ref_init() == 0

    def _ok(self, rc, what):
        if rc != 0:
            raise RuntimeError(f"{what}: {self.lib.ref_last_error().decode()}")

    def fr_constant(self, which):
        out = np.zeros(4, np.uint64)
        self._ok(self.lib.ref_fr_constant(ctypes.c_int(which), _p(out)), "fr_constant")
        return out

    def poseidon_hash2(self, left, right):
        out = np.zeros(4, np.uint64)
        self._ok(self.lib.ref_poseidon_hash2(_p(_arr(left)), _p(_arr(right)), _p(out)), "poseidon")
        return out

    def domain_op(self, op, data):
        d = _arr(data).copy()
        self._ok(self.lib.ref_domain_op(ctypes.c_int(op), _p(d), _U64(d.size // 4)), "domain_op")
        return d.reshape(-1, 4)

    def multiexp(self, group, bases_jac, scalars):
        out = np.zeros(12 * group, np.uint64)
        s = _arr(scalars)
        f = self.lib.ref_multiexp_g1 if group == 1 else self.lib.ref_multiexp_g2
        self._ok(f(_p(_arr(bases_jac)), _p(s), _U64(s.size // 4), _p(out)), "multiexp")
        return out

    def mul_gen(self, group, k):
        out = np.zeros(12 * group, np.uint64)
        f = self.lib.ref_g1_mul_gen if group == 1 else self.lib.ref_g2_mul_gen
        self._ok(f(_p(_arr(k)), _p(out)), "mul_gen")
        return out

    def reduced_pairing(self, p_jac, q_jac):
        """libff's reduced pairing (GT as 48 u64 Montgomery limbs) of libff Jacobian P, Q."""
        out = np.zeros(48, np.uint64)
        self._ok(self.lib.ref_reduced_pairing(_p(_arr(p_jac)), _p(_arr(q_jac)), _p(out)),
                 "reduced_pairing")
        return out

    def _circuit(self, r1cs):
        return Oracle._circuit(None, r1cs)

    def check_witness(self, r1cs, witness):
        c = self._circuit(r1cs)
        ok = ctypes.c_int()
        w = _arr(witness)
        self._ok(self.lib.ref_check_witness(ctypes.byref(c), _p(w), _U64(w.size // 4),
                                            ctypes.byref(ok)), "check_witness")
        return bool(ok.value)

    def cpu_setup(self, r1cs, pk_path, vk_path):
        c = self._circuit(r1cs)
        self._ok(self.lib.ref_cpu_setup(ctypes.byref(c), str(pk_path).encode(), str(vk_path).encode()),
                 "cpu_setup")

    def cpu_prove(self, r1cs, pk_path, witness):
        c = self._circuit(r1cs)
        g1 = np.zeros((4, 12), np.uint64)
        g2 = np.zeros(24, np.uint64)
        self._ok(self.lib.ref_cpu_prove(ctypes.byref(c), str(pk_path).encode(), _p(_arr(witness)),
                                        _p(g1), _p(g2)), "cpu_prove")
        # the shim writes affine X,Y (64 / 128 B) per point into the leading bytes
        g1a = np.zeros((4, 8), np.uint64)
        raw = g1.reshape(-1)[:32].reshape(4, 8)
        g1a[:] = raw
        return g1a, g2[:16].copy()

    def prover(self, r1cs, pk_path):
        c = self._circuit(r1cs)
        h = self.lib.ref_prover_open(ctypes.byref(c), str(pk_path).encode())
        if not h:
            raise RuntimeError(self.lib.ref_last_error().decode())
        return h

    def prover_prove(self, h, witness):
        g1 = np.zeros(32, np.uint64)
        g2 = np.zeros(16, np.uint64)
        self._ok(self.lib.ref_prover_prove(h, _p(_arr(witness)), _p(g1), _p(g2)), "prover_prove")
        return g1.reshape(4, 8), g2

    def prover_close(self, h):
        self.lib.ref_prover_close(h)

    def prover_prove_blind(self, h, witness):
        """groth16.prove.total of the reference CLI: prove, then blind_proof with the
        reference's own random r, s.  Returns (a, b, c) affine in Jacobian layout."""
        a, b, c = np.zeros(12, np.uint64), np.zeros(24, np.uint64), np.zeros(12, np.uint64)
        self._ok(self.lib.ref_prover_prove_blind(h, _p(_arr(witness)), _p(a), _p(b), _p(c)),
                 "prover_prove_blind")
        return a, b, c

    def quotient_vectors(self, r1cs, witness):
        """az, bz, cz and H of the CPU backend's prove (reference libff / libfqfft)."""
        c = self._circuit(r1cs)
        outs = [np.zeros((r1cs.rows, 4), np.uint64) for _ in range(4)]
        self._ok(self.lib.ref_quotient_vectors(ctypes.byref(c), _p(_arr(witness)),
                                               *[_p(o) for o in outs]), "quotient_vectors")
        return outs

    def seeded_pairs(self, count, density, seed):
        """The Poseidon preimages the repository's seeded generator draws (2 count Fr)."""
        out = np.zeros((2 * count, 4), np.uint64)
        self._ok(self.lib.ref_seeded_pairs(_U64(count), ctypes.c_int(density), _U64(seed), _p(out)),
                 "seeded_pairs")
        return out

    def poseidon_circuit_seeded(self, count, density, seed):
        """generate("poseidon", count, density, seed) built by the reference's own
        Poseidon gadget and R1CSManager (no part of this repository's library)."""
        d = self.poseidon_circuit_n(self.seeded_pairs(count, density, seed))
        return SimpleNamespace(**d)

    def verify(self, vk_path, public_inputs, proof_path):
        ok = ctypes.c_int()
        x = _arr(public_inputs)
        self._ok(self.lib.ref_verify(str(vk_path).encode(), _p(x), _U64(x.size // 4),
                                     str(proof_path).encode(), ctypes.byref(ok)), "verify")
        return bool(ok.value)

    def _build(self, fn, *args):
        """Two-call protocol of the ref_*_circuit builders: sizes, then arrays."""
        rows, cols, pub = _U64(), _U64(), _U64()
        nnz = (_U64 * 3)()
        self._ok(fn(*args, ctypes.byref(rows), ctypes.byref(cols), ctypes.byref(pub), nnz, None, None,
                    None, None), fn.__name__)
        rows, cols, pub = rows.value, cols.value, pub.value
        nnz = list(nnz)
        rp = np.zeros(3 * (rows + 1), np.uint32)
        ci = np.zeros(max(sum(nnz), 1), np.uint32)
        vals = np.zeros((max(sum(nnz), 1), 4), np.uint64)
        w = np.zeros((cols, 4), np.uint64)
        self._ok(fn(*args, ctypes.byref(_U64()), ctypes.byref(_U64()), ctypes.byref(_U64()),
                    (_U64 * 3)(), _p(rp), _p(ci), _p(vals), _p(w)), fn.__name__)
        out_rp, out_ci, out_v = [], [], []
        off = 0
        for k in range(3):
            out_rp.append(rp[k * (rows + 1):(k + 1) * (rows + 1)].copy())
            out_ci.append(ci[off:off + nnz[k]].copy())
            out_v.append(vals[off:off + nnz[k]].copy())
            off += nnz[k]
        return dict(rows=rows, cols=cols, public_inputs=pub, row_ptr=out_rp, col_idx=out_ci,
                    values=out_v, witness=w)

    def matmul_circuit(self, s, av, bv):
        return self._build(self.lib.ref_matmul_circuit, _U64(s), _p(_arr(av)), _p(_arr(bv)))

    def poseidon_circuit_n(self, lr):
        lr = _arr(lr)
        return self._build(self.lib.ref_poseidon_circuit_n, _U64(lr.size // 8), _p(lr))

    def sql_circuit(self, cats, amts):
        c = _arr(cats)
        return self._build(self.lib.ref_sql_circuit, _U64(c.size // 4), _p(c), _p(_arr(amts)))

    def write_vk(self, vk_parts, path):
        """Verification key artifact for keys made elsewhere; e(alpha, beta) by libff."""
        ic = _arr(vk_parts["ic"])
        self._ok(self.lib.ref_write_vk(_p(_arr(vk_parts["alpha_g1"])), _p(_arr(vk_parts["beta_g2"])),
                                       _p(_arr(vk_parts["gamma_g2"])), _p(_arr(vk_parts["delta_g2"])),
                                       _p(ic), _U64(ic.size // 12), str(path).encode()), "write_vk")

    def poseidon_circuit(self, left, right):
        rows, cols = _U64(), _U64()
        nnz = (_U64 * 3)()
        l, r = _arr(left), _arr(right)
        self._ok(self.lib.ref_poseidon_circuit(_p(l), _p(r), ctypes.byref(rows), ctypes.byref(cols),
                                               nnz, None, None, None, None), "poseidon_circuit")
        rows, cols = rows.value, cols.value
        tot = sum(nnz)
        rp = np.zeros(3 * (rows + 1), np.uint32)
        ci = np.zeros(tot, np.uint32)
        vals = np.zeros((tot, 4), np.uint64)
        w = np.zeros((cols, 4), np.uint64)
        self._ok(self.lib.ref_poseidon_circuit(_p(l), _p(r), ctypes.byref(_U64()), ctypes.byref(_U64()),
                                               (_U64 * 3)(), _p(rp), _p(ci), _p(vals), _p(w)),
                 "poseidon_circuit")
        out_rp, out_ci, out_v = [], [], []
        off = 0
        for k in range(3):
            out_rp.append(rp[k * (rows + 1):(k + 1) * (rows + 1)])
            out_ci.append(ci[off:off + nnz[k]])
            out_v.append(vals[off:off + nnz[k]])
            off += nnz[k]
        return rows, cols, out_rp, out_ci, out_v, w


def ref_available():
    return os.path.exists(REF_PATH)


REFCUDA_PATH = os.path.join(HERE, "_ref", "libnkr_ref_cuda.so")


def refcuda_available():
    return os.path.exists(REFCUDA_PATH)


class RefCuda:
    """The reference's own CUDA backend (CudaBackend::prepare / prove,
    protocols/groth16/backends/cuda/src/groth16_backend.cu:214-279) rebuilt for
    sm_100a (oracle/ref_cuda_shim.cu).  Keys must be affine-normalised."""

    def __init__(self):
        if not refcuda_available():
            raise FileNotFoundError(f"{REFCUDA_PATH} missing; run `make -C oracle refcuda`")
        self.lib = ctypes.CDLL(REFCUDA_PATH)
        self.lib.refcuda_last_error.restype = ctypes.c_char_p
        self.lib.refcuda_open.restype = _VP
        self.lib.refcuda_open.argtypes = [_VP] + [_VP] * 5
        self.lib.refcuda_prove.argtypes = [_VP, _VP, _VP, _VP, ctypes.POINTER(ctypes.c_double)]
        self.lib.refcuda_close.argtypes = [_VP]
        self.lib.refcuda_last_prepare_ms.restype = ctypes.c_double

    def open(self, r1cs, pk):
        c = Oracle._circuit(None, r1cs)
        q = [_arr(pk[k]) for k in ("a_query", "b_g1_query", "b_g2_query", "l_query", "h_query")]
        h = self.lib.refcuda_open(ctypes.byref(c), *[_p(x) for x in q])
        if not h:
            raise RuntimeError(self.lib.refcuda_last_error().decode())
        return h

    def prove(self, h, witness):
        """(g1 affine [4, 8], g2 affine [16], host wall ms of the reference's prove)"""
        g1 = np.zeros(32, np.uint64)
        g2 = np.zeros(16, np.uint64)
        ms = ctypes.c_double()
        if self.lib.refcuda_prove(h, _p(_arr(witness)), _p(g1), _p(g2), ctypes.byref(ms)) != 0:
            raise RuntimeError(self.lib.refcuda_last_error().decode())
        return g1.reshape(4, 8), g2, ms.value

    def last_prepare_ms(self):
        """host wall ms of the last open's CudaBackend::prepare (synchronised)"""
        return self.lib.refcuda_last_prepare_ms()

    def close(self, h):
        self.lib.refcuda_close(h)


DROPIN_PATH = os.path.join(HERE, "_ref", "libnkr_ref_b200.so")


class RefDropIn:
    """The reference's Groth16 code driving the B200 backend through its Backend
    interface (oracle/ref_dropin.cpp + nkr-zkp_b200/integration/b200_backend.cpp)."""

    def __init__(self):
        if not os.path.exists(DROPIN_PATH):
            raise FileNotFoundError(f"{DROPIN_PATH} missing; run `make -C oracle dropin`")
        self.lib = ctypes.CDLL(DROPIN_PATH)
        self.lib.dropin_last_error.restype = ctypes.c_char_p

    def prove_verify(self, r1cs, pk_path, vk_path, witness, gpu_setup=False):
        c = Oracle._circuit(None, r1cs)
        verified, raw_equal = ctypes.c_int(-1), ctypes.c_int(-1)
        name = ctypes.create_string_buffer(16)
        w = _arr(witness)
        rc = self.lib.dropin_prove_verify(ctypes.byref(c), str(pk_path).encode(), str(vk_path).encode(),
                                          _p(w), ctypes.c_int(1 if gpu_setup else 0),
                                          ctypes.byref(verified), ctypes.byref(raw_equal), name)
        if rc != 0:
            raise RuntimeError(self.lib.dropin_last_error().decode())
        return bool(verified.value), bool(raw_equal.value), name.value.decode()


def dropin_available():
    return os.path.exists(DROPIN_PATH)


# ---------------------------------------------------------------------------
# BinaryArchive ("LKZ1", version 1) artifacts
# ---------------------------------------------------------------------------

MAGIC = b"LKZ1"


class ArchiveWriter:
    def __init__(self, path):
        self.f = open(path, "wb")
        self.f.write(MAGIC + struct.pack("<I", 1))

    def value(self, raw: bytes):
        self.f.write(raw)

    def u64(self, v):
        self.f.write(struct.pack("<Q", v))

    def vector(self, arr):
        b = np.ascontiguousarray(arr).tobytes()
        self.f.write(struct.pack("<Q", len(b)) + b)

    def close(self):
        self.f.close()


class ArchiveReader:
    def __init__(self, path):
        self.f = open(path, "rb")
        head = self.f.read(8)
        if head[:4] != MAGIC or struct.unpack("<I", head[4:])[0] != 1:
            raise ValueError(f"{path}: not a BinaryArchive v1 file")

    def value(self, n):
        b = self.f.read(n)
        if len(b) != n:
            raise ValueError("unexpected end of file")
        return b

    def u64(self):
        return struct.unpack("<Q", self.value(8))[0]

    def vector(self, dtype, width=1):
        n = self.u64()
        a = np.frombuffer(self.value(n), dtype=dtype).copy()
        return a.reshape(-1, width) if width > 1 else a

    def close(self):
        self.f.close()


def write_circuit(path, r1cs):
    """groth16 io.cpp:33-41"""
    w = ArchiveWriter(path)
    w.u64(r1cs.public_inputs)
    w.u64(r1cs.cols)
    for k in range(3):
        w.vector(r1cs.row_ptr[k])
        w.vector(r1cs.col_idx[k])
        w.vector(r1cs.values[k])
    w.close()


def write_witness(path, witness):
    w = ArchiveWriter(path)
    w.vector(_arr(witness))
    w.close()


def read_proving_key(path):
    """io.cpp:54-61; points stay in libff Jacobian layout."""
    r = ArchiveReader(path)
    pk = {}
    pk["a_query"] = r.vector(np.uint64, 12)
    pk["b_g1_query"] = r.vector(np.uint64, 12)
    pk["b_g2_query"] = r.vector(np.uint64, 24)
    pk["l_query"] = r.vector(np.uint64, 12)
    pk["h_query"] = r.vector(np.uint64, 12)
    for name, n in (("alpha_g1", 96), ("beta_g1", 96), ("beta_g2", 192), ("delta_g1", 96),
                    ("delta_g2", 192)):
        pk[name] = np.frombuffer(r.value(n), np.uint64).copy()
    r.close()
    return pk


def write_proving_key(path, pk):
    w = ArchiveWriter(path)
    for name in ("a_query", "b_g1_query", "b_g2_query", "l_query", "h_query"):
        w.vector(_arr(pk[name]))
    for name in ("alpha_g1", "beta_g1", "beta_g2", "delta_g1", "delta_g2"):
        w.value(_arr(pk[name]).tobytes())
    w.close()


def read_verification_key(path):
    """A reference verification key artifact (common/src/io.cpp:72-77 over
    BinaryArchive: magic, version, GT, gamma G2, delta G2, ic vector)."""
    raw = open(path, "rb").read()
    assert raw[:4] == b"LKZ1", "not a BinaryArchive file"
    pos = 8
    gt = np.frombuffer(raw[pos:pos + 384], np.uint64).copy(); pos += 384
    gamma = np.frombuffer(raw[pos:pos + 192], np.uint64).copy(); pos += 192
    delta = np.frombuffer(raw[pos:pos + 192], np.uint64).copy(); pos += 192
    n = int(np.frombuffer(raw[pos:pos + 8], np.uint64)[0]); pos += 8
    ic = np.frombuffer(raw[pos:pos + n], np.uint64).copy().reshape(-1, 12)
    return {"alpha_g1_beta_g2": gt, "gamma_g2": gamma, "delta_g2": delta, "ic": ic}


def write_proof(path, a_jac, b_jac, c_jac):
    """io.cpp:92-96: raw G1, G2, G1 (libff Jacobian layout)"""
    w = ArchiveWriter(path)
    w.value(_arr(a_jac).tobytes())
    w.value(_arr(b_jac).tobytes())
    w.value(_arr(c_jac).tobytes())
    w.close()


def jac_to_affine_layout(group, jac, orc=None):
    """libff Jacobian -> affine X,Y (8 / 16 limbs), infinity as (0, 1)."""
    orc = orc or Oracle()
    return orc.to_affine(group, jac)


def affine_to_jac(group, aff):
    """affine (libff encoding) -> libff Jacobian layout with Z = 1 (or 0 for infinity)."""
    aff = _arr(aff).reshape(-1, 8 * group)
    w = 4 * group
    out = np.zeros((aff.shape[0], 12 * group), np.uint64)
    out[:, :8 * group] = aff
    one = fq_mont(1)
    z = np.zeros(w, np.uint64)
    z[:4] = one
    inf = np.all(aff[:, :w] == 0, axis=1) & np.all(aff[:, w:2 * w] == z, axis=1)
    out[:, 8 * group:] = z
    out[inf, 8 * group:] = 0
    return out


def sha256_arr(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def pk_affine(pk, orc=None):
    """A proving key dict (libff Jacobian layout) normalised to affine X,Y arrays."""
    orc = orc or Oracle()
    out = {}
    for k, v in pk.items():
        group = 2 if "g2" in k else 1
        a = orc.to_affine(group, v)
        out[k] = a.reshape(-1) if np.asarray(v).ndim == 1 else a
    return out
