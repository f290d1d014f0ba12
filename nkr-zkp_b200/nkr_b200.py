"""ctypes binding of libnkr_b200.so (the C ABI in include/nkr_b200.h).

Python mirror of the reference's Groth16 backend interface for the prove path
(protocols/groth16/common/include/groth16/backend.hpp:11-28): `Backend.name()`,
`prepare(circuit, proving_key)` and `prove(circuit, proving_key, witness)`
returning a RawProof, plus the operator-level NTT / SpMV / MSM calls
(operators/cuda/include/nkr/operators/cuda.hpp).  Buffers are numpy arrays in
the reference's libff byte layouts (Fr = 4 x uint64 Montgomery; G1 Jacobian =
12 x uint64; G2 Jacobian = 24 x uint64).

There is no CPU fallback: importing this module fails loudly if the CUDA
library has not been built, and every compute call raises if no sm_100 GPU is
usable.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libnkr_b200.so")

if not os.path.exists(LIB_PATH):
    raise ImportError(
        f"{LIB_PATH} is missing: build it with `python nkr-zkp_b200/build.py` "
        "(there is no CPU fallback for the B200 backend)")

# more hardware work queues than the default 8, so the many streams of concurrent
# prove slots do not alias onto a few queues (read when the CUDA context is created)
os.environ.setdefault("CUDA_DEVICE_MAX_CONNECTIONS", "32")

_lib = ctypes.CDLL(LIB_PATH)

OK, EINVAL, ECUDA, ENOMEM, ENODEV, ETIMEOUT, EBUSY = range(7)
_VP = ctypes.c_void_p
_U64 = ctypes.c_uint64


class Circuit(ctypes.Structure):
    _fields_ = [("rows", _U64), ("cols", _U64), ("public_inputs", _U64),
                ("row_ptr", _VP * 3), ("col_idx", _VP * 3), ("values", _VP * 3)]


class ProvingKey(ctypes.Structure):
    _fields_ = [(n, _VP) for n in ("a_query", "b_g1_query", "b_g2_query", "l_query", "h_query",
                                   "alpha_g1", "beta_g1", "delta_g1", "beta_g2", "delta_g2")]


class RawProofC(ctypes.Structure):
    _fields_ = [("ar", ctypes.c_uint8 * 96), ("bs1", ctypes.c_uint8 * 96),
                ("zk", ctypes.c_uint8 * 96), ("qz", ctypes.c_uint8 * 96),
                ("bs2", ctypes.c_uint8 * 192)]


class ProofC(ctypes.Structure):
    _fields_ = [("a", ctypes.c_uint8 * 96), ("b", ctypes.c_uint8 * 192), ("c", ctypes.c_uint8 * 96)]


class VerificationKeyC(ctypes.Structure):
    _fields_ = [("alpha_g1_beta_g2", _VP), ("gamma_g2", _VP), ("delta_g2", _VP), ("ic", _VP),
                ("n_ic", _U64)]


class StageTimes(ctypes.Structure):
    _fields_ = [(n, ctypes.c_float) for n in
                ("spmv_ms", "quotient_ms", "witness_msms_ms", "quotient_msm_ms", "total_ms",
                 "msm_a_end_ms", "msm_b_g1_end_ms", "msm_b_g2_end_ms", "msm_l_end_ms",
                 "msm_h_end_ms")] + [("msm_phase_ms", ctypes.c_float * 20)]


_MSM_NAMES = ("a", "b_g1", "b_g2", "l", "h")
_PHASE_NAMES = ("l1_start", "l1_end", "fixup_end", "reduce_first_end")


class MsmStats(ctypes.Structure):
    _fields_ = [("total_ms", ctypes.c_float), ("acc_ms", ctypes.c_float), ("entries", _U64),
                ("tasks", _U64), ("window_bits", ctypes.c_uint32), ("windows", ctypes.c_uint32),
                ("buckets", ctypes.c_uint32), ("sort_ms", ctypes.c_float), ("fixup_ms", ctypes.c_float),
                ("reduce_first_ms", ctypes.c_float), ("reduce_levels_ms", ctypes.c_float)]


_SIGS = {
    "nkr_b200_launch_count": (_U64, []),
    "nkr_b200_msm_bases_stats": (ctypes.c_int, [_VP, ctypes.POINTER(MsmStats)]),
    "nkr_b200_open": (ctypes.c_int, [ctypes.c_int, ctypes.POINTER(_VP)]),
    "nkr_b200_close": (None, [_VP]),
    "nkr_b200_last_error": (ctypes.c_char_p, []),
    "nkr_b200_backend_name": (ctypes.c_char_p, []),
    "nkr_b200_prepare": (ctypes.c_int, [_VP, ctypes.POINTER(Circuit), ctypes.POINTER(ProvingKey),
                                        ctypes.POINTER(_VP)]),
    "nkr_b200_prepare_file": (ctypes.c_int, [_VP, ctypes.POINTER(Circuit), ctypes.c_char_p,
                                             ctypes.POINTER(_VP)]),
    "nkr_b200_pk_file_info": (ctypes.c_int, [ctypes.c_char_p, ctypes.POINTER(_U64),
                                             ctypes.POINTER(_U64)]),
    "nkr_b200_write_proving_key": (ctypes.c_int, [ctypes.c_char_p, ctypes.POINTER(ProvingKey),
                                                  _U64, _U64]),
    "nkr_b200_key_free": (None, [_VP]),
    "nkr_b200_key_device_bytes": (_U64, [_VP]),
    "nkr_b200_prove": (ctypes.c_int, [_VP, _VP, _U64, ctypes.POINTER(RawProofC)]),
    "nkr_b200_tune_save": (ctypes.c_int, [_VP, ctypes.c_char_p]),
    "nkr_b200_tune_load": (ctypes.c_int, [_VP, ctypes.c_char_p, ctypes.POINTER(ctypes.c_int)]),
    "nkr_b200_vk_prepare": (ctypes.c_int, [_VP, ctypes.POINTER(VerificationKeyC),
                                           ctypes.POINTER(_VP)]),
    "nkr_b200_verify_batch": (ctypes.c_int, [_VP, _VP, _U64, _VP, _U64, _VP]),
    "nkr_b200_vk_free": (None, [_VP]),
    "nkr_b200_reduced_pairing": (ctypes.c_int, [_VP, _VP, _VP, _U64, _VP]),
    "nkr_b200_blind": (ctypes.c_int, [_VP, ctypes.POINTER(RawProofC), _VP, _VP,
                                      ctypes.POINTER(ProofC)]),
    "nkr_b200_key_intermediates": (ctypes.c_int, [_VP, _VP, _VP, _VP, _VP]),
    "nkr_b200_key_stage_times": (ctypes.c_int, [_VP, ctypes.POINTER(StageTimes)]),
    "nkr_b200_prove_batch": (ctypes.c_int, [ctypes.POINTER(_VP), ctypes.POINTER(_VP), ctypes.c_int,
                                            ctypes.POINTER(RawProofC)]),
    "nkr_b200_prove_batch_lists": (ctypes.c_int, [ctypes.POINTER(_VP), ctypes.POINTER(_VP), ctypes.c_int,
                                            ctypes.POINTER(RawProofC)]),
    "nkr_b200_ntt": (ctypes.c_int, [_VP, ctypes.c_int, _VP, _U64]),
    "nkr_b200_tune_ntt": (ctypes.c_int, [_VP, _U64, ctypes.POINTER(ctypes.c_int),
                                         ctypes.POINTER(ctypes.c_int)]),
    "nkr_b200_ntt_device": (ctypes.c_int, [_VP, ctypes.c_int, _VP, _VP, _U64, _VP,
                                           ctypes.POINTER(ctypes.c_float)]),
    "nkr_b200_server_create": (ctypes.c_int, [_VP, ctypes.c_int, ctypes.c_int, ctypes.POINTER(_VP)]),
    "nkr_b200_server_add_key": (ctypes.c_int, [_VP, _VP, ctypes.POINTER(ctypes.c_int)]),
    "nkr_b200_server_submit": (ctypes.c_int, [_VP, ctypes.c_int, _VP, ctypes.POINTER(_U64)]),
    "nkr_b200_server_wait": (ctypes.c_int, [_VP, _U64, ctypes.POINTER(RawProofC),
                                            ctypes.POINTER(ctypes.c_double),
                                            ctypes.POINTER(ctypes.c_double)]),
    "nkr_b200_server_slots": (ctypes.c_int, [_VP, ctypes.c_int, ctypes.POINTER(ctypes.c_int)]),
    "nkr_b200_server_set_ageing": (ctypes.c_int, [_VP, ctypes.c_double]),
    "nkr_b200_server_stats": (ctypes.c_int, [_VP, ctypes.POINTER(_U64), ctypes.POINTER(_U64),
                                             ctypes.POINTER(_U64)]),
    "nkr_b200_server_destroy": (None, [_VP]),
    "nkr_b200_set_autotune": (ctypes.c_int, [_VP, ctypes.c_int]),
    "nkr_b200_tune_msm": (ctypes.c_int, [_VP, _U64, ctypes.POINTER(ctypes.c_int),
                                          ctypes.POINTER(ctypes.c_float)]),
    "nkr_b200_ntt_noalloc": (ctypes.c_int, [ctypes.c_int, ctypes.c_int, _VP, _VP, _U64, _VP]),
    "nkr_b200_spmv": (ctypes.c_int, [_VP, _U64, _U64, _VP, _VP, _VP, _VP, _VP]),
    "nkr_b200_msm_g1": (ctypes.c_int, [_VP, _VP, _VP, _U64, _VP]),
    "nkr_b200_msm_g2": (ctypes.c_int, [_VP, _VP, _VP, _U64, _VP]),
    "nkr_b200_msm_bases_create": (ctypes.c_int, [_VP, ctypes.c_int, _VP, _U64, ctypes.POINTER(_VP)]),
    "nkr_b200_msm_bases_run": (ctypes.c_int, [_VP, _VP, _U64, _VP, ctypes.POINTER(ctypes.c_float)]),
    "nkr_b200_msm_bases_free": (None, [_VP]),
    "nkr_b200_field_op": (ctypes.c_int, [_VP, ctypes.c_int, ctypes.c_int, _VP, _VP, _VP, _U64]),
    "nkr_b200_group_op": (ctypes.c_int, [_VP, ctypes.c_int, ctypes.c_int, _VP, _VP, _VP, _U64]),
    "nkr_b200_bench_mul": (ctypes.c_int, [_VP, ctypes.c_int, ctypes.POINTER(ctypes.c_double),
                                          ctypes.POINTER(ctypes.c_double)]),
    "nkr_b200_r1cs_generate": (ctypes.c_int, [ctypes.c_char_p, _U64, ctypes.c_int, _U64,
                                              ctypes.POINTER(_VP)]),
    "nkr_b200_r1cs_info": (ctypes.c_int, [_VP, ctypes.POINTER(_U64)]),
    "nkr_b200_r1cs_view": (ctypes.c_int, [_VP, ctypes.POINTER(Circuit), ctypes.POINTER(_VP)]),
    "nkr_b200_r1cs_free": (None, [_VP]),
    "nkr_b200_poseidon_hash2": (ctypes.c_int, [_VP, _VP, _VP]),
    "nkr_b200_poseidon_parameters": (ctypes.c_int, [_VP, _VP]),
}
for _name, (_res, _args) in _SIGS.items():
    _f = getattr(_lib, _name)
    _f.restype = _res
    _f.argtypes = _args


class B200Error(RuntimeError):
    def __init__(self, status, where):
        msg = _lib.nkr_b200_last_error().decode(errors="replace")
        super().__init__(f"{where}: status {status}: {msg}")
        self.status = status


def _check(status, where):
    if status != OK:
        raise B200Error(status, where)


def _ptr(a):
    return a.ctypes.data_as(_VP) if a is not None else None


def _fr(a):
    a = np.ascontiguousarray(a, dtype=np.uint64)
    assert a.size % 4 == 0
    return a


def lib():
    return _lib


def backend_name():
    return _lib.nkr_b200_backend_name().decode()


def launch_count():
    """Kernels launched by the library so far in this process."""
    return int(_lib.nkr_b200_launch_count())


# ---------------------------------------------------------------------------
# circuits (generated or given as numpy CSR arrays)
# ---------------------------------------------------------------------------

class R1CS:
    """A circuit in the reference CSR layout plus its witness (numpy arrays)."""

    def __init__(self, rows, cols, public_inputs, row_ptr, col_idx, values, witness):
        self.rows, self.cols, self.public_inputs = int(rows), int(cols), int(public_inputs)
        self.row_ptr = [np.ascontiguousarray(x, dtype=np.uint32) for x in row_ptr]
        self.col_idx = [np.ascontiguousarray(x, dtype=np.uint32) for x in col_idx]
        self.values = [_fr(x).reshape(-1, 4) for x in values]
        self.witness = None if witness is None else _fr(witness).reshape(-1, 4)

    def c_circuit(self):
        c = Circuit()
        c.rows, c.cols, c.public_inputs = self.rows, self.cols, self.public_inputs
        for k in range(3):
            c.row_ptr[k] = self.row_ptr[k].ctypes.data
            c.col_idx[k] = self.col_idx[k].ctypes.data if self.col_idx[k].size else None
            c.values[k] = self.values[k].ctypes.data if self.values[k].size else None
        return c


def generate(kind, param, density=0, seed=1):
    """Seeded restatement of groth16-gen (kind: matmul, poseidon, sql-aggregate, fibonacci)."""
    h = _VP()
    _check(_lib.nkr_b200_r1cs_generate(kind.encode(), param, density, seed, ctypes.byref(h)),
           f"generate {kind} {param}")
    try:
        sizes = (_U64 * 8)()
        _check(_lib.nkr_b200_r1cs_info(h, sizes), "r1cs_info")
        rows, cols, pub, ncons, nvars, na, nb, nc = list(sizes)
        view = Circuit()
        wit = _VP()
        _check(_lib.nkr_b200_r1cs_view(h, ctypes.byref(view), ctypes.byref(wit)), "r1cs_view")

        def arr(ptr, count, dtype, width=1):
            if count == 0:
                return np.zeros((0, width) if width > 1 else 0, dtype=dtype)
            buf = (ctypes.c_uint8 * (count * width * np.dtype(dtype).itemsize)).from_address(ptr)
            a = np.frombuffer(buf, dtype=dtype).copy()
            return a.reshape(-1, width) if width > 1 else a

        nnz = [na, nb, nc]
        rp = [arr(view.row_ptr[k], rows + 1, np.uint32) for k in range(3)]
        ci = [arr(view.col_idx[k], nnz[k], np.uint32) for k in range(3)]
        vals = [arr(view.values[k], nnz[k], np.uint64, 4) for k in range(3)]
        w = arr(wit.value, cols, np.uint64, 4)
        r = R1CS(rows, cols, pub, rp, ci, vals, w)
        r.constraints, r.variables = ncons, nvars
        return r
    finally:
        _lib.nkr_b200_r1cs_free(h)


def poseidon_hash2(left, right):
    out = np.zeros(4, np.uint64)
    _check(_lib.nkr_b200_poseidon_hash2(_ptr(_fr(left)), _ptr(_fr(right)), _ptr(out)), "poseidon")
    return out


NTT_NOALLOC_MAX = 1 << 16


def ntt_noalloc(device, op, in_ptr, out_ptr, n, stream_ptr=0):
    """nkr_b200_ntt_noalloc on device pointers (enqueued on stream_ptr, not waited for)."""
    _check(_lib.nkr_b200_ntt_noalloc(device, op, in_ptr, out_ptr, n, stream_ptr or None),
           f"ntt_noalloc op {op}")


def poseidon_parameters():
    rc = np.zeros((195, 4), np.uint64)
    mds = np.zeros((9, 4), np.uint64)
    _check(_lib.nkr_b200_poseidon_parameters(_ptr(rc), _ptr(mds)), "poseidon_parameters")
    return rc, mds


# ---------------------------------------------------------------------------
# device context, keys, operators
# ---------------------------------------------------------------------------

class Context:
    """One GPU (nkr_b200_open)."""

    def __init__(self, device=0):
        h = _VP()
        _check(_lib.nkr_b200_open(device, ctypes.byref(h)), "nkr_b200_open")
        self.h = h

    def close(self):
        if self.h:
            _lib.nkr_b200_close(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # operator-level entry points -------------------------------------------
    def tune_save(self, path):
        """Write the measured MSM window widths of this context (nkr_b200_tune_save)."""
        _check(_lib.nkr_b200_tune_save(self.h, str(path).encode()), "nkr_b200_tune_save")

    def tune_load(self, path):
        """Load widths measured earlier on this device model; returns the size classes read."""
        n = ctypes.c_int()
        _check(_lib.nkr_b200_tune_load(self.h, str(path).encode(), ctypes.byref(n)), "nkr_b200_tune_load")
        return n.value

    def ntt(self, op, data):
        d = _fr(data).copy()
        _check(_lib.nkr_b200_ntt(self.h, op, _ptr(d), d.size // 4), f"ntt op {op}")
        return d.reshape(-1, 4)

    def ntt_device(self, op, in_ptr, out_ptr, n, stream_ptr=None, timed=False):
        """Domain op on device vectors (result in out_ptr, in_ptr overwritten); with
        timed, waits and returns the device milliseconds."""
        ms = ctypes.c_float()
        _check(_lib.nkr_b200_ntt_device(self.h, op, in_ptr, out_ptr, n, stream_ptr,
                                        ctypes.byref(ms) if timed else None), f"ntt_device op {op}")
        return ms.value if timed else None

    def tune_ntt(self, n):
        """(max stages per pass, butterflies per thread) chosen for 2^k-point NTTs."""
        a, b = ctypes.c_int(), ctypes.c_int()
        _check(_lib.nkr_b200_tune_ntt(self.h, n, ctypes.byref(a), ctypes.byref(b)), "tune_ntt")
        return a.value, b.value

    def spmv(self, rows, cols, row_ptr, col_idx, values, z):
        y = np.zeros((rows, 4), np.uint64)
        rp = np.ascontiguousarray(row_ptr, np.uint32)
        ci = np.ascontiguousarray(col_idx, np.uint32)
        vv = _fr(values)
        zz = _fr(z)
        _check(_lib.nkr_b200_spmv(self.h, rows, cols, _ptr(rp), _ptr(ci) if ci.size else None,
                                  _ptr(vv) if vv.size else None, _ptr(zz), _ptr(y)), "spmv")
        return y

    def msm(self, group, bases_jac, scalars):
        b = np.ascontiguousarray(bases_jac, np.uint64)
        s = _fr(scalars)
        out = np.zeros(12 if group == 1 else 24, np.uint64)
        f = _lib.nkr_b200_msm_g1 if group == 1 else _lib.nkr_b200_msm_g2
        _check(f(self.h, _ptr(b), _ptr(s), s.size // 4, _ptr(out)), f"msm g{group}")
        return out

    def field_op(self, field, op, a, b=None):
        w = 8 if field in (2, 4) else 4
        a = np.ascontiguousarray(a, np.uint64).reshape(-1, w)
        bb = None if b is None else np.ascontiguousarray(b, np.uint64).reshape(-1, w)
        out = np.zeros_like(a)
        _check(_lib.nkr_b200_field_op(self.h, field, op, _ptr(a), _ptr(bb), _ptr(out), a.shape[0]),
               f"field_op {field} {op}")
        return out

    def group_op(self, group, op, a, b=None):
        w = 12 if group == 1 else 24
        a = np.ascontiguousarray(a, np.uint64).reshape(-1, w)
        bb = None if b is None else np.ascontiguousarray(b, np.uint64)
        out = np.zeros_like(a)
        _check(_lib.nkr_b200_group_op(self.h, group, op, _ptr(a), _ptr(bb), _ptr(out), a.shape[0]),
               f"group_op {group} {op}")
        return out

    def set_autotune(self, enable):
        _check(_lib.nkr_b200_set_autotune(self.h, int(bool(enable))), "set_autotune")

    def tune_msm(self, n):
        """(window bits, measured ms at that size class) for an MSM of n points."""
        c = ctypes.c_int()
        ms = ctypes.c_float()
        _check(_lib.nkr_b200_tune_msm(self.h, n, ctypes.byref(c), ctypes.byref(ms)), "tune_msm")
        return c.value, ms.value

    def bench_mul(self, field):
        rate, ms = ctypes.c_double(), ctypes.c_double()
        _check(_lib.nkr_b200_bench_mul(self.h, field, ctypes.byref(rate), ctypes.byref(ms)),
               "bench_mul")
        return rate.value, ms.value


class MsmBases:
    """Resident MSM bases (per-window copies built once), then MSMs with new scalars."""

    def __init__(self, ctx, group, bases_jac):
        self.ctx, self.group = ctx, group
        b = np.ascontiguousarray(bases_jac, np.uint64)
        self.n = b.size // (12 if group == 1 else 24)
        h = _VP()
        _check(_lib.nkr_b200_msm_bases_create(ctx.h, group, _ptr(b), self.n, ctypes.byref(h)),
               "msm_bases_create")
        self.h = h

    def run(self, scalars, scalars_ptr=None):
        out = np.zeros(12 if self.group == 1 else 24, np.uint64)
        ms = ctypes.c_float()
        ptr = scalars_ptr if scalars_ptr is not None else _ptr(_fr(scalars))
        _check(_lib.nkr_b200_msm_bases_run(self.h, ptr, self.n, _ptr(out), ctypes.byref(ms)),
               "msm_bases_run")
        return out, ms.value

    def stats(self):
        s = MsmStats()
        _check(_lib.nkr_b200_msm_bases_stats(self.h, ctypes.byref(s)), "msm_bases_stats")
        return {n: getattr(s, n) for n, _ in MsmStats._fields_}

    def free(self):
        if self.h:
            _lib.nkr_b200_msm_bases_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def reduced_pairing(ctx, p_g1, q_g2):
    """libff's reduced pairing of count (P, Q) pairs on the device: P G1 libff Jacobian
    (count x 12 u64), Q G2 (count x 24 u64) -> GT (count x 48 u64, alt_bn128_Fq12)."""
    p = np.ascontiguousarray(p_g1, dtype=np.uint64).reshape(-1, 12)
    q = np.ascontiguousarray(q_g2, dtype=np.uint64).reshape(-1, 24)
    if p.shape[0] != q.shape[0]:
        raise ValueError("as many G1 as G2 points are needed")
    out = np.zeros((p.shape[0], 48), np.uint64)
    _check(_lib.nkr_b200_reduced_pairing(ctx.h, _ptr(p), _ptr(q), p.shape[0], _ptr(out)),
           "nkr_b200_reduced_pairing")
    return out


class VerifyingKey:
    """A verification key prepared on the device (nkr_b200_vk_prepare); verify_batch
    is the reference's verify (protocol.cpp:96-108) for many proofs at once."""

    def __init__(self, ctx, alpha_g1_beta_g2, gamma_g2, delta_g2, ic):
        self.ctx = ctx
        self._keep = [np.ascontiguousarray(x, dtype=np.uint64) for x in
                      (alpha_g1_beta_g2, gamma_g2, delta_g2, ic)]
        gt, g, d, icv = self._keep
        self.n_ic = icv.size // 12
        c = VerificationKeyC(gt.ctypes.data, g.ctypes.data, d.ctypes.data, icv.ctypes.data, self.n_ic)
        h = _VP()
        _check(_lib.nkr_b200_vk_prepare(ctx.h, ctypes.byref(c), ctypes.byref(h)), "nkr_b200_vk_prepare")
        self.h = h

    def verify_batch(self, public_inputs, proofs):
        """public_inputs: count x n_public x 4 u64 (Fr Montgomery); proofs: count x 48 u64
        (A, B, C libff Jacobian) -> bool array of verdicts."""
        pr = np.ascontiguousarray(proofs, dtype=np.uint64).reshape(-1, 48)
        count = pr.shape[0]
        if count == 0:
            return np.zeros(0, bool)
        x = np.ascontiguousarray(public_inputs, dtype=np.uint64).reshape(count, -1)
        n_public = x.shape[1] // 4
        acc = np.zeros(count, np.uint8)
        _check(_lib.nkr_b200_verify_batch(self.h, _ptr(x) if x.size else None, n_public, _ptr(pr),
                                          count, _ptr(acc)), "nkr_b200_verify_batch")
        return acc.astype(bool)

    def free(self):
        if self.h:
            _lib.nkr_b200_vk_free(self.h)
            self.h = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


def raw_to_arrays(raw):
    g1 = [np.frombuffer(bytes(getattr(raw, f)), np.uint64).copy() for f in ("ar", "bs1", "zk", "qz")]
    g2 = np.frombuffer(bytes(raw.bs2), np.uint64).copy()
    return g1, g2


class Backend:
    """The B200 backend behind NKR-ZKP's Backend interface (prepare / prove).

    Mirrors protocols/groth16/common/include/groth16/backend.hpp:11-28: prepare()
    makes the circuit and proving key resident; prove() returns the raw proof
    {ar, bs1, zk, qz, bs2} affine-normalised in libff layout.
    """

    def __init__(self, ctx):
        self.ctx = ctx
        self.key = None
        self._keep = None

    @staticmethod
    def name():
        return backend_name()

    def prepare(self, r1cs, pk):
        """pk: dict with a_query, b_g1_query, b_g2_query, l_query, h_query (uint64 arrays in
        libff Jacobian layout) and alpha_g1, beta_g1, delta_g1, beta_g2, delta_g2."""
        c = r1cs.c_circuit()
        keep = {k: np.ascontiguousarray(v, np.uint64) for k, v in pk.items()}
        p = ProvingKey()
        for name, _ in ProvingKey._fields_:
            setattr(p, name, keep[name].ctypes.data)
        h = _VP()
        _check(_lib.nkr_b200_prepare(self.ctx.h, ctypes.byref(c), ctypes.byref(p), ctypes.byref(h)),
               "nkr_b200_prepare")
        self.free()
        self.key = h
        self._keep = keep
        self.cols = r1cs.cols
        self.rows = r1cs.rows

    def prepare_file(self, r1cs, pk_path):
        """prepare() from a proving-key artifact file (BinaryArchive, no 1 GiB limit)."""
        c = r1cs.c_circuit()
        h = _VP()
        _check(_lib.nkr_b200_prepare_file(self.ctx.h, ctypes.byref(c), str(pk_path).encode(),
                                          ctypes.byref(h)), "nkr_b200_prepare_file")
        self.free()
        self.key = h
        self._keep = None
        self.cols = r1cs.cols
        self.rows = r1cs.rows

    def prove(self, witness, witness_ptr=None):
        raw = RawProofC()
        if witness_ptr is None:
            w = _fr(witness)
            _check(_lib.nkr_b200_prove(self.key, _ptr(w), w.size // 4, ctypes.byref(raw)),
                   "nkr_b200_prove")
        else:
            _check(_lib.nkr_b200_prove(self.key, witness_ptr, self.cols, ctypes.byref(raw)),
                   "nkr_b200_prove")
        return raw

    def blind(self, raw, r, s):
        proof = ProofC()
        _check(_lib.nkr_b200_blind(self.key, ctypes.byref(raw), _ptr(_fr(r)), _ptr(_fr(s)),
                                   ctypes.byref(proof)), "nkr_b200_blind")
        return proof

    def intermediates(self):
        az, bz, cz, h = (np.zeros((self.rows, 4), np.uint64) for _ in range(4))
        _check(_lib.nkr_b200_key_intermediates(self.key, _ptr(az), _ptr(bz), _ptr(cz), _ptr(h)),
               "intermediates")
        return az, bz, cz, h

    def stage_times(self):
        t = StageTimes()
        _check(_lib.nkr_b200_key_stage_times(self.key, ctypes.byref(t)), "stage_times")
        out = {n: getattr(t, n) for n, _ in StageTimes._fields_ if n != "msm_phase_ms"}
        for i, m in enumerate(_MSM_NAMES):
            for j, ph in enumerate(_PHASE_NAMES):
                out[f"msm_{m}_{ph}_ms"] = t.msm_phase_ms[4 * i + j]
        return out

    def device_bytes(self):
        return int(_lib.nkr_b200_key_device_bytes(self.key))

    def free(self):
        if self.key:
            _lib.nkr_b200_key_free(self.key)
            self.key = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass


class SetupOut(ctypes.Structure):
    _fields_ = [(n, _VP) for n in ("a_query", "b_g1_query", "l_query", "b_g2_query", "h_query", "ic",
                                   "alpha_g1", "beta_g1", "delta_g1", "beta_g2", "delta_g2",
                                   "gamma_g2")]


_lib.nkr_b200_setup.restype = ctypes.c_int
_lib.nkr_b200_setup.argtypes = [_VP, ctypes.POINTER(Circuit), _VP, ctypes.POINTER(SetupOut)]


def setup(ctx, r1cs, toxic):
    """GPU setup with toxic waste Fr[5] = (t, alpha, beta, gamma, delta).

    Returns (pk, vk_parts): pk in the proving-key dict layout Backend.prepare takes
    (libff Jacobian arrays); vk_parts holds ic, gamma_g2, delta_g2, alpha_g1, beta_g2 and
    alpha_g1_beta_g2 (e(alpha, beta), computed on the device)."""
    cols, rows = r1cs.cols, r1cs.rows
    arrs = {
        "a_query": np.zeros((cols, 12), np.uint64), "b_g1_query": np.zeros((cols, 12), np.uint64),
        "l_query": np.zeros((cols, 12), np.uint64), "b_g2_query": np.zeros((cols, 24), np.uint64),
        "h_query": np.zeros((rows, 12), np.uint64),
        "ic": np.zeros((r1cs.public_inputs + 1, 12), np.uint64),
        "alpha_g1": np.zeros(12, np.uint64), "beta_g1": np.zeros(12, np.uint64),
        "delta_g1": np.zeros(12, np.uint64), "beta_g2": np.zeros(24, np.uint64),
        "delta_g2": np.zeros(24, np.uint64), "gamma_g2": np.zeros(24, np.uint64),
    }
    out = SetupOut()
    for name, _ in SetupOut._fields_:
        setattr(out, name, arrs[name].ctypes.data)
    c = r1cs.c_circuit()
    tox = _fr(np.stack([np.asarray(t, np.uint64) for t in toxic]))
    _check(_lib.nkr_b200_setup(ctx.h, ctypes.byref(c), _ptr(tox), ctypes.byref(out)), "nkr_b200_setup")
    pk = {k: arrs[k] for k in ("a_query", "b_g1_query", "b_g2_query", "l_query", "h_query",
                               "alpha_g1", "beta_g1", "delta_g1", "beta_g2", "delta_g2")}
    vk = {k: arrs[k] for k in ("ic", "gamma_g2", "delta_g2", "alpha_g1", "beta_g2")}
    # the key's e(alpha, beta), as the reference's setup stores it (libff's GT value)
    vk["alpha_g1_beta_g2"] = reduced_pairing(ctx, vk["alpha_g1"], vk["beta_g2"])[0]
    return pk, vk


def pk_file_info(path):
    """(rows, cols) of a proving-key artifact file; reads no GPU."""
    rows, cols = _U64(), _U64()
    _check(_lib.nkr_b200_pk_file_info(str(path).encode(), ctypes.byref(rows), ctypes.byref(cols)),
           "nkr_b200_pk_file_info")
    return rows.value, cols.value


def write_proving_key(path, pk, rows, cols):
    """Writes a proving-key dict (libff Jacobian arrays) as a BinaryArchive artifact."""
    keep = {k: np.ascontiguousarray(v, np.uint64) for k, v in pk.items()}
    p = ProvingKey()
    for name, _ in ProvingKey._fields_:
        setattr(p, name, keep[name].ctypes.data)
    _check(_lib.nkr_b200_write_proving_key(str(path).encode(), ctypes.byref(p), rows, cols),
           "nkr_b200_write_proving_key")


def prove_batch(backends, witnesses=None, witness_ptrs=None, lists=False):
    """Batched prove (nkr_b200_prove_batch, or nkr_b200_prove_batch_lists with
    cross-proof launches when lists): numpy witnesses, or raw pointers (pinned
    host or device memory) in witness_ptrs."""
    n = len(backends)
    keys = (_VP * n)(*[b.key for b in backends])
    if witness_ptrs is None:
        ws = [_fr(w) for w in witnesses]
        witness_ptrs = [w.ctypes.data for w in ws]
    wp = (_VP * n)(*witness_ptrs)
    out = (RawProofC * n)()
    f = _lib.nkr_b200_prove_batch_lists if lists else _lib.nkr_b200_prove_batch
    _check(f(keys, wp, n, out), "prove_batch")
    return list(out)


class Server:
    """Request server (nkr_b200_server_*): continuous batching over resident keys.
    Witness arrays are kept referenced until their request is waited for."""

    def __init__(self, ctx, max_inflight=8, max_slots_per_key=4):
        h = _VP()
        _check(_lib.nkr_b200_server_create(ctx.h, max_inflight, max_slots_per_key, ctypes.byref(h)),
               "server_create")
        self.h = h
        self._pending = {}

    def add_key(self, backend):
        kid = ctypes.c_int()
        _check(_lib.nkr_b200_server_add_key(self.h, backend.key, ctypes.byref(kid)), "server_add_key")
        return kid.value

    def submit(self, key_id, witness=None, witness_ptr=None):
        keep = None
        if witness_ptr is None:
            keep = _fr(witness)
            witness_ptr = keep.ctypes.data
        rid = _U64()
        _check(_lib.nkr_b200_server_submit(self.h, key_id, witness_ptr, ctypes.byref(rid)), "server_submit")
        self._pending[rid.value] = keep
        return rid.value

    def wait(self, rid):
        """(RawProofC, latency ms, queue ms)"""
        raw = RawProofC()
        lat, q = ctypes.c_double(), ctypes.c_double()
        st = _lib.nkr_b200_server_wait(self.h, rid, ctypes.byref(raw), ctypes.byref(lat), ctypes.byref(q))
        self._pending.pop(rid, None)
        _check(st, "server_wait")
        return raw, lat.value, q.value

    def slots(self, key_id):
        n = ctypes.c_int()
        _check(_lib.nkr_b200_server_slots(self.h, key_id, ctypes.byref(n)), "server_slots")
        return n.value

    def set_ageing(self, age_factor):
        _check(_lib.nkr_b200_server_set_ageing(self.h, float(age_factor)), "server_set_ageing")

    def stats(self):
        c, f, a = _U64(), _U64(), _U64()
        _check(_lib.nkr_b200_server_stats(self.h, ctypes.byref(c), ctypes.byref(f), ctypes.byref(a)),
               "server_stats")
        return {"completed": c.value, "failed": f.value, "aged": a.value}

    def close(self):
        if self.h:
            _lib.nkr_b200_server_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
