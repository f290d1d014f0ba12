"""The reference's own GPU prove path (CudaBackend, protocols/groth16/backends/
cuda/src/groth16_backend.cu:214-279) rebuilt unchanged for sm_100a, run beside
this backend on the same circuit, keys and witness on the same B200.

Both calls go host to host: witness in host memory, raw proof back on the host
(nkr_b200_prove; CudaBackend::prove, which uploads the witness and combines the
MSM windows on the host).  The reference CPU backend stays the parity oracle;
the reference GPU path's own result is reported, not required to match (its
bucket accumulation adds equal points without a doubling branch,
operators/cuda/include/msm/msm_kernel.cuh:9,51-55)."""
import json
import os
import statistics
import time

import numpy as np
import pytest

import nkr_b200 as nk
import oracle as O

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def refcuda():
    if not O.refcuda_available():
        pytest.skip("oracle/_ref/libnkr_ref_cuda.so (the reference CUDA backend) is not built here")
    return O.RefCuda()


@pytest.mark.parametrize("kind,param,dens", [("matmul", 8, 2), ("poseidon", 2048, 2)])
def test_b200_prove_faster_than_reference_cuda(ctx, refcuda, kind, param, dens):
    r1 = nk.generate(kind, param, dens, seed=3)
    toxic = O.random_fr(5, np.random.default_rng(17))
    pk, _ = nk.setup(ctx, r1, toxic)           # affine-normalised keys (Z = 1)
    # prepare (key upload and device layout) from host keys, timed on both sides;
    # ours twice: the first prepare of a size class also runs the autotuners
    prep = []
    for _ in range(2):
        be = nk.Backend(ctx)
        t0 = time.perf_counter()
        be.prepare(r1, pk)
        prep.append((time.perf_counter() - t0) * 1e3)
        if len(prep) == 1:
            be.free()
    h = refcuda.open(r1, pk)
    ref_prep = refcuda.last_prepare_ms()
    try:
        ours, theirs = [], []
        for i in range(5):
            g1r, g2r, ms = refcuda.prove(h, r1.witness)
            if i:
                theirs.append(ms)
            t0 = time.perf_counter()
            raw = be.prove(r1.witness)
            if i:
                ours.append((time.perf_counter() - t0) * 1e3)
    finally:
        refcuda.close(h)
    g1, g2 = nk.raw_to_arrays(raw)
    same = bool(np.array_equal(np.stack([x[:8] for x in g1]), g1r) and np.array_equal(g2[:16], g2r))
    res = {"circuit": f"{kind} {param}", "rows": r1.rows,
           "b200_ms": round(statistics.median(ours), 3),
           "reference_cuda_ms": round(statistics.median(theirs), 3),
           "speedup": round(statistics.median(theirs) / statistics.median(ours), 2),
           "reference_cuda_raw_proof_equal": same,
           "b200_prepare_ms": {"first": round(prep[0], 1), "tuned": round(prep[1], 1)},
           "reference_cuda_prepare_ms": round(ref_prep, 1)}
    print(json.dumps(res))
    out = os.environ.get("NKR_B200_REFCUDA_LOG")
    if out:
        with open(out, "a") as f:
            f.write(json.dumps(res) + "\n")
    be.free()
    assert statistics.median(ours) < statistics.median(theirs)
