"""NTT / domain operations on the B200 against libfqfft's semantics (the oracle
restates basic_radix2_domain; golden digests come from the reference's own
libfqfft).  Bit-exact: outputs are unique field vectors."""
import json
import os

import numpy as np
import pytest

import oracle as O
from conftest import GOLDEN

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("logn", [1, 2, 3, 5, 8, 10, 11, 12, 16])
def test_domain_ops_match_oracle(ctx, orc, logn, rng):
    n = 1 << logn
    x = O.random_fr(n, rng)
    x[0] = 0
    for op in range(5):
        assert np.array_equal(ctx.ntt(op, x), orc.domain_op(op, x)), f"op {op} n 2^{logn}"


def test_domain_ops_golden(ctx):
    g = json.load(open(os.path.join(GOLDEN, "domain_ops.json")))
    x = O.random_fr(g["n"], np.random.default_rng(g["seed"]))
    for op, digest in g["ops"].items():
        assert O.sha256_arr(ctx.ntt(int(op), x)) == digest, f"op {op}"


@pytest.mark.parametrize("logn", [20, 24])
def test_full_vectors_match_oracle_at_benchmark_sizes(ctx, orc, logn, rng):
    """Every output element against the oracle's serial libfqfft restatement:
    all five domain ops at 2^20 (the prove's domain), the FFT at 2^24."""
    n = 1 << logn
    x = O.random_fr(n, rng)
    for op in (range(5) if logn == 20 else (0,)):
        assert np.array_equal(ctx.ntt(op, x), orc.domain_op(op, x)), f"op {op} n 2^{logn}"


@pytest.mark.parametrize("logn", [20, 22, 24])
def test_large_round_trips_and_spot_values(ctx, logn, rng):
    """Size-independent properties at the benchmark sizes: inverse pairs are
    identities, linearity holds, and sampled outputs equal the definition
    sum_i a_i w^(ij)."""
    n = 1 << logn
    x = O.random_fr(n, rng)
    f = ctx.ntt(0, x)
    assert np.array_equal(ctx.ntt(1, f), x)
    c = ctx.ntt(2, x)
    assert np.array_equal(ctx.ntt(3, c), x)
    # linearity: FFT(x + y) = FFT(x) + FFT(y) on a sample of coordinates
    y = O.random_fr(n, rng)
    fy = ctx.ntt(0, y)
    s = np.stack([O.fr_mont((O.fr_int(x[i]) + O.fr_int(y[i])) % O.R) for i in range(n)]) if logn <= 20 else None
    if s is not None:
        fs = ctx.ntt(0, s)
        for j in rng.integers(0, n, 8):
            assert O.fr_int(fs[j]) == (O.fr_int(f[j]) + O.fr_int(fy[j])) % O.R
    # definition at two sampled points (w = 5^((r-1)/2^28) squared down)
    w = pow(pow(5, (O.R - 1) >> 28, O.R), 1 << (28 - logn), O.R)
    xi = [O.fr_int(v) for v in x] if logn <= 20 else None
    if xi is not None:
        for j in (1, int(rng.integers(2, n))):
            wj = pow(w, j, O.R)
            acc, p = 0, 1
            for a in xi:
                acc = (acc + a * p) % O.R
                p = p * wj % O.R
            assert O.fr_int(f[j]) == acc


@pytest.mark.parametrize("logn", [16, 24])
def test_sparse_input_matches_definition_at_full_size(ctx, logn, rng):
    """FFT and cosetFFT of a vector with 48 nonzero coefficients, checked at sampled
    outputs against sum_i a_i w^(ij) (and a_i (g w^j)^i for the coset), any size."""
    n = 1 << logn
    x = np.zeros((n, 4), np.uint64)
    pos = rng.choice(n, 48, replace=False)
    x[pos] = O.random_fr(48, rng)
    w = pow(pow(5, (O.R - 1) >> 28, O.R), 1 << (28 - logn), O.R)
    nz = [(int(i), O.fr_int(x[i])) for i in pos]
    f, c = ctx.ntt(0, x), ctx.ntt(2, x)
    for j in [0, 1, n - 1] + [int(v) for v in rng.integers(0, n, 5)]:
        wj = pow(w, j, O.R)
        assert O.fr_int(f[j]) == sum(a * pow(wj, i, O.R) for i, a in nz) % O.R
        gw = 5 * wj % O.R
        assert O.fr_int(c[j]) == sum(a * pow(gw, i, O.R) for i, a in nz) % O.R


@pytest.mark.parametrize("logn", [4, 16, 20])
def test_device_entry_point_equals_host_entry_point(ctx, logn, rng):
    import torch
    n = 1 << logn
    x = O.random_fr(n, rng)
    xd = torch.from_numpy(x.view(np.int64).reshape(-1)).to("cuda:0")
    for op in range(5):
        work, out = xd.clone(), torch.empty_like(xd)
        stream = torch.cuda.current_stream().cuda_stream   # orders the op after the clone
        ms = ctx.ntt_device(op, work.data_ptr(), out.data_ptr(), n, stream_ptr=stream, timed=True)
        assert ms > 0
        got = out.cpu().numpy().view(np.uint64).reshape(n, 4)
        assert np.array_equal(got, ctx.ntt(op, x)), f"op {op}"


def test_device_entry_point_rejects_bad_buffers(ctx):
    import torch
    import nkr_b200 as nk
    n = 1 << 10
    xd = torch.zeros(4 * n * 2, dtype=torch.int64, device="cuda:0")
    with pytest.raises(nk.B200Error, match="overlap"):
        ctx.ntt_device(0, xd.data_ptr(), xd.data_ptr() + 64, n)
    host = np.zeros((n, 4), np.uint64)
    with pytest.raises(nk.B200Error, match="device memory"):
        ctx.ntt_device(0, host.ctypes.data, xd.data_ptr() + n * 32, n)
    with pytest.raises(nk.B200Error, match="power of two"):
        ctx.ntt_device(0, xd.data_ptr(), xd.data_ptr() + n * 32, 1000)


@pytest.mark.parametrize("logn", [10, 16, 20])
def test_tuned_tile_shape_is_in_range_and_exact(ctx, logn, rng):
    """The NTT tile tuner picks a shape from its candidate set; the transforms
    it drives stay bit-exact (inverse pairs are identities)."""
    n = 1 << logn
    stages, bpt = ctx.tune_ntt(n)
    if logn < 14:
        assert (stages, bpt) == (10, 1)
    else:
        assert 7 <= stages <= 10 and bpt in (1, 2, 4)
    x = O.random_fr(n, rng)
    assert np.array_equal(ctx.ntt(1, ctx.ntt(0, x)), x)
    assert np.array_equal(ctx.ntt(3, ctx.ntt(2, x)), x)
