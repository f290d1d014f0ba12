"""nkr_b200_ntt_noalloc: the domain ops on device buffers with no device allocation
(scratch in a fixed array inside the library).  Its outputs must equal those of
nkr_b200_ntt, the allocating entry point, for every op, on calls made back to back
on one stream, in place and out of place.  The file name sorts last so the GPU
test also runs after every other test of a full session."""
import ctypes

import numpy as np
import pytest

import nkr_b200 as nk
import oracle as O

SIZES = [1, 5, 10, 11, 16]  # log2 n: one pass, two passes (11), the maximum (16)


def _status(op, n, in_ptr=1, out_ptr=1):
    return nk.lib().nkr_b200_ntt_noalloc(0, op, ctypes.c_void_p(in_ptr), ctypes.c_void_p(out_ptr),
                                         n, None)


def test_rejects_bad_arguments_before_touching_a_device():
    for n in (nk.NTT_NOALLOC_MAX * 2, 1 << 28, 0, 1, 3, 1000):
        assert _status(0, n) == nk.EINVAL, n
    msg = nk.lib().nkr_b200_last_error().decode()
    assert "power of two in [2, 65536]" in msg
    assert _status(5, 16) == nk.EINVAL
    assert _status(0, 16, in_ptr=0) == nk.EINVAL


@pytest.mark.gpu
def test_matches_allocating_ntt_on_consecutive_calls(ctx):
    import torch

    dev = torch.device("cuda:0")
    stream = torch.cuda.current_stream(dev)
    rng = np.random.default_rng(2024)
    cases = []
    for logn in SIZES:
        n = 1 << logn
        for op in range(5):
            xs = [O.random_fr(n, rng) for _ in range(2)]
            want = [ctx.ntt(op, x) for x in xs]  # the allocating entry point
            dins = [torch.from_numpy(x.view(np.int64).copy()).to(dev) for x in xs]
            douts = [torch.zeros_like(d) for d in dins]
            cases.append((logn, op, want, dins, douts))
    torch.cuda.synchronize()

    def run_all(in_place):
        for logn, op, want, dins, douts in cases:
            for d_in, d_out in zip(dins, douts):
                if in_place:
                    d_out.copy_(d_in)
                src = d_out if in_place else d_in
                nk.ntt_noalloc(0, op, src.data_ptr(), d_out.data_ptr(), 1 << logn,
                               stream.cuda_stream)
        torch.cuda.synchronize()
        for logn, op, want, dins, douts in cases:
            for k, (w, d_out) in enumerate(zip(want, douts)):
                got = d_out.cpu().numpy().view(np.uint64).reshape(-1, 4)
                assert np.array_equal(got, w), f"op {op} n 2^{logn} call {k} in_place={in_place}"

    run_all(False)  # first use on the device: builds the scratch tables
    free_before = torch.cuda.mem_get_info(dev)[0]
    run_all(False)
    run_all(True)
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info(dev)[0] == free_before, "device memory changed across calls"


@pytest.mark.gpu
def test_rejects_oversize_and_host_buffers_on_gpu(ctx):
    import torch

    n = nk.NTT_NOALLOC_MAX * 2
    d = torch.zeros(n * 4, dtype=torch.int64, device="cuda:0")
    with pytest.raises(nk.B200Error, match="power of two"):
        nk.ntt_noalloc(0, 0, d.data_ptr(), d.data_ptr(), n)
    host = np.zeros((16, 4), np.uint64)
    with pytest.raises(nk.B200Error, match="device memory"):
        nk.ntt_noalloc(0, 0, host.ctypes.data, d.data_ptr(), 16)
    torch.cuda.synchronize()
