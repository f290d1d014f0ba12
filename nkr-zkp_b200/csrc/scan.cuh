// Device-wide exclusive prefix sum of u32 values (three kernels: block totals,
// scan of the totals, block scans plus offsets).  The input is read through a
// functor so callers can scan a derived quantity (e.g. ceil(count / K)) without
// materialising it.  out has n + 1 entries; out[n] is the total.
#pragma once

#include <cstdint>

#include "common.cuh"

namespace nkr {

constexpr int kScanThreads = 1024;
constexpr int kScanItems = 4;
constexpr int kScanTile = kScanThreads * kScanItems;

__device__ __forceinline__ uint32_t warp_incl_scan(uint32_t v)
{
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, v, d);
        if (lane >= d) v += y;
    }
    return v;
}

// Exclusive scan of one value per thread across the block; returns the
// exclusive prefix and writes the block total to *total.
__device__ __forceinline__ uint32_t block_excl_scan(uint32_t v, uint32_t *total)
{
    __shared__ uint32_t warp_sums[32];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const uint32_t incl = warp_incl_scan(v);
    if (lane == 31) warp_sums[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        const int nw = blockDim.x >> 5;
        uint32_t s = lane < nw ? warp_sums[lane] : 0;
        s = warp_incl_scan(s);
        warp_sums[lane] = s;
    }
    __syncthreads();
    const uint32_t before = warp ? warp_sums[warp - 1] : 0;
    *total = warp_sums[(blockDim.x >> 5) - 1];
    __syncthreads();
    return before + incl - v;
}

template <class Load>
__global__ void __launch_bounds__(kScanThreads) k_scan_totals(Load load, uint64_t n,
                                                               uint32_t *block_totals)
{
    const uint64_t base = uint64_t(blockIdx.x) * kScanTile + uint64_t(threadIdx.x) * kScanItems;
    uint32_t s = 0;
#pragma unroll
    for (int i = 0; i < kScanItems; ++i)
        if (base + i < n) s += load(base + i);
    uint32_t total;
    block_excl_scan(s, &total);
    if (threadIdx.x == 0) block_totals[blockIdx.x] = total;
}

// single block: exclusive scan of nb <= kScanTile block totals, in place
__global__ void __launch_bounds__(kScanThreads) k_scan_block_totals(uint32_t *totals, uint32_t nb);

template <class Load>
__global__ void __launch_bounds__(kScanThreads) k_scan_apply(Load load, uint64_t n,
                                                              const uint32_t *block_offsets,
                                                              uint32_t *out)
{
    const uint64_t base = uint64_t(blockIdx.x) * kScanTile + uint64_t(threadIdx.x) * kScanItems;
    uint32_t v[kScanItems];
    uint32_t s = 0;
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
        v[i] = base + i < n ? load(base + i) : 0;
        s += v[i];
    }
    uint32_t total;
    uint32_t run = block_excl_scan(s, &total) + block_offsets[blockIdx.x];
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
        if (base + i < n) out[base + i] = run;
        run += v[i];
    }
    if (blockIdx.x == gridDim.x - 1 && threadIdx.x == blockDim.x - 1) out[n] = run;
}

// Scratch for a scan of up to n elements: number of u32 block totals.
inline uint64_t scan_scratch_words(uint64_t n) { return (n + kScanTile - 1) / kScanTile + 1; }

template <class Load>
int scan_exclusive(Load load, uint64_t n, uint32_t *out, uint32_t *scratch, cudaStream_t st)
{
    const uint32_t nb = static_cast<uint32_t>((n + kScanTile - 1) / kScanTile);
    if (nb == 0) {
        NKR_CUDA(cudaMemsetAsync(out, 0, sizeof(uint32_t), st));
        return NKR_B200_OK;
    }
    NKR_REQUIRE(nb <= uint32_t(kScanTile), "scan of %llu elements exceeds the two-level limit",
                (unsigned long long)n);
    k_scan_totals<<<nb, kScanThreads, 0, st>>>(load, n, scratch);
    NKR_CHECK_LAUNCH();
    k_scan_block_totals<<<1, kScanThreads, 0, st>>>(scratch, nb);
    NKR_CHECK_LAUNCH();
    k_scan_apply<<<nb, kScanThreads, 0, st>>>(load, n, scratch, out);
    NKR_CHECK_LAUNCH();
    return NKR_B200_OK;
}

struct LoadU32 {
    const uint32_t *p;
    __device__ __forceinline__ uint32_t operator()(uint64_t i) const { return p[i]; }
};

} // namespace nkr
