// Pippenger multi-scalar multiplication on G1 and G2.
//
// Reference: libff BDLO12 on the CPU (libff/algebra/scalar_multiplication/
// multiexp.tcc:165-282) and the CUDA BucketContext/MSMContext path
// (operators/cuda/include/fields/bucket.cuh:15-142, msm/msm.cuh:12-123,
// msm/msm_kernel.cuh:12-168).  The result is a canonical group element, so any
// correct bucket order is bit-exact after affine normalisation.
//
// Steps (all on the device, no host round trip):
//  1. digits: each scalar leaves Montgomery form and is cut into W signed c-bit
//     digits d in [-2^(c-1), 2^(c-1)]; bucket |d| - 1 receives the point
//     (negated when d < 0).  Counts are histogrammed with warp-aggregated atomics.
//  2. counting sort: exclusive scans give bucket offsets and, per bucket,
//     ceil(count / K1) accumulation tasks; a scatter writes (point, sign) entries.
//  3. accumulation: one thread per task sums up to K1 affine points into an XYZZ
//     accumulator (mixed add 8M + 2S, with the doubling branch).  Buckets split
//     over several tasks are finished by in-place tree levels of fan-in K2, so a
//     bucket holding a large share of all points (repeated or small scalars)
//     costs O(log n) sequential adds instead of O(n).
//  4. bucket reduction: sum_b (b + 1) S_b by chunked running sums in log levels.
//  5. windows: with resident "folded" bases the W windows share one bucket set
//     because the bases hold the copies 2^(c k) P_i (built once at prepare, HBM
//     is large); otherwise each window has its own set and a Horner pass combines
//     them.
#pragma once

#include <cstdint>

#include "common.cuh"
#include "curve.cuh"

namespace nkr {

struct MsmShape {
    uint64_t n = 0; // points
    int c = 0;      // window bits
    int W = 0;      // windows: W * c >= 255
    bool folded = false;
    uint32_t B = 0;  // buckets per set: 2^(c-1)
    uint32_t nb = 0; // total buckets: folded ? B : W * B
    int k1 = 32;     // points per accumulation task
    int k2 = 8;      // fan-in of the fix-up levels
    uint64_t entries_max() const { return uint64_t(W) * n; }
    uint64_t tasks_max() const { return (entries_max() + k1 - 1) / k1 + nb; }
};

MsmShape msm_shape(uint64_t n, bool folded, int group, int c_override = 0);

// Per-MSM device scratch, sized for a shape and reusable across calls.
struct MsmScratch {
    DevBuf canon, counts, offsets, cursor, task_off, entries, task_bucket, partials, buckets;
    DevBuf red_a, red_r, red_a2, red_r2, scan_tmp, result;
    bool timing = false;            // record events around the level-1 accumulation kernel
    cudaEvent_t ev_acc[2] = {nullptr, nullptr};
    size_t device_bytes() const
    {
        return canon.bytes + counts.bytes + offsets.bytes + cursor.bytes + task_off.bytes +
               entries.bytes + task_bucket.bytes + partials.bytes + buckets.bytes + red_a.bytes +
               red_r.bytes + red_a2.bytes + red_r2.bytes + scan_tmp.bytes + result.bytes;
    }
};

// Resident bases for one MSM: affine points, folded into W window copies when
// shape.folded (point k*n + i = 2^(c k) P_i).
struct MsmBases {
    int group = 1; // 1: G1, 2: G2
    MsmShape shape;
    DevBuf pts;
    size_t device_bytes() const { return pts.bytes; }
};

// Upload bases given in libff Jacobian layout (96 / 192 B per point) from host
// or device memory, normalise to affine and, if folded, build the window copies.
// With bitrev, point i is stored at position bitrev(i) (n a power of two), so
// scalars held in bit-reversed order pair with their own bases.
int msm_bases_build(MsmBases &b, int group, const void *jac, bool jac_on_device, uint64_t n,
                    bool folded, int c_override, bool bitrev, cudaStream_t st);

// Normalise n libff-layout Jacobian points (device) into affine (device).
int jacobian_to_affine(int group, const void *jac, void *aff, uint64_t n, cudaStream_t st);

int msm_scratch_alloc(MsmScratch &s, int group, const MsmShape &shape);

// Run one MSM: scalars Fr[n] (Montgomery, device).  The affine result is written
// to out_dev in libff Jacobian layout (Z = 1, or (0, 1, 0) for infinity).
int msm_run(const MsmBases &b, MsmScratch &s, const void *scalars_dev, void *out_dev,
            cudaStream_t st);

} // namespace nkr
