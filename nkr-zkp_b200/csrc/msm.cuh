// Pippenger multi-scalar multiplication on G1 and G2.
//
// Reference: libff BDLO12 on the CPU (libff/algebra/scalar_multiplication/
// multiexp.tcc:165-282) and the CUDA BucketContext/MSMContext path
// (operators/cuda/include/fields/bucket.cuh:15-142, msm/msm.cuh:12-123,
// msm/msm_kernel.cuh:12-168).  The result is a canonical group element, so any
// correct bucket order is bit-exact after affine normalisation.
//
// Steps (all on the device, no host round trip):
//  1. sort: each scalar leaves Montgomery form and is cut into W signed c-bit
//     digits d in [-2^(c-1), 2^(c-1)]; bucket |d| - 1 receives the point
//     (negated when d < 0).  Counts are histogrammed with warp-aggregated
//     atomics, an exclusive scan gives bucket offsets, and a scatter writes
//     (point, sign) entries in bucket order.  The sort depends only on the scalars and the
//     window shape, so MSMs over the same scalars share one sort (the three G1
//     witness MSMs of a prove; the reference shares it too, bucket.cuh:50-141).
//  2. accumulation: thread t sums the fixed segment of K1 sorted entries
//     [t K1, (t+1) K1) into XYZZ accumulators (mixed add 8M + 2S, with the
//     doubling branch), one run per bucket it crosses, so all lanes do equal
//     work whatever the bucket sizes.  A bucket spread over several segments
//     leaves one partial per segment and is finished by fix-up levels of fan-in
//     K2: each level scans, per bucket, how many groups of K2 pieces remain and
//     gives every group its own thread, so a bucket holding a large share of all
//     points (repeated or small scalars) costs O(log n) sequential additions.
//  3. bucket reduction: sum_b (b + 1) S_b in levels of 256 (G1) / 128 (G2)
//     items per block: a shared-memory suffix scan and tree sums make a level
//     about 2 log2(block) dependent additions deep.
//  4. windows: with resident "folded" bases the W windows share one bucket set
//     because the bases hold the copies 2^(c k) P_i (built once at prepare; HBM
//     is large); otherwise each window has its own set and a Horner pass
//     combines them.
//  5. output: Jacobian coordinates in the libff layout (X, Y, Z) with an
//     arbitrary Z -- no device inversion on the critical path; the host
//     normalises the few result points.
//  6. support: the witness MSMs' bases are the proving key's queries, and a
//     query point is the point at infinity for every variable absent from that
//     matrix (about 2/3 of the B query in hash circuits).  Resident bases keep
//     only the finite points and their indices; the sort gathers the scalars
//     through those indices, so no entry, lane or bucket is spent on a point
//     that adds nothing.
#pragma once

#include <cstdint>
#include <vector>

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
    // entries per level-1 segment (mixed additions per thread).  Measured slower
    // at 2^16 points: 8 or 16 (level 1 shorter, fix-ups and the first reduction
    // level longer); at 2^20: 32-48 sized to whole waves of the kernel (prove
    // 18.60 -> 18.79 ms)
    int k1 = 32;
    int k2 = 16;     // fan-in of the fix-up levels (8 and 4 measured no faster in a prove)
    uint64_t entries_max() const { return uint64_t(W) * n; }
    uint64_t segments_max() const { return (entries_max() + k1 - 1) / k1; }
    bool same_sort(const MsmShape &o) const
    {
        return n == o.n && c == o.c && W == o.W && folded == o.folded && k1 == o.k1;
    }
};

MsmShape msm_shape(uint64_t n, bool folded, int group, int c_override = 0);

// Digit sort of one scalar vector: bucket offsets and entries in bucket order.
struct MsmSort {
    DevBuf canon, counts, offsets, cursor, entries, scan_tmp;
    size_t device_bytes() const
    {
        return canon.bytes + counts.bytes + offsets.bytes + cursor.bytes + entries.bytes +
               scan_tmp.bytes;
    }
};

// Accumulation state of one MSM (partials, buckets, reduction levels, result).
struct MsmAcc {
    DevBuf partials, buckets, lead_off, red_a, red_r, red_a2, red_r2, scan_tmp, result;
    // record events at the phase boundaries: before and after the level-1
    // accumulation kernel, after the fix-up levels, after the first reduction
    // level, after the last reduction level and the final combination
    bool timing = false;
    cudaEvent_t ev_acc[5] = {};
    // added to the first reduction level's log2 buckets per thread (set before
    // msm_acc_alloc): larger levels do less work in more dependent steps
    int first_level_bias = 0;
    // G2 reduction levels on lane pairs (two lanes per item): shorter for an MSM
    // alone, but inside a prove the wider blocks crowd out the other MSMs' work
    bool lane_pairs = false;
    size_t device_bytes() const
    {
        return partials.bytes + buckets.bytes + lead_off.bytes + red_a.bytes + red_r.bytes +
               red_a2.bytes + red_r2.bytes + scan_tmp.bytes + result.bytes;
    }
};

struct MsmScratch {
    MsmSort sort;
    MsmAcc acc;
    size_t device_bytes() const { return sort.device_bytes() + acc.device_bytes(); }
};

// Resident bases for one MSM: affine points, folded into W window copies when
// shape.folded (point k*n + i = 2^(c k) P_i).
struct MsmBases {
    int group = 1; // 1: G1, 2: G2
    MsmShape shape;
    DevBuf pts;
    // support form (msm_bases_build_support): pts holds only the finite points;
    // support[i] is point i's index among the n_full original bases
    DevBuf support;
    std::vector<uint32_t> support_host;
    uint64_t n_full = 0;
    const uint32_t *gather() const { return support.p ? support.as<uint32_t>() : nullptr; }
    size_t device_bytes() const { return pts.bytes + support.bytes; }
};

// Upload bases given in libff Jacobian layout (96 / 192 B per point) from host
// or device memory, normalise to affine and, if folded, build the window copies.
// With bitrev, point i is stored at position bitrev(i) (n a power of two), so
// scalars held in bit-reversed order pair with their own bases.
int msm_bases_build(MsmBases &b, int group, const void *jac, bool jac_on_device, uint64_t n,
                    bool folded, int c_override, bool bitrev, cudaStream_t st);
// Indices of the finite points among n host bases (libff Jacobian, Z = 0 is
// infinity); one index (0) when all n are infinite.
std::vector<uint32_t> msm_support(int group, const void *jac_host, uint64_t n);
// Resident bases of the points idx (from msm_support) of n host bases; the
// scalars of this MSM are indexed by original point index through gather().
int msm_bases_build_support(MsmBases &b, int group, const void *jac_host, uint64_t n,
                            std::vector<uint32_t> idx, bool folded, int c_override, cudaStream_t st);

// Normalise n libff-layout Jacobian points (device) into affine (device).
int jacobian_to_affine(int group, const void *jac, void *aff, uint64_t n, cudaStream_t st);

int msm_sort_alloc(MsmSort &s, const MsmShape &shape);
int msm_acc_alloc(MsmAcc &a, int group, const MsmShape &shape);
int msm_scratch_alloc(MsmScratch &s, int group, const MsmShape &shape);

// Sort the scalars Fr[n] (Montgomery, device) for the shape.
// scalar i of the sort is scalars_dev[gather ? gather[i] : i]; with class_of, a
// scalar whose variable belongs to a class (class_of[v] != kNoClass, MsmDedup
// below) counts as zero (the class path adds it)
int msm_sort_run(const MsmShape &shape, MsmSort &s, const void *scalars_dev, cudaStream_t st,
                 const uint32_t *gather = nullptr, const uint32_t *class_of = nullptr);
// Accumulate / reduce with a finished sort of the same shape.  The result is
// written to out_dev in libff Jacobian layout with an arbitrary Z (or Z = 0 for
// infinity); normalise on the host (host/fr_host.hpp normalize_g1 / _g2).
int msm_acc_run(const MsmBases &b, const MsmSort &s, MsmAcc &a, void *out_dev, cudaStream_t st);
int msm_run(const MsmBases &b, MsmScratch &s, const void *scalars_dev, void *out_dev,
            cudaStream_t st);

// msm_acc_run in two parts, so that the level-1 accumulation of several MSMs of
// one group (a batch of proofs) can run as one launch over a work list: the
// level-1 kernel, then the fix-up levels, bucket reduction and final combination.
struct MsmAccJob {
    const MsmBases *bases;
    const MsmSort *sort;
    MsmAcc *acc;
};
constexpr size_t kMsmAccItemBytes = 64; // scratch per job of msm_acc_level1_list
// items_host (pinned) and items_dev: n kMsmAccItemBytes items each; the host
// items are read by the stream's copy
int msm_acc_level1_list(int group, const MsmAccJob *jobs, int n, void *items_host, void *items_dev,
                        cudaStream_t st);
int msm_acc_tail(const MsmBases &b, const MsmSort &s, MsmAcc &a, void *out_dev, cudaStream_t st);
// the level-1 kernel of msm_acc_run alone (msm_acc_tail finishes the MSM)
int msm_acc_level1(const MsmBases &b, const MsmSort &s, MsmAcc &a, cudaStream_t st);

// ---------------------------------------------------------------------------
// Repeated scalars.  A witness repeats values (constant wires, the same wire of
// every copy of a gadget: the 2^20-constraint Poseidon benchmark holds 899 K
// nonzero values of which 169 K are distinct, 829 values covering 731 K
// variables).  With classes c of variables of equal value v_c,
//     sum_i w_i P_i = sum_{i in no class} w_i P_i + sum_c v_c S_c,
//     S_c = sum_{i in c} P_i,
// so a class member costs one point addition into S_c instead of W entries of
// the digit sort; a small MSM over the classes adds the second sum.  The split is
// exact for any partition into classes of equal values, so a witness without
// repetition only pays the class-finding pass.
// ---------------------------------------------------------------------------
constexpr uint32_t kNoClass = 0xffffffffu;
constexpr uint32_t kClassMax = 4096; // classes per prove; further repeated values stay singletons
constexpr uint32_t kClassMin = 4;    // members of the smallest class (a class costs W' small-MSM entries)

// Classes of one witness (per prove slot).  A hash table of variable indices
// (linear probing on a hash of the value, full-value comparison) gives every
// nonzero value a representative; representatives with at least kClassMin
// members take class ids.
struct MsmDedup {
    DevBuf table, rep, csize, cid, class_of, values, nclass;
    uint64_t cols = 0, slots = 0;
    size_t device_bytes() const
    {
        return table.bytes + rep.bytes + csize.bytes + cid.bytes + class_of.bytes + values.bytes +
               nclass.bytes;
    }
};
int msm_dedup_alloc(MsmDedup &d, uint64_t cols);
// z: Fr[cols] (Montgomery, device).  Afterwards class_of[v] is variable v's class
// (kNoClass for zeros and singletons) and values[c] the value of class c (zero
// for unused ids).
int msm_dedup_run(MsmDedup &d, const void *z, cudaStream_t st);

// The class members of one support (n points, gather as for msm_sort_run) in
// class order: offsets[c] .. offsets[c + 1] index entries, which hold point
// indices.
struct MsmClassSort {
    DevBuf counts, offsets, cursor, entries, scan_tmp;
    uint64_t n = 0;
    size_t device_bytes() const
    {
        return counts.bytes + offsets.bytes + cursor.bytes + entries.bytes + scan_tmp.bytes;
    }
};
int msm_class_sort_alloc(MsmClassSort &s, uint64_t n);
int msm_class_sort_run(MsmClassSort &s, const MsmDedup &d, const uint32_t *gather, cudaStream_t st);

// One MSM's class path: the class sums S_c (summed like buckets: fixed segments,
// fix-up levels), normalised to affine as the bases of a small MSM over the
// class values.
struct MsmClassAcc {
    MsmShape seg;      // n = the support's points, nb = kClassMax classes, k1, k2
    DevBuf partials, buckets, lead_off, scan_tmp;
    MsmBases small;    // the class sums (affine; G2: and their psi images), non-folded
    MsmScratch small_s;
    DevBuf split;      // G2: the class values as k0 + k1 lambda (msm.cu)
    DevBuf out;        // sum_c v_c S_c, libff Jacobian layout
    size_t device_bytes() const
    {
        return partials.bytes + buckets.bytes + lead_off.bytes + scan_tmp.bytes + small.device_bytes() +
               small_s.device_bytes() + split.bytes + out.bytes;
    }
};
int msm_class_acc_alloc(MsmClassAcc &a, int group, uint64_t n);
// Class sums over bases b (its first n points: 2^0 window copies), the MSM over
// the classes, and out_dev (the MSM's result, libff Jacobian) += that sum.
int msm_class_acc_run(const MsmBases &b, const MsmClassSort &cs, const MsmDedup &d, MsmClassAcc &a,
                      void *out_dev, cudaStream_t st);
// the class-path part of msm_class_acc_run without the final addition (a.out
// holds sum_c v_c S_c), and the addition alone
int msm_class_acc_issue(const MsmBases &b, const MsmClassSort &cs, const MsmDedup &d, MsmClassAcc &a,
                        cudaStream_t st);
int msm_result_add(int group, void *out_dev, const void *add_dev, cudaStream_t st);

} // namespace nkr
