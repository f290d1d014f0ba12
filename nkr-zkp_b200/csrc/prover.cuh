// Prepared Groth16 key (circuit + proving key resident in HBM) and the prove
// orchestration.  Reference: CudaBackend::prepare / ::prove
// (protocols/groth16/backends/cuda/src/groth16_backend.cu:214-279) and the CPU
// backend's prove (backends/cpu/src/backend.cpp:156-201).
//
// Streams: after the witness upload and the SpMV, the four witness MSMs
// (a, b_g1, l on G1 and b_g2 on G2) run on their own streams while the main
// stream computes H (7 transforms) and then the H MSM; the reference runs every
// stage serially with a device sync after each.
#pragma once

#include <cstdint>

#include "common.cuh"
#include "field.cuh"
#include "msm.cuh"
#include "ntt.cuh"
#include "spmv.cuh"

struct nkr_b200_ctx {
    int device = 0;
    int sm_count = 0;
    cudaStream_t stream = nullptr; // operator-level calls
};

namespace nkr {

enum { kMsmA = 0, kMsmB1 = 1, kMsmL = 2, kMsmH = 3, kMsmB2 = 4, kNumMsm = 5 };

} // namespace nkr

struct nkr_b200_key {
    nkr_b200_ctx *ctx = nullptr;
    uint64_t rows = 0, cols = 0, public_inputs = 0;
    int logn = 0;
    nkr::CsrDevice mat[3];
    nkr::NttTables ntt;
    nkr::MsmBases bases[nkr::kNumMsm];
    // digit sorts of the witness: one per distinct support among the 4 witness MSMs
    // (B1 and B2 always share one); sort g runs on the stream of MSM sort_stream[g]
    nkr::MsmSort sort_w[4];
    int n_sorts = 0;
    int sort_of[nkr::kNumMsm] = {};
    int sort_stream[4] = {};
    nkr::MsmSort sort_h;               // digit sort of H
    nkr::MsmAcc acc[nkr::kNumMsm];
    nkr::DevBuf z, az, bz, cz, h;
    nkr::DevBuf out;      // 4 G1 + 1 G2 results, libff Jacobian layout (96 * 4 + 192 B)
    nkr::DevBuf pk_const; // alpha_g1, beta_g1, delta_g1 (G1 affine) and beta_g2, delta_g2 (G2 affine)
    nkr::DevBuf blind_io; // r, s in; proof out
    cudaStream_t st[nkr::kNumMsm] = {};
    cudaEvent_t ev_z = nullptr, ev_sorted[4] = {}, ev_done[nkr::kNumMsm] = {};
    cudaEvent_t ev_t[5] = {};
    void *pinned_in = nullptr;  // witness staging (cols * 32 B)
    void *pinned_out = nullptr; // results staging (576 B + proof)
    nkr_b200_stage_times times{};
    bool have_times = false;
};

namespace nkr {

// Issue one full prove on the key's streams, witness already in key->z.
// Results land in key->out (device, Jacobian with arbitrary Z).  No host
// synchronisation.
int prove_issue(nkr_b200_key *key, bool timed);

// Affine-normalise the 4 G1 + 1 G2 result points (576 B, libff layout) in place.
void normalize_raw(void *raw576);

} // namespace nkr
