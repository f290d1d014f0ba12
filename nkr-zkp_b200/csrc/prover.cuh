// Prepared Groth16 key (circuit + proving key resident in HBM) and the prove
// orchestration.  Reference: CudaBackend::prepare / ::prove
// (protocols/groth16/backends/cuda/src/groth16_backend.cu:214-279) and the CPU
// backend's prove (backends/cpu/src/backend.cpp:156-201).
//
// A key holds what every proof of the circuit reads (CSR matrices, NTT tables,
// folded MSM bases) once.  Everything one proof writes lives in a prove slot:
// witness and quotient vectors, digit sorts, bucket scratch, result points,
// five streams and their events, and a CUDA graph of the whole prove.  Slot 0
// serves nkr_b200_prove; batches and the request server add slots so several
// proofs of one key are in flight at once.
//
// Streams of a slot: after the witness upload and the SpMV, the four witness
// MSMs (a, b_g1, l on G1 and b_g2 on G2) run on their own streams while the
// main stream computes H (7 transforms) and then the H MSM; the reference runs
// every stage serially with a device sync after each.  The witness's repeated
// values are found once per prove, and each witness MSM sums the bases of every
// class of equal values on a class stream of higher priority (msm.cuh).
#pragma once

#include <cstdint>
#include <memory>
#include <vector>

#include "common.cuh"
#include "field.cuh"
#include "msm.cuh"
#include "ntt.cuh"
#include "spmv.cuh"

struct nkr_b200_ctx {
    int device = 0;
    int sm_count = 0;
    cudaStream_t stream = nullptr; // operator-level calls
    // MSM window autotuner: measured best window bits per log2 point count
    // (0 = not measured yet); off: the cost model of msm_shape decides
    bool autotune = true;
    int msm_window[33] = {};
    float msm_window_ms[33] = {};
};

namespace nkr {
// Window bits for an MSM of n points: measured once per power-of-two size class
// on this device when autotuning is on (synthetic bases, uniform scalars),
// else 0 (the cost model).  Sizes above 2^22 take the 2^22 offset from the model.
int tuned_window_bits(nkr_b200_ctx *ctx, uint64_t n, int *c);
} // namespace nkr

namespace nkr {

enum { kMsmA = 0, kMsmB1 = 1, kMsmL = 2, kMsmH = 3, kMsmB2 = 4, kNumMsm = 5 };
constexpr size_t kOutBytes = 4 * 96 + 192; // ar, bs1, zk, qz (G1) + bs2 (G2), libff layout
constexpr size_t kBlindStage = 1280;       // pinned staging of one blinding, after the results

struct ProveSlot {
    MsmSort sort_w[4]; // witness digit sorts, one per distinct support
    MsmSort sort_h;    // digit sort of H
    MsmAcc acc[kNumMsm];
    // repeated witness values (msm.cuh): the witness's classes, and each
    // class-path MSM's class members, class sums and small MSM
    MsmDedup dedup;
    MsmClassSort csort[kNumMsm];
    MsmClassAcc cacc[kNumMsm];
    cudaStream_t cls[kNumMsm] = {}; // class-path streams (class sums, MSM over the classes)
    cudaEvent_t ev_dedup = nullptr, ev_cls[kNumMsm] = {};
    DevBuf z, az, bz, cz, h;
    DevBuf spmv_prod[3]; // SpMV products of the non-unit terms, per matrix
    DevBuf out; // 4 G1 + 1 G2 results, libff Jacobian layout (kOutBytes)
    DevBuf glv_tab; // slot 0: ar and bs1 of its last prove, tabulated for blinding (blind.cu)
    cudaStream_t st[kNumMsm] = {};
    // higher-priority streams: each MSM's fix-up and reduction levels (tail[k]),
    // and the quotient chain with the H digit sort (chain)
    cudaStream_t tail[kNumMsm] = {};
    cudaStream_t chain = nullptr;
    cudaEvent_t ev_l1[kNumMsm] = {}, ev_hsorted = nullptr;
    cudaEvent_t ev_z = nullptr, ev_sorted[4] = {}, ev_done[kNumMsm] = {};
    cudaEvent_t ev_t[5] = {};
    cudaEvent_t ev_msm_end[kNumMsm] = {}; // timed proves: each MSM's end on its stream
    // the prove as a graph (witness already in z); kernels launched per replay
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t graph_exec = nullptr;
    unsigned long long graph_kernels = 0;
    // pinned staging: witness double buffer (pageable inputs) and results
    void *pinned_wit[2] = {nullptr, nullptr};
    cudaEvent_t ev_wit[2] = {nullptr, nullptr};
    int wit_next = 0;
    void *pinned_out = nullptr; // kOutBytes + kBlindStage (blinding)
    cudaStream_t main() const { return st[kMsmH]; }
    ~ProveSlot();
};

} // namespace nkr

struct nkr_b200_key {
    nkr_b200_ctx *ctx = nullptr;
    uint64_t rows = 0, cols = 0, public_inputs = 0;
    int logn = 0;
    nkr::CsrDevice mat[3];
    nkr::NttTables ntt;
    nkr::MsmBases bases[nkr::kNumMsm];
    // witness MSMs with identical supports share a digit sort: MSM k uses sort
    // sort_of[k], which runs on the stream of MSM sort_stream[g]
    int n_sorts = 0;
    int sort_of[nkr::kNumMsm] = {};
    int sort_stream[4] = {};
    // the witness MSMs take repeated witness values through the class path (their
    // sorts leave class members out)
    bool classes[nkr::kNumMsm] = {};
    nkr::DevBuf pk_const; // alpha_g1, beta_g1, delta_g1 (G1 affine) and beta_g2, delta_g2 (G2 affine)
    nkr::DevBuf blind_io;  // raw proof and scalars in, proof out (blind.cu)
    nkr::DevBuf blind_tab; // fixed-base tables of alpha1, beta1, delta1 (G1) and delta2 (G2)
    std::vector<std::unique_ptr<nkr::ProveSlot>> slots; // slots[0]: nkr_b200_prove
    uint64_t slot_bytes = 0;                            // device bytes of one slot
    nkr_b200_stage_times times{};
    bool have_times = false;
};

namespace nkr {

// Adds one prove slot to the key (device buffers, streams, pinned staging).
int slot_add(nkr_b200_key *key);
// Issue one full prove on a slot's streams, witness already in slot->z.
// Results land in slot->out (device, Jacobian with arbitrary Z).  No host
// synchronisation; with timed, events bracket the stages on the main stream;
// with blind_tables (slot 0, nkr_b200_prove) the slot's GLV tables of ar and bs1
// are computed for a following blinding (the captured graphs of batches and the
// server leave them out).
int prove_issue(nkr_b200_key *key, ProveSlot *slot, bool timed, bool blind_tables);
// Captures prove_issue into the slot's graph (once).
int slot_capture(nkr_b200_key *key, ProveSlot *slot);
// Queues the witness upload (device, pinned or pageable host memory) on the
// slot's main stream; pageable input goes through the slot's pinned double buffer.
int slot_upload_witness(nkr_b200_key *key, ProveSlot *slot, const void *witness);
// Replays the slot's graph on its main stream.
// Replays the slot's captured prove graph into `launch` (default: the slot's main
// stream); the graph's kernels run at that stream's priority.
int slot_launch(ProveSlot *slot, cudaStream_t launch = nullptr);
// Blinding buffers and the fixed-base tables of the key's alpha1, beta1, delta1
// and delta2 (pk_const already resident); synchronises st.
int blind_tables_build(nkr_b200_key *key, cudaStream_t st);
// Device bytes of a slot's GLV tables, and their computation from the slot's
// ar and bs1 (queued on st once both MSMs are final).
size_t glv_tables_bytes();
int glv_tables_issue(ProveSlot *slot, cudaStream_t st);
// Affine-normalise the 4 G1 + 1 G2 result points (576 B, libff layout) in place.
void normalize_raw(void *raw576);
void raw_from_bytes(const void *raw576, nkr_b200_raw_proof *res);

} // namespace nkr
