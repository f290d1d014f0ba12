// Groth16 prepare / prove orchestration on one B200 (design notes in
// prover.cuh); the blinding kernels live in blind.cu, verification in verify.cu.
#include <algorithm>
#include <cstring>
#include <vector>

#include "../host/fr_host.hpp"
#include "prover.cuh"

namespace nkr {

namespace {

constexpr size_t kOutOffset[kNumMsm] = {0, 96, 192, 288, 384}; // A, B1, L, H, B2
// issue order of the witness MSMs: the G2 MSM (longest) first
constexpr int kWitnessOrder[4] = {kMsmB2, kMsmA, kMsmB1, kMsmL};

} // namespace

void normalize_raw(void *raw576)
{
    uint8_t *o = static_cast<uint8_t *>(raw576);
    for (int i = 0; i < 4; ++i) host::normalize_g1(o + 96 * i);
    host::normalize_g2(o + 384);
}

void raw_from_bytes(const void *raw576, nkr_b200_raw_proof *res)
{
    const uint8_t *o = static_cast<const uint8_t *>(raw576);
    std::memcpy(res->ar, o + 0, 96);
    std::memcpy(res->bs1, o + 96, 96);
    std::memcpy(res->zk, o + 192, 96);
    std::memcpy(res->qz, o + 288, 96);
    std::memcpy(res->bs2, o + 384, 192);
}

namespace {

cudaMemcpyKind copy_kind_from(const void *p)
{
    cudaPointerAttributes attr{};
    if (cudaPointerGetAttributes(&attr, p) != cudaSuccess) {
        cudaGetLastError();
        return cudaMemcpyHostToDevice;
    }
    return attr.type == cudaMemoryTypeDevice || attr.type == cudaMemoryTypeManaged
               ? cudaMemcpyDeviceToDevice
               : cudaMemcpyHostToDevice;
}

bool is_pageable(const void *p)
{
    cudaPointerAttributes attr{};
    if (cudaPointerGetAttributes(&attr, p) != cudaSuccess) {
        cudaGetLastError();
        return true;
    }
    return attr.type == cudaMemoryTypeUnregistered;
}

} // namespace

ProveSlot::~ProveSlot()
{
    for (auto s : st)
        if (s) cudaStreamSynchronize(s);
    if (graph_exec) cudaGraphExecDestroy(graph_exec);
    if (graph) cudaGraphDestroy(graph);
    for (auto s : tail)
        if (s) cudaStreamSynchronize(s);
    for (auto s : cls)
        if (s) cudaStreamSynchronize(s);
    if (chain) cudaStreamSynchronize(chain);
    for (int k = 0; k < kNumMsm; ++k) {
        if (st[k]) cudaStreamDestroy(st[k]);
        if (tail[k]) cudaStreamDestroy(tail[k]);
        if (cls[k]) cudaStreamDestroy(cls[k]);
        if (ev_done[k]) cudaEventDestroy(ev_done[k]);
        if (ev_l1[k]) cudaEventDestroy(ev_l1[k]);
        if (ev_cls[k]) cudaEventDestroy(ev_cls[k]);
    }
    if (chain) cudaStreamDestroy(chain);
    for (cudaEvent_t e : {ev_z, ev_wit[0], ev_wit[1], ev_hsorted, ev_dedup})
        if (e) cudaEventDestroy(e);
    for (auto e : ev_sorted)
        if (e) cudaEventDestroy(e);
    for (auto e : ev_t)
        if (e) cudaEventDestroy(e);
    for (auto e : ev_msm_end)
        if (e) cudaEventDestroy(e);
    for (auto &a : acc)
        for (auto e : a.ev_acc)
            if (e) cudaEventDestroy(e);
    for (auto p : pinned_wit)
        if (p) cudaFreeHost(p);
    if (pinned_out) cudaFreeHost(pinned_out);
}

// Stream priority of a key's slots: smaller circuits run at higher priority.
// Levels above the lowest (B200 has five): 2^16 and below 5, 2^17 4, 2^18 3,
// 2^19..2^20 2, 2^21..2^22 1, 2^23 and up 0.  When proofs of several keys share
// the GPU (batches, the request server) the block scheduler then starts the
// blocks of shorter proofs first, so a small request is not held behind a large
// one; a proof alone runs as before.
static int slot_stream_priority(int logn)
{
    int least = 0, greatest = 0;
    if (cudaDeviceGetStreamPriorityRange(&least, &greatest) != cudaSuccess) {
        cudaGetLastError();
        return 0;
    }
    const int levels = least - greatest; // priorities run from least (0) down to greatest (< 0)
    const int above = logn <= 16 ? 5 : logn == 17 ? 4 : logn == 18 ? 3 : logn <= 20 ? 2 : logn <= 22 ? 1 : 0;
    return least - (above < levels ? above : levels);
}

int slot_add(nkr_b200_key *key)
{
    NKR_CUDA(cudaSetDevice(key->ctx->device));
    auto slot = std::make_unique<ProveSlot>();
    ProveSlot *sl = slot.get();
    // One priority for all streams of a slot.  Measured on a 2^20 prove (19.6 ms):
    // a higher priority for the main stream alone is slower (the H chain finishes
    // early but the H MSM then crowds out the witness MSMs); one or two levels more
    // for the G2 MSM's stream end it at 12.0 instead of 19.8 ms while the others end
    // later (20.05 vs 19.98 ms); the quotient chain one or two levels higher ends at
    // 6.4 instead of 14.8 ms but the prove takes 20.2-20.6 ms (the level-1 kernels of
    // several MSMs then share the SMs and all finish later); the fix-up and reduction
    // levels one or two levels higher finish early but take SM slots from the level-1
    // kernels (20.1-20.2 ms).  Running the level-1 kernels one after another on one
    // stream, in any order, with or without waiting for the quotient chain, took
    // 20.2-22.4 ms.
    const int prio = slot_stream_priority(key->logn);
    int least = 0, greatest = 0;
    if (cudaDeviceGetStreamPriorityRange(&least, &greatest) != cudaSuccess) cudaGetLastError();
    const int cls_prio = prio - 2 < greatest ? greatest : prio - 2;
    for (int k = 0; k < kNumMsm; ++k) {
        NKR_CUDA(cudaStreamCreateWithPriority(&sl->st[k], cudaStreamNonBlocking, prio));
        NKR_CUDA(cudaStreamCreateWithPriority(&sl->tail[k], cudaStreamNonBlocking, prio));
        // the class path is a chain of small, latency-bound launches: two priority
        // levels above the slot's level-1 kernels, so its blocks do not queue
        // behind theirs (cls[kMsmH] carries the class finding)
        NKR_CUDA(cudaStreamCreateWithPriority(&sl->cls[k], cudaStreamNonBlocking, cls_prio));
        NKR_CUDA(cudaEventCreateWithFlags(&sl->ev_cls[k], cudaEventDisableTiming));
        NKR_CUDA(cudaEventCreateWithFlags(&sl->ev_done[k], cudaEventDisableTiming));
        NKR_CUDA(cudaEventCreateWithFlags(&sl->ev_l1[k], cudaEventDisableTiming));
    }
    NKR_CUDA(cudaStreamCreateWithPriority(&sl->chain, cudaStreamNonBlocking, prio));
    NKR_CUDA(cudaEventCreateWithFlags(&sl->ev_hsorted, cudaEventDisableTiming));
    NKR_CUDA(cudaEventCreateWithFlags(&sl->ev_dedup, cudaEventDisableTiming));
    NKR_CUDA(cudaEventCreateWithFlags(&sl->ev_z, cudaEventDisableTiming));
    for (auto &e : sl->ev_sorted) NKR_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    for (auto &e : sl->ev_wit) NKR_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    for (auto &e : sl->ev_t) NKR_CUDA(cudaEventCreate(&e));
    for (auto &e : sl->ev_msm_end) NKR_CUDA(cudaEventCreate(&e));
    for (auto &a : sl->acc)
        for (auto &e : a.ev_acc) NKR_CUDA(cudaEventCreate(&e));
    size_t bytes = 0;
    for (int g = 0; g < key->n_sorts; ++g) {
        NKR_TRY(msm_sort_alloc(sl->sort_w[g], key->bases[key->sort_stream[g]].shape));
        bytes += sl->sort_w[g].device_bytes();
    }
    NKR_TRY(msm_sort_alloc(sl->sort_h, key->bases[kMsmH].shape));
    bytes += sl->sort_h.device_bytes();
    NKR_TRY(msm_dedup_alloc(sl->dedup, key->cols));
    bytes += sl->dedup.device_bytes();
    for (int k = 0; k < kNumMsm; ++k) {
        if (!key->classes[k]) continue;
        NKR_TRY(msm_class_sort_alloc(sl->csort[k], key->bases[k].shape.n));
        bytes += sl->csort[k].device_bytes();
        NKR_TRY(msm_class_acc_alloc(sl->cacc[k], key->bases[k].group, key->bases[k].shape.n));
        bytes += sl->cacc[k].device_bytes();
    }
    for (int k = 0; k < kNumMsm; ++k) {
        // The G1 witness MSMs' reductions run beside other MSMs' level-1 work, so
        // their first level takes twice the buckets per thread (less work, more
        // dependent steps); the H MSM ends the prove and the G2 MSM's levels are
        // long chains, so both keep the latency-optimal width.  Measured at 2^20
        // (four runs each): 19.48 vs 19.55 ms; the G2 MSM at half the width, 19.63.
        sl->acc[k].first_level_bias = (k == kMsmA || k == kMsmB1 || k == kMsmL) ? 1 : 0;
        NKR_TRY(msm_acc_alloc(sl->acc[k], key->bases[k].group, key->bases[k].shape));
        bytes += sl->acc[k].device_bytes();
    }
    NKR_TRY(sl->z.alloc(key->cols * 32, "witness"));
    NKR_TRY(sl->az.alloc(key->rows * 32, "az"));
    NKR_TRY(sl->bz.alloc(key->rows * 32, "bz"));
    NKR_TRY(sl->cz.alloc(key->rows * 32, "cz"));
    NKR_TRY(sl->h.alloc(key->rows * 32, "H"));
    NKR_TRY(sl->out.alloc(kOutBytes, "proof points"));
    // slot 0 (nkr_b200_prove) keeps the GLV tables of its last proof for the
    // blinding; zeroed, they describe the point at infinity until the first prove
    if (key->slots.empty()) {
        NKR_TRY(sl->glv_tab.alloc(glv_tables_bytes(), "blinding GLV tables"));
        NKR_CUDA(cudaMemset(sl->glv_tab.p, 0, sl->glv_tab.bytes));
    }
    bytes += sl->z.bytes + 4 * sl->az.bytes + sl->out.bytes + sl->glv_tab.bytes;
    for (int k = 0; k < 3; ++k) {
        NKR_TRY(sl->spmv_prod[k].alloc(std::max<uint64_t>(key->mat[k].nu, 1) * 32, "SpMV products"));
        bytes += sl->spmv_prod[k].bytes;
    }
    if (cudaHostAlloc(&sl->pinned_out, kOutBytes + kBlindStage, cudaHostAllocDefault) != cudaSuccess) {
        cudaGetLastError();
        set_error("pinned host allocation failed");
        return NKR_B200_ENOMEM;
    }
    key->slot_bytes = bytes;
    key->slots.push_back(std::move(slot));
    return NKR_B200_OK;
}

int prove_issue(nkr_b200_key *key, ProveSlot *sl, bool timed, bool blind_tables)
{
    cudaStream_t s0 = sl->main();
    const uint64_t rows = key->rows;
    Fr *z = sl->z.as<Fr>();
    Fr *az = sl->az.as<Fr>(), *bz = sl->bz.as<Fr>(), *cz = sl->cz.as<Fr>(), *h = sl->h.as<Fr>();
    uint8_t *out = sl->out.as<uint8_t>();
    if (timed) NKR_CUDA(cudaEventRecord(sl->ev_t[0], s0));
    for (auto &a : sl->acc) a.timing = timed; // phase events of each MSM (timed proves only)
    const CsrDevice *mats[3] = {&key->mat[0], &key->mat[1], &key->mat[2]};
    Fr *ys[3] = {az, bz, cz};
    Fr *prods[3] = {sl->spmv_prod[0].as<Fr>(), sl->spmv_prod[1].as<Fr>(), sl->spmv_prod[2].as<Fr>()};
    NKR_TRY(spmv_multi(mats, 3, z, ys, prods, s0));
    NKR_CUDA(cudaEventRecord(sl->ev_z, s0));
    if (timed) NKR_CUDA(cudaEventRecord(sl->ev_t[1], s0));
    // witness MSMs on their own streams, overlapping the H chain; one digit sort
    // of z (gathered through the bases' support) per distinct support
    // classes of repeated witness values (main stream), then the digit sorts
    // without the class members and the class members of each support
    NKR_CUDA(cudaStreamWaitEvent(sl->cls[kMsmH], sl->ev_z, 0));
    NKR_TRY(msm_dedup_run(sl->dedup, z, sl->cls[kMsmH]));
    NKR_CUDA(cudaEventRecord(sl->ev_dedup, sl->cls[kMsmH]));
    for (int g = 0; g < key->n_sorts; ++g) {
        const int o = key->sort_stream[g];
        const bool cls = key->classes[o];
        NKR_CUDA(cudaStreamWaitEvent(sl->st[o], cls ? sl->ev_dedup : sl->ev_z, 0));
        NKR_TRY(msm_sort_run(key->bases[o].shape, sl->sort_w[g], z, sl->st[o], key->bases[o].gather(),
                             cls ? sl->dedup.class_of.as<uint32_t>() : nullptr));
        NKR_CUDA(cudaEventRecord(sl->ev_sorted[g], sl->st[o]));
    }
    // level 1 on the MSM's stream, the fix-up and reduction levels on its tail
    // stream; a class-path MSM runs its class sums and the MSM over the classes on
    // its class stream (once the classes are known), beside its level 1 and tail, and
    // its tail ends with the addition of the two results
    auto msm_issue = [&](int k, const MsmSort &so, cudaStream_t s_l1) -> int {
        if (key->classes[k]) {
            NKR_CUDA(cudaStreamWaitEvent(sl->cls[k], sl->ev_dedup, 0));
            NKR_TRY(msm_class_sort_run(sl->csort[k], sl->dedup, key->bases[k].gather(), sl->cls[k]));
            NKR_TRY(msm_class_acc_issue(key->bases[k], sl->csort[k], sl->dedup, sl->cacc[k], sl->cls[k]));
            NKR_CUDA(cudaEventRecord(sl->ev_cls[k], sl->cls[k]));
        }
        NKR_TRY(msm_acc_level1(key->bases[k], so, sl->acc[k], s_l1));
        NKR_CUDA(cudaEventRecord(sl->ev_l1[k], s_l1));
        NKR_CUDA(cudaStreamWaitEvent(sl->tail[k], sl->ev_l1[k], 0));
        NKR_TRY(msm_acc_tail(key->bases[k], so, sl->acc[k], out + kOutOffset[k], sl->tail[k]));
        if (key->classes[k]) {
            NKR_CUDA(cudaStreamWaitEvent(sl->tail[k], sl->ev_cls[k], 0));
            NKR_TRY(msm_result_add(key->bases[k].group, out + kOutOffset[k], sl->cacc[k].out.p, sl->tail[k]));
        }
        if (timed) NKR_CUDA(cudaEventRecord(sl->ev_msm_end[k], sl->tail[k]));
        NKR_CUDA(cudaEventRecord(sl->ev_done[k], sl->tail[k]));
        return NKR_B200_OK;
    };
    // H = icosetFFT((cosetFFT(iFFT(a)) * cosetFFT(iFFT(b)) - cosetFFT(iFFT(c))) / Z(g))
    auto chain_issue = [&]() -> int {
        const NttTables &T = key->ntt;
        const Fr *cst = T.consts.as<Fr>();
        cudaStream_t sc = sl->chain;
        NKR_CUDA(cudaStreamWaitEvent(sc, sl->ev_z, 0));
        for (Fr *v : {az, bz, cz}) {
            NKR_TRY(ntt_dif(T, v, true, nullptr, nullptr, nullptr, sc));
            NKR_TRY(ntt_dit(T, v, false, T.t1.as<Fr>(), nullptr, nullptr, sc));
        }
        NKR_TRY(fr_quotient_pointwise(az, bz, cz, h, rows, cst + kConstZinv, sc));
        NKR_TRY(ntt_dif(T, h, true, nullptr, T.t2.as<Fr>(), nullptr, sc));
        if (timed) NKR_CUDA(cudaEventRecord(sl->ev_t[2], sc));
        NKR_TRY(msm_sort_run(key->bases[kMsmH].shape, sl->sort_h, h, sc));
        NKR_CUDA(cudaEventRecord(sl->ev_hsorted, sc));
        return NKR_B200_OK;
    };
    for (int k : kWitnessOrder) {
        const int g = key->sort_of[k];
        if (key->sort_stream[g] != k) NKR_CUDA(cudaStreamWaitEvent(sl->st[k], sl->ev_sorted[g], 0));
        NKR_TRY(msm_issue(k, sl->sort_w[g], sl->st[k]));
    }
    NKR_TRY(chain_issue());
    NKR_CUDA(cudaStreamWaitEvent(s0, sl->ev_hsorted, 0));
    NKR_TRY(msm_issue(kMsmH, sl->sort_h, s0));
    // ar and bs1 tabulated for the blinding, behind both MSMs on A's tail stream
    if (blind_tables) {
        NKR_CUDA(cudaStreamWaitEvent(sl->tail[kMsmA], sl->ev_done[kMsmB1], 0));
        NKR_TRY(glv_tables_issue(sl, sl->tail[kMsmA]));
        NKR_CUDA(cudaEventRecord(sl->ev_done[kMsmA], sl->tail[kMsmA]));
    }
    NKR_CUDA(cudaStreamWaitEvent(s0, sl->ev_done[kMsmH], 0));
    if (timed) NKR_CUDA(cudaEventRecord(sl->ev_t[3], s0));
    for (int k : kWitnessOrder) NKR_CUDA(cudaStreamWaitEvent(s0, sl->ev_done[k], 0));
    if (timed) NKR_CUDA(cudaEventRecord(sl->ev_t[4], s0));
    return NKR_B200_OK;
}

int slot_capture(nkr_b200_key *key, ProveSlot *sl)
{
    if (sl->graph_exec) return NKR_B200_OK;
    NKR_CUDA(cudaSetDevice(key->ctx->device));
    for (auto s : sl->st) NKR_CUDA(cudaStreamSynchronize(s));
    for (auto s : sl->tail) NKR_CUDA(cudaStreamSynchronize(s));
    for (auto s : sl->cls) NKR_CUDA(cudaStreamSynchronize(s));
    NKR_CUDA(cudaStreamSynchronize(sl->chain));
    cudaStream_t s0 = sl->main();
    const unsigned long long before = g_kernel_launches.load();
    NKR_CUDA(cudaStreamBeginCapture(s0, cudaStreamCaptureModeRelaxed));
    const int s = prove_issue(key, sl, false, false);
    cudaGraph_t g = nullptr;
    const cudaError_t e = cudaStreamEndCapture(s0, &g);
    // capturing records kernels, it launches none
    g_kernel_launches.fetch_sub(g_kernel_launches.load() - before);
    if (s != NKR_B200_OK || e != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        cudaGetLastError();
        if (s == NKR_B200_OK) set_error("prove graph capture failed: %s", cudaGetErrorString(e));
        return s != NKR_B200_OK ? s : NKR_B200_ECUDA;
    }
    size_t nn = 0;
    NKR_CUDA(cudaGraphGetNodes(g, nullptr, &nn));
    std::vector<cudaGraphNode_t> nodes(nn);
    NKR_CUDA(cudaGraphGetNodes(g, nodes.data(), &nn));
    unsigned long long kernels = 0;
    for (auto nd : nodes) {
        cudaGraphNodeType t;
        NKR_CUDA(cudaGraphNodeGetType(nd, &t));
        kernels += t == cudaGraphNodeTypeKernel;
    }
    cudaGraphExec_t ex = nullptr;
    const cudaError_t ei = cudaGraphInstantiate(&ex, g, 0);
    if (ei != cudaSuccess) {
        cudaGraphDestroy(g);
        set_error("prove graph instantiation failed: %s", cudaGetErrorString(ei));
        return NKR_B200_ECUDA;
    }
    sl->graph = g;
    sl->graph_exec = ex;
    sl->graph_kernels = kernels;
    return NKR_B200_OK;
}

int slot_upload_witness(nkr_b200_key *key, ProveSlot *sl, const void *witness)
{
    const size_t bytes = key->cols * 32;
    cudaStream_t s0 = sl->main();
    if (!is_pageable(witness)) {
        NKR_CUDA(cudaMemcpyAsync(sl->z.p, witness, bytes, copy_kind_from(witness), s0));
        return NKR_B200_OK;
    }
    // pageable: stage through the slot's pinned double buffer so the copy is asynchronous
    const int b = sl->wit_next;
    sl->wit_next ^= 1;
    if (!sl->pinned_wit[b] && cudaHostAlloc(&sl->pinned_wit[b], bytes, cudaHostAllocDefault) != cudaSuccess) {
        cudaGetLastError();
        sl->pinned_wit[b] = nullptr;
        set_error("pinned witness staging allocation failed");
        return NKR_B200_ENOMEM;
    }
    NKR_CUDA(cudaEventSynchronize(sl->ev_wit[b]));
    std::memcpy(sl->pinned_wit[b], witness, bytes);
    NKR_CUDA(cudaMemcpyAsync(sl->z.p, sl->pinned_wit[b], bytes, cudaMemcpyHostToDevice, s0));
    NKR_CUDA(cudaEventRecord(sl->ev_wit[b], s0));
    return NKR_B200_OK;
}

int slot_launch(ProveSlot *sl, cudaStream_t launch)
{
    NKR_CUDA(cudaGraphLaunch(sl->graph_exec, launch ? launch : sl->main()));
    g_kernel_launches.fetch_add(sl->graph_kernels, std::memory_order_relaxed);
    return NKR_B200_OK;
}

int key_prepare(nkr_b200_ctx *ctx, const nkr_b200_circuit *c, const nkr_b200_proving_key *pk,
                nkr_b200_key **out)
{
    NKR_REQUIRE(ctx && c && pk && out, "null argument");
    const int logn = log2_exact(c->rows);
    NKR_REQUIRE(logn >= 1 && logn <= 28, "constraint count %llu must be a power of two in [2, 2^28]",
                (unsigned long long)c->rows);
    NKR_REQUIRE(c->cols >= 1 && c->public_inputs + 1 <= c->cols,
                "public input count exceeds the variable count");
    for (int k = 0; k < 3; ++k)
        NKR_REQUIRE(c->row_ptr[k] && (c->row_ptr[k][c->rows] == 0 || (c->col_idx[k] && c->values[k])),
                    "matrix %d has null CSR arrays", k);
    NKR_REQUIRE(pk->a_query && pk->b_g1_query && pk->b_g2_query && pk->l_query && pk->h_query &&
                    pk->alpha_g1 && pk->beta_g1 && pk->delta_g1 && pk->beta_g2 && pk->delta_g2,
                "proving key has null arrays");
    NKR_CUDA(cudaSetDevice(ctx->device));
    auto *key = new nkr_b200_key();
    key->ctx = ctx;
    key->rows = c->rows;
    key->cols = c->cols;
    key->public_inputs = c->public_inputs;
    key->logn = logn;
    auto fail = [&](int s) {
        nkr_b200_key_free(key);
        return s;
    };
    int s = NKR_B200_OK;
#define NKR_PREP(expr)                                                                          \
    do {                                                                                        \
        s = (expr);                                                                             \
        if (s != NKR_B200_OK) return fail(s);                                                   \
    } while (0)
    cudaStream_t st = ctx->stream;
    for (int k = 0; k < 3; ++k)
        NKR_PREP(csr_upload(key->mat[k], c->rows, c->cols, c->row_ptr[k], c->col_idx[k],
                            c->values[k], st));
    NKR_PREP(ntt_tables_build(key->ntt, logn, st));
    // proving key: normalise (hazard: CPU-setup keys are unnormalised Jacobian), fold
    // windows; witness queries keep only their finite points (variables present in the matrix)
    // window widths from the autotuner (per support size; 0 = cost model)
    const void *wq[4] = {pk->a_query, pk->b_g1_query, pk->l_query, pk->b_g2_query};
    const int wk[4] = {kMsmA, kMsmB1, kMsmL, kMsmB2};
    for (int j = 0; j < 4; ++j) {
        const int group = wk[j] == kMsmB2 ? 2 : 1;
        std::vector<uint32_t> idx = msm_support(group, wq[j], c->cols);
        int cw = 0;
        NKR_PREP(tuned_window_bits(ctx, idx.size(), &cw));
        NKR_PREP(msm_bases_build_support(key->bases[wk[j]], group, wq[j], c->cols, std::move(idx), true,
                                         cw, st));
    }
    int ch = 0;
    NKR_PREP(tuned_window_bits(ctx, c->rows, &ch));
    NKR_PREP(msm_bases_build(key->bases[kMsmH], 1, pk->h_query, false, c->rows, true, ch, true, st));
    // MSMs with the same support (and so the same window shape) and the same use
    // of the class path share a digit sort
    for (int k : kWitnessOrder) key->classes[k] = true;
    key->n_sorts = 0;
    for (int k : kWitnessOrder) {
        int g = -1;
        for (int h = 0; h < key->n_sorts && g < 0; ++h) {
            const int ho = key->sort_stream[h];
            const MsmBases &o = key->bases[ho];
            if (o.shape.same_sort(key->bases[k].shape) && o.support_host == key->bases[k].support_host &&
                key->classes[ho] == key->classes[k])
                g = h;
        }
        if (g < 0) {
            g = key->n_sorts++;
            key->sort_stream[g] = k;
        }
        key->sort_of[k] = g;
    }
    // PK constants: libff Jacobian -> affine
    {
        DevBuf stage;
        NKR_PREP(stage.alloc(3 * 96 + 2 * 192, "pk constant upload"));
        uint8_t *sp = stage.as<uint8_t>();
        const void *g1s[3] = {pk->alpha_g1, pk->beta_g1, pk->delta_g1};
        const void *g2s[2] = {pk->beta_g2, pk->delta_g2};
        for (int i = 0; i < 3; ++i)
            if (cudaMemcpyAsync(sp + 96 * i, g1s[i], 96, cudaMemcpyHostToDevice, st) != cudaSuccess)
                return fail(NKR_B200_ECUDA);
        for (int i = 0; i < 2; ++i)
            if (cudaMemcpyAsync(sp + 288 + 192 * i, g2s[i], 192, cudaMemcpyHostToDevice, st) !=
                cudaSuccess)
                return fail(NKR_B200_ECUDA);
        NKR_PREP(key->pk_const.alloc(3 * sizeof(G1Affine) + 2 * sizeof(G2Affine), "pk constants"));
        NKR_PREP(jacobian_to_affine(1, sp, key->pk_const.p, 3, st));
        NKR_PREP(jacobian_to_affine(2, sp + 288, key->pk_const.as<uint8_t>() + 3 * sizeof(G1Affine), 2,
                                    st));
        if (cudaStreamSynchronize(st) != cudaSuccess) {
            set_error("prepare: %s", cudaGetErrorString(cudaGetLastError()));
            return fail(NKR_B200_ECUDA);
        }
    }
    NKR_PREP(blind_tables_build(key, st));
    NKR_PREP(slot_add(key));
#undef NKR_PREP
    *out = key;
    return NKR_B200_OK;
}

int key_prove(nkr_b200_key *key, const void *witness, uint64_t n, nkr_b200_raw_proof *res)
{
    NKR_REQUIRE(key && witness && res, "null argument");
    NKR_REQUIRE(n == key->cols, "witness has %llu elements, the circuit has %llu columns",
                (unsigned long long)n, (unsigned long long)key->cols);
    NKR_CUDA(cudaSetDevice(key->ctx->device));
    ProveSlot *sl = key->slots[0].get();
    cudaStream_t s0 = sl->main();
    // s0 is ordered after the previous prove's joins, so z is free to overwrite
    NKR_CUDA(cudaMemcpyAsync(sl->z.p, witness, n * 32, copy_kind_from(witness), s0));
    NKR_TRY(prove_issue(key, sl, true, true));
    NKR_CUDA(cudaMemcpyAsync(sl->pinned_out, sl->out.p, kOutBytes, cudaMemcpyDeviceToHost, s0));
    NKR_CUDA(cudaStreamSynchronize(s0));
    normalize_raw(sl->pinned_out);
    raw_from_bytes(sl->pinned_out, res);
    float ms[4];
    for (int i = 0; i < 4; ++i) NKR_CUDA(cudaEventElapsedTime(&ms[i], sl->ev_t[i], sl->ev_t[i + 1]));
    key->times.spmv_ms = ms[0];
    key->times.quotient_ms = ms[1];
    key->times.quotient_msm_ms = ms[2];
    NKR_CUDA(cudaEventElapsedTime(&key->times.total_ms, sl->ev_t[0], sl->ev_t[4]));
    key->times.witness_msms_ms = key->times.total_ms - ms[0];
    float *ends[kNumMsm];
    ends[kMsmA] = &key->times.msm_a_end_ms;
    ends[kMsmB1] = &key->times.msm_b_g1_end_ms;
    ends[kMsmB2] = &key->times.msm_b_g2_end_ms;
    ends[kMsmL] = &key->times.msm_l_end_ms;
    ends[kMsmH] = &key->times.msm_h_end_ms;
    for (int k = 0; k < kNumMsm; ++k)
        NKR_CUDA(cudaEventElapsedTime(ends[k], sl->ev_t[0], sl->ev_msm_end[k]));
    // phases in the public MSM order A, B_G1, B_G2, L, H
    const int order[kNumMsm] = {kMsmA, kMsmB1, kMsmB2, kMsmL, kMsmH};
    for (int i = 0; i < kNumMsm; ++i)
        for (int j = 0; j < 4; ++j)
            NKR_CUDA(cudaEventElapsedTime(&key->times.msm_phase_ms[i][j], sl->ev_t[0],
                                          sl->acc[order[i]].ev_acc[j]));
    key->have_times = true;
    return NKR_B200_OK;
}

int key_intermediates(nkr_b200_key *key, void *az, void *bz, void *cz, void *h)
{
    NKR_REQUIRE(key, "null key");
    NKR_CUDA(cudaSetDevice(key->ctx->device));
    ProveSlot *sl = key->slots[0].get();
    cudaStream_t s0 = sl->main();
    const uint64_t rows = key->rows;
    DevBuf tmp;
    NKR_TRY(tmp.alloc(4 * rows * 32, "intermediate scratch"));
    Fr *t = tmp.as<Fr>();
    // the SpMV is a pure function of the resident witness: recompute az, bz, cz
    const CsrDevice *mats[3] = {&key->mat[0], &key->mat[1], &key->mat[2]};
    Fr *ys[3] = {t, t + rows, t + 2 * rows};
    Fr *prods[3] = {sl->spmv_prod[0].as<Fr>(), sl->spmv_prod[1].as<Fr>(), sl->spmv_prod[2].as<Fr>()};
    NKR_TRY(spmv_multi(mats, 3, sl->z.as<Fr>(), ys, prods, s0));
    // H is held in bit-reversed order; return it in natural order
    NKR_TRY(ntt_bitrev_permute(sl->h.as<Fr>(), t + 3 * rows, rows, nullptr, nullptr, s0));
    void *dst[4] = {az, bz, cz, h};
    for (int i = 0; i < 4; ++i)
        if (dst[i]) NKR_CUDA(cudaMemcpyAsync(dst[i], t + i * rows, rows * 32, cudaMemcpyDeviceToHost, s0));
    NKR_CUDA(cudaStreamSynchronize(s0));
    return NKR_B200_OK;
}

namespace {

constexpr int kMaxSlotsPerKey = 4;
constexpr size_t kSlotHeadroom = size_t(1) << 30; // free HBM kept after admitting a slot

// Grows the key's slots toward `want` while free HBM admits another one.
int admit_slots(nkr_b200_key *key, int want)
{
    NKR_CUDA(cudaSetDevice(key->ctx->device));
    while (int(key->slots.size()) < want) {
        size_t free_b = 0, total_b = 0;
        NKR_CUDA(cudaMemGetInfo(&free_b, &total_b));
        if (free_b < key->slot_bytes + kSlotHeadroom) break;
        NKR_TRY(slot_add(key));
    }
    return NKR_B200_OK;
}

} // namespace

namespace {

// One wave of a batch: at most one proof per prove slot, all proofs' stages
// aligned so that the work of every proof in a stage runs as one launch over a
// device work list.  Per proof (on its slot's streams): witness upload, SpMV,
// the witness digit sorts; then, across the wave, the level-1 bucket
// accumulation of every G1 witness MSM in one launch (stream bw) and of every
// G2 MSM in another (stream bw2); per proof the fix-up and reduction levels.
// Across the wave on stream bq: the quotient chains, each NTT pass of every
// proof's transforms in one launch and the pointwise step of all proofs in one;
// per proof the digit sort of H; the level-1 accumulation of every H MSM in one
// launch; per proof the H MSM's remaining levels, the join of the witness MSMs
// and the result download.
struct WaveProof {
    nkr_b200_key *key;
    ProveSlot *slot;
    const void *witness;
    uint8_t *result; // pinned host, kOutBytes
};

struct WaveScratch {
    cudaStream_t bq = nullptr, bw = nullptr, bw2 = nullptr; // chains + H, G1 witness, G2 witness
    cudaEvent_t ev_wacc = nullptr, ev_wacc2 = nullptr, ev_chain = nullptr, ev_hacc = nullptr;
    std::vector<cudaEvent_t> ev_ready, ev_hsort; // per proof and witness MSM / per proof
    DevBuf ntt_items, q_items, w_items, h_items;
    // pinned host staging of the work lists: three NTT lists, quotient, witness
    // and H accumulation lists (the copies read it asynchronously)
    uint8_t *stage = nullptr;
    size_t ntt_bytes = 0, q_bytes = 0, w_bytes = 0, h_bytes = 0;
    NttPassItem *stage_ntt(int call) { return reinterpret_cast<NttPassItem *>(stage + call * ntt_bytes); }
    QuotientItem *stage_q() { return reinterpret_cast<QuotientItem *>(stage + 3 * ntt_bytes); }
    uint8_t *stage_w() { return stage + 3 * ntt_bytes + q_bytes; }
    uint8_t *stage_h() { return stage + 3 * ntt_bytes + q_bytes + w_bytes; }
    ~WaveScratch()
    {
        if (stage) {
            if (bq) cudaStreamSynchronize(bq);
            if (bw) cudaStreamSynchronize(bw);
            if (bw2) cudaStreamSynchronize(bw2);
            cudaFreeHost(stage);
        }
        for (cudaStream_t st : {bq, bw, bw2})
            if (st) {
                cudaStreamSynchronize(st);
                cudaStreamDestroy(st);
            }
        for (cudaEvent_t e : {ev_wacc, ev_wacc2, ev_chain, ev_hacc})
            if (e) cudaEventDestroy(e);
        for (auto e : ev_ready)
            if (e) cudaEventDestroy(e);
        for (auto e : ev_hsort)
            if (e) cudaEventDestroy(e);
    }
    int init(size_t max_wave)
    {
        NKR_CUDA(cudaStreamCreateWithFlags(&bq, cudaStreamNonBlocking));
        NKR_CUDA(cudaStreamCreateWithFlags(&bw, cudaStreamNonBlocking));
        NKR_CUDA(cudaStreamCreateWithFlags(&bw2, cudaStreamNonBlocking));
        for (cudaEvent_t *e : {&ev_wacc, &ev_wacc2, &ev_chain, &ev_hacc})
            NKR_CUDA(cudaEventCreateWithFlags(e, cudaEventDisableTiming));
        ev_ready.assign(max_wave * 4, nullptr);
        ev_hsort.assign(max_wave, nullptr);
        for (auto &e : ev_ready) NKR_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        for (auto &e : ev_hsort) NKR_CUDA(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
        ntt_bytes = 8 * 3 * max_wave * sizeof(NttPassItem);
        q_bytes = max_wave * sizeof(QuotientItem);
        w_bytes = 4 * max_wave * kMsmAccItemBytes;
        h_bytes = max_wave * kMsmAccItemBytes;
        NKR_TRY(ntt_items.alloc(ntt_bytes, "batch NTT work list"));
        NKR_TRY(q_items.alloc(q_bytes, "batch quotient work list"));
        NKR_TRY(w_items.alloc(w_bytes, "batch accumulation work list"));
        NKR_TRY(h_items.alloc(h_bytes, "batch accumulation work list"));
        if (cudaHostAlloc(reinterpret_cast<void **>(&stage), 3 * ntt_bytes + q_bytes + w_bytes + h_bytes,
                          cudaHostAllocDefault) != cudaSuccess) {
            cudaGetLastError();
            stage = nullptr;
            set_error("pinned work-list staging allocation failed");
            return NKR_B200_ENOMEM;
        }
        return NKR_B200_OK;
    }
};

int run_wave(const std::vector<WaveProof> &wave, WaveScratch &ws)
{
    const size_t P = wave.size();
    // the previous wave's work-list copies have read the staging area
    NKR_CUDA(cudaStreamSynchronize(ws.bq));
    NKR_CUDA(cudaStreamSynchronize(ws.bw));
    NKR_CUDA(cudaStreamSynchronize(ws.bw2));
    // per proof: upload, SpMV, witness sorts
    for (size_t p = 0; p < P; ++p) {
        nkr_b200_key *key = wave[p].key;
        ProveSlot *sl = wave[p].slot;
        cudaStream_t s0 = sl->main();
        NKR_TRY(slot_upload_witness(key, sl, wave[p].witness));
        const CsrDevice *mats[3] = {&key->mat[0], &key->mat[1], &key->mat[2]};
        Fr *ys[3] = {sl->az.as<Fr>(), sl->bz.as<Fr>(), sl->cz.as<Fr>()};
        Fr *prods[3] = {sl->spmv_prod[0].as<Fr>(), sl->spmv_prod[1].as<Fr>(), sl->spmv_prod[2].as<Fr>()};
        NKR_TRY(spmv_multi(mats, 3, sl->z.as<Fr>(), ys, prods, s0));
        NKR_CUDA(cudaEventRecord(sl->ev_z, s0));
        for (int g = 0; g < key->n_sorts; ++g) {
            const int o = key->sort_stream[g];
            NKR_CUDA(cudaStreamWaitEvent(sl->st[o], sl->ev_z, 0));
            NKR_TRY(msm_sort_run(key->bases[o].shape, sl->sort_w[g], sl->z.p, sl->st[o],
                                 key->bases[o].gather()));
            NKR_CUDA(cudaEventRecord(sl->ev_sorted[g], sl->st[o]));
        }
        for (int i = 0; i < 4; ++i) {
            const int k = kWitnessOrder[i];
            const int g = key->sort_of[k];
            if (key->sort_stream[g] != k) NKR_CUDA(cudaStreamWaitEvent(sl->st[k], sl->ev_sorted[g], 0));
            NKR_CUDA(cudaEventRecord(ws.ev_ready[4 * p + i], sl->st[k]));
        }
    }
    // witness MSMs: level 1 of the wave's G1 MSMs in one launch (stream bw) and of
    // its G2 MSMs in another (stream bw2)
    std::vector<MsmAccJob> g1, g2;
    for (size_t p = 0; p < P; ++p) {
        nkr_b200_key *key = wave[p].key;
        ProveSlot *sl = wave[p].slot;
        for (int i = 0; i < 4; ++i) {
            const int k = kWitnessOrder[i];
            const bool is_g1 = key->bases[k].group == 1;
            NKR_CUDA(cudaStreamWaitEvent(is_g1 ? ws.bw : ws.bw2, ws.ev_ready[4 * p + i], 0));
            MsmAccJob j{&key->bases[k], &sl->sort_w[key->sort_of[k]], &sl->acc[k]};
            (is_g1 ? g1 : g2).push_back(j);
        }
    }
    uint8_t *wi = ws.w_items.as<uint8_t>();
    uint8_t *wh = ws.stage_w();
    NKR_TRY(msm_acc_level1_list(1, g1.data(), int(g1.size()), wh, wi, ws.bw));
    NKR_TRY(msm_acc_level1_list(2, g2.data(), int(g2.size()), wh + g1.size() * kMsmAccItemBytes,
                                wi + g1.size() * kMsmAccItemBytes, ws.bw2));
    NKR_CUDA(cudaEventRecord(ws.ev_wacc, ws.bw));
    NKR_CUDA(cudaEventRecord(ws.ev_wacc2, ws.bw2));
    for (size_t p = 0; p < P; ++p) {
        nkr_b200_key *key = wave[p].key;
        ProveSlot *sl = wave[p].slot;
        uint8_t *out = sl->out.as<uint8_t>();
        for (int k : kWitnessOrder) {
            NKR_CUDA(cudaStreamWaitEvent(sl->st[k], key->bases[k].group == 1 ? ws.ev_wacc : ws.ev_wacc2, 0));
            NKR_TRY(msm_acc_tail(key->bases[k], sl->sort_w[key->sort_of[k]], sl->acc[k],
                                 out + kOutOffset[k], sl->st[k]));
            NKR_CUDA(cudaEventRecord(sl->ev_done[k], sl->st[k]));
        }
    }
    // quotient chains: every pass of every proof's transforms in one launch
    std::vector<NttJob> jobs;
    std::vector<QuotientItem> qi;
    for (size_t p = 0; p < P; ++p) {
        ProveSlot *sl = wave[p].slot;
        NKR_CUDA(cudaStreamWaitEvent(ws.bq, sl->ev_z, 0));
    }
    NttPassItem *ni = ws.ntt_items.as<NttPassItem>();
    for (size_t p = 0; p < P; ++p) {
        const NttTables &T = wave[p].key->ntt;
        ProveSlot *sl = wave[p].slot;
        for (Fr *v : {sl->az.as<Fr>(), sl->bz.as<Fr>(), sl->cz.as<Fr>()})
            jobs.push_back(NttJob{&T, v, nullptr, nullptr, nullptr});
    }
    NKR_TRY(ntt_run_list(jobs.data(), int(jobs.size()), true, true, ws.stage_ntt(0), ni, ws.bq)); // iFFT (DIF)
    for (size_t p = 0; p < P; ++p)
        for (int v = 0; v < 3; ++v) jobs[3 * p + v].pre = wave[p].key->ntt.t1.as<Fr>();
    NKR_TRY(ntt_run_list(jobs.data(), int(jobs.size()), false, false, ws.stage_ntt(1), ni, ws.bq)); // cosetFFT
    for (size_t p = 0; p < P; ++p) {
        const NttTables &T = wave[p].key->ntt;
        ProveSlot *sl = wave[p].slot;
        qi.push_back(QuotientItem{sl->az.as<Fr>(), sl->bz.as<Fr>(), sl->cz.as<Fr>(), sl->h.as<Fr>(),
                                  T.consts.as<Fr>() + kConstZinv, wave[p].key->rows});
    }
    std::copy(qi.begin(), qi.end(), ws.stage_q());
    NKR_TRY(fr_quotient_list(ws.stage_q(), int(qi.size()), ws.q_items.as<QuotientItem>(), ws.bq));
    jobs.clear();
    for (size_t p = 0; p < P; ++p)
        jobs.push_back(NttJob{&wave[p].key->ntt, wave[p].slot->h.as<Fr>(), nullptr,
                              wave[p].key->ntt.t2.as<Fr>(), nullptr});
    NKR_TRY(ntt_run_list(jobs.data(), int(jobs.size()), true, true, ws.stage_ntt(2), ni, ws.bq)); // icosetFFT
    NKR_CUDA(cudaEventRecord(ws.ev_chain, ws.bq));
    // H: per proof the sort, then level 1 of every H MSM in one launch
    std::vector<MsmAccJob> hj;
    for (size_t p = 0; p < P; ++p) {
        nkr_b200_key *key = wave[p].key;
        ProveSlot *sl = wave[p].slot;
        cudaStream_t s0 = sl->main();
        NKR_CUDA(cudaStreamWaitEvent(s0, ws.ev_chain, 0));
        NKR_TRY(msm_sort_run(key->bases[kMsmH].shape, sl->sort_h, sl->h.p, s0));
        NKR_CUDA(cudaEventRecord(ws.ev_hsort[p], s0));
        NKR_CUDA(cudaStreamWaitEvent(ws.bq, ws.ev_hsort[p], 0));
        hj.push_back(MsmAccJob{&key->bases[kMsmH], &sl->sort_h, &sl->acc[kMsmH]});
    }
    NKR_TRY(msm_acc_level1_list(1, hj.data(), int(hj.size()), ws.stage_h(), ws.h_items.p, ws.bq));
    NKR_CUDA(cudaEventRecord(ws.ev_hacc, ws.bq));
    for (size_t p = 0; p < P; ++p) {
        nkr_b200_key *key = wave[p].key;
        ProveSlot *sl = wave[p].slot;
        cudaStream_t s0 = sl->main();
        NKR_CUDA(cudaStreamWaitEvent(s0, ws.ev_hacc, 0));
        NKR_TRY(msm_acc_tail(key->bases[kMsmH], sl->sort_h, sl->acc[kMsmH],
                             sl->out.as<uint8_t>() + kOutOffset[kMsmH], s0));
        for (int k : kWitnessOrder) NKR_CUDA(cudaStreamWaitEvent(s0, sl->ev_done[k], 0));
        NKR_CUDA(cudaMemcpyAsync(wave[p].result, sl->out.p, kOutBytes, cudaMemcpyDeviceToHost, s0));
    }
    return NKR_B200_OK;
}

} // namespace

int key_prove_batch_lists(nkr_b200_key *const *keys, const void *const *witnesses, int count,
                          nkr_b200_raw_proof *out)
{
    NKR_REQUIRE(keys && witnesses && out && count >= 0, "null argument");
    if (count == 0) return NKR_B200_OK;
    std::vector<nkr_b200_key *> distinct;
    std::vector<int> per_key;
    for (int i = 0; i < count; ++i) {
        NKR_REQUIRE(keys[i] && witnesses[i], "null key or witness at %d", i);
        NKR_REQUIRE(keys[i]->ctx == keys[0]->ctx, "batch keys belong to different contexts");
        size_t j = 0;
        while (j < distinct.size() && distinct[j] != keys[i]) ++j;
        if (j == distinct.size()) {
            distinct.push_back(keys[i]);
            per_key.push_back(0);
        }
        ++per_key[j];
    }
    NKR_CUDA(cudaSetDevice(keys[0]->ctx->device));
    size_t max_wave = 0;
    for (size_t j = 0; j < distinct.size(); ++j) {
        NKR_TRY(admit_slots(distinct[j], std::min(per_key[j], kMaxSlotsPerKey)));
        max_wave += distinct[j]->slots.size();
    }
    max_wave = std::min<size_t>(max_wave, size_t(count));
    void *res = nullptr;
    if (cudaHostAlloc(&res, size_t(count) * kOutBytes, cudaHostAllocDefault) != cudaSuccess) {
        cudaGetLastError();
        set_error("pinned result allocation failed");
        return NKR_B200_ENOMEM;
    }
    int status = NKR_B200_OK;
    {
        WaveScratch ws;
        status = ws.init(max_wave);
        // waves: proofs in order, each on the next free slot of its key; a proof
        // whose key has no free slot left starts the next wave
        std::vector<WaveProof> wave;
        std::vector<size_t> used(distinct.size(), 0);
        for (int i = 0; i < count && status == NKR_B200_OK; ++i) {
            const size_t j = size_t(std::find(distinct.begin(), distinct.end(), keys[i]) - distinct.begin());
            if (used[j] == distinct[j]->slots.size()) {
                status = run_wave(wave, ws);
                wave.clear();
                std::fill(used.begin(), used.end(), size_t(0));
            }
            if (status != NKR_B200_OK) break;
            wave.push_back(WaveProof{keys[i], distinct[j]->slots[used[j]++].get(), witnesses[i],
                                     static_cast<uint8_t *>(res) + size_t(i) * kOutBytes});
        }
        if (status == NKR_B200_OK && !wave.empty()) status = run_wave(wave, ws);
        for (auto *key : distinct)
            for (auto &sl : key->slots)
                for (auto st : sl->st)
                    if (cudaStreamSynchronize(st) != cudaSuccess && status == NKR_B200_OK) {
                        set_error("batch: %s", cudaGetErrorString(cudaGetLastError()));
                        status = NKR_B200_ECUDA;
                    }
    }
    if (status == NKR_B200_OK)
        for (int i = 0; i < count; ++i) {
            uint8_t *o = static_cast<uint8_t *>(res) + size_t(i) * kOutBytes;
            normalize_raw(o);
            raw_from_bytes(o, &out[i]);
        }
    cudaFreeHost(res);
    return status;
}

int key_prove_batch(nkr_b200_key *const *keys, const void *const *witnesses, int count,
                    nkr_b200_raw_proof *out)
{
    NKR_REQUIRE(keys && witnesses && out && count >= 0, "null argument");
    std::vector<nkr_b200_key *> distinct;
    std::vector<int> per_key;
    for (int i = 0; i < count; ++i) {
        NKR_REQUIRE(keys[i] && witnesses[i], "null key or witness at %d", i);
        size_t j = 0;
        while (j < distinct.size() && distinct[j] != keys[i]) ++j;
        if (j == distinct.size()) {
            distinct.push_back(keys[i]);
            per_key.push_back(0);
        }
        ++per_key[j];
    }
    // slots: up to kMaxSlotsPerKey proofs of one key in flight, admitted by free HBM;
    // each slot replays its captured prove graph
    for (size_t j = 0; j < distinct.size(); ++j) {
        NKR_TRY(admit_slots(distinct[j], std::min(per_key[j], kMaxSlotsPerKey)));
        for (auto &sl : distinct[j]->slots) NKR_TRY(slot_capture(distinct[j], sl.get()));
    }
    void *res = nullptr;
    if (count) {
        NKR_CUDA(cudaSetDevice(keys[0]->ctx->device));
        if (cudaHostAlloc(&res, size_t(count) * kOutBytes, cudaHostAllocDefault) != cudaSuccess) {
            cudaGetLastError();
            set_error("pinned result allocation failed");
            return NKR_B200_ENOMEM;
        }
    }
    std::vector<size_t> next(distinct.size(), 0);
    std::vector<ProveSlot *> used;
    int status = NKR_B200_OK;
    for (int i = 0; i < count && status == NKR_B200_OK; ++i) {
        nkr_b200_key *key = keys[i];
        const size_t j = size_t(std::find(distinct.begin(), distinct.end(), key) - distinct.begin());
        ProveSlot *sl = key->slots[next[j]++ % key->slots.size()].get();
        if (cudaSetDevice(key->ctx->device) != cudaSuccess) {
            set_error("cudaSetDevice failed");
            status = NKR_B200_ECUDA;
            break;
        }
        status = slot_upload_witness(key, sl, witnesses[i]);
        if (status == NKR_B200_OK) status = slot_launch(sl);
        if (status == NKR_B200_OK &&
            cudaMemcpyAsync(static_cast<uint8_t *>(res) + size_t(i) * kOutBytes, sl->out.p, kOutBytes,
                            cudaMemcpyDeviceToHost, sl->main()) != cudaSuccess) {
            set_error("result download failed");
            status = NKR_B200_ECUDA;
        }
        if (std::find(used.begin(), used.end(), sl) == used.end()) used.push_back(sl);
    }
    for (ProveSlot *sl : used)
        if (cudaStreamSynchronize(sl->main()) != cudaSuccess && status == NKR_B200_OK) {
            set_error("batch: %s", cudaGetErrorString(cudaGetLastError()));
            status = NKR_B200_ECUDA;
        }
    if (status == NKR_B200_OK)
        for (int i = 0; i < count; ++i) {
            uint8_t *o = static_cast<uint8_t *>(res) + size_t(i) * kOutBytes;
            normalize_raw(o);
            raw_from_bytes(o, &out[i]);
        }
    if (res) cudaFreeHost(res);
    return status;
}

} // namespace nkr

void nkr_b200_key_free(nkr_b200_key *key)
{
    if (!key) return;
    if (key->ctx) cudaSetDevice(key->ctx->device);
    key->slots.clear();
    delete key;
}

uint64_t nkr_b200_key_device_bytes(const nkr_b200_key *key)
{
    if (!key) return 0;
    uint64_t b = key->ntt.device_bytes() + key->pk_const.bytes + key->blind_io.bytes +
                 key->blind_tab.bytes;
    for (int k = 0; k < 3; ++k)
        b += key->mat[k].row_ptr.bytes + key->mat[k].col.bytes + key->mat[k].nu_col.bytes +
             key->mat[k].nu_val.bytes;
    for (int k = 0; k < nkr::kNumMsm; ++k) b += key->bases[k].device_bytes();
    b += key->slot_bytes * key->slots.size();
    return b;
}
