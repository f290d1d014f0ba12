// Prove request server: continuous batching of Groth16 proves over resident keys.
//
// The reference proves one request at a time per process (app/prove.cpp:70-88;
// its bench runs one process per GPU, scripts/bench/runner.py:420-428).  Here
// one server owns a set of prepared keys; callers submit (key, witness) requests
// from any thread and wait for them.  Slot streams carry a priority by circuit
// size (prover.cu, slot_stream_priority), so among the requests in flight the
// block scheduler serves smaller proofs first.  A scheduler thread
//   - admits the oldest waiting request whose key has a free prove slot, adding
//     a slot to the key when free HBM admits one (kServerHeadroom kept free) and
//     the key has fewer than its slot cap (key_slot_cap),
//   - uploads the witness and replays the slot's captured prove graph on the
//     slot's streams, so requests of different keys (and several of one key)
//     overlap on the device while earlier ones are still running,
//   - polls the slots' completion events, normalises finished raw proofs and
//     wakes their waiters,
//   - ages waiting requests: one that waited longer than age_factor times its
//     key's recent service time (an average over its completed requests) is
//     launched into a stream of the device's highest priority instead of the
//     slot's own, so the block scheduler no longer serves it after every
//     smaller proof (captured graphs run at the priority of the stream they are
//     launched into).  Without ageing, the largest circuit's requests absorb the
//     priority given to the small ones and their tail latency exceeds that of a
//     plain FIFO queue.
// A request's result does not depend on what else is in flight: every slot has
// its own buffers and the resident key data is read only.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <thread>
#include <vector>

#include "prover.cuh"

namespace nkr {

namespace {

constexpr size_t kServerHeadroom = size_t(2) << 30;

using Clock = std::chrono::steady_clock;

struct Request {
    uint64_t id = 0;
    int key_id = 0;
    bool aged = false;
    const void *witness = nullptr;
    Clock::time_point t_submit, t_start, t_done;
    bool done = false;
    int status = NKR_B200_OK;
    std::string error;
    nkr_b200_raw_proof raw{};
};

struct SlotState {
    ProveSlot *slot = nullptr;
    cudaEvent_t ev_finish = nullptr;
    cudaEvent_t ev_ready = nullptr;   // the witness upload, for an aged launch
    cudaStream_t urgent = nullptr;    // highest-priority launch stream (made on first use)
    Request *req = nullptr; // in flight on this slot
};

struct KeyState {
    nkr_b200_key *key = nullptr;
    std::vector<SlotState> slots;
    double service_ms = 0; // running average of t_done - t_start (0: none completed yet)
};

} // namespace

} // namespace nkr

struct nkr_b200_server {
    nkr_b200_ctx *ctx = nullptr;
    int max_inflight = 8;
    int max_slots_per_key = 4;
    double age_factor = 0.5; // 0: no ageing
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::vector<nkr::KeyState> keys;
    std::deque<nkr::Request *> waiting;
    std::map<uint64_t, std::unique_ptr<nkr::Request>> requests;
    uint64_t next_id = 1;
    int inflight = 0;
    bool stop = false;
    std::thread worker;
    // statistics
    uint64_t completed = 0, failed = 0, aged = 0;
    double busy_first_ms = -1, busy_last_ms = 0;
    nkr::Clock::time_point t0 = nkr::Clock::now();
};

namespace nkr {

namespace {

double ms_since(const Clock::time_point &a, const Clock::time_point &b)
{
    return std::chrono::duration<double, std::milli>(b - a).count();
}

// Requests of one key that may be on the GPU at once.  A proof of 2^19 rows or
// more fills the GPU by itself; running several of them side by side makes
// every one of them finish late (processor sharing among equal jobs: two
// together both end at about twice the time, one after the other end at one
// and two times), so such keys prove one request at a time and the rest wait in
// arrival order.  Smaller keys take up to max_slots_per_key.
int key_slot_cap(const nkr_b200_server *sv, const nkr_b200_key *key)
{
    return key->logn >= 19 ? 1 : sv->max_slots_per_key;
}

// The slot's highest-priority launch stream (created on first use) and the event
// that orders it after the witness upload on the slot's main stream.
int aged_stream(SlotState *st, cudaStream_t *out)
{
    if (!st->urgent) {
        int least = 0, greatest = 0;
        NKR_CUDA(cudaDeviceGetStreamPriorityRange(&least, &greatest));
        NKR_CUDA(cudaStreamCreateWithPriority(&st->urgent, cudaStreamNonBlocking, greatest));
        NKR_CUDA(cudaEventCreateWithFlags(&st->ev_ready, cudaEventDisableTiming));
    }
    *out = st->urgent;
    return NKR_B200_OK;
}

// Start request r on a free slot of its key; returns false when none can be had.
bool try_start(nkr_b200_server *sv, Request *r)
{
    KeyState &ks = sv->keys[r->key_id];
    SlotState *free_slot = nullptr;
    for (auto &s : ks.slots)
        if (!s.req) {
            free_slot = &s;
            break;
        }
    if (!free_slot && int(ks.slots.size()) < key_slot_cap(sv, ks.key)) {
        // the key's existing slots first (slot 0 is always resident), then new
        // ones while free HBM admits them
        nkr_b200_key *key = ks.key;
        ProveSlot *sl = nullptr;
        if (ks.slots.size() < key->slots.size()) {
            sl = key->slots[ks.slots.size()].get();
        } else {
            size_t free_b = 0, total_b = 0;
            if (cudaMemGetInfo(&free_b, &total_b) == cudaSuccess &&
                free_b >= key->slot_bytes + kServerHeadroom && slot_add(key) == NKR_B200_OK)
                sl = key->slots.back().get();
            cudaGetLastError();
        }
        if (sl && slot_capture(key, sl) == NKR_B200_OK) {
            SlotState st;
            st.slot = sl;
            if (cudaEventCreateWithFlags(&st.ev_finish, cudaEventDisableTiming) == cudaSuccess) {
                ks.slots.push_back(st);
                free_slot = &ks.slots.back();
            }
        }
    }
    if (!free_slot) return false;
    ProveSlot *sl = free_slot->slot;
    r->t_start = Clock::now();
    r->aged = sv->age_factor > 0 && ks.service_ms > 0 &&
              ms_since(r->t_submit, r->t_start) > sv->age_factor * ks.service_ms;
    int s = slot_upload_witness(ks.key, sl, r->witness);
    cudaStream_t launch = sl->main();
    if (s == NKR_B200_OK && r->aged) {
        s = aged_stream(free_slot, &launch);
        if (s == NKR_B200_OK && (cudaEventRecord(free_slot->ev_ready, sl->main()) != cudaSuccess ||
                                 cudaStreamWaitEvent(launch, free_slot->ev_ready, 0) != cudaSuccess))
            s = NKR_B200_ECUDA;
    }
    if (s == NKR_B200_OK) s = slot_launch(sl, launch);
    if (s == NKR_B200_OK &&
        cudaMemcpyAsync(sl->pinned_out, sl->out.p, kOutBytes, cudaMemcpyDeviceToHost, launch) !=
            cudaSuccess)
        s = NKR_B200_ECUDA;
    if (s == NKR_B200_OK && cudaEventRecord(free_slot->ev_finish, launch) != cudaSuccess)
        s = NKR_B200_ECUDA;
    if (s == NKR_B200_OK && r->aged) ++sv->aged;
    if (s != NKR_B200_OK) {
        r->status = s;
        r->error = get_error();
        r->done = true;
        r->t_done = Clock::now();
        ++sv->failed;
        sv->cv_done.notify_all();
        return true;
    }
    free_slot->req = r;
    ++sv->inflight;
    return true;
}

void worker_loop(nkr_b200_server *sv)
{
    cudaSetDevice(sv->ctx->device);
    std::unique_lock<std::mutex> lk(sv->mu);
    while (true) {
        // admit: oldest first; a request whose key has no free slot does not
        // block requests of other keys behind it
        for (auto it = sv->waiting.begin(); it != sv->waiting.end() && sv->inflight < sv->max_inflight;) {
            if (try_start(sv, *it))
                it = sv->waiting.erase(it);
            else
                ++it;
        }
        // complete
        bool any = false;
        for (auto &ks : sv->keys)
            for (auto &s : ks.slots) {
                if (!s.req) continue;
                const cudaError_t q = cudaEventQuery(s.ev_finish);
                if (q == cudaErrorNotReady) continue;
                Request *r = s.req;
                s.req = nullptr;
                --sv->inflight;
                any = true;
                r->t_done = Clock::now();
                if (q != cudaSuccess) {
                    r->status = NKR_B200_ECUDA;
                    r->error = cudaGetErrorString(q);
                    ++sv->failed;
                } else {
                    normalize_raw(s.slot->pinned_out);
                    raw_from_bytes(s.slot->pinned_out, &r->raw);
                    ++sv->completed;
                    const double svc = ms_since(r->t_start, r->t_done);
                    ks.service_ms = ks.service_ms > 0 ? 0.75 * ks.service_ms + 0.25 * svc : svc;
                }
                r->done = true;
                const double t_ms = ms_since(sv->t0, r->t_done);
                sv->busy_last_ms = t_ms;
            }
        if (any) sv->cv_done.notify_all();
        if (sv->stop && sv->inflight == 0 && sv->waiting.empty()) break;
        if (sv->inflight == 0 && sv->waiting.empty()) {
            sv->cv_work.wait(lk, [&] { return sv->stop || !sv->waiting.empty(); });
        } else {
            // device work in flight: poll again shortly
            lk.unlock();
            std::this_thread::sleep_for(std::chrono::microseconds(50));
            lk.lock();
        }
    }
}

} // namespace

} // namespace nkr

using nkr::Clock;

extern "C" {

int nkr_b200_server_create(nkr_b200_ctx *ctx, int max_inflight, int max_slots_per_key,
                           nkr_b200_server **out)
{
    NKR_REQUIRE(ctx && out, "null argument");
    NKR_REQUIRE(max_inflight >= 1 && max_slots_per_key >= 1, "server limits must be positive");
    auto *sv = new nkr_b200_server();
    sv->ctx = ctx;
    sv->max_inflight = max_inflight;
    sv->max_slots_per_key = max_slots_per_key;
    sv->worker = std::thread(nkr::worker_loop, sv);
    *out = sv;
    return NKR_B200_OK;
}

int nkr_b200_server_add_key(nkr_b200_server *sv, nkr_b200_key *key, int *key_id)
{
    NKR_REQUIRE(sv && key && key_id, "null argument");
    NKR_REQUIRE(key->ctx == sv->ctx, "key belongs to another context");
    std::lock_guard<std::mutex> g(sv->mu);
    for (size_t i = 0; i < sv->keys.size(); ++i)
        NKR_REQUIRE(sv->keys[i].key != key, "key already added (id %zu)", i);
    nkr::KeyState ks;
    ks.key = key;
    sv->keys.push_back(ks);
    *key_id = int(sv->keys.size() - 1);
    return NKR_B200_OK;
}

int nkr_b200_server_submit(nkr_b200_server *sv, int key_id, const void *witness, uint64_t *request_id)
{
    NKR_REQUIRE(sv && witness && request_id, "null argument");
    std::lock_guard<std::mutex> g(sv->mu);
    NKR_REQUIRE(!sv->stop, "server is stopping");
    NKR_REQUIRE(key_id >= 0 && key_id < int(sv->keys.size()), "unknown key id %d", key_id);
    auto r = std::make_unique<nkr::Request>();
    r->id = sv->next_id++;
    r->key_id = key_id;
    r->witness = witness;
    r->t_submit = Clock::now();
    sv->waiting.push_back(r.get());
    *request_id = r->id;
    sv->requests[r->id] = std::move(r);
    sv->cv_work.notify_one();
    return NKR_B200_OK;
}

int nkr_b200_server_wait(nkr_b200_server *sv, uint64_t request_id, nkr_b200_raw_proof *out,
                         double *latency_ms, double *queue_ms)
{
    NKR_REQUIRE(sv && out, "null argument");
    std::unique_lock<std::mutex> lk(sv->mu);
    auto it = sv->requests.find(request_id);
    NKR_REQUIRE(it != sv->requests.end(), "unknown request id %llu", (unsigned long long)request_id);
    nkr::Request *r = it->second.get();
    sv->cv_done.wait(lk, [&] { return r->done; });
    const int status = r->status;
    if (status == NKR_B200_OK) {
        *out = r->raw;
    } else {
        nkr::set_error("request %llu failed: %s", (unsigned long long)request_id, r->error.c_str());
    }
    if (latency_ms) *latency_ms = nkr::ms_since(r->t_submit, r->t_done);
    if (queue_ms) *queue_ms = nkr::ms_since(r->t_submit, r->t_start);
    sv->requests.erase(it);
    return status;
}

int nkr_b200_server_set_ageing(nkr_b200_server *sv, double age_factor)
{
    NKR_REQUIRE(sv && age_factor >= 0, "bad argument");
    std::lock_guard<std::mutex> g(sv->mu);
    sv->age_factor = age_factor;
    return NKR_B200_OK;
}

int nkr_b200_server_stats(nkr_b200_server *sv, uint64_t *completed, uint64_t *failed, uint64_t *aged)
{
    NKR_REQUIRE(sv, "null argument");
    std::lock_guard<std::mutex> g(sv->mu);
    if (completed) *completed = sv->completed;
    if (failed) *failed = sv->failed;
    if (aged) *aged = sv->aged;
    return NKR_B200_OK;
}

int nkr_b200_server_slots(nkr_b200_server *sv, int key_id, int *slots)
{
    NKR_REQUIRE(sv && slots, "null argument");
    std::lock_guard<std::mutex> g(sv->mu);
    NKR_REQUIRE(key_id >= 0 && key_id < int(sv->keys.size()), "unknown key id %d", key_id);
    *slots = int(sv->keys[key_id].slots.size());
    return NKR_B200_OK;
}

void nkr_b200_server_destroy(nkr_b200_server *sv)
{
    if (!sv) return;
    {
        std::lock_guard<std::mutex> g(sv->mu);
        sv->stop = true;
        sv->cv_work.notify_all();
    }
    if (sv->worker.joinable()) sv->worker.join();
    cudaSetDevice(sv->ctx->device);
    for (auto &ks : sv->keys)
        for (auto &s : ks.slots) {
            if (s.ev_finish) cudaEventDestroy(s.ev_finish);
            if (s.ev_ready) cudaEventDestroy(s.ev_ready);
            if (s.urgent) cudaStreamDestroy(s.urgent);
        }
    delete sv;
}

} // extern "C"
