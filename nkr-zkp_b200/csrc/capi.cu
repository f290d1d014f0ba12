// extern "C" surface of libnkr_b200.so (declarations and reference mapping in
// include/nkr_b200.h).  Every entry point converts failures to a status code
// plus a thread-local message; nothing here exits the process.
#include <cstdarg>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>

#include "../host/fr_host.hpp"
#include "msm.cuh"
#include "ntt.cuh"
#include "ops.cuh"
#include "prover.cuh"
#include "scan.cuh"
#include "spmv.cuh"

namespace nkr {

std::atomic<unsigned long long> g_kernel_launches{0};

namespace {
thread_local char g_err[1024] = "";
std::mutex g_table_mu;
std::map<std::pair<int, int>, std::unique_ptr<NttTables>> g_tables; // (device, logn)
} // namespace

void set_error(const char *fmt, ...)
{
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(g_err, sizeof(g_err), fmt, ap);
    va_end(ap);
}

const char *get_error() { return g_err; }

int device_alloc(void **p, size_t bytes, const char *what)
{
    // Admission against free HBM for large buffers, keeping 512 MiB of headroom for
    // the runtime and other tenants of the GPU.  Buffers under 64 MiB skip the
    // query (cudaMemGetInfo costs about as much as the allocation itself, and a
    // small key's prove slot makes ~90 of them): a failing cudaMalloc still
    // reports NKR_B200_ENOMEM.
    cudaError_t e;
    if (bytes >= (size_t(64) << 20)) {
        size_t free_b = 0, total_b = 0;
        e = cudaMemGetInfo(&free_b, &total_b);
        if (e != cudaSuccess) {
            set_error("cudaMemGetInfo: %s", cudaGetErrorString(e));
            return NKR_B200_ECUDA;
        }
        const size_t reserve = size_t(512) << 20;
        if (bytes + reserve > free_b) {
            set_error("device memory admission refused for %s: need %zu B, %zu B free", what, bytes,
                      free_b);
            return NKR_B200_ENOMEM;
        }
    }
    e = cudaMalloc(p, bytes);
    if (e != cudaSuccess) {
        cudaGetLastError();
        set_error("cudaMalloc(%zu) for %s: %s", bytes, what, cudaGetErrorString(e));
        return NKR_B200_ENOMEM;
    }
    return NKR_B200_OK;
}

__global__ void __launch_bounds__(kScanThreads) k_scan_block_totals(uint32_t *totals, uint32_t nb)
{
    const uint32_t base = threadIdx.x * kScanItems;
    uint32_t v[kScanItems], s = 0;
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
        v[i] = base + i < nb ? totals[base + i] : 0;
        s += v[i];
    }
    uint32_t total;
    uint32_t run = block_excl_scan(s, &total);
#pragma unroll
    for (int i = 0; i < kScanItems; ++i) {
        if (base + i < nb) totals[base + i] = run;
        run += v[i];
    }
}

int get_tables(nkr_b200_ctx *ctx, int logn, const NttTables **out)
{
    std::lock_guard<std::mutex> g(g_table_mu);
    auto &slot = g_tables[{ctx->device, logn}];
    if (!slot) {
        auto t = std::make_unique<NttTables>();
        NKR_TRY(ntt_tables_build(*t, logn, ctx->stream));
        slot = std::move(t);
    }
    *out = slot.get();
    return NKR_B200_OK;
}

int key_prepare(nkr_b200_ctx *, const nkr_b200_circuit *, const nkr_b200_proving_key *,
                nkr_b200_key **);
int key_prove(nkr_b200_key *, const void *, uint64_t, nkr_b200_raw_proof *);
int key_blind(nkr_b200_key *, const nkr_b200_raw_proof *, const void *, const void *,
              nkr_b200_proof *);
int key_intermediates(nkr_b200_key *, void *, void *, void *, void *);
int key_prove_batch(nkr_b200_key *const *, const void *const *, int, nkr_b200_raw_proof *);
int key_prove_batch_lists(nkr_b200_key *const *, const void *const *, int, nkr_b200_raw_proof *);

int ctx_check(nkr_b200_ctx *ctx)
{
    NKR_REQUIRE(ctx != nullptr, "null context");
    NKR_CUDA(cudaSetDevice(ctx->device));
    return NKR_B200_OK;
}

} // namespace nkr

struct nkr_b200_msm_bases {
    nkr_b200_ctx *ctx;
    nkr::MsmBases bases;
    nkr::MsmScratch scratch;
    nkr::DevBuf scalars;
    nkr_b200_msm_stats last{};
};

using namespace nkr;

extern "C" {

const char *nkr_b200_last_error(void) { return get_error(); }
uint64_t nkr_b200_launch_count(void) { return g_kernel_launches.load(); }
const char *nkr_b200_backend_name(void) { return "b200"; }

int nkr_b200_open(int device, nkr_b200_ctx **out)
{
    NKR_REQUIRE(out != nullptr, "null output handle");
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || count == 0) {
        cudaGetLastError();
        set_error("no CUDA device available (%s)", cudaGetErrorString(e));
        return NKR_B200_ENODEV;
    }
    NKR_REQUIRE(device >= 0 && device < count, "device %d out of range (%d devices)", device, count);
    cudaDeviceProp prop{};
    NKR_CUDA(cudaGetDeviceProperties(&prop, device));
    if (prop.major != 10) {
        set_error("device %d is sm_%d%d; this library is built for sm_100a only", device,
                  prop.major, prop.minor);
        return NKR_B200_ENODEV;
    }
    NKR_CUDA(cudaSetDevice(device));
    auto *ctx = new nkr_b200_ctx();
    ctx->device = device;
    ctx->sm_count = prop.multiProcessorCount;
    if (cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking) != cudaSuccess) {
        delete ctx;
        set_error("stream creation failed");
        return NKR_B200_ECUDA;
    }
    *out = ctx;
    return NKR_B200_OK;
}

void nkr_b200_close(nkr_b200_ctx *ctx)
{
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    {
        std::lock_guard<std::mutex> g(g_table_mu);
        for (auto it = g_tables.begin(); it != g_tables.end();)
            if (it->first.first == ctx->device)
                it = g_tables.erase(it);
            else
                ++it;
    }
    cudaStreamDestroy(ctx->stream);
    delete ctx;
}

int nkr_b200_prepare(nkr_b200_ctx *ctx, const nkr_b200_circuit *circuit,
                     const nkr_b200_proving_key *pk, nkr_b200_key **out)
{
    NKR_TRY(ctx_check(ctx));
    return key_prepare(ctx, circuit, pk, out);
}

int nkr_b200_prove(nkr_b200_key *key, const void *witness, uint64_t n, nkr_b200_raw_proof *out)
{
    return key_prove(key, witness, n, out);
}

int nkr_b200_blind(nkr_b200_key *key, const nkr_b200_raw_proof *raw, const void *r, const void *s,
                   nkr_b200_proof *out)
{
    return key_blind(key, raw, r, s, out);
}

int nkr_b200_key_intermediates(nkr_b200_key *key, void *az, void *bz, void *cz, void *h)
{
    return key_intermediates(key, az, bz, cz, h);
}

int nkr_b200_key_stage_times(const nkr_b200_key *key, nkr_b200_stage_times *out)
{
    NKR_REQUIRE(key && out, "null argument");
    NKR_REQUIRE(key->have_times, "no timed prove on this key yet");
    *out = key->times;
    return NKR_B200_OK;
}

int nkr_b200_prove_batch(nkr_b200_key *const *keys, const void *const *witnesses, int count,
                         nkr_b200_raw_proof *out)
{
    return key_prove_batch(keys, witnesses, count, out);
}

int nkr_b200_prove_batch_lists(nkr_b200_key *const *keys, const void *const *witnesses, int count,
                               nkr_b200_raw_proof *out)
{
    return key_prove_batch_lists(keys, witnesses, count, out);
}

int nkr_b200_ntt(nkr_b200_ctx *ctx, int op, void *data, uint64_t n)
{
    NKR_TRY(ctx_check(ctx));
    NKR_REQUIRE(data != nullptr, "null data");
    NKR_REQUIRE(op >= 0 && op <= 4, "ntt op %d unknown", op);
    const int logn = log2_exact(n);
    NKR_REQUIRE(logn >= 1 && logn <= 28, "NTT size %llu must be a power of two in [2, 2^28]",
                (unsigned long long)n);
    const NttTables *T;
    NKR_TRY(get_tables(ctx, logn, &T));
    cudaStream_t st = ctx->stream;
    DevBuf a, b;
    NKR_TRY(a.alloc(n * 32, "ntt data"));
    NKR_TRY(b.alloc(n * 32, "ntt scratch"));
    NKR_CUDA(cudaMemcpyAsync(a.p, data, n * 32, cudaMemcpyHostToDevice, st));
    const Fr *c = T->consts.as<Fr>();
    Fr *pa = a.as<Fr>(), *pb = b.as<Fr>();
    Fr *res = pb;
    switch (op) {
    case 0: // FFT
        NKR_TRY(ntt_dif(*T, pa, false, nullptr, nullptr, nullptr, st));
        NKR_TRY(ntt_bitrev_permute(pa, pb, n, nullptr, nullptr, st));
        break;
    case 1: // iFFT
        NKR_TRY(ntt_dif(*T, pa, true, nullptr, nullptr, nullptr, st));
        NKR_TRY(ntt_bitrev_permute(pa, pb, n, nullptr, c + kConstNinv, st));
        break;
    case 2: // cosetFFT
        NKR_TRY(ntt_dif(*T, pa, false, T->gpow.as<Fr>(), nullptr, nullptr, st));
        NKR_TRY(ntt_bitrev_permute(pa, pb, n, nullptr, nullptr, st));
        break;
    case 3: // icosetFFT
        NKR_TRY(ntt_dif(*T, pa, true, nullptr, nullptr, nullptr, st));
        NKR_TRY(ntt_bitrev_permute(pa, pb, n, T->t2.as<Fr>(), nullptr, st));
        break;
    case 4: // divide_by_Z_on_coset
        NKR_TRY(fr_scale_const(pa, n, c + kConstZinv, st));
        res = pa;
        break;
    }
    NKR_CUDA(cudaMemcpyAsync(data, res, n * 32, cudaMemcpyDeviceToHost, st));
    NKR_CUDA(cudaStreamSynchronize(st));
    return NKR_B200_OK;
}

int nkr_b200_ntt_device(nkr_b200_ctx *ctx, int op, void *in, void *out, uint64_t n, void *stream,
                        float *device_ms)
{
    NKR_TRY(ctx_check(ctx));
    NKR_REQUIRE(in && out, "null data");
    NKR_REQUIRE(op >= 0 && op <= 4, "ntt op %d unknown", op);
    const int logn = log2_exact(n);
    NKR_REQUIRE(logn >= 1 && logn <= 28, "NTT size %llu must be a power of two in [2, 2^28]",
                (unsigned long long)n);
    const uint8_t *ib = static_cast<const uint8_t *>(in), *ob = static_cast<const uint8_t *>(out);
    NKR_REQUIRE(ib + n * 32 <= ob || ob + n * 32 <= ib, "in and out overlap");
    for (const void *p : {static_cast<const void *>(in), static_cast<const void *>(out)}) {
        cudaPointerAttributes attr{};
        const cudaError_t e = cudaPointerGetAttributes(&attr, p);
        if (e != cudaSuccess) cudaGetLastError();
        NKR_REQUIRE(e == cudaSuccess && attr.type == cudaMemoryTypeDevice &&
                        attr.device == ctx->device,
                    "ntt_device buffers must be device memory of device %d", ctx->device);
    }
    const NttTables *T;
    NKR_TRY(get_tables(ctx, logn, &T));
    // NULL is CUDA's legacy default stream, so work the caller queued there (for
    // instance the copy that filled `in`) is ordered before the transform
    cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : cudaStreamLegacy;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    if (device_ms) {
        NKR_CUDA(cudaEventCreate(&e0));
        NKR_CUDA(cudaEventCreate(&e1));
        NKR_CUDA(cudaEventRecord(e0, st));
    }
    const Fr *c = T->consts.as<Fr>();
    Fr *pa = static_cast<Fr *>(in), *pb = static_cast<Fr *>(out);
    switch (op) {
    case 0:
        NKR_TRY(ntt_dif(*T, pa, false, nullptr, nullptr, nullptr, st));
        NKR_TRY(ntt_bitrev_permute(pa, pb, n, nullptr, nullptr, st));
        break;
    case 1:
        NKR_TRY(ntt_dif(*T, pa, true, nullptr, nullptr, nullptr, st));
        NKR_TRY(ntt_bitrev_permute(pa, pb, n, nullptr, c + kConstNinv, st));
        break;
    case 2:
        NKR_TRY(ntt_dif(*T, pa, false, T->gpow.as<Fr>(), nullptr, nullptr, st));
        NKR_TRY(ntt_bitrev_permute(pa, pb, n, nullptr, nullptr, st));
        break;
    case 3:
        NKR_TRY(ntt_dif(*T, pa, true, nullptr, nullptr, nullptr, st));
        NKR_TRY(ntt_bitrev_permute(pa, pb, n, T->t2.as<Fr>(), nullptr, st));
        break;
    case 4:
        NKR_TRY(fr_scale_const(pa, n, c + kConstZinv, st));
        NKR_CUDA(cudaMemcpyAsync(pb, pa, n * 32, cudaMemcpyDeviceToDevice, st));
        break;
    }
    if (device_ms) {
        NKR_CUDA(cudaEventRecord(e1, st));
        NKR_CUDA(cudaEventSynchronize(e1));
        NKR_CUDA(cudaEventElapsedTime(device_ms, e0, e1));
        cudaEventDestroy(e0);
        cudaEventDestroy(e1);
    }
    return NKR_B200_OK;
}

int nkr_b200_domain_constants(nkr_b200_ctx *ctx, uint64_t n, void *omega, void *coset)
{
    NKR_TRY(ctx_check(ctx));
    NKR_REQUIRE(omega && coset, "null output");
    const int logn = log2_exact(n);
    NKR_REQUIRE(logn >= 1 && logn <= 28, "domain size %llu must be a power of two in [2, 2^28]",
                (unsigned long long)n);
    const NttTables *T;
    NKR_TRY(get_tables(ctx, logn, &T));
    Fr c[kConstGinv + 1];
    NKR_CUDA(cudaMemcpyAsync(c, T->consts.p, sizeof c, cudaMemcpyDeviceToHost, ctx->stream));
    NKR_CUDA(cudaStreamSynchronize(ctx->stream));
    std::memcpy(omega, &c[kConstOmega], 32);
    std::memcpy(coset, &c[kConstG], 32);
    return NKR_B200_OK;
}

int nkr_b200_quotient_device(nkr_b200_ctx *ctx, const void *a, const void *b, const void *c,
                             void *out, uint64_t n, void *stream)
{
    NKR_TRY(ctx_check(ctx));
    NKR_REQUIRE(a && b && c && out, "null data");
    const int logn = log2_exact(n);
    NKR_REQUIRE(logn >= 1 && logn <= 28, "quotient size %llu must be a power of two in [2, 2^28]",
                (unsigned long long)n);
    for (const void *p : {a, b, c, static_cast<const void *>(out)}) {
        cudaPointerAttributes attr{};
        const cudaError_t e = cudaPointerGetAttributes(&attr, p);
        if (e != cudaSuccess) cudaGetLastError();
        NKR_REQUIRE(e == cudaSuccess && attr.type == cudaMemoryTypeDevice &&
                        attr.device == ctx->device,
                    "quotient buffers must be device memory of device %d", ctx->device);
    }
    const NttTables *T;
    NKR_TRY(get_tables(ctx, logn, &T));
    cudaStream_t st = stream ? static_cast<cudaStream_t>(stream) : cudaStreamLegacy;
    // element-wise: out may be a, b or c
    return fr_quotient_pointwise(static_cast<const Fr *>(a), static_cast<const Fr *>(b),
                                 static_cast<const Fr *>(c), static_cast<Fr *>(out), n,
                                 T->consts.as<Fr>() + kConstZinv, st);
}

int nkr_b200_spmv(nkr_b200_ctx *ctx, uint64_t rows, uint64_t cols, const uint32_t *row_ptr,
                  const uint32_t *col_idx, const void *values, const void *z, void *y)
{
    NKR_TRY(ctx_check(ctx));
    NKR_REQUIRE(z && y, "null vector");
    cudaStream_t st = ctx->stream;
    CsrDevice m;
    NKR_TRY(csr_upload(m, rows, cols, row_ptr, col_idx, values, st));
    DevBuf dz, dy;
    NKR_TRY(dz.alloc(std::max<uint64_t>(cols, 1) * 32, "spmv z"));
    NKR_TRY(dy.alloc(rows * 32, "spmv y"));
    NKR_CUDA(cudaMemcpyAsync(dz.p, z, cols * 32, cudaMemcpyHostToDevice, st));
    DevBuf prod;
    NKR_TRY(prod.alloc(std::max<uint64_t>(m.nu, 1) * 32, "spmv products"));
    const CsrDevice *mats[1] = {&m};
    Fr *ys[1] = {dy.as<Fr>()};
    Fr *prods[1] = {prod.as<Fr>()};
    NKR_TRY(spmv_multi(mats, 1, dz.as<Fr>(), ys, prods, st));
    NKR_CUDA(cudaMemcpyAsync(y, dy.p, rows * 32, cudaMemcpyDeviceToHost, st));
    NKR_CUDA(cudaStreamSynchronize(st));
    return NKR_B200_OK;
}

static int msm_plain(nkr_b200_ctx *ctx, int group, const void *bases, const void *scalars,
                     uint64_t n, void *out)
{
    NKR_TRY(ctx_check(ctx));
    NKR_REQUIRE(out && (n == 0 || (bases && scalars)), "null argument");
    cudaStream_t st = ctx->stream;
    MsmBases b;
    NKR_TRY(msm_bases_build(b, group, bases, false, n, false, 0, false, st));
    MsmScratch s;
    s.acc.lane_pairs = true; // an MSM alone: latency-bound reduction levels
    NKR_TRY(msm_scratch_alloc(s, group, b.shape));
    DevBuf ds;
    NKR_TRY(ds.alloc(std::max<uint64_t>(n, 1) * 32, "msm scalars"));
    if (n) NKR_CUDA(cudaMemcpyAsync(ds.p, scalars, n * 32, cudaMemcpyHostToDevice, st));
    NKR_TRY(msm_run(b, s, ds.p, s.acc.result.p, st));
    NKR_CUDA(cudaMemcpyAsync(out, s.acc.result.p, group == 1 ? 96 : 192, cudaMemcpyDeviceToHost, st));
    NKR_CUDA(cudaStreamSynchronize(st));
    if (group == 1)
        host::normalize_g1(out);
    else
        host::normalize_g2(out);
    return NKR_B200_OK;
}

int nkr_b200_msm_g1(nkr_b200_ctx *ctx, const void *bases, const void *scalars, uint64_t n, void *out)
{
    return msm_plain(ctx, 1, bases, scalars, n, out);
}

int nkr_b200_msm_g2(nkr_b200_ctx *ctx, const void *bases, const void *scalars, uint64_t n, void *out)
{
    return msm_plain(ctx, 2, bases, scalars, n, out);
}

int nkr_b200_msm_bases_create(nkr_b200_ctx *ctx, int group, const void *bases, uint64_t n,
                              nkr_b200_msm_bases **out)
{
    NKR_TRY(ctx_check(ctx));
    NKR_REQUIRE(out && (n == 0 || bases), "null argument");
    auto h = std::make_unique<nkr_b200_msm_bases>();
    h->ctx = ctx;
    std::vector<uint32_t> idx = msm_support(group, bases, n);
    int c = 0;
    NKR_TRY(tuned_window_bits(ctx, idx.size(), &c));
    NKR_TRY(msm_bases_build_support(h->bases, group, bases, n, std::move(idx), true, c, ctx->stream));
    NKR_TRY(msm_scratch_alloc(h->scratch, group, h->bases.shape));
    for (auto &e : h->scratch.acc.ev_acc) NKR_CUDA(cudaEventCreate(&e));
    h->scratch.acc.timing = true;
    h->scratch.acc.lane_pairs = true; // MSMs alone: latency-bound reduction levels
    NKR_TRY(h->scalars.alloc(std::max<uint64_t>(n, 1) * 32, "msm scalars"));
    *out = h.release();
    return NKR_B200_OK;
}

int nkr_b200_msm_bases_run(nkr_b200_msm_bases *b, const void *scalars, uint64_t n, void *out,
                           float *device_ms)
{
    NKR_REQUIRE(b && out, "null argument");
    NKR_REQUIRE(n == b->bases.n_full, "scalar count %llu does not match the %llu bases",
                (unsigned long long)n, (unsigned long long)b->bases.n_full);
    NKR_TRY(ctx_check(b->ctx));
    cudaStream_t st = b->ctx->stream;
    cudaMemoryType mt = cudaMemoryTypeUnregistered;
    {
        cudaPointerAttributes attr{};
        if (cudaPointerGetAttributes(&attr, scalars) == cudaSuccess)
            mt = attr.type;
        else
            cudaGetLastError();
    }
    const void *src = scalars;
    if (mt != cudaMemoryTypeDevice) {
        if (n) NKR_CUDA(cudaMemcpyAsync(b->scalars.p, scalars, n * 32, cudaMemcpyHostToDevice, st));
        src = b->scalars.p;
    }
    cudaEvent_t e0, e1;
    NKR_CUDA(cudaEventCreate(&e0));
    NKR_CUDA(cudaEventCreate(&e1));
    NKR_CUDA(cudaEventRecord(e0, st));
    const int s = msm_run(b->bases, b->scratch, src, b->scratch.acc.result.p, st);
    NKR_CUDA(cudaEventRecord(e1, st));
    NKR_CUDA(cudaMemcpyAsync(out, b->scratch.acc.result.p, b->bases.group == 1 ? 96 : 192,
                             cudaMemcpyDeviceToHost, st));
    NKR_CUDA(cudaStreamSynchronize(st));
    float total = 0.f;
    cudaEventElapsedTime(&total, e0, e1);
    if (device_ms) *device_ms = total;
    if (s == NKR_B200_OK) {
        if (b->bases.group == 1)
            host::normalize_g1(out);
        else
            host::normalize_g2(out);
        b->last.total_ms = total;
        const cudaEvent_t *ev = b->scratch.acc.ev_acc;
        NKR_CUDA(cudaEventElapsedTime(&b->last.sort_ms, e0, ev[0]));
        NKR_CUDA(cudaEventElapsedTime(&b->last.acc_ms, ev[0], ev[1]));
        NKR_CUDA(cudaEventElapsedTime(&b->last.fixup_ms, ev[1], ev[2]));
        NKR_CUDA(cudaEventElapsedTime(&b->last.reduce_first_ms, ev[2], ev[3]));
        NKR_CUDA(cudaEventElapsedTime(&b->last.reduce_levels_ms, ev[3], ev[4]));
        uint32_t entries = 0, tasks = 0;
        const uint32_t nb = b->bases.shape.nb;
        NKR_CUDA(cudaMemcpy(&entries, b->scratch.sort.offsets.as<uint32_t>() + nb, 4, cudaMemcpyDeviceToHost));
        tasks = uint32_t((uint64_t(entries) + b->bases.shape.k1 - 1) / b->bases.shape.k1);
        b->last.entries = entries;
        b->last.tasks = tasks;
        b->last.window_bits = uint32_t(b->bases.shape.c);
        b->last.windows = uint32_t(b->bases.shape.W);
        b->last.buckets = nb;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return s;
}

int nkr_b200_msm_bases_stats(const nkr_b200_msm_bases *b, nkr_b200_msm_stats *out)
{
    NKR_REQUIRE(b && out, "null argument");
    *out = b->last;
    return NKR_B200_OK;
}

void nkr_b200_msm_bases_free(nkr_b200_msm_bases *b)
{
    if (!b) return;
    cudaSetDevice(b->ctx->device);
    cudaStreamSynchronize(b->ctx->stream);
    for (auto &e : b->scratch.acc.ev_acc)
        if (e) cudaEventDestroy(e);
    delete b;
}

int nkr_b200_tune_ntt(nkr_b200_ctx *ctx, uint64_t n, int *max_stages, int *bfly_per_thread)
{
    NKR_TRY(ctx_check(ctx));
    NKR_REQUIRE(max_stages && bfly_per_thread, "null argument");
    const int logn = log2_exact(n);
    NKR_REQUIRE(logn >= 1 && logn <= 28, "NTT size %llu must be a power of two in [2, 2^28]",
                (unsigned long long)n);
    const NttTables *T;
    NKR_TRY(get_tables(ctx, logn, &T));
    *max_stages = T->max_stages;
    *bfly_per_thread = T->bfly_per_thread;
    return NKR_B200_OK;
}

int nkr_b200_set_autotune(nkr_b200_ctx *ctx, int enable)
{
    NKR_REQUIRE(ctx, "null context");
    ctx->autotune = enable != 0;
    return NKR_B200_OK;
}

int nkr_b200_tune_msm(nkr_b200_ctx *ctx, uint64_t n, int *window_bits, float *ms)
{
    NKR_TRY(ctx_check(ctx));
    NKR_REQUIRE(window_bits, "null argument");
    int c = 0;
    NKR_TRY(tuned_window_bits(ctx, n, &c));
    if (c == 0) c = msm_shape(n, true, 1).c;
    *window_bits = c;
    if (ms) {
        int lg = 0;
        while ((uint64_t(1) << lg) < n) ++lg;
        *ms = lg < 33 ? ctx->msm_window_ms[lg] : 0.f;
    }
    return NKR_B200_OK;
}

int nkr_b200_field_op(nkr_b200_ctx *ctx, int field, int op, const void *a, const void *b, void *out,
                      uint64_t n)
{
    NKR_TRY(ctx_check(ctx));
    NKR_REQUIRE(a && out, "null argument");
    NKR_REQUIRE(field >= 0 && field <= 4, "field %d unknown", field);
    const size_t esz = (field == 2 || field == 4) ? 64 : 32; // Fq2 elements are 64 B
    cudaStream_t st = ctx->stream;
    DevBuf da, db, dout;
    NKR_TRY(da.alloc(std::max<uint64_t>(n, 1) * esz, "field op a"));
    NKR_TRY(db.alloc(std::max<uint64_t>(n, 1) * esz, "field op b"));
    NKR_TRY(dout.alloc(std::max<uint64_t>(n, 1) * esz, "field op out"));
    NKR_CUDA(cudaMemcpyAsync(da.p, a, n * esz, cudaMemcpyHostToDevice, st));
    if (b) NKR_CUDA(cudaMemcpyAsync(db.p, b, n * esz, cudaMemcpyHostToDevice, st));
    NKR_TRY(field_op_device(field, op, da.p, b ? db.p : nullptr, dout.p, n, st));
    NKR_CUDA(cudaMemcpyAsync(out, dout.p, n * esz, cudaMemcpyDeviceToHost, st));
    NKR_CUDA(cudaStreamSynchronize(st));
    return NKR_B200_OK;
}

int nkr_b200_group_op(nkr_b200_ctx *ctx, int group, int op, const void *a, const void *b, void *out,
                      uint64_t n)
{
    NKR_TRY(ctx_check(ctx));
    NKR_REQUIRE(a && out && (op == 1 || b), "null argument");
    const size_t psz = group == 1 ? 96 : 192;
    const size_t bsz = op == 2 ? 32 : psz;
    cudaStream_t st = ctx->stream;
    DevBuf da, db, dout;
    NKR_TRY(da.alloc(std::max<uint64_t>(n, 1) * psz, "group op a"));
    NKR_TRY(db.alloc(std::max<uint64_t>(n, 1) * bsz, "group op b"));
    NKR_TRY(dout.alloc(std::max<uint64_t>(n, 1) * psz, "group op out"));
    NKR_CUDA(cudaMemcpyAsync(da.p, a, n * psz, cudaMemcpyHostToDevice, st));
    if (b) NKR_CUDA(cudaMemcpyAsync(db.p, b, n * bsz, cudaMemcpyHostToDevice, st));
    NKR_TRY(group_op_device(group, op, da.p, db.p, dout.p, n, st));
    NKR_CUDA(cudaMemcpyAsync(out, dout.p, n * psz, cudaMemcpyDeviceToHost, st));
    NKR_CUDA(cudaStreamSynchronize(st));
    return NKR_B200_OK;
}

int nkr_b200_bench_mul(nkr_b200_ctx *ctx, int field, double *muls_per_s, double *ms)
{
    NKR_TRY(ctx_check(ctx));
    NKR_REQUIRE(muls_per_s && ms, "null argument");
    return bench_mul_device(field, ctx->sm_count, muls_per_s, ms, ctx->stream);
}

} // extern "C"
