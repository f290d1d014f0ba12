// MSM window autotuner.  The window width c trades accumulation work (about
// n * ceil(255 / c) mixed additions) against bucket reduction and fix-up work
// (about 2^(c-1) buckets, each a few dependent full additions).  The cost model
// in msm_shape weighs the two by product counts; the reduction is latency
// bound, so its real cost per bucket depends on the part and the size.  The
// tuner times the whole MSM (sort + accumulation + reduction) on this device for
// the model's c and its neighbours, once per power-of-two size class, and keeps
// the fastest.  Any c gives the same (canonical) result.
#define NKR_FIELD_MUL_OUTLINE 1
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "msm.cuh"
#include "prover.cuh"

namespace nkr {

namespace {

constexpr int kTuneMinLog = 10;   // smaller MSMs use the model
constexpr int kTuneMaxLog = 22;   // larger sizes extrapolate from 2^22
constexpr int kTunePoints = 1024; // distinct synthetic bases, tiled

__device__ __forceinline__ uint64_t mix64(uint64_t x)
{
    x += 0x9e3779b97f4a7c15ull;
    x = (x ^ (x >> 30)) * 0xbf58476d1ce4e5b9ull;
    x = (x ^ (x >> 27)) * 0x94d049bb133111ebull;
    return x ^ (x >> 31);
}

// 252 random bits per scalar (below r): a valid Montgomery representative
__global__ void k_tune_scalars(Fr *s, uint64_t n, uint64_t seed)
{
    const uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    Fr v;
    for (int j = 0; j < 4; ++j) {
        const uint64_t w = mix64(seed ^ (i * 4 + j));
        v.v[2 * j] = uint32_t(w);
        v.v[2 * j + 1] = uint32_t(w >> 32);
    }
    v.v[7] &= 0x0fffffffu;
    s[i] = v;
}

// tab[j] = k_j G1 with pseudo-random k_j (affine)
__global__ void k_tune_points(G1Affine *tab, int count, uint64_t seed)
{
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j >= count) return;
    uint32_t k[8];
    for (int q = 0; q < 4; ++q) {
        const uint64_t w = mix64(seed ^ (uint64_t(j) * 4 + q));
        k[2 * q] = uint32_t(w);
        k[2 * q + 1] = uint32_t(w >> 32);
    }
    k[7] &= 0x0fffffffu;
    k[0] |= 1u;
    const G1Affine g{Fq::one(), Fq::one() + Fq::one()}; // (1, 2)
    tab[j] = xyzz_to_affine(xyzz_mul_canon(g, k));
}

// libff Jacobian rows (X, Y, Z = 1) of the tiled table
__global__ void k_tune_jac(const G1Affine *tab, int count, Fq *jac, uint64_t n)
{
    const uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const G1Affine a = tab[i % uint64_t(count)];
    jac[3 * i] = a.x;
    jac[3 * i + 1] = a.y;
    jac[3 * i + 2] = Fq::one();
}

bool autotune_enabled(const nkr_b200_ctx *ctx)
{
    const char *e = std::getenv("NKR_B200_AUTOTUNE");
    if (e && std::strcmp(e, "0") == 0) return false;
    return ctx->autotune;
}

int measure(nkr_b200_ctx *ctx, int lg)
{
    cudaStream_t st = ctx->stream;
    const uint64_t n = uint64_t(1) << lg;
    DevBuf tab, jac, sc;
    NKR_TRY(tab.alloc(kTunePoints * sizeof(G1Affine), "tuner bases"));
    NKR_TRY(jac.alloc(n * 96, "tuner bases"));
    NKR_TRY(sc.alloc(n * sizeof(Fr), "tuner scalars"));
    k_tune_points<<<blocks_for(kTunePoints, 64), 64, 0, st>>>(tab.as<G1Affine>(), kTunePoints, 0x5eedull);
    NKR_CHECK_LAUNCH();
    k_tune_jac<<<blocks_for(n, 256), 256, 0, st>>>(tab.as<G1Affine>(), kTunePoints, jac.as<Fq>(), n);
    NKR_CHECK_LAUNCH();
    k_tune_scalars<<<blocks_for(n, 256), 256, 0, st>>>(sc.as<Fr>(), n, 0x5ca1ull + lg);
    NKR_CHECK_LAUNCH();
    cudaEvent_t e0, e1;
    NKR_CUDA(cudaEventCreate(&e0));
    NKR_CUDA(cudaEventCreate(&e1));
    const int c0 = msm_shape(n, true, 1).c;
    int best_c = c0;
    float best = 1e30f;
    int status = NKR_B200_OK;
    for (int c = c0 - 3; c <= c0 + 1 && status == NKR_B200_OK; ++c) {
        if (c < 6 || c > 22) continue;
        MsmBases b;
        MsmScratch s;
        status = msm_bases_build(b, 1, jac.p, true, n, true, c, false, st);
        if (status == NKR_B200_OK) status = msm_scratch_alloc(s, 1, b.shape);
        if (status != NKR_B200_OK) break;
        float t_min = 1e30f;
        for (int rep = 0; rep < 4 && status == NKR_B200_OK; ++rep) {
            cudaEventRecord(e0, st);
            status = msm_run(b, s, sc.p, s.acc.result.p, st);
            cudaEventRecord(e1, st);
            if (cudaEventSynchronize(e1) != cudaSuccess) {
                set_error("tuner: %s", cudaGetErrorString(cudaGetLastError()));
                status = NKR_B200_ECUDA;
                break;
            }
            float ms = 0.f;
            cudaEventElapsedTime(&ms, e0, e1);
            if (rep > 0 && ms < t_min) t_min = ms; // rep 0 warms up
        }
        if (t_min < best) {
            best = t_min;
            best_c = c;
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (status != NKR_B200_OK) return status;
    ctx->msm_window[lg] = best_c;
    ctx->msm_window_ms[lg] = best;
    return NKR_B200_OK;
}

} // namespace

int tuned_window_bits(nkr_b200_ctx *ctx, uint64_t n, int *c)
{
    *c = 0;
    if (!autotune_enabled(ctx)) return NKR_B200_OK;
    int lg = 0;
    while ((uint64_t(1) << lg) < n) ++lg;
    if (lg < kTuneMinLog) return NKR_B200_OK;
    NKR_CUDA(cudaSetDevice(ctx->device));
    const int lm = lg > kTuneMaxLog ? kTuneMaxLog : lg;
    if (!ctx->msm_window[lm]) NKR_TRY(measure(ctx, lm));
    if (lg == lm) {
        *c = ctx->msm_window[lm];
    } else {
        const int off = ctx->msm_window[lm] - msm_shape(uint64_t(1) << lm, true, 1).c;
        int v = msm_shape(n, true, 1).c + off;
        *c = v < 6 ? 6 : v > 22 ? 22 : v;
    }
    return NKR_B200_OK;
}

} // namespace nkr

// Tuned widths persist across processes: the reference's CLI proves once per
// process (app/prove.cpp:70-88), and every process would otherwise measure the
// same size classes again (about 1.6 s for a 2^20 key's classes).  Text file:
//   nkr-b200-tune 1
//   device <cudaDeviceProp::name>
//   sms <multiprocessor count>
//   msm <log2 size class> <window bits> <ms>     (one line per measured class)
namespace nkr {

namespace {

int device_identity(const nkr_b200_ctx *ctx, char *name, size_t len)
{
    cudaDeviceProp prop{};
    NKR_CUDA(cudaGetDeviceProperties(&prop, ctx->device));
    std::snprintf(name, len, "%s", prop.name);
    return NKR_B200_OK;
}

} // namespace

} // namespace nkr

extern "C" {

int nkr_b200_tune_save(nkr_b200_ctx *ctx, const char *path)
{
    NKR_REQUIRE(ctx && path, "null argument");
    char name[256];
    NKR_TRY(nkr::device_identity(ctx, name, sizeof name));
    FILE *f = std::fopen(path, "w");
    NKR_REQUIRE(f, "%s: cannot open for writing", path);
    bool ok = std::fprintf(f, "nkr-b200-tune 1\ndevice %s\nsms %d\n", name, ctx->sm_count) > 0;
    for (int lg = 0; lg < 33 && ok; ++lg)
        if (ctx->msm_window[lg])
            ok = std::fprintf(f, "msm %d %d %.6f\n", lg, ctx->msm_window[lg], ctx->msm_window_ms[lg]) > 0;
    ok = (std::fclose(f) == 0) && ok;
    NKR_REQUIRE(ok, "%s: write failed", path);
    return NKR_B200_OK;
}

int nkr_b200_tune_load(nkr_b200_ctx *ctx, const char *path, int *loaded)
{
    NKR_REQUIRE(ctx && path, "null argument");
    if (loaded) *loaded = 0;
    char name[256];
    NKR_TRY(nkr::device_identity(ctx, name, sizeof name));
    FILE *f = std::fopen(path, "r");
    NKR_REQUIRE(f, "%s: cannot open", path);
    char line[512];
    int version = 0, sms = -1, n = 0, window[33] = {};
    float ms[33] = {};
    bool same_device = false, bad = false;
    while (std::fgets(line, sizeof line, f)) {
        line[std::strcspn(line, "\r\n")] = 0;
        int lg = 0, c = 0;
        float t = 0.f;
        if (std::sscanf(line, "nkr-b200-tune %d", &version) == 1) continue;
        if (std::strncmp(line, "device ", 7) == 0) {
            same_device = std::strcmp(line + 7, name) == 0;
        } else if (std::sscanf(line, "sms %d", &sms) == 1) {
        } else if (std::sscanf(line, "msm %d %d %f", &lg, &c, &t) == 3) {
            if (lg < 0 || lg > 32 || c < 6 || c > 22) bad = true;
            else {
                window[lg] = c;
                ms[lg] = t;
                ++n;
            }
        } else if (line[0]) {
            bad = true;
        }
    }
    std::fclose(f);
    NKR_REQUIRE(version == 1 && !bad, "%s: not a tuning file of this library", path);
    NKR_REQUIRE(same_device && sms == ctx->sm_count, "%s: measured on another device", path);
    for (int lg = 0; lg < 33; ++lg)
        if (window[lg]) {
            ctx->msm_window[lg] = window[lg];
            ctx->msm_window_ms[lg] = ms[lg];
        }
    if (loaded) *loaded = n;
    return NKR_B200_OK;
}

} // extern "C"
