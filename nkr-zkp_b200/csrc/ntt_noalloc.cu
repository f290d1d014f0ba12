// nkr_b200_ntt_noalloc: the libfqfft domain ops of nkr_b200_ntt on caller-owned
// device buffers, with every byte of scratch in one fixed-size array in this file.
//
// Who needs it: a caller that has already given the device's memory to its own
// pool (a serving process whose caching allocator holds most of the 180 GB) can
// see cudaMalloc fail or fragment that pool, and a caller that keeps several
// streams busy cannot afford cudaFree, which waits for the whole device.  This
// entry point calls neither, nor any routine that allocates device memory: the
// twiddle tables and the working vector live in g_ntt_scratch below.
//
// Limit: n = 2^k Fr elements with 1 <= k <= 16 (65,536 elements); larger sizes
// are rejected with NKR_B200_EINVAL.  The array is 5 * 2^16 Fr (10 MiB) plus
// 17 * 8 Fr of per-size constants.
//
// Set-up: the first call on a device (with that device current) looks up the
// array's device address with cudaGetSymbolAddress, builds the tables in it on the
// caller's stream and waits for that stream; later calls only enqueue work.  Make
// the first call on each device before capturing any stream.  The address and the
// tables belong to the device's context: the set-up is keyed by the context's
// unique id, so after cudaDeviceReset (a new primary context, the module and its
// array loaded afresh) the next call runs the set-up again.
//
// Memory: with lazily loaded modules (CUDA's default) the 10 MiB array is placed
// on a device when this library's kernels are first used there; with eager
// loading (CUDA_MODULE_LOADING=EAGER) every context the library is loaded into
// holds it, whether or not this entry point is called.
//
// Sharing: every call on a device uses the same working vector.  Calls ordered on
// one stream are safe; two calls in flight at once (two streams, or two host
// threads) overwrite each other's working vector and give wrong results.  No part
// of the array has to start at zero: the set-up writes every table entry a call
// reads, and a call writes the working vector before reading it.
#include <atomic>
#include <mutex>

#include "ntt.cuh"

namespace nkr {

namespace {

constexpr int kLogMax = 16;
constexpr uint64_t kMax = uint64_t(1) << kLogMax;
// layout in Fr (32 B) units
constexpr uint64_t kTwFwd = 0;          // stage twiddles of w, built for 2^16
constexpr uint64_t kTwInv = kMax;       // same for w^-1
constexpr uint64_t kGpow = 2 * kMax;    // g^i, i < 2^16 (natural order)
constexpr uint64_t kGinvPow = 3 * kMax; // g^-i
constexpr uint64_t kWork = 4 * kMax;    // working vector (also a table-build temporary)
constexpr uint64_t kConsts = 5 * kMax;  // Fr[8] per logn in [0, 16], NttTables::consts layout
constexpr uint64_t kScratchFr = kConsts + 8 * (kLogMax + 1);

static __device__ __align__(256) uint4 g_ntt_scratch[kScratchFr * 2]; // 2 x 16 B per Fr

constexpr int kMaxDevices = 64;
std::mutex g_setup_mu;
std::atomic<Fr *> g_base[kMaxDevices];
std::atomic<unsigned long long> g_ctx_id[kMaxDevices]; // context the tables were built in

// The unique id of the current context (driver cuCtxGetCurrent + cuCtxGetId,
// reached through the runtime's entry-point query: the library links no libcuda).
int current_ctx_id(unsigned long long *id)
{
    using GetCurrent = int (*)(void **);
    using GetId = int (*)(void *, unsigned long long *);
    static GetCurrent get_current = nullptr;
    static GetId get_id = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void *f = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_current = reinterpret_cast<GetCurrent>(f);
        f = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_id = reinterpret_cast<GetId>(f);
    });
    void *ctx = nullptr;
    if (!get_current || !get_id || get_current(&ctx) != 0 || !ctx || get_id(ctx, id) != 0) {
        set_error("ntt_noalloc: the current CUDA context could not be identified");
        return NKR_B200_ECUDA;
    }
    return NKR_B200_OK;
}

// Builds the tables in the array of the current device (context ctx_id); returns
// its Fr base.
int setup_device(int device, unsigned long long ctx_id, cudaStream_t st, Fr **out)
{
    std::lock_guard<std::mutex> lock(g_setup_mu);
    Fr *b = g_base[device].load(std::memory_order_acquire);
    if (b && g_ctx_id[device].load(std::memory_order_acquire) == ctx_id) {
        *out = b;
        return NKR_B200_OK;
    }
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_ntt_scratch);
    if (e != cudaSuccess || p == nullptr) {
        set_error("ntt_noalloc: cudaGetSymbolAddress of the scratch array failed on device %d: %s",
                  device, cudaGetErrorString(e));
        return NKR_B200_ECUDA;
    }
    b = static_cast<Fr *>(p);
    Fr *c = b + kConsts;
    Fr *top = c + 8 * kLogMax;
    NKR_TRY(ntt_constants_into(kLogMax, top, st));
    NKR_TRY(fr_powers_into(top + kConstOmega, b + kWork, kMax / 2, st));
    NKR_TRY(ntt_stage_twiddles_into(b + kWork, b + kTwFwd, kLogMax, st));
    NKR_TRY(fr_powers_into(top + kConstOmegaInv, b + kWork, kMax / 2, st));
    NKR_TRY(ntt_stage_twiddles_into(b + kWork, b + kTwInv, kLogMax, st));
    NKR_TRY(fr_powers_into(top + kConstG, b + kGpow, kMax, st));
    NKR_TRY(fr_powers_into(top + kConstGinv, b + kGinvPow, kMax, st));
    for (int lg = 1; lg < kLogMax; ++lg) NKR_TRY(ntt_constants_into(lg, c + 8 * lg, st));
    NKR_CUDA(cudaStreamSynchronize(st));
    g_ctx_id[device].store(ctx_id, std::memory_order_release);
    g_base[device].store(b, std::memory_order_release);
    *out = b;
    return NKR_B200_OK;
}

int check_device_ptr(const void *p, int device, const char *what)
{
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
        cudaGetLastError();
        set_error("ntt_noalloc: %s is not a CUDA pointer", what);
        return NKR_B200_EINVAL;
    }
    NKR_REQUIRE((a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged) &&
                    a.device == device,
                "ntt_noalloc: %s must be device memory of device %d", what, device);
    return NKR_B200_OK;
}

struct DeviceRestore {
    int prev = -1;
    ~DeviceRestore()
    {
        if (prev >= 0) cudaSetDevice(prev);
    }
};

int ntt_noalloc(int device, int op, const void *in, void *out, uint64_t n, cudaStream_t st)
{
    NKR_REQUIRE(op >= 0 && op <= 4, "ntt op %d unknown", op);
    NKR_REQUIRE(in != nullptr && out != nullptr, "null buffer");
    const int logn = log2_exact(n);
    NKR_REQUIRE(logn >= 1 && logn <= kLogMax,
                "ntt_noalloc: n = %llu must be a power of two in [2, %llu] (the fixed scratch "
                "array holds tables for 2^%d elements)",
                (unsigned long long)n, (unsigned long long)kMax, kLogMax);
    int count = 0;
    NKR_CUDA(cudaGetDeviceCount(&count));
    if (device < 0 || device >= count || device >= kMaxDevices) {
        set_error("ntt_noalloc: device %d not present (%d devices)", device, count);
        return NKR_B200_ENODEV;
    }
    DeviceRestore restore;
    NKR_CUDA(cudaGetDevice(&restore.prev));
    NKR_CUDA(cudaSetDevice(device));
    NKR_TRY(check_device_ptr(in, device, "in"));
    NKR_TRY(check_device_ptr(out, device, "out"));
    unsigned long long ctx_id = 0;
    NKR_TRY(current_ctx_id(&ctx_id));
    Fr *b = g_base[device].load(std::memory_order_acquire);
    if (!b || g_ctx_id[device].load(std::memory_order_acquire) != ctx_id)
        NKR_TRY(setup_device(device, ctx_id, st, &b));
    const Fr *c = b + kConsts + 8 * logn;
    Fr *work = b + kWork;
    const Fr *src = static_cast<const Fr *>(in);
    if (op == 4) { // divide_by_Z_on_coset: scale by (g^n - 1)^-1
        NKR_CUDA(cudaMemcpyAsync(work, src, n * sizeof(Fr), cudaMemcpyDeviceToDevice, st));
        NKR_TRY(fr_scale_const(work, n, c + kConstZinv, st));
    } else {
        // natural -> bit-reversed with the input-side scale, then DIT back to natural
        const bool inverse = op == 1 || op == 3;
        NKR_TRY(ntt_bitrev_permute(src, work, n, op == 2 ? b + kGpow : nullptr,
                                   inverse ? c + kConstNinv : nullptr, st));
        NKR_TRY(ntt_dit_raw(logn, b + (inverse ? kTwInv : kTwFwd), work, nullptr,
                            op == 3 ? b + kGinvPow : nullptr, nullptr, st));
    }
    NKR_CUDA(cudaMemcpyAsync(out, work, n * sizeof(Fr), cudaMemcpyDeviceToDevice, st));
    return NKR_B200_OK;
}

} // namespace

} // namespace nkr

extern "C" int nkr_b200_ntt_noalloc(int device, int op, const void *in, void *out, uint64_t n,
                                    void *stream)
{
    return nkr::ntt_noalloc(device, op, in, out, n, static_cast<cudaStream_t>(stream));
}
