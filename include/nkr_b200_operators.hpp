/*
 * nkr_b200_operators.hpp -- the reference's operator-level CUDA API on top of the
 * C ABI in nkr_b200.h, header-only C++.
 *
 * A caller written against the reference's operators/cuda contexts keeps its code
 * and swaps the include:
 *   NTTContext<FieldT, HostFT>       operators/cuda/include/ntt/ntt.cuh:22-208
 *   BucketContext<FieldT, HostFT>    operators/cuda/include/fields/bucket.cuh:15-142
 *   MSMContext<FieldT, AffT, ProjT, XYZZT, HostFT, HostPT, elastic>
 *                                    operators/cuda/include/msm/msm.cuh:12-123
 * (all three gathered by nkr/operators/cuda.hpp:1-23).  Same class names, template
 * parameters, constructors, member functions, argument meaning and data layouts:
 * device vectors of 32-byte Fr Montgomery elements, host points in libff's
 * Jacobian layout (96 B for G1, 192 B for G2).  The device-side type parameters
 * (FieldT, AffT, ProjT, XYZZT) only have to have the reference's sizes; the
 * arithmetic is this library's.
 *
 * What differs, on purpose:
 *   - errors throw nkr_b200::operators::Error (a std::runtime_error carrying the
 *     library's message) where the reference calls exit() (utils/cuda_check.cuh);
 *   - MSMContext's window_bits is advisory: the library measures the window width
 *     per size on the device (nkr_b200_tune_msm) where the reference fixes 8, 11 or
 *     13 bits (backends/cuda/src/groth16_backend.cu:17-25); `elastic` is accepted
 *     and unused (the library keeps every window's base copies resident);
 *   - BucketContext::process() leaves the scalars in Montgomery form: the digit
 *     sort runs inside each MSMContext::msm call (the reference's process() sorts
 *     up front and converts the scalars out of Montgomery form in place);
 *   - NTTContext takes only the domain the library implements -- libfqfft's
 *     root of unity for n and the multiplicative generator 5 as the coset, the
 *     only values the reference's Groth16 backend passes (groth16_backend.cu:87)
 *     -- and throws std::invalid_argument for any other omega or coset; it keeps
 *     no omega power table, so omega_powers() is not provided.
 * Every call is synchronous with respect to the host, as the reference's are.
 * Work runs on the legacy default stream of the current device, so device writes
 * the caller queued there (or made with cudaMemcpy) are ordered before it.
 */
#ifndef NKR_B200_OPERATORS_HPP
#define NKR_B200_OPERATORS_HPP

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>
#include <cstring>
#include <mutex>
#include <stdexcept>
#include <string>

#include "nkr_b200.h"

namespace nkr_b200 {
namespace operators {

class Error : public std::runtime_error {
public:
    using std::runtime_error::runtime_error;
};

inline void check(int status, const char *what)
{
    if (status != NKR_B200_OK)
        throw Error(std::string(what) + ": " + nkr_b200_last_error());
}

inline void check_cuda(cudaError_t e, const char *what)
{
    if (e != cudaSuccess) throw Error(std::string(what) + ": " + cudaGetErrorString(e));
}

// The library context of the current CUDA device, opened on first use and kept
// for the life of the process (the reference's contexts likewise act on the
// current device with no handle).
inline nkr_b200_ctx *device_context()
{
    constexpr int kMaxDevices = 64;
    static std::mutex mu;
    static nkr_b200_ctx *ctxs[kMaxDevices] = {};
    int dev = 0;
    check_cuda(cudaGetDevice(&dev), "cudaGetDevice");
    if (dev < 0 || dev >= kMaxDevices) throw Error("device index out of range");
    std::lock_guard<std::mutex> lock(mu);
    if (!ctxs[dev]) check(nkr_b200_open(dev, &ctxs[dev]), "nkr_b200_open");
    return ctxs[dev];
}

// A device array owned by one of the contexts below.
template <typename T>
class DeviceArray {
    T *p_ = nullptr;

public:
    DeviceArray() = default;
    explicit DeviceArray(size_t n)
    {
        check_cuda(cudaMalloc(reinterpret_cast<void **>(&p_), n * sizeof(T)), "cudaMalloc");
    }
    DeviceArray(const DeviceArray &) = delete;
    DeviceArray &operator=(const DeviceArray &) = delete;
    ~DeviceArray()
    {
        if (p_) cudaFree(p_);
    }
    T *get() const { return p_; }
};

template <typename FieldT, typename HostFT>
class NTTContext {
    static_assert(sizeof(FieldT) == 32 && sizeof(HostFT) == 32,
                  "Fr elements are 32 bytes (4 x u64 Montgomery)");
    size_t scale;
    nkr_b200_ctx *ctx;
    DeviceArray<FieldT> buffer; // the transform's output before it returns into poly

    void check_domain(const void *omega, const void *coset)
    {
        unsigned char w[32], g[32];
        check(nkr_b200_domain_constants(ctx, scale, w, g), "nkr_b200_domain_constants");
        if (std::memcmp(w, omega, 32) != 0)
            throw std::invalid_argument("NTTContext: omega is not libfqfft's root of unity for this size");
        if (std::memcmp(g, coset, 32) != 0)
            throw std::invalid_argument("NTTContext: coset is not the multiplicative generator 5");
    }

    void run(int op, FieldT *poly)
    {
        check(nkr_b200_ntt_device(ctx, op, poly, buffer.get(), scale, nullptr, nullptr),
              "nkr_b200_ntt_device");
        check_cuda(cudaMemcpyAsync(poly, buffer.get(), scale * sizeof(FieldT),
                                   cudaMemcpyDeviceToDevice, cudaStreamLegacy),
                   "cudaMemcpyAsync");
        check_cuda(cudaStreamSynchronize(cudaStreamLegacy), "cudaStreamSynchronize");
    }

    static size_t checked_scale(size_t s)
    {
        if (s < 2 || (s & (s - 1)) != 0)
            throw std::invalid_argument("NTTContext: scale must be a power of 2, at least 2");
        return s;
    }

public:
    NTTContext(size_t scale_, HostFT omega, HostFT coset)
        : scale(checked_scale(scale_)), ctx(device_context()), buffer(scale)
    {
        check_domain(&omega, &coset);
    }

    NTTContext(size_t scale_, const HostFT *omega_powers, const HostFT *coset_powers,
               const HostFT *inverse_omega_powers, const HostFT *inverse_coset_powers)
        : scale(checked_scale(scale_)), ctx(device_context()), buffer(scale)
    {
        (void)inverse_omega_powers;
        (void)inverse_coset_powers;
        check_domain(&omega_powers[1], &coset_powers[1]);
    }

    // FFT (inverse = false) or inverse FFT with the 1/n scale, in place on the
    // device vector poly of `scale` elements, natural order in and out
    void ntt(FieldT *poly, bool inverse = false) { run(inverse ? 1 : 0, poly); }
    void intt(FieldT *poly) { run(1, poly); }
    // poly_i g^i, then the FFT
    void coset_ntt(FieldT *poly) { run(2, poly); }
    // the inverse FFT, then poly_i g^-i
    void coset_intt(FieldT *poly) { run(3, poly); }
    // polyA = (polyA polyB - polyC) / (g^scale - 1)
    void A_times_B_minus_C_divided_by_Z(FieldT *polyA, FieldT *polyB, FieldT *polyC)
    {
        check(nkr_b200_quotient_device(ctx, polyA, polyB, polyC, polyA, scale, nullptr),
              "nkr_b200_quotient_device");
        check_cuda(cudaStreamSynchronize(cudaStreamLegacy), "cudaStreamSynchronize");
    }
};

template <typename FieldT, typename HostFT, typename key_t = uint16_t>
class BucketContext {
    static_assert(sizeof(FieldT) == 32 && sizeof(HostFT) == 32,
                  "Fr elements are 32 bytes (4 x u64 Montgomery)");
    DeviceArray<FieldT> storage;

    static size_t ceil_div(size_t a, size_t b) { return (a + b - 1) / b; }

public:
    FieldT *scalars; // device, `scale` Fr Montgomery
    size_t scale;
    size_t window_bits;
    size_t windows_count, buckets_count;

    BucketContext(size_t scale_, size_t window_bits_)
        : storage(scale_ ? scale_ : 1), scalars(storage.get()), scale(scale_), window_bits(window_bits_),
          windows_count(ceil_div(254, window_bits_ ? window_bits_ : 1)),
          buckets_count(size_t(1) << window_bits_)
    {
    }

    void load_scalars(const HostFT *host_scalars)
    {
        check_cuda(cudaMemcpy(scalars, host_scalars, scale * sizeof(FieldT), cudaMemcpyHostToDevice),
                   "cudaMemcpy");
    }
    void load_scalars(FieldT *device_scalars)
    {
        check_cuda(cudaMemcpy(scalars, device_scalars, scale * sizeof(FieldT),
                              cudaMemcpyDeviceToDevice),
                   "cudaMemcpy");
    }
    // The digit sort is part of every MSMContext::msm call; nothing to do here.
    void process(bool from = true, bool extraction = true, bool sort = true, bool scatter = true)
    {
        (void)from;
        (void)extraction;
        (void)sort;
        (void)scatter;
    }
};

template <typename FieldT, typename AffT, typename ProjT, typename XYZZT, typename HostFT,
          typename HostPT, size_t elastic = 2>
class MSMContext {
    static_assert(sizeof(HostPT) == 96 || sizeof(HostPT) == 192,
                  "host points are libff Jacobian G1 (96 B) or G2 (192 B)");
    static constexpr int kGroup = sizeof(HostPT) == 96 ? 1 : 2;
    nkr_b200_ctx *ctx;
    nkr_b200_msm_bases *bases = nullptr;

public:
    size_t scale;
    size_t window_bits;

    MSMContext(size_t scale_, size_t window_bits_)
        : ctx(device_context()), scale(scale_), window_bits(window_bits_)
    {
    }
    MSMContext(const MSMContext &) = delete;
    MSMContext &operator=(const MSMContext &) = delete;
    ~MSMContext()
    {
        if (bases) nkr_b200_msm_bases_free(bases);
    }

    // scale points in libff Jacobian layout (host memory; need not be normalised)
    void load_bases(const HostPT *host_bases)
    {
        if (bases) {
            nkr_b200_msm_bases_free(bases);
            bases = nullptr;
        }
        check(nkr_b200_msm_bases_create(ctx, kGroup, host_bases, scale, &bases),
              "nkr_b200_msm_bases_create");
    }

    // sum_i scalars_i bases_i over the bucket context's device scalars; the result
    // (affine-normalised, libff Jacobian layout) goes to *result when given
    template <typename BucketT>
    void msm(BucketT &bkt_ctx, HostPT *result = 0)
    {
        if (!bases) throw Error("MSMContext::msm before load_bases");
        if (bkt_ctx.scale != scale) throw std::invalid_argument("MSMContext: scalar count differs");
        unsigned char out[sizeof(HostPT)];
        check(nkr_b200_msm_bases_run(bases, bkt_ctx.scalars, scale, out, nullptr),
              "nkr_b200_msm_bases_run");
        if (result) std::memcpy(static_cast<void *>(result), out, sizeof(HostPT));
    }
};

} // namespace operators
} // namespace nkr_b200

#endif
