// Shared host-side plumbing for the B200 backend: status codes with a
// thread-local message (no exit() in library code), CUDA error propagation,
// owning device buffers, and launch helpers.
#pragma once

#include <cuda_runtime.h>

#include <atomic>
#include <cstdarg>
#include <cstdint>
#include <cstdio>
#include <string>
#include <utility>

#include "../../include/nkr_b200.h"

namespace nkr {

void set_error(const char *fmt, ...);
const char *get_error();

#define NKR_CUDA(call)                                                                          \
    do {                                                                                        \
        cudaError_t nkr_e_ = (call);                                                            \
        if (nkr_e_ != cudaSuccess) {                                                            \
            ::nkr::set_error("%s:%d: %s: %s", __FILE__, __LINE__, #call,                       \
                             cudaGetErrorString(nkr_e_));                                       \
            return NKR_B200_ECUDA;                                                              \
        }                                                                                       \
    } while (0)

#define NKR_TRY(expr)                                                                           \
    do {                                                                                        \
        int nkr_s_ = (expr);                                                                    \
        if (nkr_s_ != NKR_B200_OK) return nkr_s_;                                               \
    } while (0)

// Every kernel launch is followed by exactly one NKR_CHECK_LAUNCH(): it counts
// the launch (nkr_b200_launch_count) and surfaces launch errors.
extern std::atomic<unsigned long long> g_kernel_launches;
#define NKR_CHECK_LAUNCH()                                                                      \
    do {                                                                                        \
        ::nkr::g_kernel_launches.fetch_add(1, std::memory_order_relaxed);                       \
        NKR_CUDA(cudaGetLastError());                                                           \
    } while (0)

#define NKR_REQUIRE(cond, ...)                                                                  \
    do {                                                                                        \
        if (!(cond)) {                                                                          \
            ::nkr::set_error(__VA_ARGS__);                                                      \
            return NKR_B200_EINVAL;                                                             \
        }                                                                                       \
    } while (0)

// Device allocation with an explicit admission check against free HBM.
int device_alloc(void **p, size_t bytes, const char *what);

// Owning device buffer (moved, never copied).
struct DevBuf {
    void *p = nullptr;
    size_t bytes = 0;
    DevBuf() = default;
    DevBuf(const DevBuf &) = delete;
    DevBuf &operator=(const DevBuf &) = delete;
    DevBuf(DevBuf &&o) noexcept : p(o.p), bytes(o.bytes)
    {
        o.p = nullptr;
        o.bytes = 0;
    }
    DevBuf &operator=(DevBuf &&o) noexcept
    {
        if (this != &o) {
            release();
            p = o.p;
            bytes = o.bytes;
            o.p = nullptr;
            o.bytes = 0;
        }
        return *this;
    }
    ~DevBuf() { release(); }
    void release()
    {
        if (p) cudaFree(p);
        p = nullptr;
        bytes = 0;
    }
    int alloc(size_t n, const char *what)
    {
        if (n <= bytes && p) return NKR_B200_OK;
        release();
        if (n == 0) return NKR_B200_OK;
        int s = device_alloc(&p, n, what);
        if (s == NKR_B200_OK) bytes = n;
        return s;
    }
    template <class T>
    T *as() const
    {
        return static_cast<T *>(p);
    }
};

inline unsigned blocks_for(uint64_t n, unsigned threads)
{
    return static_cast<unsigned>((n + threads - 1) / threads);
}

inline int log2_exact(uint64_t n)
{
    if (n == 0 || (n & (n - 1))) return -1;
    int k = 0;
    while ((uint64_t(1) << k) < n) ++k;
    return k;
}

} // namespace nkr
