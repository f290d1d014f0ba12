// Host-side BN254 scalar field Fr (4 x u64 Montgomery limbs, the libff byte
// layout) for circuit and witness generation.  Not on the prove hot path.
#pragma once

#include <cstdint>
#include <cstring>
#include <random>

namespace nkr::host {

struct Fr {
    uint64_t v[4];
    bool operator==(const Fr &o) const { return std::memcmp(v, o.v, 32) == 0; }
    bool operator!=(const Fr &o) const { return !(*this == o); }
    bool is_zero() const { return (v[0] | v[1] | v[2] | v[3]) == 0; }
};

constexpr uint64_t kR[4] = {0x43e1f593f0000001ull, 0x2833e84879b97091ull, 0xb85045b68181585dull,
                            0x30644e72e131a029ull};
constexpr uint64_t kInv = 0xc2e1f593efffffffull; // -r^-1 mod 2^64
constexpr Fr kOne = {{0xac96341c4ffffffbull, 0x36fc76959f60cd29ull, 0x666ea36f7879462eull,
                      0x0e0a77c19a07df2full}};
constexpr Fr kR2 = {{0x1bb8e645ae216da7ull, 0x53fe3ab1e35c59e3ull, 0x8c49833d53bb8085ull,
                     0x0216d0b17f4e44a5ull}};

inline bool geq_r(const uint64_t *a)
{
    for (int i = 3; i >= 0; --i) {
        if (a[i] > kR[i]) return true;
        if (a[i] < kR[i]) return false;
    }
    return true;
}

inline void sub_r(uint64_t *a)
{
    unsigned __int128 b = 0;
    for (int i = 0; i < 4; ++i) {
        const unsigned __int128 d = (unsigned __int128)a[i] - kR[i] - (uint64_t)b;
        a[i] = (uint64_t)d;
        b = (d >> 64) ? 1 : 0;
    }
}

inline Fr operator+(const Fr &a, const Fr &b)
{
    Fr r;
    unsigned __int128 c = 0;
    for (int i = 0; i < 4; ++i) {
        c = (unsigned __int128)a.v[i] + b.v[i] + (uint64_t)(c >> 64);
        r.v[i] = (uint64_t)c;
    }
    if (geq_r(r.v)) sub_r(r.v);
    return r;
}

inline Fr operator-(const Fr &a, const Fr &b)
{
    Fr r;
    unsigned __int128 br = 0;
    for (int i = 0; i < 4; ++i) {
        const unsigned __int128 d = (unsigned __int128)a.v[i] - b.v[i] - (uint64_t)br;
        r.v[i] = (uint64_t)d;
        br = (d >> 64) ? 1 : 0;
    }
    if (br) {
        unsigned __int128 c = 0;
        for (int i = 0; i < 4; ++i) {
            c = (unsigned __int128)r.v[i] + kR[i] + (uint64_t)(c >> 64);
            r.v[i] = (uint64_t)c;
        }
    }
    return r;
}

inline Fr operator-(const Fr &a) { return Fr{{0, 0, 0, 0}} - a; }

// CIOS Montgomery product
inline Fr operator*(const Fr &a, const Fr &b)
{
    uint64_t t[6] = {0, 0, 0, 0, 0, 0};
    for (int i = 0; i < 4; ++i) {
        unsigned __int128 c = 0;
        for (int j = 0; j < 4; ++j) {
            c = (unsigned __int128)a.v[j] * b.v[i] + t[j] + (uint64_t)(c >> 64);
            t[j] = (uint64_t)c;
        }
        c = (unsigned __int128)t[4] + (uint64_t)(c >> 64);
        t[4] = (uint64_t)c;
        t[5] = (uint64_t)(c >> 64);
        const uint64_t m = t[0] * kInv;
        c = (unsigned __int128)m * kR[0] + t[0];
        for (int j = 1; j < 4; ++j) {
            c = (unsigned __int128)m * kR[j] + t[j] + (uint64_t)(c >> 64);
            t[j - 1] = (uint64_t)c;
        }
        c = (unsigned __int128)t[4] + (uint64_t)(c >> 64);
        t[3] = (uint64_t)c;
        t[4] = t[5] + (uint64_t)(c >> 64);
    }
    Fr r;
    std::memcpy(r.v, t, 32);
    if (t[4] || geq_r(r.v)) sub_r(r.v);
    return r;
}

inline Fr& operator+=(Fr &a, const Fr &b) { return a = a + b; }
inline Fr& operator*=(Fr &a, const Fr &b) { return a = a * b; }

inline Fr zero() { return Fr{{0, 0, 0, 0}}; }
inline Fr one() { return kOne; }

// canonical integer (< r) -> Montgomery
inline Fr from_canonical(const uint64_t c[4])
{
    Fr x;
    std::memcpy(x.v, c, 32);
    return x * kR2;
}
inline Fr from_u64(uint64_t v)
{
    const uint64_t c[4] = {v, 0, 0, 0};
    return from_canonical(c);
}
inline void to_canonical(const Fr &a, uint64_t out[4])
{
    const Fr one_int = {{1, 0, 0, 0}};
    const Fr c = a * one_int;
    std::memcpy(out, c.v, 32);
}

inline Fr pow(const Fr &a, const uint64_t e[4])
{
    Fr acc = kOne;
    for (int i = 255; i >= 0; --i) {
        acc = acc * acc;
        if ((e[i / 64] >> (i % 64)) & 1) acc = acc * a;
    }
    return acc;
}

inline Fr inverse(const Fr &a)
{
    const uint64_t e[4] = {kR[0] - 2, kR[1], kR[2], kR[3]};
    return pow(a, e);
}

// Uniform element: random 254-bit limbs with rejection of values >= r, taken
// as the Montgomery representation (a bijection), as libff's
// Fp_model::random_element does (libff/algebra/fields/fp.tcc:719-744).
inline Fr random_element(std::mt19937_64 &rng)
{
    Fr r;
    do {
        for (int i = 0; i < 4; ++i) r.v[i] = rng();
        r.v[3] &= (uint64_t(1) << 62) - 1; // clear bits above the modulus' top bit (253)
    } while (geq_r(r.v));
    return r;
}

} // namespace nkr::host
