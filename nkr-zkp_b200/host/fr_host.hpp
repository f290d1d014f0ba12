// Host-side BN254 prime fields (4 x u64 Montgomery limbs, the libff byte
// layout): Fr for circuit / witness generation and the setup's scalar part, Fq
// and Fq2 for normalising the few projective points the GPU returns.  Not on
// the prove hot path.
#pragma once

#include <cstdint>
#include <cstring>
#include <random>

namespace nkr::host {

struct FrMod {
    static constexpr uint64_t M[4] = {0x43e1f593f0000001ull, 0x2833e84879b97091ull,
                                      0xb85045b68181585dull, 0x30644e72e131a029ull};
    static constexpr uint64_t INV = 0xc2e1f593efffffffull; // -r^-1 mod 2^64
    static constexpr uint64_t ONE[4] = {0xac96341c4ffffffbull, 0x36fc76959f60cd29ull,
                                        0x666ea36f7879462eull, 0x0e0a77c19a07df2full};
    static constexpr uint64_t R2[4] = {0x1bb8e645ae216da7ull, 0x53fe3ab1e35c59e3ull,
                                       0x8c49833d53bb8085ull, 0x0216d0b17f4e44a5ull};
};

struct FqMod {
    static constexpr uint64_t M[4] = {0x3c208c16d87cfd47ull, 0x97816a916871ca8dull,
                                      0xb85045b68181585dull, 0x30644e72e131a029ull};
    static constexpr uint64_t INV = 0x87d20782e4866389ull; // -p^-1 mod 2^64
    static constexpr uint64_t ONE[4] = {0xd35d438dc58f0d9dull, 0x0a78eb28f5c70b3dull,
                                        0x666ea36f7879462cull, 0x0e0a77c19a07df2full};
    static constexpr uint64_t R2[4] = {0xf32cfc5b538afa89ull, 0xb5e71911d44501fbull,
                                       0x47ab1eff0a417ff6ull, 0x06d89f71cab8351full};
};

template <class Mod>
struct Fp64 {
    uint64_t v[4];
    bool operator==(const Fp64 &o) const { return std::memcmp(v, o.v, 32) == 0; }
    bool operator!=(const Fp64 &o) const { return !(*this == o); }
    bool is_zero() const { return (v[0] | v[1] | v[2] | v[3]) == 0; }
    static Fp64 zero() { return Fp64{{0, 0, 0, 0}}; }
    static Fp64 one() { return Fp64{{Mod::ONE[0], Mod::ONE[1], Mod::ONE[2], Mod::ONE[3]}}; }
};

template <class Mod>
inline bool geq_mod(const uint64_t *a)
{
    for (int i = 3; i >= 0; --i) {
        if (a[i] > Mod::M[i]) return true;
        if (a[i] < Mod::M[i]) return false;
    }
    return true;
}

template <class Mod>
inline void sub_mod(uint64_t *a)
{
    unsigned __int128 b = 0;
    for (int i = 0; i < 4; ++i) {
        const unsigned __int128 d = (unsigned __int128)a[i] - Mod::M[i] - (uint64_t)b;
        a[i] = (uint64_t)d;
        b = (d >> 64) ? 1 : 0;
    }
}

template <class Mod>
inline Fp64<Mod> operator+(const Fp64<Mod> &a, const Fp64<Mod> &b)
{
    Fp64<Mod> r;
    unsigned __int128 c = 0;
    for (int i = 0; i < 4; ++i) {
        c = (unsigned __int128)a.v[i] + b.v[i] + (uint64_t)(c >> 64);
        r.v[i] = (uint64_t)c;
    }
    if (geq_mod<Mod>(r.v)) sub_mod<Mod>(r.v);
    return r;
}

template <class Mod>
inline Fp64<Mod> operator-(const Fp64<Mod> &a, const Fp64<Mod> &b)
{
    Fp64<Mod> r;
    unsigned __int128 br = 0;
    for (int i = 0; i < 4; ++i) {
        const unsigned __int128 d = (unsigned __int128)a.v[i] - b.v[i] - (uint64_t)br;
        r.v[i] = (uint64_t)d;
        br = (d >> 64) ? 1 : 0;
    }
    if (br) {
        unsigned __int128 c = 0;
        for (int i = 0; i < 4; ++i) {
            c = (unsigned __int128)r.v[i] + Mod::M[i] + (uint64_t)(c >> 64);
            r.v[i] = (uint64_t)c;
        }
    }
    return r;
}

template <class Mod>
inline Fp64<Mod> operator-(const Fp64<Mod> &a)
{
    return Fp64<Mod>::zero() - a;
}

// CIOS Montgomery product
template <class Mod>
inline Fp64<Mod> operator*(const Fp64<Mod> &a, const Fp64<Mod> &b)
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
        const uint64_t m = t[0] * Mod::INV;
        c = (unsigned __int128)m * Mod::M[0] + t[0];
        for (int j = 1; j < 4; ++j) {
            c = (unsigned __int128)m * Mod::M[j] + t[j] + (uint64_t)(c >> 64);
            t[j - 1] = (uint64_t)c;
        }
        c = (unsigned __int128)t[4] + (uint64_t)(c >> 64);
        t[3] = (uint64_t)c;
        t[4] = t[5] + (uint64_t)(c >> 64);
    }
    Fp64<Mod> r;
    std::memcpy(r.v, t, 32);
    if (t[4] || geq_mod<Mod>(r.v)) sub_mod<Mod>(r.v);
    return r;
}

template <class Mod>
inline Fp64<Mod> &operator+=(Fp64<Mod> &a, const Fp64<Mod> &b)
{
    return a = a + b;
}
template <class Mod>
inline Fp64<Mod> &operator*=(Fp64<Mod> &a, const Fp64<Mod> &b)
{
    return a = a * b;
}

template <class Mod>
inline Fp64<Mod> pow(const Fp64<Mod> &a, const uint64_t e[4])
{
    Fp64<Mod> acc = Fp64<Mod>::one();
    for (int i = 255; i >= 0; --i) {
        acc = acc * acc;
        if ((e[i / 64] >> (i % 64)) & 1) acc = acc * a;
    }
    return acc;
}

// Fermat inverse; 0 maps to 0
template <class Mod>
inline Fp64<Mod> inverse(const Fp64<Mod> &a)
{
    const uint64_t e[4] = {Mod::M[0] - 2, Mod::M[1], Mod::M[2], Mod::M[3]};
    return pow(a, e);
}

using Fr = Fp64<FrMod>;
using Fq = Fp64<FqMod>;

constexpr const uint64_t *kR = FrMod::M;
inline bool geq_r(const uint64_t *a) { return geq_mod<FrMod>(a); }
inline void sub_r(uint64_t *a) { sub_mod<FrMod>(a); }
inline Fr zero() { return Fr::zero(); }
inline Fr one() { return Fr::one(); }

// canonical integer (< r) -> Montgomery
inline Fr from_canonical(const uint64_t c[4])
{
    Fr x;
    std::memcpy(x.v, c, 32);
    const Fr r2 = {{FrMod::R2[0], FrMod::R2[1], FrMod::R2[2], FrMod::R2[3]}};
    return x * r2;
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

// Jacobian (X, Y, Z) in libff layout -> affine-normalised (Z = 1), or (0, 1, 0)
// for infinity.  G1: 3 Fq; G2: 3 Fq2 with Fq2 = {c0, c1} and u^2 = -1.
inline void normalize_g1(void *p96)
{
    Fq *p = static_cast<Fq *>(p96);
    if (p[2].is_zero()) {
        p[0] = Fq::zero();
        p[1] = Fq::one();
        return;
    }
    const Fq zi = inverse(p[2]);
    const Fq zi2 = zi * zi;
    p[0] = p[0] * zi2;
    p[1] = p[1] * (zi2 * zi);
    p[2] = Fq::one();
}

inline void fq2_mul(const Fq *a, const Fq *b, Fq *o)
{
    const Fq r0 = a[0] * b[0] - a[1] * b[1];
    const Fq r1 = a[0] * b[1] + a[1] * b[0];
    o[0] = r0;
    o[1] = r1;
}

inline void normalize_g2(void *p192)
{
    Fq *p = static_cast<Fq *>(p192); // X = p[0..1], Y = p[2..3], Z = p[4..5]
    if (p[4].is_zero() && p[5].is_zero()) {
        p[0] = p[1] = p[3] = Fq::zero();
        p[2] = Fq::one();
        return;
    }
    const Fq n = p[4] * p[4] + p[5] * p[5];
    const Fq ni = inverse(n);
    const Fq zi[2] = {p[4] * ni, -(p[5] * ni)};
    Fq zi2[2], zi3[2];
    fq2_mul(zi, zi, zi2);
    fq2_mul(zi2, zi, zi3);
    fq2_mul(p, zi2, p);
    fq2_mul(p + 2, zi3, p + 2);
    p[4] = Fq::one();
    p[5] = Fq::zero();
}

} // namespace nkr::host
