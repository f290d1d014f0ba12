// Fq in five 52-bit limbs with products on the double-precision FMA pipe.
//
// The Montgomery product of field.cuh is bound by the integer multiply (IMAD)
// pipe and, for one warp alone, by its long carry chains (about a microsecond
// of latency per product).  B200 also has a full-rate FP64 pipe, and a double
// FMA computes a 52 x 52-bit limb product exactly when the high half is taken
// with round toward zero against a 2^104 offset and the low half as the exact
// remainder (Emmart, Zheng and Weems, "Faster modular exponentiation using
// double precision floating point arithmetic on the GPU", ARITH 2018):
//     h = fma_rz(a, b, 2^104)              = 2^104 + floor(a b / 2^52) 2^52
//     l = fma(a, b, (2^104 + 2^52) - h)    = 2^52 + (a b mod 2^52)
// Both results hold their integer in the mantissa, so their bit patterns minus
// the offsets' bit patterns are the integers; the 25 limb products of a x b
// are independent, columns are summed as 64-bit integers and the offsets are
// removed once per column.  The reduction is word-serial Montgomery with
// 52-bit words (q = t * (-p^-1) mod 2^52 by integer multiply; q * p by FMA,
// of whose lowest limb product only the high half is formed).
//
// Representation: limbs are uint64 integers < 2^52, values canonical (< p),
// Montgomery form with R' = 2^260.  In memory these values are stored in the
// 8 x 32-bit layout of Fq (to52 / from52 only move bits); the MSM keeps all of
// its buffers in the R' domain and converts at entry (bases) and exit (result).
#pragma once

#include <cstdint>

#include "field.cuh"

namespace nkr {

struct Fq52 {
    uint64_t l[5];
    static constexpr bool kCanonical = true; // products end with the conditional subtraction
    __device__ __forceinline__ static Fq52 zero() { return {{0, 0, 0, 0, 0}}; }
    // 2^260 mod p
    __device__ __forceinline__ static Fq52 one()
    {
        return {{0x20880f6fce4b4ull, 0x49baa989a8455ull, 0x18f014a498908ull, 0x724f85a9201d8ull,
                 0x1f16424e1bb7ull}};
    }
    __device__ __forceinline__ bool is_zero() const
    {
        return (l[0] | l[1] | l[2] | l[3] | l[4]) == 0;
    }
    __device__ __forceinline__ bool operator==(const Fq52 &o) const
    {
        return ((l[0] ^ o.l[0]) | (l[1] ^ o.l[1]) | (l[2] ^ o.l[2]) | (l[3] ^ o.l[3]) |
                (l[4] ^ o.l[4])) == 0;
    }
    __device__ __forceinline__ bool operator!=(const Fq52 &o) const { return !(*this == o); }
};

namespace f52 {

constexpr uint64_t kMask = (uint64_t(1) << 52) - 1;
constexpr uint64_t kBias52 = 0x4330000000000000ull;  // bit pattern of 2^52
constexpr uint64_t kBias104 = 0x4670000000000000ull; // bit pattern of 2^104
// p in 52-bit limbs and -p^-1 mod 2^52
__host__ __device__ constexpr uint64_t p_limb(int k)
{
    return k == 0 ? 0x8c16d87cfd47ull
           : k == 1 ? 0x916871ca8d3c2ull
           : k == 2 ? 0x181585d97816aull
           : k == 3 ? 0xa029b85045b68ull
                    : 0x30644e72e131ull;
}
constexpr uint64_t kPinv = 0x20782e4866389ull;
// 2p in 52-bit limbs
__host__ __device__ constexpr uint64_t p2_limb(int k)
{
    return k == 0 ? 0x1182db0f9fa8eull
           : k == 1 ? 0x22d0e3951a784ull
           : k == 2 ? 0x302b0bb2f02d5ull
           : k == 3 ? 0x405370a08b6d0ull
                    : 0x60c89ce5c263ull;
}
template <int M> // M p in limbs, M = 1 or 2
__host__ __device__ constexpr uint64_t mp_limb(int k)
{
    return M == 1 ? p_limb(k) : p2_limb(k);
}

__device__ __forceinline__ double to_double(uint64_t v) // v < 2^52, exact
{
    return __longlong_as_double(static_cast<long long>(kBias52 | v)) - 0x1p52;
}

// a b = hi 2^52 + lo for integers a, b < 2^52 held in doubles; returns the
// offset bit patterns (kBias52 + lo, kBias104 + hi)
__device__ __forceinline__ void mul_wide(double a, double b, uint64_t &lo_b, uint64_t &hi_b)
{
    const double h = __fma_rz(a, b, 0x1p104);
    const double c = (0x1p104 + 0x1p52) - h;
    const double l = __fma_rn(a, b, c);
    hi_b = static_cast<uint64_t>(__double_as_longlong(h));
    lo_b = static_cast<uint64_t>(__double_as_longlong(l));
}


// s (five 52-bit limbs, value < 2 M p) minus M p when s >= M p
template <int M>
__device__ __forceinline__ void sub_mp_if_ge(uint64_t *s)
{
    uint64_t d[5];
    int64_t borrow = 0;
#pragma unroll
    for (int k = 0; k < 5; ++k) {
        const int64_t t = int64_t(s[k]) - int64_t(mp_limb<M>(k)) + borrow;
        d[k] = uint64_t(t) & kMask;
        borrow = t >> 52;
    }
    if (borrow == 0) {
#pragma unroll
        for (int k = 0; k < 5; ++k) s[k] = d[k];
    }
}
// s (value < 2p) minus p when s >= p
__device__ __forceinline__ void sub_p_if_ge(uint64_t *s) { sub_mp_if_ge<1>(s); }

} // namespace f52

#ifdef NKR_FIELD_MUL_OUTLINE
#define NKR_MUL52_ATTR inline __noinline__ // inline: one definition across translation units
#else
#define NKR_MUL52_ATTR __forceinline__
#endif

// N independent products r[k] = a[k] b[k] 2^-260 mod p.  The word-serial
// Montgomery result t = (a b + q p) / 2^260 with q < 2^260 is below
// a b / 2^260 + p: for a, b < 2p that is under 1.05 p, so the canonical type
// (T::kCanonical) ends with one conditional subtraction of p and the lazily
// reduced type (Fq52L, values in [0, 2p)) skips it.  The N computations share no
// data, so the scheduler interleaves their dependency chains (the word-serial
// reduction is one long chain per product).
template <int N, class T>
__device__ __forceinline__ void mul52_body(const T *const *a, const T *const *b, T *const *r)
{
    using namespace f52;
    double ad[N][5], bd[N][5], pd[5];
#pragma unroll
    for (int i = 0; i < 5; ++i) pd[i] = double(p_limb(i)); // exact, folded at compile time
#pragma unroll
    for (int k = 0; k < N; ++k)
#pragma unroll
        for (int i = 0; i < 5; ++i) {
            ad[k][i] = to_double(a[k]->l[i]);
            bd[k][i] = to_double(b[k]->l[i]);
        }
    uint64_t C[N][10];
    uint64_t bias[10];
#pragma unroll
    for (int j = 0; j < 10; ++j) {
        bias[j] = 0;
#pragma unroll
        for (int k = 0; k < N; ++k) C[k][j] = 0;
    }
#pragma unroll
    for (int i = 0; i < 5; ++i)
#pragma unroll
        for (int j = 0; j < 5; ++j) {
#pragma unroll
            for (int k = 0; k < N; ++k) {
                uint64_t lo, hi;
                mul_wide(ad[k][i], bd[k][j], lo, hi);
                C[k][i + j] += lo;
                C[k][i + j + 1] += hi;
            }
            bias[i + j] += kBias52;
            bias[i + j + 1] += kBias104;
        }
#pragma unroll
    for (int i = 0; i < 5; ++i) {
        uint64_t t[N];
        double q[N];
#pragma unroll
        for (int k = 0; k < N; ++k) {
            t[k] = C[k][i] - bias[i]; // the column's integer value
            // q = t (-p^-1) mod 2^52 on the integer multiply pipe (the low 64 bits
            // of a 52 x 52-bit product), leaving the FP64 pipe to the limb
            // products: 160 instead of 180 FP64 instructions per product, 1.5%
            // off a 2^20 prove
            q[k] = to_double(((t[k] & kMask) * kPinv) & kMask);
        }
#pragma unroll
        for (int k = 0; k < N; ++k) {
            uint64_t lo, hi;
            // t + q p0 is 0 mod 2^52 and the low 52 bits of t and of q p0 are
            // each below 2^52, so they sum to 0 (t's are 0) or to 2^52: the carry
            // into the next column needs only the high half of q p0 (one FMA
            // instead of two FMAs and a subtraction)
            hi = static_cast<uint64_t>(__double_as_longlong(__fma_rz(q[k], pd[0], 0x1p104)));
            C[k][i + 1] += hi + (t[k] >> 52) + ((t[k] & kMask) != 0 ? 1u : 0u);
#pragma unroll
            for (int j = 1; j < 5; ++j) {
                mul_wide(q[k], pd[j], lo, hi);
                C[k][i + j] += lo;
                if (i + j + 1 < 10) C[k][i + j + 1] += hi;
            }
        }
        bias[i + 1] += kBias104;
#pragma unroll
        for (int j = 1; j < 5; ++j) {
            bias[i + j] += kBias52;
            if (i + j + 1 < 10) bias[i + j + 1] += kBias104;
        }
    }
#pragma unroll
    for (int k = 0; k < N; ++k) {
        uint64_t carry = 0;
#pragma unroll
        for (int j = 5; j < 10; ++j) {
            const uint64_t v = C[k][j] - bias[j] + carry;
            r[k]->l[j - 5] = v & kMask;
            carry = v >> 52;
        }
        if constexpr (T::kCanonical) sub_p_if_ge(r[k]->l); // the result is below 2p
    }
}

__device__ NKR_MUL52_ATTR Fq52 mul52(Fq52 a, Fq52 b)
{
    Fq52 r;
    const Fq52 *pa[1] = {&a}, *pb[1] = {&b};
    Fq52 *pr[1] = {&r};
    mul52_body<1>(pa, pb, pr);
    return r;
}

struct Fq52Pair {
    Fq52 x, y;
};

// (a b, c d) in one call: two independent products with interleaved chains.
// Operands and results travel by value so the call passes them in registers
// (reference parameters would go through the thread's local-memory stack).
__device__ NKR_MUL52_ATTR Fq52Pair mul52x2v(Fq52 a, Fq52 b, Fq52 c, Fq52 d)
{
    Fq52Pair r;
    const Fq52 *pa[2] = {&a, &c}, *pb[2] = {&b, &d};
    Fq52 *pr[2] = {&r.x, &r.y};
    mul52_body<2>(pa, pb, pr);
    return r;
}

struct Fq52Triple {
    Fq52 x, y, z;
};

// (a b, c d, e f) in one call: the three products of a Karatsuba Fq2 product
__device__ NKR_MUL52_ATTR Fq52Triple mul52x3v(Fq52 a, Fq52 b, Fq52 c, Fq52 d, Fq52 e, Fq52 f)
{
    Fq52Triple r;
    const Fq52 *pa[3] = {&a, &c, &e}, *pb[3] = {&b, &d, &f};
    Fq52 *pr[3] = {&r.x, &r.y, &r.z};
    mul52_body<3>(pa, pb, pr);
    return r;
}

__device__ __forceinline__ void mul52x2(const Fq52 &a, const Fq52 &b, const Fq52 &c, const Fq52 &d,
                                        Fq52 &ab, Fq52 &cd)
{
    const Fq52Pair r = mul52x2v(a, b, c, d);
    ab = r.x;
    cd = r.y;
}

__device__ __forceinline__ Fq52 operator*(const Fq52 &a, const Fq52 &b) { return mul52(a, b); }
__device__ __forceinline__ Fq52 sqr(const Fq52 &a) { return mul52(a, a); }
// x = a b, y = c d (curve formulas issue independent products in pairs)
__device__ __forceinline__ void mul2(const Fq52 &a, const Fq52 &b, const Fq52 &c, const Fq52 &d,
                                     Fq52 &x, Fq52 &y)
{
    mul52x2(a, b, c, d, x, y);
}
template <>
struct HasPairedMul<Fq52> {
    static constexpr bool value = true;
};

__device__ __forceinline__ Fq52 operator+(const Fq52 &a, const Fq52 &b)
{
    Fq52 r;
    uint64_t c = 0;
#pragma unroll
    for (int k = 0; k < 5; ++k) {
        const uint64_t t = a.l[k] + b.l[k] + c;
        r.l[k] = t & f52::kMask;
        c = t >> 52;
    }
    f52::sub_p_if_ge(r.l);
    return r;
}

__device__ __forceinline__ Fq52 operator-(const Fq52 &a, const Fq52 &b)
{
    Fq52 r;
    int64_t br = 0;
#pragma unroll
    for (int k = 0; k < 5; ++k) {
        const int64_t t = int64_t(a.l[k]) - int64_t(b.l[k]) + br;
        r.l[k] = uint64_t(t) & f52::kMask;
        br = t >> 52;
    }
    if (br) { // a < b: add p back
        uint64_t c = 0;
#pragma unroll
        for (int k = 0; k < 5; ++k) {
            const uint64_t t = r.l[k] + f52::p_limb(k) + c;
            r.l[k] = t & f52::kMask;
            c = t >> 52;
        }
    }
    return r;
}

__device__ __forceinline__ Fq52 neg(const Fq52 &a) { return Fq52::zero() - a; }
__device__ __forceinline__ Fq52 dbl(const Fq52 &a) { return a + a; }

// ---------------------------------------------------------------------------
// Fq52L: the same limbs and R' domain, lazily reduced -- every value is in
// [0, 2p), not canonical.  A product of two such values is already below
// 1.05 p (mul52_body), so it skips the conditional subtraction of p that ends a
// canonical product (about 40 of its 362 instructions); additions and
// subtractions work modulo 2p at the cost of their canonical forms.  Zero tests
// accept 0 and p.  MSM kernels compute in this type and canonicalise once, when a
// value leaves for memory (canon()).
// ---------------------------------------------------------------------------
struct Fq52L {
    uint64_t l[5];
    static constexpr bool kCanonical = false;
    Fq52L() = default;
    __device__ __forceinline__ Fq52L(const Fq52 &c) // a canonical value is in range
    {
#pragma unroll
        for (int k = 0; k < 5; ++k) l[k] = c.l[k];
    }
    __device__ __forceinline__ static Fq52L zero() { return Fq52::zero(); }
    __device__ __forceinline__ static Fq52L one() { return Fq52::one(); }
    __device__ __forceinline__ bool is_zero() const // 0 or p
    {
        return (l[0] | l[1] | l[2] | l[3] | l[4]) == 0 ||
               ((l[0] ^ f52::p_limb(0)) | (l[1] ^ f52::p_limb(1)) | (l[2] ^ f52::p_limb(2)) |
                (l[3] ^ f52::p_limb(3)) | (l[4] ^ f52::p_limb(4))) == 0;
    }
    __device__ __forceinline__ Fq52 canon() const
    {
        Fq52 r;
#pragma unroll
        for (int k = 0; k < 5; ++k) r.l[k] = l[k];
        f52::sub_p_if_ge(r.l);
        return r;
    }
    __device__ __forceinline__ bool operator==(const Fq52L &o) const { return canon() == o.canon(); }
    __device__ __forceinline__ bool operator!=(const Fq52L &o) const { return !(*this == o); }
};

__device__ NKR_MUL52_ATTR Fq52L mul52L(Fq52L a, Fq52L b)
{
    Fq52L r;
    const Fq52L *pa[1] = {&a}, *pb[1] = {&b};
    Fq52L *pr[1] = {&r};
    mul52_body<1>(pa, pb, pr);
    return r;
}

struct Fq52LPair {
    Fq52L x, y;
};

// (a b, c d) in one call, lazily reduced (as mul52x2v)
__device__ NKR_MUL52_ATTR Fq52LPair mul52Lx2v(Fq52L a, Fq52L b, Fq52L c, Fq52L d)
{
    Fq52LPair r;
    const Fq52L *pa[2] = {&a, &c}, *pb[2] = {&b, &d};
    Fq52L *pr[2] = {&r.x, &r.y};
    mul52_body<2>(pa, pb, pr);
    return r;
}

__device__ __forceinline__ Fq52L operator*(const Fq52L &a, const Fq52L &b) { return mul52L(a, b); }
__device__ __forceinline__ Fq52L sqr(const Fq52L &a) { return mul52L(a, a); }

__device__ __forceinline__ void mul2(const Fq52L &a, const Fq52L &b, const Fq52L &c, const Fq52L &d,
                                     Fq52L &x, Fq52L &y)
{
    const Fq52LPair r = mul52Lx2v(a, b, c, d);
    x = r.x;
    y = r.y;
}
template <>
struct HasPairedMul<Fq52L> {
    static constexpr bool value = true;
};

// (a + b) mod 2p for a, b in [0, 2p)
__device__ __forceinline__ Fq52L operator+(const Fq52L &a, const Fq52L &b)
{
    Fq52L r;
    uint64_t c = 0;
#pragma unroll
    for (int k = 0; k < 5; ++k) {
        const uint64_t t = a.l[k] + b.l[k] + c;
        r.l[k] = t & f52::kMask;
        c = t >> 52;
    }
    f52::sub_mp_if_ge<2>(r.l);
    return r;
}

// (a - b) mod 2p for a, b in [0, 2p)
__device__ __forceinline__ Fq52L operator-(const Fq52L &a, const Fq52L &b)
{
    Fq52L r;
    int64_t br = 0;
#pragma unroll
    for (int k = 0; k < 5; ++k) {
        const int64_t t = int64_t(a.l[k]) - int64_t(b.l[k]) + br;
        r.l[k] = uint64_t(t) & f52::kMask;
        br = t >> 52;
    }
    if (br) { // a < b: add 2p back
        uint64_t c = 0;
#pragma unroll
        for (int k = 0; k < 5; ++k) {
            const uint64_t t = r.l[k] + f52::p2_limb(k) + c;
            r.l[k] = t & f52::kMask;
            c = t >> 52;
        }
    }
    return r;
}

__device__ __forceinline__ Fq52L neg(const Fq52L &a) { return Fq52L::zero() - a; }
__device__ __forceinline__ Fq52L dbl(const Fq52L &a) { return a + a; }

// Fq2 = Fq[u] / (u^2 + 1) over Fq52 (Karatsuba, as Fq2 in field.cuh)
struct Fq2x52 {
    Fq52 c0, c1;
    __device__ __forceinline__ static Fq2x52 zero() { return {Fq52::zero(), Fq52::zero()}; }
    __device__ __forceinline__ static Fq2x52 one() { return {Fq52::one(), Fq52::zero()}; }
    __device__ __forceinline__ bool is_zero() const { return c0.is_zero() && c1.is_zero(); }
    __device__ __forceinline__ bool operator==(const Fq2x52 &o) const
    {
        return c0 == o.c0 && c1 == o.c1;
    }
    __device__ __forceinline__ bool operator!=(const Fq2x52 &o) const { return !(*this == o); }
};

__device__ __forceinline__ Fq2x52 operator+(const Fq2x52 &a, const Fq2x52 &b)
{
    return {a.c0 + b.c0, a.c1 + b.c1};
}
__device__ __forceinline__ Fq2x52 operator-(const Fq2x52 &a, const Fq2x52 &b)
{
    return {a.c0 - b.c0, a.c1 - b.c1};
}
__device__ __forceinline__ Fq2x52 neg(const Fq2x52 &a) { return {neg(a.c0), neg(a.c1)}; }
__device__ __forceinline__ Fq2x52 dbl(const Fq2x52 &a) { return {dbl(a.c0), dbl(a.c1)}; }
// Karatsuba, the three base-field products in one call (the FP64 Fq2 form serves
// latency-bound single-thread chains, where one call of three interleaved
// products takes far less than a pair and a single)
__device__ __forceinline__ Fq2x52 operator*(const Fq2x52 &a, const Fq2x52 &b)
{
    const Fq52Triple t = mul52x3v(a.c0, b.c0, a.c1, b.c1, a.c0 + a.c1, b.c0 + b.c1);
    return {t.x - t.y, t.z - t.x - t.y};
}
__device__ __forceinline__ Fq2x52 sqr(const Fq2x52 &a)
{
    Fq52 p, q;
    mul52x2(a.c0 + a.c1, a.c0 - a.c1, a.c0, a.c1, p, q);
    return {p, q + q};
}

// Fermat inverse a^(p-2); R' products keep the R' domain.  0 maps to 0.
__device__ inline Fq52 inverse(const Fq52 &a)
{
    const uint32_t e[8] = {FqParams::P0 - 2u, FqParams::P1, FqParams::P2, FqParams::P3,
                           FqParams::P4,      FqParams::P5, FqParams::P6, FqParams::P7};
    Fq52 acc = Fq52::one();
    for (int i = 255; i >= 0; --i) {
        acc = sqr(acc);
        if ((e[i >> 5] >> (i & 31)) & 1) acc = acc * a;
    }
    return acc;
}

// 1 / (a0 + a1 u) = (a0 - a1 u) / (a0^2 + a1^2)
__device__ inline Fq2x52 inverse(const Fq2x52 &a)
{
    const Fq52 ni = inverse(sqr(a.c0) + sqr(a.c1));
    return {a.c0 * ni, neg(a.c1) * ni};
}

// ---------------------------------------------------------------------------
// storage <-> compute: bits only (the stored value is already in the R' domain)
// ---------------------------------------------------------------------------

__device__ __forceinline__ Fq52 to52(const Fq &x)
{
    uint64_t w[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) w[i] = uint64_t(x.v[2 * i]) | (uint64_t(x.v[2 * i + 1]) << 32);
    Fq52 r;
    r.l[0] = w[0] & f52::kMask;
    r.l[1] = ((w[0] >> 52) | (w[1] << 12)) & f52::kMask;
    r.l[2] = ((w[1] >> 40) | (w[2] << 24)) & f52::kMask;
    r.l[3] = ((w[2] >> 28) | (w[3] << 36)) & f52::kMask;
    r.l[4] = w[3] >> 16;
    return r;
}

__device__ __forceinline__ Fq from52(const Fq52 &x)
{
    uint64_t w[4];
    w[0] = x.l[0] | (x.l[1] << 52);
    w[1] = (x.l[1] >> 12) | (x.l[2] << 40);
    w[2] = (x.l[2] >> 24) | (x.l[3] << 28);
    w[3] = (x.l[3] >> 36) | (x.l[4] << 16);
    Fq r;
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        r.v[2 * i] = uint32_t(w[i]);
        r.v[2 * i + 1] = uint32_t(w[i] >> 32);
    }
    return r;
}

__device__ __forceinline__ Fq52 to_compute(const Fq &x) { return to52(x); }
__device__ __forceinline__ Fq2x52 to_compute(const Fq2 &x) { return {to52(x.c0), to52(x.c1)}; }
__device__ __forceinline__ Fq to_storage(const Fq52 &x) { return from52(x); }
__device__ __forceinline__ Fq2 to_storage(const Fq2x52 &x) { return {from52(x.c0), from52(x.c1)}; }

template <class S>
struct Compute;
template <>
struct Compute<Fq> {
    using type = Fq52;
};
template <>
struct Compute<Fq2> {
    using type = Fq2x52;
};

// Montgomery domain changes: x 2^256 -> x 2^260 (times 2^264 mod p) and back
// (times 2^256 mod p), each one R' product
__device__ __forceinline__ Fq52 r256_to_r260(const Fq52 &x)
{
    return mul52(x, Fq52{{0xb0f2afaec667aull, 0xed9626b0fffbdull, 0x9e2a0fcad825aull,
                          0xe357276f48b70ull, 0xd791464ef86ull}});
}
__device__ __forceinline__ Fq52 r260_to_r256(const Fq52 &x)
{
    return mul52(x, Fq52{{0xd438dc58f0d9dull, 0x28f5c70b3dd35ull, 0x879462c0a78ebull,
                          0xdf2f666ea36f7ull, 0xe0a77c19a07ull}});
}
__device__ __forceinline__ Fq2x52 r256_to_r260(const Fq2x52 &x)
{
    return {r256_to_r260(x.c0), r256_to_r260(x.c1)};
}
__device__ __forceinline__ Fq2x52 r260_to_r256(const Fq2x52 &x)
{
    return {r260_to_r256(x.c0), r260_to_r256(x.c1)};
}

} // namespace nkr
