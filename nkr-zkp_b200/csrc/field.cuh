// BN254 base field Fq and scalar field Fr on sm_100a.
//
// Representation: 8 x 32-bit little-endian limbs in Montgomery form
// (R = 2^256), always fully reduced (< modulus).  The byte image is identical
// to libff's Fp_model<4, modulus>::mont_repr on x86-64, so device buffers are
// bit-for-bit the reference's host vectors (reference: libff
// algebra/fields/fp.hpp:40-42, CUDA mont_t layout operators/cuda/include/fields/
// mont_t.cuh:45).
//
// Multiplication is CIOS Montgomery: per limb of b, one carry chain adds the
// low halves of a*b_i, one adds the high halves, then the reduction by
// m = t0 * (-p^-1) repeats the pair of chains with the modulus as immediates.
// Because p < 2^254, the running value stays below 2p and 9 words suffice.
#pragma once

#include <cstdint>

namespace nkr {

// True for a field type whose products have a paired form mul2 (two independent
// products in one call; field52.cuh).  The curve formulas issue their products in
// pairs only for such fields and keep their original order otherwise.
template <class F>
struct HasPairedMul {
    static constexpr bool value = false;
};

struct FqParams {
    static constexpr uint32_t P0 = 0xd87cfd47u, P1 = 0x3c208c16u, P2 = 0x6871ca8du,
                              P3 = 0x97816a91u, P4 = 0x8181585du, P5 = 0xb85045b6u,
                              P6 = 0xe131a029u, P7 = 0x30644e72u;
    static constexpr uint32_t INV = 0xe4866389u; // -p^-1 mod 2^32
    static constexpr uint32_t O0 = 0xc58f0d9du, O1 = 0xd35d438du, O2 = 0xf5c70b3du, O3 = 0x0a78eb28u, O4 = 0x7879462cu, O5 = 0x666ea36fu, O6 = 0x9a07df2fu, O7 = 0x0e0a77c1u;
    static constexpr uint32_t Q0 = 0x538afa89u, Q1 = 0xf32cfc5bu, Q2 = 0xd44501fbu, Q3 = 0xb5e71911u, Q4 = 0x0a417ff6u, Q5 = 0x47ab1effu, Q6 = 0xcab8351fu, Q7 = 0x06d89f71u;
};

struct FrParams {
    static constexpr uint32_t P0 = 0xf0000001u, P1 = 0x43e1f593u, P2 = 0x79b97091u,
                              P3 = 0x2833e848u, P4 = 0x8181585du, P5 = 0xb85045b6u,
                              P6 = 0xe131a029u, P7 = 0x30644e72u;
    static constexpr uint32_t INV = 0xefffffffu;
    static constexpr uint32_t O0 = 0x4ffffffbu, O1 = 0xac96341cu, O2 = 0x9f60cd29u, O3 = 0x36fc7695u, O4 = 0x7879462eu, O5 = 0x666ea36fu, O6 = 0x9a07df2fu, O7 = 0x0e0a77c1u;
    static constexpr uint32_t Q0 = 0xae216da7u, Q1 = 0x1bb8e645u, Q2 = 0xe35c59e3u, Q3 = 0x53fe3ab1u, Q4 = 0x53bb8085u, Q5 = 0x8c49833du, Q6 = 0x7f4e44a5u, Q7 = 0x0216d0b1u;
};

template <class P>
struct alignas(32) Fp {
    uint32_t v[8];

    __device__ __forceinline__ static Fp zero()
    {
        Fp r;
#pragma unroll
        for (int i = 0; i < 8; ++i) r.v[i] = 0;
        return r;
    }
    __device__ __forceinline__ static Fp one()
    {
        return {{P::O0, P::O1, P::O2, P::O3, P::O4, P::O5, P::O6, P::O7}};
    }
    __device__ __forceinline__ static Fp r2()
    {
        return {{P::Q0, P::Q1, P::Q2, P::Q3, P::Q4, P::Q5, P::Q6, P::Q7}};
    }
    __device__ __forceinline__ bool is_zero() const
    {
        uint32_t x = v[0];
#pragma unroll
        for (int i = 1; i < 8; ++i) x |= v[i];
        return x == 0;
    }
    __device__ __forceinline__ bool operator==(const Fp &o) const
    {
        uint32_t x = 0;
#pragma unroll
        for (int i = 0; i < 8; ++i) x |= v[i] ^ o.v[i];
        return x == 0;
    }
    __device__ __forceinline__ bool operator!=(const Fp &o) const { return !(*this == o); }
};

using Fq = Fp<FqParams>;
using Fr = Fp<FrParams>;

// ---------------------------------------------------------------------------
// conditional subtraction of the modulus: r = (t >= p) ? t - p : t
// ---------------------------------------------------------------------------
template <class P>
__device__ __forceinline__ void reduce_once(uint32_t *t)
{
    uint32_t s0, s1, s2, s3, s4, s5, s6, s7, br;
    asm("sub.cc.u32  %0, %9,  %17;\n\t"
        "subc.cc.u32 %1, %10, %18;\n\t"
        "subc.cc.u32 %2, %11, %19;\n\t"
        "subc.cc.u32 %3, %12, %20;\n\t"
        "subc.cc.u32 %4, %13, %21;\n\t"
        "subc.cc.u32 %5, %14, %22;\n\t"
        "subc.cc.u32 %6, %15, %23;\n\t"
        "subc.cc.u32 %7, %16, %24;\n\t"
        "subc.u32    %8, 0, 0;"
        : "=r"(s0), "=r"(s1), "=r"(s2), "=r"(s3), "=r"(s4), "=r"(s5), "=r"(s6), "=r"(s7),
          "=r"(br)
        : "r"(t[0]), "r"(t[1]), "r"(t[2]), "r"(t[3]), "r"(t[4]), "r"(t[5]), "r"(t[6]),
          "r"(t[7]), "n"(P::P0), "n"(P::P1), "n"(P::P2), "n"(P::P3), "n"(P::P4), "n"(P::P5),
          "n"(P::P6), "n"(P::P7));
    // br == 0xffffffff when t < p (keep t), 0 when t >= p (take t - p)
    const bool keep = br != 0;
    t[0] = keep ? t[0] : s0;
    t[1] = keep ? t[1] : s1;
    t[2] = keep ? t[2] : s2;
    t[3] = keep ? t[3] : s3;
    t[4] = keep ? t[4] : s4;
    t[5] = keep ? t[5] : s5;
    t[6] = keep ? t[6] : s6;
    t[7] = keep ? t[7] : s7;
}

template <class P>
__device__ __forceinline__ Fp<P> operator+(const Fp<P> &a, const Fp<P> &b)
{
    Fp<P> r;
    asm("add.cc.u32  %0, %8,  %16;\n\t"
        "addc.cc.u32 %1, %9,  %17;\n\t"
        "addc.cc.u32 %2, %10, %18;\n\t"
        "addc.cc.u32 %3, %11, %19;\n\t"
        "addc.cc.u32 %4, %12, %20;\n\t"
        "addc.cc.u32 %5, %13, %21;\n\t"
        "addc.cc.u32 %6, %14, %22;\n\t"
        "addc.u32    %7, %15, %23;"
        : "=r"(r.v[0]), "=r"(r.v[1]), "=r"(r.v[2]), "=r"(r.v[3]), "=r"(r.v[4]), "=r"(r.v[5]),
          "=r"(r.v[6]), "=r"(r.v[7])
        : "r"(a.v[0]), "r"(a.v[1]), "r"(a.v[2]), "r"(a.v[3]), "r"(a.v[4]), "r"(a.v[5]),
          "r"(a.v[6]), "r"(a.v[7]), "r"(b.v[0]), "r"(b.v[1]), "r"(b.v[2]), "r"(b.v[3]),
          "r"(b.v[4]), "r"(b.v[5]), "r"(b.v[6]), "r"(b.v[7]));
    reduce_once<P>(r.v);
    return r;
}

template <class P>
__device__ __forceinline__ Fp<P> operator-(const Fp<P> &a, const Fp<P> &b)
{
    Fp<P> r;
    uint32_t br;
    asm("sub.cc.u32  %0, %9,  %17;\n\t"
        "subc.cc.u32 %1, %10, %18;\n\t"
        "subc.cc.u32 %2, %11, %19;\n\t"
        "subc.cc.u32 %3, %12, %20;\n\t"
        "subc.cc.u32 %4, %13, %21;\n\t"
        "subc.cc.u32 %5, %14, %22;\n\t"
        "subc.cc.u32 %6, %15, %23;\n\t"
        "subc.cc.u32 %7, %16, %24;\n\t"
        "subc.u32    %8, 0, 0;"
        : "=r"(r.v[0]), "=r"(r.v[1]), "=r"(r.v[2]), "=r"(r.v[3]), "=r"(r.v[4]), "=r"(r.v[5]),
          "=r"(r.v[6]), "=r"(r.v[7]), "=r"(br)
        : "r"(a.v[0]), "r"(a.v[1]), "r"(a.v[2]), "r"(a.v[3]), "r"(a.v[4]), "r"(a.v[5]),
          "r"(a.v[6]), "r"(a.v[7]), "r"(b.v[0]), "r"(b.v[1]), "r"(b.v[2]), "r"(b.v[3]),
          "r"(b.v[4]), "r"(b.v[5]), "r"(b.v[6]), "r"(b.v[7]));
    // on borrow add p back (br is an all-ones mask)
    asm("add.cc.u32  %0, %0, %8;\n\t"
        "addc.cc.u32 %1, %1, %9;\n\t"
        "addc.cc.u32 %2, %2, %10;\n\t"
        "addc.cc.u32 %3, %3, %11;\n\t"
        "addc.cc.u32 %4, %4, %12;\n\t"
        "addc.cc.u32 %5, %5, %13;\n\t"
        "addc.cc.u32 %6, %6, %14;\n\t"
        "addc.u32    %7, %7, %15;"
        : "+r"(r.v[0]), "+r"(r.v[1]), "+r"(r.v[2]), "+r"(r.v[3]), "+r"(r.v[4]), "+r"(r.v[5]),
          "+r"(r.v[6]), "+r"(r.v[7])
        : "r"(P::P0 & br), "r"(P::P1 & br), "r"(P::P2 & br), "r"(P::P3 & br), "r"(P::P4 & br),
          "r"(P::P5 & br), "r"(P::P6 & br), "r"(P::P7 & br));
    return r;
}

template <class P>
__device__ __forceinline__ Fp<P> neg(const Fp<P> &a)
{
    return Fp<P>::zero() - a;
}

template <class P>
__device__ __forceinline__ Fp<P> dbl(const Fp<P> &a)
{
    return a + a;
}

// One CIOS round: t[0..8] += a * bi; m = t0 * inv; t += m * p; t >>= 32.
#define NKR_CIOS_ROUND(bi)                                                                     \
    asm("mad.lo.cc.u32  %0, %9,  %17, %0;\n\t"                                                 \
        "madc.lo.cc.u32 %1, %10, %17, %1;\n\t"                                                 \
        "madc.lo.cc.u32 %2, %11, %17, %2;\n\t"                                                 \
        "madc.lo.cc.u32 %3, %12, %17, %3;\n\t"                                                 \
        "madc.lo.cc.u32 %4, %13, %17, %4;\n\t"                                                 \
        "madc.lo.cc.u32 %5, %14, %17, %5;\n\t"                                                 \
        "madc.lo.cc.u32 %6, %15, %17, %6;\n\t"                                                 \
        "madc.lo.cc.u32 %7, %16, %17, %7;\n\t"                                                 \
        "addc.u32       %8, %8, 0;\n\t"                                                        \
        "mad.hi.cc.u32  %1, %9,  %17, %1;\n\t"                                                 \
        "madc.hi.cc.u32 %2, %10, %17, %2;\n\t"                                                 \
        "madc.hi.cc.u32 %3, %11, %17, %3;\n\t"                                                 \
        "madc.hi.cc.u32 %4, %12, %17, %4;\n\t"                                                 \
        "madc.hi.cc.u32 %5, %13, %17, %5;\n\t"                                                 \
        "madc.hi.cc.u32 %6, %14, %17, %6;\n\t"                                                 \
        "madc.hi.cc.u32 %7, %15, %17, %7;\n\t"                                                 \
        "madc.hi.u32    %8, %16, %17, %8;"                                                     \
        : "+r"(t0), "+r"(t1), "+r"(t2), "+r"(t3), "+r"(t4), "+r"(t5), "+r"(t6), "+r"(t7),      \
          "+r"(t8)                                                                             \
        : "r"(a.v[0]), "r"(a.v[1]), "r"(a.v[2]), "r"(a.v[3]), "r"(a.v[4]), "r"(a.v[5]),        \
          "r"(a.v[6]), "r"(a.v[7]), "r"(bi));                                                  \
    {                                                                                          \
        const uint32_t m = t0 * P::INV;                                                        \
        asm("mad.lo.cc.u32  %0, %9, %10, %0;\n\t"                                              \
            "madc.lo.cc.u32 %1, %9, %11, %1;\n\t"                                              \
            "madc.lo.cc.u32 %2, %9, %12, %2;\n\t"                                              \
            "madc.lo.cc.u32 %3, %9, %13, %3;\n\t"                                              \
            "madc.lo.cc.u32 %4, %9, %14, %4;\n\t"                                              \
            "madc.lo.cc.u32 %5, %9, %15, %5;\n\t"                                              \
            "madc.lo.cc.u32 %6, %9, %16, %6;\n\t"                                              \
            "madc.lo.cc.u32 %7, %9, %17, %7;\n\t"                                              \
            "addc.u32       %8, %8, 0;\n\t"                                                    \
            "mad.hi.cc.u32  %1, %9, %10, %1;\n\t"                                              \
            "madc.hi.cc.u32 %2, %9, %11, %2;\n\t"                                              \
            "madc.hi.cc.u32 %3, %9, %12, %3;\n\t"                                              \
            "madc.hi.cc.u32 %4, %9, %13, %4;\n\t"                                              \
            "madc.hi.cc.u32 %5, %9, %14, %5;\n\t"                                              \
            "madc.hi.cc.u32 %6, %9, %15, %6;\n\t"                                              \
            "madc.hi.cc.u32 %7, %9, %16, %7;\n\t"                                              \
            "madc.hi.u32    %8, %9, %17, %8;"                                                  \
            : "+r"(t0), "+r"(t1), "+r"(t2), "+r"(t3), "+r"(t4), "+r"(t5), "+r"(t6), "+r"(t7),  \
              "+r"(t8)                                                                         \
            : "r"(m), "n"(P::P0), "n"(P::P1), "n"(P::P2), "n"(P::P3), "n"(P::P4), "n"(P::P5),  \
              "n"(P::P6), "n"(P::P7));                                                         \
    }                                                                                          \
    t0 = t1;                                                                                   \
    t1 = t2;                                                                                   \
    t2 = t3;                                                                                   \
    t3 = t4;                                                                                   \
    t4 = t5;                                                                                   \
    t5 = t6;                                                                                   \
    t6 = t7;                                                                                   \
    t7 = t8;                                                                                   \
    t8 = 0;

// Translation units whose kernels chain many products (curve arithmetic) define
// NKR_FIELD_MUL_OUTLINE before including this header: the product body then
// exists once per kernel instead of once per call site, which keeps the hot
// loop inside the instruction cache (inlined, one XYZZ addition is several
// thousand instructions).  Elementwise kernels keep it inlined.
// NKR_MUL_ATTR_FN is the same for non-template functions, which also need
// `inline` to be defined in every translation unit that includes the header.
#ifdef NKR_FIELD_MUL_OUTLINE
#define NKR_MUL_ATTR __noinline__
#define NKR_MUL_ATTR_FN inline __noinline__
#else
#define NKR_MUL_ATTR __forceinline__
#define NKR_MUL_ATTR_FN __forceinline__
#endif

template <class P>
__device__ __forceinline__ uint32_t mod_word(int j)
{
    switch (j) {
    case 0: return P::P0;
    case 1: return P::P1;
    case 2: return P::P2;
    case 3: return P::P3;
    case 4: return P::P4;
    case 5: return P::P5;
    case 6: return P::P6;
    default: return P::P7;
    }
}

// The library's Montgomery product: CIOS with 64-bit accumulation of the
// 32 x 32 -> 64 partial products.  On sm_100a it issues fewer multiply-pipe
// instructions than explicit 32-bit carry chains (mont_mul_cc below) and
// measures 14% faster in the throughput microbenchmark (nkr_b200_bench_mul);
// both forms are bit-identical.
template <class P, int N>
__device__ __forceinline__ void mont_mul_body(const Fp<P> *const *a, const Fp<P> *const *b,
                                              Fp<P> *const *r)
{
    uint32_t t[N][10];
#pragma unroll
    for (int k = 0; k < N; ++k)
#pragma unroll
        for (int j = 0; j < 10; ++j) t[k][j] = 0;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
#pragma unroll
        for (int k = 0; k < N; ++k) {
            uint64_t c = 0;
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                const uint64_t p = uint64_t(a[k]->v[j]) * b[k]->v[i] + t[k][j] + c;
                t[k][j] = uint32_t(p);
                c = p >> 32;
            }
            uint64_t s = uint64_t(t[k][8]) + c;
            t[k][8] = uint32_t(s);
            t[k][9] = uint32_t(s >> 32);
            const uint32_t m = t[k][0] * P::INV;
            c = (uint64_t(m) * P::P0 + t[k][0]) >> 32;
#pragma unroll
            for (int j = 1; j < 8; ++j) {
                const uint64_t p = uint64_t(m) * mod_word<P>(j) + t[k][j] + c;
                t[k][j - 1] = uint32_t(p);
                c = p >> 32;
            }
            s = uint64_t(t[k][8]) + c;
            t[k][7] = uint32_t(s);
            t[k][8] = t[k][9] + uint32_t(s >> 32);
        }
    }
#pragma unroll
    for (int k = 0; k < N; ++k) {
#pragma unroll
        for (int i = 0; i < 8; ++i) r[k]->v[i] = t[k][i];
        reduce_once<P>(r[k]->v);
    }
}

// Operands travel by value: an out-of-line call (NKR_FIELD_MUL_OUTLINE) then
// passes them in registers instead of through the thread's local-memory stack
// (measured 10% faster G2 MSMs than reference parameters).
template <class P>
__device__ NKR_MUL_ATTR Fp<P> operator*(Fp<P> a, Fp<P> b)
{
    Fp<P> r;
    const Fp<P> *pa[1] = {&a}, *pb[1] = {&b};
    Fp<P> *pr[1] = {&r};
    mont_mul_body<P, 1>(pa, pb, pr);
    return r;
}

// The same product with explicit PTX carry chains (two chains per limb of b
// for the low / high halves, then the reduction pair); kept for comparison.
template <class P>
__device__ __forceinline__ Fp<P> mont_mul_cc(const Fp<P> &a, const Fp<P> &b)
{
    uint32_t t0 = 0, t1 = 0, t2 = 0, t3 = 0, t4 = 0, t5 = 0, t6 = 0, t7 = 0, t8 = 0;
    NKR_CIOS_ROUND(b.v[0])
    NKR_CIOS_ROUND(b.v[1])
    NKR_CIOS_ROUND(b.v[2])
    NKR_CIOS_ROUND(b.v[3])
    NKR_CIOS_ROUND(b.v[4])
    NKR_CIOS_ROUND(b.v[5])
    NKR_CIOS_ROUND(b.v[6])
    NKR_CIOS_ROUND(b.v[7])
    Fp<P> r;
    r.v[0] = t0;
    r.v[1] = t1;
    r.v[2] = t2;
    r.v[3] = t3;
    r.v[4] = t4;
    r.v[5] = t5;
    r.v[6] = t6;
    r.v[7] = t7;
    (void)t8;
    reduce_once<P>(r.v);
    return r;
}

template <class P>
__device__ __forceinline__ Fp<P> sqr(const Fp<P> &a)
{
    return a * a;
}

// Montgomery -> canonical integer (same limb layout)
template <class P>
__device__ __forceinline__ Fp<P> from_mont(const Fp<P> &a)
{
    Fp<P> one;
    one.v[0] = 1;
#pragma unroll
    for (int i = 1; i < 8; ++i) one.v[i] = 0;
    return a * one;
}

// canonical integer (< p) -> Montgomery
template <class P>
__device__ __forceinline__ Fp<P> to_mont(const Fp<P> &a)
{
    return a * Fp<P>::r2();
}

// a^e for a small public exponent given as 8 limbs (left-to-right square-and-multiply)
template <class P>
__device__ Fp<P> pow_limbs(const Fp<P> &a, const uint32_t *e)
{
    Fp<P> acc = Fp<P>::one();
    for (int i = 255; i >= 0; --i) {
        acc = sqr(acc);
        if ((e[i >> 5] >> (i & 31)) & 1) acc = acc * a;
    }
    return acc;
}

// Fermat inverse: a^(p-2).  0 maps to 0.
template <class P>
__device__ Fp<P> inverse(const Fp<P> &a)
{
    const uint32_t e[8] = {P::P0 - 2u, P::P1, P::P2, P::P3, P::P4, P::P5, P::P6, P::P7};
    return pow_limbs(a, e);
}

// ---------------------------------------------------------------------------
// Fq2 = Fq[u] / (u^2 + 1)  (libff alt_bn128_Fq2, non_residue = -1)
// ---------------------------------------------------------------------------
struct alignas(32) Fq2 {
    Fq c0, c1;
    __device__ __forceinline__ static Fq2 zero() { return {Fq::zero(), Fq::zero()}; }
    __device__ __forceinline__ static Fq2 one() { return {Fq::one(), Fq::zero()}; }
    __device__ __forceinline__ bool is_zero() const { return c0.is_zero() && c1.is_zero(); }
    __device__ __forceinline__ bool operator==(const Fq2 &o) const
    {
        return c0 == o.c0 && c1 == o.c1;
    }
    __device__ __forceinline__ bool operator!=(const Fq2 &o) const { return !(*this == o); }
};

__device__ __forceinline__ Fq2 operator+(const Fq2 &a, const Fq2 &b)
{
    return {a.c0 + b.c0, a.c1 + b.c1};
}
__device__ __forceinline__ Fq2 operator-(const Fq2 &a, const Fq2 &b)
{
    return {a.c0 - b.c0, a.c1 - b.c1};
}
__device__ __forceinline__ Fq2 neg(const Fq2 &a) { return {neg(a.c0), neg(a.c1)}; }
__device__ __forceinline__ Fq2 dbl(const Fq2 &a) { return {dbl(a.c0), dbl(a.c1)}; }

// Karatsuba with 3 Montgomery products (one three-product call measured slower:
// more registers and a three times larger body)
__device__ __forceinline__ Fq2 operator*(const Fq2 &a, const Fq2 &b)
{
    const Fq v0 = a.c0 * b.c0;
    const Fq v1 = a.c1 * b.c1;
    const Fq s = (a.c0 + a.c1) * (b.c0 + b.c1);
    return {v0 - v1, s - v0 - v1};
}

// (a0 + a1 u)^2 = (a0 + a1)(a0 - a1) + 2 a0 a1 u
__device__ __forceinline__ Fq2 sqr(const Fq2 &a)
{
    const Fq p = (a.c0 + a.c1) * (a.c0 - a.c1);
    const Fq q = a.c0 * a.c1;
    return {p, q + q};
}

namespace lazy {
// 256 x 256 -> 512-bit schoolbook product, 64-bit accumulation of the partial
// products (t[16], little-endian words)
__device__ __forceinline__ void mul_wide(const uint32_t *a, const uint32_t *b, uint32_t *t)
{
#pragma unroll
    for (int j = 0; j < 16; ++j) t[j] = 0;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        uint64_t c = 0;
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            const uint64_t p = uint64_t(a[j]) * b[i] + t[i + j] + c;
            t[i + j] = uint32_t(p);
            c = p >> 32;
        }
        t[i + 8] = uint32_t(c);
    }
}

// Montgomery reduction T R^-1 mod p of a 512-bit T < p R (R = 2^256): eight
// word rows clear t[0..7]; the row carry out of t[i + 8] enters row i + 1.  The
// result is below 2p before the final conditional subtraction.
__device__ __forceinline__ Fq redc_wide(uint32_t *t)
{
    uint32_t hi = 0;
#pragma unroll
    for (int i = 0; i < 8; ++i) {
        const uint32_t m = t[i] * FqParams::INV;
        uint64_t c = (uint64_t(m) * FqParams::P0 + t[i]) >> 32;
#pragma unroll
        for (int j = 1; j < 8; ++j) {
            const uint64_t p = uint64_t(m) * mod_word<FqParams>(j) + t[i + j] + c;
            t[i + j] = uint32_t(p);
            c = p >> 32;
        }
        const uint64_t s = uint64_t(t[i + 8]) + c + hi;
        t[i + 8] = uint32_t(s);
        hi = uint32_t(s >> 32);
    }
    Fq r;
#pragma unroll
    for (int i = 0; i < 8; ++i) r.v[i] = t[8 + i];
    reduce_once<FqParams>(r.v);
    return r;
}

// p^2 for BN254's base field, 16 little-endian words
__device__ __forceinline__ uint32_t p2_word(int k)
{
    constexpr uint32_t w[16] = {0x275d69b1u, 0x3b5458a2u, 0x09eac101u, 0xa602072du,
                                0x6d96cadcu, 0x4a50189cu, 0x7a1242c8u, 0x04689e95u,
                                0x34c6b38du, 0x26edfa5cu, 0x16375606u, 0xb00b8551u,
                                0x0348d21cu, 0x599a6f7cu, 0x763cbf9cu, 0x0925c4b8u};
    return w[k];
}
} // namespace lazy

// Fq2 with the lazily reduced product below: same layout and values as Fq2, its
// arithmetic closed over the type.  It is the compute type of the G2 bucket
// reduction levels, whose long dependent chains gain from the shorter product
// (at 2^18 points: first level 0.41 -> 0.36 ms, block levels 1.50 -> 1.22 ms);
// the G2 accumulation keeps Fq2, where the larger product body costs registers:
// 255 with spills at 2 blocks per SM (4% slower), 100 B of spills at the 3-block
// budget of the shared-memory accumulator (3.86 instead of 3.25 ms at 2^18).
struct Fq2L : Fq2 {
    Fq2L() = default;
    __device__ __forceinline__ Fq2L(const Fq2 &a) : Fq2(a) {}
    __device__ __forceinline__ static Fq2L zero() { return Fq2::zero(); }
    __device__ __forceinline__ static Fq2L one() { return Fq2::one(); }
};
__device__ __forceinline__ Fq2L operator+(const Fq2L &a, const Fq2L &b)
{
    return static_cast<const Fq2 &>(a) + static_cast<const Fq2 &>(b);
}
__device__ __forceinline__ Fq2L operator-(const Fq2L &a, const Fq2L &b)
{
    return static_cast<const Fq2 &>(a) - static_cast<const Fq2 &>(b);
}
__device__ __forceinline__ Fq2L neg(const Fq2L &a) { return neg(static_cast<const Fq2 &>(a)); }
__device__ __forceinline__ Fq2L dbl(const Fq2L &a) { return dbl(static_cast<const Fq2 &>(a)); }
__device__ __forceinline__ Fq2L sqr(const Fq2L &a) { return sqr(static_cast<const Fq2 &>(a)); }

// Fq2 product with lazy reduction: the Karatsuba products are formed as 512-bit
// integers and combined before reduction, 3 schoolbook products and 2
// Montgomery reductions instead of 3 Montgomery products (18% fewer
// multiply-pipe instructions):
//   c0 = REDC(a0 b0 + p^2 - a1 b1)                          T in [0, 2 p^2)
//   c1 = REDC((a0 + a1)(b0 + b1) - a0 b0 - a1 b1)           T = a0 b1 + a1 b0 in [0, 2 p^2)
// with a0 + a1 and b0 + b1 unreduced (< 2p < 2^255) and 2 p^2 < p R, so each
// reduction lands below 2p and one conditional subtraction makes it canonical:
// the result equals the 3-product form bit for bit.
__device__ NKR_MUL_ATTR_FN Fq2L operator*(Fq2L a, Fq2L b)
{
    uint32_t v0[16], v1[16], t[16], w[16];
    lazy::mul_wide(a.c0.v, b.c0.v, v0);
    lazy::mul_wide(a.c1.v, b.c1.v, v1);
    {
        int64_t c0 = 0, c1 = 0;
#pragma unroll
        for (int k = 0; k < 16; ++k) {
            const int64_t d = int64_t(v0[k]) + lazy::p2_word(k) - int64_t(v1[k]) + c0;
            t[k] = uint32_t(d);
            c0 = d >> 32;
            const int64_t e = int64_t(v0[k]) + int64_t(v1[k]) + c1;
            w[k] = uint32_t(e);
            c1 = e >> 32;
        }
    }
    Fq2 r;
    r.c0 = lazy::redc_wide(t);
    uint32_t sa[8], sb[8];
    {
        uint64_t ca = 0, cb = 0;
#pragma unroll
        for (int k = 0; k < 8; ++k) {
            const uint64_t x = uint64_t(a.c0.v[k]) + a.c1.v[k] + ca;
            sa[k] = uint32_t(x);
            ca = x >> 32;
            const uint64_t y = uint64_t(b.c0.v[k]) + b.c1.v[k] + cb;
            sb[k] = uint32_t(y);
            cb = y >> 32;
        }
    }
    lazy::mul_wide(sa, sb, t);
    {
        int64_t c = 0;
#pragma unroll
        for (int k = 0; k < 16; ++k) {
            const int64_t d = int64_t(t[k]) - int64_t(w[k]) + c;
            t[k] = uint32_t(d);
            c = d >> 32;
        }
    }
    r.c1 = lazy::redc_wide(t);
    return r;
}


__device__ inline Fq2 inverse(const Fq2 &a)
{
    const Fq n = sqr(a.c0) + sqr(a.c1);
    const Fq ni = inverse(n);
    return {a.c0 * ni, neg(a.c1) * ni};
}

} // namespace nkr
