// The BN254 (alt_bn128) reduced pairing exactly as libff computes it, for
// Groth16 verification on the device (protocol.cpp:96-108 compares GT values
// against the verification key's libff-computed e(alpha, beta), so the values
// must be libff's bit for bit, not merely a pairing).
//
// Tower (libff alt_bn128): Fq2 = Fq[u]/(u^2 + 1), Fq6 = Fq2[v]/(v^3 - xi) with
// xi = 9 + u, Fq12 = Fq6[w]/(w^2 - v); G2 lives on the D-type twist
// y^2 = x^3 + 3/xi, untwisted by (x, y) -> (x w^2, y w^3) (w^6 = xi).
//
// Miller loop: the optimal ate loop over L = 6z + 2 (z = 4965661367192848881),
// left to right from the bit below the top one, then the lines through pi(Q)
// and -pi^2(Q) (libff alt_bn128_pairing.cpp, ate_miller_loop).  Lines are
// computed in affine twist coordinates: for slope lam' on the twist the line
// at P = (xP, yP) is yP - lam' xP w + (lam' xT - yT) v w (its vertical-line and
// projective-scale factors lie in proper subfields and vanish in the final
// exponentiation, so the value after it equals libff's).
//
// Final exponentiation: f^((q^6 - 1)(q^2 + 1) k (q^4 - q^2 + 1)/r) with
// k = 2z(6z^2 + 3z + 1): libff's last chunk (Fuentes-Castaneda et al.) computes
// this multiple of the exact hard-part exponent, and GT values must match its.
// Here the easy part is conj(f) / f and the rest one square-and-multiply
// exponentiation by the constant E = (q^2 + 1) k (q^4 - q^2 + 1)/r.
#pragma once

#include "curve.cuh"

namespace nkr {

struct Fq6 {
    Fq2 c0, c1, c2;
};
struct Fq12 {
    Fq6 c0, c1;
};

// ---------------------------------------------------------------------------
// Fq2 helpers
// ---------------------------------------------------------------------------

// a (9 + u) = (9 a0 - a1) + (a0 + 9 a1) u
__device__ __forceinline__ Fq2 mul_xi(const Fq2 &a)
{
    const Fq2 n = dbl(dbl(dbl(a))) + a;
    return {n.c0 - a.c1, a.c0 + n.c1};
}
__device__ __forceinline__ Fq2 mul_fq(const Fq2 &a, const Fq &s) { return {a.c0 * s, a.c1 * s}; }
__device__ __forceinline__ Fq2 conj(const Fq2 &a) { return {a.c0, neg(a.c1)}; }

// ---------------------------------------------------------------------------
// Fq6
// ---------------------------------------------------------------------------

__device__ __forceinline__ Fq6 fq6_zero() { return {Fq2::zero(), Fq2::zero(), Fq2::zero()}; }
__device__ __forceinline__ Fq6 operator+(const Fq6 &a, const Fq6 &b)
{
    return {a.c0 + b.c0, a.c1 + b.c1, a.c2 + b.c2};
}
__device__ __forceinline__ Fq6 operator-(const Fq6 &a, const Fq6 &b)
{
    return {a.c0 - b.c0, a.c1 - b.c1, a.c2 - b.c2};
}
__device__ __forceinline__ Fq6 neg(const Fq6 &a) { return {neg(a.c0), neg(a.c1), neg(a.c2)}; }
// a v
__device__ __forceinline__ Fq6 mul_v(const Fq6 &a) { return {mul_xi(a.c2), a.c0, a.c1}; }

// Karatsuba: 6 Fq2 products
__device__ inline Fq6 operator*(const Fq6 &a, const Fq6 &b)
{
    const Fq2 t0 = a.c0 * b.c0, t1 = a.c1 * b.c1, t2 = a.c2 * b.c2;
    return {t0 + mul_xi((a.c1 + a.c2) * (b.c1 + b.c2) - t1 - t2),
            (a.c0 + a.c1) * (b.c0 + b.c1) - t0 - t1 + mul_xi(t2),
            (a.c0 + a.c2) * (b.c0 + b.c2) - t0 - t2 + t1};
}

__device__ inline Fq6 inverse(const Fq6 &a)
{
    const Fq2 t0 = sqr(a.c0) - mul_xi(a.c1 * a.c2);
    const Fq2 t1 = mul_xi(sqr(a.c2)) - a.c0 * a.c1;
    const Fq2 t2 = sqr(a.c1) - a.c0 * a.c2;
    const Fq2 d = a.c0 * t0 + mul_xi(a.c2 * t1 + a.c1 * t2);
    const Fq2 di = inverse(d);
    return {t0 * di, t1 * di, t2 * di};
}

// ---------------------------------------------------------------------------
// Fq12
// ---------------------------------------------------------------------------

__device__ __forceinline__ Fq12 fq12_one() { return {{Fq2::one(), Fq2::zero(), Fq2::zero()}, fq6_zero()}; }

__device__ inline Fq12 operator*(const Fq12 &a, const Fq12 &b)
{
    const Fq6 t0 = a.c0 * b.c0, t1 = a.c1 * b.c1;
    return {t0 + mul_v(t1), (a.c0 + a.c1) * (b.c0 + b.c1) - t0 - t1};
}

// (a0 + a1 w)^2 = (a0 + a1)(a0 + v a1) - t - v t + 2 t w, t = a0 a1
__device__ inline Fq12 sqr(const Fq12 &a)
{
    const Fq6 t = a.c0 * a.c1;
    return {(a.c0 + a.c1) * (a.c0 + mul_v(a.c1)) - t - mul_v(t), t + t};
}

__device__ __forceinline__ Fq12 conj(const Fq12 &a) { return {a.c0, neg(a.c1)}; }

__device__ inline Fq12 inverse(const Fq12 &a)
{
    const Fq6 t = inverse(a.c0 * a.c0 - mul_v(a.c1 * a.c1));
    return {a.c0 * t, neg(a.c1 * t)};
}

__device__ __forceinline__ bool operator==(const Fq12 &a, const Fq12 &b)
{
    return a.c0.c0 == b.c0.c0 && a.c0.c1 == b.c0.c1 && a.c0.c2 == b.c0.c2 && a.c1.c0 == b.c1.c0 &&
           a.c1.c1 == b.c1.c1 && a.c1.c2 == b.c1.c2;
}

// f times the line yP + a w + b v w (a = -lam xP, b = lam xT - yT):
// (f0 + f1 w)(L0 + L1 w) = (f0 L0 + v f1 L1) + (f0 L1 + f1 L0) w with L0 = yP,
// L1 = a + b v
__device__ __forceinline__ Fq6 mul_by_ab(const Fq6 &f, const Fq2 &a, const Fq2 &b)
{
    // (f0 + f1 v + f2 v^2)(a + b v)
    return {f.c0 * a + mul_xi(f.c2 * b), f.c0 * b + f.c1 * a, f.c1 * b + f.c2 * a};
}
__device__ __forceinline__ Fq6 mul_by_fq(const Fq6 &f, const Fq &s)
{
    return {mul_fq(f.c0, s), mul_fq(f.c1, s), mul_fq(f.c2, s)};
}
__device__ inline Fq12 mul_by_line(const Fq12 &f, const Fq &yP, const Fq2 &a, const Fq2 &b)
{
    return {mul_by_fq(f.c0, yP) + mul_v(mul_by_ab(f.c1, a, b)),
            mul_by_ab(f.c0, a, b) + mul_by_fq(f.c1, yP)};
}

// ---------------------------------------------------------------------------
// constants
// ---------------------------------------------------------------------------

// L = 6z + 2 (65 bits)
constexpr uint64_t kAteLoopLo = 0x9d797039be763ba8ull; // bits 0..63
constexpr int kAteTopBit = 64;                           // bit 64 is set
__device__ __forceinline__ bool ate_bit(int i) { return (kAteLoopLo >> i) & 1ull; }
// doubling steps (bits 63..0), addition steps (set bits among them), 2 final lines
constexpr int kAteLines = 64 + 36 + 2;

// Frobenius on the twist: pi(x, y) = (conj(x) gx1, conj(y) gy1) with
// gx1 = xi^((q-1)/3), gy1 = xi^((q-1)/2); pi^2(x, y) = (x gx2, y gy2) with
// gx2 = xi^((q^2-1)/3), gy2 = xi^((q^2-1)/2) = -1 (all Montgomery, R = 2^256)
__device__ __forceinline__ Fq fq_from_u64(uint64_t w0, uint64_t w1, uint64_t w2, uint64_t w3)
{
    Fq r;
    const uint64_t w[4] = {w0, w1, w2, w3};
#pragma unroll
    for (int i = 0; i < 4; ++i) {
        r.v[2 * i] = uint32_t(w[i]);
        r.v[2 * i + 1] = uint32_t(w[i] >> 32);
    }
    return r;
}
__device__ __forceinline__ Fq2 frob_gx1()
{
    return {fq_from_u64(0xb5773b104563ab30ull, 0x347f91c8a9aa6454ull, 0x7a007127242e0991ull,
                        0x1956bcd8118214ecull),
            fq_from_u64(0x6e849f1ea0aa4757ull, 0xaa1c7b6d89f89141ull, 0xb6e713cdfae0ca3aull,
                        0x26694fbb4e82ebc3ull)};
}
__device__ __forceinline__ Fq2 frob_gy1()
{
    return {fq_from_u64(0xe4bbdd0c2936b629ull, 0xbb30f162e133bacbull, 0x31a9d1b6f9645366ull,
                        0x253570bea500f8ddull),
            fq_from_u64(0xa1d77ce45ffe77c7ull, 0x07affd117826d1dbull, 0x6d16bd27bb7edc6bull,
                        0x2c87200285defeccull)};
}
__device__ __forceinline__ Fq frob_gx2()
{
    return fq_from_u64(0x3350c88e13e80b9cull, 0x7dce557cdb5e56b9ull, 0x6001b4b8b615564aull,
                       0x2682e617020217e0ull);
}

// E = (q^2 + 1) k (q^4 - q^2 + 1) / r, k = 2z(6z^2 + 3z + 1): 1458 bits
constexpr int kFinalExpWords = 23;
__constant__ const uint64_t kFinalExp[kFinalExpWords] = {
    0xd6c08a23dc23c528ull, 0x8ed5c03899fb6979ull, 0x187e5473cb82d214ull, 0x8c7064b37ae3153full,
    0xbdc6c32436e64b50ull, 0x4f3af528bbd1d49cull, 0xf0df440eaea08563ull, 0x24a265eec7377203ull,
    0x0db2a8cde71e9e84ull, 0xd9f7471d95e4d462ull, 0x188d608e076e2860ull, 0xe423711720687169ull,
    0x3fcfd06577665e73ull, 0x9b14073211496f79ull, 0x6c7e4e2444dcfebdull, 0xb57bcf7f0afba769ull,
    0xff5f7a0bb44be320ull, 0xe923f03ab1100164ull, 0xd93136646b4d81ebull, 0x1cf27bc8b3f4b0a9ull,
    0x06d165820287b280ull, 0x0db1120bab2f06a5ull, 0x0003b3d6150ca882ull};

__device__ inline Fq12 final_exponentiation(const Fq12 &f)
{
    const Fq12 g = conj(f) * inverse(f); // f^(q^6 - 1)
    Fq12 acc = fq12_one();
    bool started = false;
    for (int w = kFinalExpWords - 1; w >= 0; --w) {
        const uint64_t e = kFinalExp[w];
        for (int b = 63; b >= 0; --b) {
            if (started) acc = sqr(acc);
            if ((e >> b) & 1ull) {
                acc = started ? acc * g : g;
                started = true;
            }
        }
    }
    return acc;
}

// ---------------------------------------------------------------------------
// Miller loop pieces
// ---------------------------------------------------------------------------

// One line of a Miller loop on the twist: slope lam and c = lam xT - yT.
struct AteLine {
    Fq2 lam, c;
};

// The line through T and itself (tangent), T <- 2T; T affine, not infinity
__device__ __forceinline__ AteLine ate_double(Affine<Fq2> &t)
{
    const Fq2 xx = sqr(t.x);
    const Fq2 lam = (xx + dbl(xx)) * inverse(dbl(t.y));
    const AteLine l{lam, lam * t.x - t.y};
    const Fq2 x3 = sqr(lam) - dbl(t.x);
    t.y = lam * (t.x - x3) - t.y;
    t.x = x3;
    return l;
}

// The line through T and Q, T <- T + Q
__device__ __forceinline__ AteLine ate_add(Affine<Fq2> &t, const Affine<Fq2> &q)
{
    const Fq2 lam = (q.y - t.y) * inverse(q.x - t.x);
    const AteLine l{lam, lam * t.x - t.y};
    const Fq2 x3 = sqr(lam) - t.x - q.x;
    t.y = lam * (t.x - x3) - t.y;
    t.x = x3;
    return l;
}

__device__ __forceinline__ Affine<Fq2> twist_frobenius(const Affine<Fq2> &q)
{
    return {conj(q.x) * frob_gx1(), conj(q.y) * frob_gy1()};
}

// -pi^2(Q): (x gx2, -y gy2) = (x gx2, y) since gy2 = -1
__device__ __forceinline__ Affine<Fq2> twist_neg_frobenius2(const Affine<Fq2> &q)
{
    return {mul_fq(q.x, frob_gx2()), q.y};
}

// The kAteLines lines of the Miller loop of Q, in loop order (Q not infinity).
__device__ inline void ate_lines(const Affine<Fq2> &q, AteLine *out)
{
    Affine<Fq2> t = q;
    int s = 0;
    for (int i = kAteTopBit - 1; i >= 0; --i) {
        out[s++] = ate_double(t);
        if (ate_bit(i)) out[s++] = ate_add(t, q);
    }
    out[s++] = ate_add(t, twist_frobenius(q));
    Affine<Fq2> t2 = t;
    out[s++] = ate_add(t2, twist_neg_frobenius2(q));
}

__device__ __forceinline__ Fq12 apply_line(const Fq12 &f, const AteLine &l, const Affine<Fq> &p)
{
    return mul_by_line(f, p.y, neg(mul_fq(l.lam, p.x)), l.c);
}

} // namespace nkr
