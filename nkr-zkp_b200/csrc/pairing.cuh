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
// exponentiation, so the value after it equals libff's); a per-call point runs
// in homogeneous coordinates with Fq2-scaled lines (no inversion per step).
//
// Final exponentiation: f^((q^6 - 1)(q^2 + 1) k (q^4 - q^2 + 1)/r) with
// k = 2z(6z^2 + 3z + 1): libff's last chunk (Fuentes-Castaneda et al.) computes
// this multiple of the exact hard-part exponent, and GT values must match its.
// Here the easy part is conj(f) / f times its q^2-Frobenius, and the hard part
// libff's addition chain (three exponentiations by -z, Frobenius maps).
#pragma once

#include "curve.cuh"

// The Fq12-level operations are compiled out of line: inlined, one verification
// is a single function of several hundred thousand instructions (ptxas runs for
// minutes and the frame spills kilobytes); out of line, each body exists once.
#define NKR_PAIR_FN inline __noinline__

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

__device__ NKR_PAIR_FN Fq12 operator*(const Fq12 &a, const Fq12 &b)
{
    const Fq6 t0 = a.c0 * b.c0, t1 = a.c1 * b.c1;
    return {t0 + mul_v(t1), (a.c0 + a.c1) * (b.c0 + b.c1) - t0 - t1};
}

// (a0 + a1 w)^2 = (a0 + a1)(a0 + v a1) - t - v t + 2 t w, t = a0 a1
__device__ NKR_PAIR_FN Fq12 sqr(const Fq12 &a)
{
    const Fq6 t = a.c0 * a.c1;
    return {(a.c0 + a.c1) * (a.c0 + mul_v(a.c1)) - t - mul_v(t), t + t};
}

__device__ __forceinline__ Fq12 conj(const Fq12 &a) { return {a.c0, neg(a.c1)}; }

__device__ NKR_PAIR_FN Fq12 inverse(const Fq12 &a)
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
__device__ NKR_PAIR_FN Fq12 mul_by_line(const Fq12 &f, const Fq &yP, const Fq2 &a, const Fq2 &b)
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

// Frobenius maps x -> x^(q^k), k = 1, 2, 3.  The coefficient of v^i w^j is that of
// w^m, m = 2i + j (w^2 = v), and (a w^m)^(q^k) = conj^k(a) xi^(m (q^k - 1)/6) w^m;
// kFrobGamma[(k - 1) * 5 + m - 1] = xi^(m (q^k - 1)/6) (Fq2, Montgomery limbs).
__constant__ const uint64_t kFrobGamma[15][2][4] = {
    {{0xaf9ba69633144907ull, 0xca6b1d7387afb78aull, 0x11bded5ef08a2087ull, 0x02f34d751a1f3a7cull}, {0xa222ae234c492d72ull, 0xd00f02a4565de15bull, 0xdc2ff3a253dfc926ull, 0x10a75716b3899551ull}}, // k = 1, m = 1
    {{0xb5773b104563ab30ull, 0x347f91c8a9aa6454ull, 0x7a007127242e0991ull, 0x1956bcd8118214ecull}, {0x6e849f1ea0aa4757ull, 0xaa1c7b6d89f89141ull, 0xb6e713cdfae0ca3aull, 0x26694fbb4e82ebc3ull}}, // k = 1, m = 2
    {{0xe4bbdd0c2936b629ull, 0xbb30f162e133bacbull, 0x31a9d1b6f9645366ull, 0x253570bea500f8ddull}, {0xa1d77ce45ffe77c7ull, 0x07affd117826d1dbull, 0x6d16bd27bb7edc6bull, 0x2c87200285defeccull}}, // k = 1, m = 3
    {{0x7361d77f843abe92ull, 0xa5bb2bd3273411fbull, 0x9c941f314b3e2399ull, 0x15df9cddbb9fd3ecull}, {0x5dddfd154bd8c949ull, 0x62cb29a5a4445b60ull, 0x37bc870a0c7dd2b9ull, 0x24830a9d3171f0fdull}}, // k = 1, m = 4
    {{0xc970692f41690fe7ull, 0xe240342127694b0bull, 0x32bee66b83c459e8ull, 0x12aabced0ab08841ull}, {0x0d485d2340aebfa9ull, 0x05193418ab2fcc57ull, 0xd3b0a40b8a4910f5ull, 0x2f21ebb535d2925aull}}, // k = 1, m = 5
    {{0xca8d800500fa1bf2ull, 0xf0c5d61468b39769ull, 0x0e201271ad0d4418ull, 0x04290f65bad856e6ull}, {0x0000000000000000ull, 0x0000000000000000ull, 0x0000000000000000ull, 0x0000000000000000ull}}, // k = 2, m = 1
    {{0x3350c88e13e80b9cull, 0x7dce557cdb5e56b9ull, 0x6001b4b8b615564aull, 0x2682e617020217e0ull}, {0x0000000000000000ull, 0x0000000000000000ull, 0x0000000000000000ull, 0x0000000000000000ull}}, // k = 2, m = 2
    {{0x68c3488912edefaaull, 0x8d087f6872aabf4full, 0x51e1a24709081231ull, 0x2259d6b14729c0faull}, {0x0000000000000000ull, 0x0000000000000000ull, 0x0000000000000000ull, 0x0000000000000000ull}}, // k = 2, m = 3
    {{0x71930c11d782e155ull, 0xa6bb947cffbe3323ull, 0xaa303344d4741444ull, 0x2c3b3f0d26594943ull}, {0x0000000000000000ull, 0x0000000000000000ull, 0x0000000000000000ull, 0x0000000000000000ull}}, // k = 2, m = 4
    {{0x08cfc388c494f1abull, 0x19b315148d1373d4ull, 0x584e90fdcb6c0213ull, 0x09e1685bdf2f8849ull}, {0x0000000000000000ull, 0x0000000000000000ull, 0x0000000000000000ull, 0x0000000000000000ull}}, // k = 2, m = 5
    {{0x365316184e46d97dull, 0x0af7129ed4c96d9full, 0x659da72fca1009b5ull, 0x08116d8983a20d23ull}, {0xb1df4af7c39c1939ull, 0x3d9f02878a73bf7full, 0x9b2220928caf0ae0ull, 0x26684515eff054a6ull}}, // k = 3, m = 1
    {{0xc9af22f716ad6badull, 0xb311782a4aa662b2ull, 0x19eeaf64e248c7f4ull, 0x20273e77e3439f82ull}, {0xacc02860f7ce93acull, 0x3933d5817ba76b4cull, 0x69e6188b446c8467ull, 0x0a46036d4417cc55ull}}, // k = 3, m = 2
    {{0x5764af0aaf46471eull, 0xdc50792e873e0fc1ull, 0x86a673ff881d04f6ull, 0x0b2eddb43c30a74cull}, {0x9a490f32787e8580ull, 0x8fd16d7ff04af8b1ull, 0x4b39888ec6027bf2ull, 0x03dd2e705b52a15dull}}, // k = 3, m = 3
    {{0x448a93a57b6762dfull, 0xbfd62df528fdeadfull, 0xd858f5d00e9bd47aull, 0x06b03d4d3476ec58ull}, {0x2b19daf4bcc936d1ull, 0xa1a54e7a56f4299full, 0xb533eee05adeaef1ull, 0x170c812b84dda0b2ull}}, // k = 3, m = 4
    {{0xe0bc4b2275cf559full, 0xc238b945c154e60full, 0x803982a5929a7d5eull, 0x15ce052df7e4a37eull}, {0x2d28efbdbf3799a7ull, 0x9b097e3c1ad60773ull, 0x982d4113af4a535bull, 0x24e18991e3056063ull}}, // k = 3, m = 5
};

__device__ __forceinline__ Fq2 frob_gamma(int k, int m)
{
    const uint64_t(*g)[4] = kFrobGamma[(k - 1) * 5 + m - 1];
    return {fq_from_u64(g[0][0], g[0][1], g[0][2], g[0][3]), fq_from_u64(g[1][0], g[1][1], g[1][2], g[1][3])};
}

__device__ __forceinline__ Fq2 frob_coeff(const Fq2 &a, int k, int m)
{
    const Fq2 b = (k & 1) ? conj(a) : a;
    return m ? b * frob_gamma(k, m) : b;
}

__device__ NKR_PAIR_FN Fq12 frobenius(const Fq12 &x, int k)
{
    return {{frob_coeff(x.c0.c0, k, 0), frob_coeff(x.c0.c1, k, 2), frob_coeff(x.c0.c2, k, 4)},
            {frob_coeff(x.c1.c0, k, 1), frob_coeff(x.c1.c1, k, 3), frob_coeff(x.c1.c2, k, 5)}};
}

// x^(-z) for x in the cyclotomic subgroup (inverse = conjugate), z = 0x44e992b44a6909f1
constexpr uint64_t kZ = 0x44e992b44a6909f1ull;
__device__ NKR_PAIR_FN Fq12 exp_by_neg_z(const Fq12 &x)
{
    Fq12 r = x;
    for (int b = 61; b >= 0; --b) { // bit 62, the top one, is r = x
        r = sqr(r);
        if ((kZ >> b) & 1ull) r = r * x;
    }
    return conj(r);
}

// f^((q^6 - 1)(q^2 + 1)) (the easy part), then libff's last chunk
// (alt_bn128_pairing.cpp:152-224, Fuentes-Castaneda et al.): the same addition
// chain, so the result is libff's GT value: elt^(2z(6z^2 + 3z + 1)(q^4 - q^2 + 1)/r)
__device__ NKR_PAIR_FN Fq12 final_exponentiation(const Fq12 &f)
{
    const Fq12 c = conj(f) * inverse(f);
    const Fq12 elt = frobenius(c, 2) * c;
    const Fq12 A = exp_by_neg_z(elt);
    const Fq12 B = sqr(A);
    const Fq12 C = sqr(B);
    const Fq12 D = C * B;
    const Fq12 E = exp_by_neg_z(D);
    const Fq12 F = sqr(E);
    const Fq12 G = exp_by_neg_z(F);
    const Fq12 K = conj(G) * E * conj(D); // 12z^3 + 6z^2 + 6z
    const Fq12 L = K * B;                 // 12z^3 + 6z^2 + 4z
    const Fq12 N = K * E * elt;           // 12z^3 + 12z^2 + 6z + 1
    const Fq12 R = frobenius(K, 2) * (frobenius(L, 1) * N);
    return frobenius(conj(elt) * L, 3) * R;
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

// The Miller loop of a point Q that changes per call (a proof's B) runs T in
// homogeneous coordinates (x = X/Z, y = Y/Z) so that no step inverts.  Its lines
// are the affine ones times an Fq2 factor (2YZ^2 for a doubling, xQ Z - X for an
// addition), which the final exponentiation removes: line = c0 + a w + b v w,
// c0 already multiplied by yP.
struct G2Proj {
    Fq2 x, y, z;
};
struct ProjLine {
    Fq2 c0, a, b;
};

// tangent at T, T <- 2T: with A = 3X^2, B = 2YZ (slope A/B),
// 2T = ((A^2 Z - 2X B^2) B, A (3X B^2 - A^2 Z) - Y B^3, B^3 Z)
__device__ NKR_PAIR_FN ProjLine proj_double(G2Proj &t, const Affine<Fq> &p)
{
    const Fq2 xx = sqr(t.x);
    const Fq2 a = xx + dbl(xx);
    const Fq2 b = dbl(t.y * t.z);
    const Fq2 b2 = sqr(b), b3 = b2 * b;
    const Fq2 a2z = sqr(a) * t.z;
    const Fq2 xb2 = t.x * b2;
    const ProjLine l{mul_fq(b * t.z, p.y), neg(mul_fq(a * t.z, p.x)), a * t.x - t.y * b};
    const Fq2 x3 = (a2z - dbl(xb2)) * b;
    const Fq2 y3 = a * (xb2 + dbl(xb2) - a2z) - t.y * b3;
    t = {x3, y3, b3 * t.z};
    return l;
}

// line through T and affine Q, T <- T + Q: with N = yQ Z - Y, D = xQ Z - X (slope N/D),
// T + Q = ((N^2 Z - (X + xQ Z) D^2) D, N ((2X + xQ Z) D^2 - N^2 Z) - Y D^3, D^3 Z)
__device__ NKR_PAIR_FN ProjLine proj_add(G2Proj &t, const Affine<Fq2> &q, const Affine<Fq> &p)
{
    const Fq2 n = q.y * t.z - t.y;
    const Fq2 xqz = q.x * t.z;
    const Fq2 d = xqz - t.x;
    const Fq2 d2 = sqr(d), d3 = d2 * d;
    const Fq2 n2z = sqr(n) * t.z;
    const ProjLine l{mul_fq(d, p.y), neg(mul_fq(n, p.x)), n * q.x - q.y * d};
    const Fq2 x3 = (n2z - (t.x + xqz) * d2) * d;
    const Fq2 y3 = n * ((dbl(t.x) + xqz) * d2 - n2z) - t.y * d3;
    t = {x3, y3, d3 * t.z};
    return l;
}

__device__ __forceinline__ Fq6 mul_by_fq2(const Fq6 &f, const Fq2 &s) { return {f.c0 * s, f.c1 * s, f.c2 * s}; }

__device__ NKR_PAIR_FN Fq12 apply_proj_line(const Fq12 &f, const ProjLine &l)
{
    return {mul_by_fq2(f.c0, l.c0) + mul_v(mul_by_ab(f.c1, l.a, l.b)),
            mul_by_ab(f.c0, l.a, l.b) + mul_by_fq2(f.c1, l.c0)};
}

} // namespace nkr
