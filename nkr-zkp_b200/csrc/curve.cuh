// BN254 G1 (y^2 = x^3 + 3 over Fq) and G2 (the sextic twist over Fq2), a = 0.
//
// Storage forms:
//   Affine<F>  {x, y}; infinity uses libff's to_affine_coordinates encoding
//              (x = 0, y = 1), which is not on either curve.  Byte image equals
//              the first 2/3 of a libff alt_bn128_G1 / G2 (X, Y) with Z = 1.
//   Xyzz<F>    {X, Y, ZZ, ZZZ} with x = X/ZZ, y = Y/ZZZ; infinity <=> ZZ = 0.
//              Bucket accumulators use it: mixed addition costs 8M + 2S.
//
// Every addition handles the equal-x cases (P == Q doubles, P == -Q gives
// infinity).  The reference CUDA bucket add assumes distinct points
// (operators/cuda/include/curves/xyzz_t.cuh:431-469, used under WRONG_FOR_SPEED
// in msm/msm_kernel.cuh:9,51-55); this file does not take that shortcut.
#pragma once

#include "field.cuh"

namespace nkr {

template <class F>
struct Affine {
    F x, y;
    __device__ __forceinline__ static Affine inf() { return {F::zero(), F::one()}; }
    __device__ __forceinline__ bool is_inf() const { return x.is_zero() && y == F::one(); }
};

template <class F>
struct Xyzz {
    F x, y, zz, zzz;
    __device__ __forceinline__ static Xyzz inf() { return {F::zero(), F::one(), F::zero(), F::zero()}; }
    __device__ __forceinline__ bool is_inf() const { return zz.is_zero(); }
};

using G1Affine = Affine<Fq>;
using G2Affine = Affine<Fq2>;
using G1Xyzz = Xyzz<Fq>;
using G2Xyzz = Xyzz<Fq2>;

template <class F>
__device__ __forceinline__ F times3(const F &a)
{
    return dbl(a) + a;
}

// 2 * P for affine P (mdbl-2008-s-1); P not infinity
template <class F>
__device__ __forceinline__ Xyzz<F> xyzz_from_affine_dbl(const Affine<F> &p)
{
    if (p.y.is_zero()) return Xyzz<F>::inf();
    const F u = dbl(p.y);
    const F v = sqr(u);
    const F w = u * v;
    const F s = p.x * v;
    const F m = times3(sqr(p.x));
    Xyzz<F> r;
    r.x = sqr(m) - dbl(s);
    r.y = m * (s - r.x) - w * p.y;
    r.zz = v;
    r.zzz = w;
    return r;
}

// x = a b, y = c d.  Fields with a paired product (field52.cuh) overload this so
// the two independent products share one call and interleave their chains.
template <class F>
__device__ __forceinline__ void mul2(const F &a, const F &b, const F &c, const F &d, F &x, F &y)
{
    x = a * b;
    y = c * d;
}

// 2 * P (dbl-2008-s-1): 6M + 3S, as four independent pairs and one single
// product where the field has a paired product
template <class F>
__device__ __forceinline__ Xyzz<F> xyzz_dbl(const Xyzz<F> &p)
{
    if (p.is_inf() || p.y.is_zero()) return Xyzz<F>::inf();
    const F u = dbl(p.y);
    Xyzz<F> r;
    if constexpr (HasPairedMul<F>::value) {
        F v, xx, w, s, my, wy;
        mul2(u, u, p.x, p.x, v, xx);
        mul2(u, v, p.x, v, w, s);
        mul2(v, p.zz, w, p.zzz, r.zz, r.zzz);
        const F m = times3(xx);
        r.x = sqr(m) - dbl(s);
        mul2(m, s - r.x, w, p.y, my, wy);
        r.y = my - wy;
    } else {
        const F v = sqr(u);
        const F w = u * v;
        const F s = p.x * v;
        const F m = times3(sqr(p.x));
        r.x = sqr(m) - dbl(s);
        r.y = m * (s - r.x) - w * p.y;
        r.zz = v * p.zz;
        r.zzz = w * p.zzz;
    }
    return r;
}

// acc + q for affine q (madd-2008-s): 8M + 2S, as five independent pairs where
// the field has a paired product; q may be infinity
template <class F>
__device__ __forceinline__ Xyzz<F> xyzz_add_affine(const Xyzz<F> &acc, const Affine<F> &q)
{
    if (q.is_inf()) return acc;
    if (acc.is_inf()) return {q.x, q.y, F::one(), F::one()};
    if constexpr (HasPairedMul<F>::value) {
        F u2, s2;
        mul2(q.x, acc.zz, q.y, acc.zzz, u2, s2);
        const F p = u2 - acc.x;
        const F r = s2 - acc.y;
        if (p.is_zero()) {
            if (r.is_zero()) return xyzz_from_affine_dbl(q);
            return Xyzz<F>::inf();
        }
        F pp, rr, ppp, qq, y1ppp, ry;
        mul2(p, p, r, r, pp, rr);
        mul2(p, pp, acc.x, pp, ppp, qq);
        Xyzz<F> o;
        mul2(acc.zzz, ppp, acc.y, ppp, o.zzz, y1ppp);
        o.x = rr - ppp - dbl(qq);
        mul2(r, qq - o.x, acc.zz, pp, ry, o.zz);
        o.y = ry - y1ppp;
        return o;
    } else {
        const F u2 = q.x * acc.zz;
        const F s2 = q.y * acc.zzz;
        const F p = u2 - acc.x;
        const F r = s2 - acc.y;
        if (p.is_zero()) {
            if (r.is_zero()) return xyzz_from_affine_dbl(q);
            return Xyzz<F>::inf();
        }
        const F pp = sqr(p);
        const F ppp = p * pp;
        const F qq = acc.x * pp;
        Xyzz<F> o;
        o.x = sqr(r) - ppp - dbl(qq);
        o.y = r * (qq - o.x) - acc.y * ppp;
        o.zz = acc.zz * pp;
        o.zzz = acc.zzz * ppp;
        return o;
    }
}

// a + b (add-2008-s): 12M + 2S, as seven independent pairs where the field has a
// paired product
template <class F>
__device__ __forceinline__ Xyzz<F> xyzz_add(const Xyzz<F> &a, const Xyzz<F> &b)
{
    if (a.is_inf()) return b;
    if (b.is_inf()) return a;
    if constexpr (HasPairedMul<F>::value) {
        F u1, u2, s1, s2;
        mul2(a.x, b.zz, b.x, a.zz, u1, u2);
        mul2(a.y, b.zzz, b.y, a.zzz, s1, s2);
        const F p = u2 - u1;
        const F r = s2 - s1;
        if (p.is_zero()) {
            if (r.is_zero()) return xyzz_dbl(a);
            return Xyzz<F>::inf();
        }
        F pp, rr, ppp, qq, zz_ab, zzz_ab, ry, s1ppp;
        mul2(p, p, r, r, pp, rr);
        mul2(p, pp, u1, pp, ppp, qq);
        mul2(a.zz, b.zz, a.zzz, b.zzz, zz_ab, zzz_ab);
        Xyzz<F> o;
        o.x = rr - ppp - dbl(qq);
        mul2(r, qq - o.x, s1, ppp, ry, s1ppp);
        o.y = ry - s1ppp;
        mul2(zz_ab, pp, zzz_ab, ppp, o.zz, o.zzz);
        return o;
    } else {
        const F u1 = a.x * b.zz;
        const F u2 = b.x * a.zz;
        const F s1 = a.y * b.zzz;
        const F s2 = b.y * a.zzz;
        const F p = u2 - u1;
        const F r = s2 - s1;
        if (p.is_zero()) {
            if (r.is_zero()) return xyzz_dbl(a);
            return Xyzz<F>::inf();
        }
        const F pp = sqr(p);
        const F ppp = p * pp;
        const F qq = u1 * pp;
        Xyzz<F> o;
        o.x = sqr(r) - ppp - dbl(qq);
        o.y = r * (qq - o.x) - s1 * ppp;
        o.zz = a.zz * b.zz * pp;
        o.zzz = a.zzz * b.zzz * ppp;
        return o;
    }
}

template <class F>
__device__ __forceinline__ Affine<F> affine_neg(const Affine<F> &p)
{
    if (p.is_inf()) return p;
    return {p.x, neg(p.y)};
}

template <class F>
__device__ __forceinline__ Xyzz<F> xyzz_neg(const Xyzz<F> &p)
{
    return {p.x, neg(p.y), p.zz, p.zzz};
}

// XYZZ -> affine with one field inversion
template <class F>
__device__ inline Affine<F> xyzz_to_affine(const Xyzz<F> &p)
{
    if (p.is_inf()) return Affine<F>::inf();
    const F t = inverse(p.zz * p.zzz); // 1 / (ZZ ZZZ)
    const F izz = t * p.zzz;            // 1 / ZZ
    const F izzz = t * p.zz;            // 1 / ZZZ
    return {p.x * izz, p.y * izzz};
}

// k * P for a canonical 256-bit scalar (8 limbs), double-and-add from the top
template <class F>
__device__ inline Xyzz<F> xyzz_mul_canon(const Affine<F> &p, const uint32_t *k)
{
    Xyzz<F> acc = Xyzz<F>::inf();
    for (int i = 255; i >= 0; --i) {
        acc = xyzz_dbl(acc);
        if ((k[i >> 5] >> (i & 31)) & 1) acc = xyzz_add_affine(acc, p);
    }
    return acc;
}

} // namespace nkr
