// Pippenger MSM kernels (design notes in msm.cuh).
//
// The curve arithmetic here chains many field products per thread, so the
// product is compiled out of line (one body per kernel) to keep the hot loops
// resident in the instruction cache.
#define NKR_FIELD_MUL_OUTLINE 1
#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <type_traits>

#include "field52.cuh"
#include "msm.cuh"
#include "pairing.cuh" // twist_frobenius: the endomorphism psi of G2
#include "scan.cuh"

namespace nkr {

// --------------------------------------------------------------------------
// lane pairs.  The bucket reduction levels are chains of dependent additions
// run by few threads, so there each addition is computed by two lanes: the
// curve formulas issue their products in independent pairs (mul2), and a lane
// pair computes one product of each pair and exchanges the results.  Everything
// else is computed by both lanes alike, so a pair stays converged.
// --------------------------------------------------------------------------
template <class B>
struct Pair2 : B {
    using base = B;
    Pair2() = default;
    __device__ __forceinline__ Pair2(const B &b) : B(b) {}
    __device__ __forceinline__ static Pair2 zero() { return B::zero(); }
    __device__ __forceinline__ static Pair2 one() { return B::one(); }
};
template <class B>
__device__ __forceinline__ Pair2<B> operator+(const Pair2<B> &a, const Pair2<B> &b)
{
    return static_cast<const B &>(a) + static_cast<const B &>(b);
}
template <class B>
__device__ __forceinline__ Pair2<B> operator-(const Pair2<B> &a, const Pair2<B> &b)
{
    return static_cast<const B &>(a) - static_cast<const B &>(b);
}
template <class B>
__device__ __forceinline__ Pair2<B> operator*(const Pair2<B> &a, const Pair2<B> &b)
{
    return static_cast<const B &>(a) * static_cast<const B &>(b);
}
template <class B>
__device__ __forceinline__ Pair2<B> dbl(const Pair2<B> &a) { return dbl(static_cast<const B &>(a)); }
template <class B>
__device__ __forceinline__ Pair2<B> sqr(const Pair2<B> &a) { return sqr(static_cast<const B &>(a)); }

__device__ __forceinline__ Fq52 shfl_xor1(unsigned mask, const Fq52 &a)
{
    Fq52 r;
#pragma unroll
    for (int j = 0; j < 5; ++j) r.l[j] = __shfl_xor_sync(mask, a.l[j], 1);
    return r;
}
__device__ __forceinline__ Fq52L shfl_xor1(unsigned mask, const Fq52L &a)
{
    Fq52L r;
#pragma unroll
    for (int j = 0; j < 5; ++j) r.l[j] = __shfl_xor_sync(mask, a.l[j], 1);
    return r;
}
__device__ __forceinline__ Fq2 shfl_xor1(unsigned mask, const Fq2 &a)
{
    Fq2 r;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
        r.c0.v[j] = __shfl_xor_sync(mask, a.c0.v[j], 1);
        r.c1.v[j] = __shfl_xor_sync(mask, a.c1.v[j], 1);
    }
    return r;
}

// the pair of lanes (2j, 2j + 1) of the calling lane
__device__ __forceinline__ unsigned pair_mask() { return 3u << ((threadIdx.x & 31u) & 30u); }

// x = a b, y = c d: the even lane computes a b, the odd lane c d
template <class B>
__device__ __forceinline__ void mul2(const Pair2<B> &a, const Pair2<B> &b, const Pair2<B> &c,
                                     const Pair2<B> &d, Pair2<B> &x, Pair2<B> &y)
{
    const bool odd = threadIdx.x & 1u;
    const B m = static_cast<const B &>(odd ? c : a) * static_cast<const B &>(odd ? d : b);
    const B o = shfl_xor1(pair_mask(), m);
    x = odd ? o : m;
    y = odd ? m : o;
}
template <class B>
struct HasPairedMul<Pair2<B>> {
    static constexpr bool value = true;
};

namespace {

// --------------------------------------------------------------------------
// signed digits
// --------------------------------------------------------------------------

// bits [off, off + c) of a canonical 256-bit integer (c <= 24)
__device__ __forceinline__ uint32_t window_bits(const Fr &s, int off, int c)
{
    const int limb = off >> 5, sh = off & 31;
    if (limb >= 8) return 0;
    uint64_t w = s.v[limb];
    if (limb + 1 < 8) w |= uint64_t(s.v[limb + 1]) << 32;
    return uint32_t(w >> sh) & ((1u << c) - 1u);
}

// Walks the signed digits of one scalar; calls f(k, has, bucket_in_set, negative)
// for every window.  Digits: v = bits + carry; v > 2^(c-1) -> v - 2^c.
template <class Fn>
__device__ __forceinline__ void for_each_digit(const Fr &s, int c, int W, Fn &&f)
{
    uint32_t carry = 0;
    const uint32_t half = 1u << (c - 1), full = 1u << c;
    for (int k = 0; k < W; ++k) {
        const uint32_t v = window_bits(s, k * c, c) + carry;
        bool has, negd = false;
        uint32_t mag;
        if (v > half) {
            carry = 1;
            mag = full - v;
            negd = mag != 0;
            has = mag != 0;
        } else {
            carry = 0;
            mag = v;
            has = v != 0;
        }
        f(k, has, mag - 1u, negd);
    }
}

// Lanes of this warp whose scalar equals this lane's (all eight words): equal
// scalars have equal digits, so one lane per group updates the bucket counters
// for the whole group.  Matching once per scalar replaces a match per digit
// (repeated scalars are what makes buckets hot in sparse witnesses; distinct
// uniform scalars form groups of one).
__device__ __forceinline__ unsigned equal_scalar_lanes(unsigned mask, const Fr &s)
{
    unsigned peers = mask;
#pragma unroll
    for (int w = 0; w < 8; w += 2)
        peers &= __match_any_sync(mask, uint64_t(s.v[w]) | (uint64_t(s.v[w + 1]) << 32));
    return peers;
}

__global__ void k_digits_count(const Fr *__restrict__ scalars, const uint32_t *__restrict__ gather,
                               const uint32_t *__restrict__ class_of, uint64_t n, int c, int W,
                               bool folded, uint32_t B, Fr *__restrict__ canon,
                               uint32_t *__restrict__ counts)
{
    const uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    const bool live = i < n;
    Fr s = Fr::zero();
    if (live) {
        const uint64_t v = gather ? gather[i] : i;
        // a class member's scalar is added by the class path (zero: no digits here)
        if (!class_of || class_of[v] == kNoClass) s = from_mont(scalars[v]);
        canon[i] = s;
    }
    const int lane = threadIdx.x & 31;
    const unsigned act = __ballot_sync(0xffffffffu, live);
    if (!live) return;
    const unsigned peers = equal_scalar_lanes(act, s);
    if (lane != __ffs(peers) - 1) return;
    const uint32_t group = uint32_t(__popc(peers));
    for_each_digit(s, c, W, [&](int k, bool has, uint32_t b, bool) {
        if (has) atomicAdd(&counts[(folded ? 0u : uint32_t(k) * B) + b], group);
    });
}

__global__ void k_scatter(const Fr *__restrict__ canon, uint64_t n, int c, int W, bool folded,
                          uint32_t B, uint32_t *__restrict__ cursor, uint32_t *__restrict__ entries)
{
    const uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    const bool live = i < n;
    const int lane = threadIdx.x & 31;
    const unsigned act = __ballot_sync(0xffffffffu, live);
    if (!live) return;
    const Fr s = canon[i];
    const unsigned peers = equal_scalar_lanes(act, s);
    const int leader = __ffs(peers) - 1;
    const uint32_t group = uint32_t(__popc(peers));
    const uint32_t rank = __popc(peers & ((1u << lane) - 1u));
    for_each_digit(s, c, W, [&](int k, bool has, uint32_t b, bool negd) {
        // the group's lanes agree on every digit, so they take this branch together
        if (has) {
            const uint32_t bucket = (folded ? 0u : uint32_t(k) * B) + b;
            uint32_t base = 0;
            if (lane == leader) base = atomicAdd(&cursor[bucket], group);
            base = __shfl_sync(peers, base, leader);
            const uint32_t point = folded ? uint32_t(uint64_t(k) * n + i) : uint32_t(i);
            entries[base + rank] = point | (negd ? 0x80000000u : 0u);
        }
    });
}

// --------------------------------------------------------------------------
// storage vs compute.  G1 arithmetic runs on the FP64 pipe (Fq52, R' = 2^260):
// every G1 MSM buffer (bases, partials, buckets, reduction items) holds R'-domain
// values in the 8 x 32-bit layout of Fq, converted at entry (bases) and exit
// (result).  G2 arithmetic stays on the integer pipe (Fq2, R = 2^256): measured,
// its FP64 form (Fq2 products as three interleaved 52-bit products) needs all 255
// registers and ran 34% slower at 2^18 points; with the accumulator in shared
// memory as for G1 (254 registers, bases in R' from prepare, flushes leaving R')
// the level-1 kernel took 7.96 instead of 3.48 ms.  The same holds for the G2
// reduction levels alone, although they are latency bound (a 32-bit product is
// one long carry chain): in the FP64 form they spill 600 B per thread and took
// 1.81 instead of 1.53 ms at 2^18; with the three Karatsuba products of an Fq2
// product interleaved in one 32-bit call they took 1.66 ms, no faster.  Moving one
// Karatsuba product of every Fq2 product to the FP64 pipe ((16 x) y 2^-260 =
// x y 2^-256) relieves the integer multiply pipe but costs four doublings, limb
// conversions and spills at 255 registers: the G2 accumulation took 4.01 instead
// of 3.48 ms at 2^18.
// --------------------------------------------------------------------------

template <class F>
struct MsmArith;
template <>
struct MsmArith<Fq> {
    using type = Fq52L;
};
template <>
struct MsmArith<Fq2> {
    using type = Fq2;
};
template <class F>
using CF = typename MsmArith<F>::type;

// Compute type and shape of the bucket reduction levels (first level, block
// levels, final combination): latency-bound chains of dependent additions, with
// LANES lanes per item.  G2 computes in the lazily reduced Fq2 product (Fq2L,
// field.cuh), 128 items per block; an MSM alone (MsmAcc::lane_pairs) runs it on
// lane pairs (Pair2): at 2^18 points the block levels 1.21 -> 0.85 ms and the
// first level 0.36 -> 0.28 ms.  Inside a prove the G2 levels overlap the other
// MSMs' level-1 kernels, and there the pairs' 256-thread blocks, which take a
// whole SM's registers, cost more than they save (2^20 prove 19.09 vs 18.97 ms),
// so a prove keeps one lane per item.  G1 keeps one lane per item and 256 items
// per block: on lane pairs (128 items per block, the register budget of a
// 256-thread block) its block levels are shorter but its first level takes
// twice the buckets per pair (2^20 MSM 4.31 vs 4.25 ms; a 2^20 prove 19.16 ms).
template <class F>
struct ReduceBase {
    using type = CF<F>;
};
template <>
struct ReduceBase<Fq2> {
    using type = Fq2L;
};
template <class F, int LANES>
struct MsmReduceArith {
    using type = typename std::conditional<LANES == 2, Pair2<typename ReduceBase<F>::type>,
                                           typename ReduceBase<F>::type>::type;
    static constexpr int lanes = LANES;
    static constexpr int items = (LANES == 1 && sizeof(F) == sizeof(Fq)) ? 256 : 128;
    static constexpr int log2_items = items == 256 ? 8 : 7;
};
template <class C>
struct BaseOf {
    using type = C;
};
template <class B>
struct BaseOf<Pair2<B>> {
    using type = B;
};

// G1 buffers hold canonical values; the lazily reduced compute values are
// canonicalised on the way out
__device__ __forceinline__ Fq52L msm_in(const Fq &x) { return to52(x); }
__device__ __forceinline__ Fq msm_out(const Fq52L &x) { return from52(x.canon()); }
__device__ __forceinline__ Fq52L msm_enter(const Fq52L &x) { return r256_to_r260(x.canon()); }
__device__ __forceinline__ Fq52L msm_leave(const Fq52L &x) { return r260_to_r256(x.canon()); }
__device__ __forceinline__ Fq2 msm_in(const Fq2 &x) { return x; }
__device__ __forceinline__ Fq2 msm_out(const Fq2 &x) { return x; }
__device__ __forceinline__ Fq2 msm_enter(const Fq2 &x) { return x; }
__device__ __forceinline__ Fq2 msm_leave(const Fq2 &x) { return x; }

template <class F>
__device__ __forceinline__ Xyzz<CF<F>> ldx(const Xyzz<F> &s)
{
    return {msm_in(s.x), msm_in(s.y), msm_in(s.zz), msm_in(s.zzz)};
}

template <class C, class F>
__device__ __forceinline__ Xyzz<C> ldr(const Xyzz<F> &s)
{
    using B = typename BaseOf<C>::type;
    return {B(msm_in(s.x)), B(msm_in(s.y)), B(msm_in(s.zz)), B(msm_in(s.zzz))};
}

template <class C>
__device__ __forceinline__ auto stx(const Xyzz<C> &c) -> Xyzz<decltype(msm_out(c.x))>
{
    return {msm_out(c.x), msm_out(c.y), msm_out(c.zz), msm_out(c.zzz)};
}

template <class F>
__device__ __forceinline__ Affine<CF<F>> lda(const Affine<F> &s)
{
    return {msm_in(s.x), msm_in(s.y)};
}

// first index in a[0, n) with a[idx] > x (a nondecreasing)
__device__ __forceinline__ uint32_t upper_bound_u32(const uint32_t *a, uint32_t n, uint32_t x)
{
    uint32_t lo = 0, hi = n;
    while (lo < hi) {
        const uint32_t mid = (lo + hi) >> 1;
        if (a[mid] <= x)
            lo = mid + 1;
        else
            hi = mid;
    }
    return lo;
}

// --------------------------------------------------------------------------
// bucket accumulation
// --------------------------------------------------------------------------

// Pieces of a bucket at level 1: the bucket's entries [off_b, off_b+1) are cut
// by the fixed segments of K1 entries; a bucket inside one segment is complete,
// otherwise it has one piece per segment it touches.  Piece k of bucket b lives
// in partial slot 2 t (the segment's first run) or 2 t + 1 (its last run).
struct Pieces {
    uint32_t t0, count;
    __device__ __forceinline__ uint64_t slot(const uint32_t off_b, uint32_t k1, uint32_t k) const
    {
        if (k == 0) return off_b == t0 * k1 ? 2ull * t0 : 2ull * t0 + 1;
        return 2ull * (t0 + k);
    }
};

__device__ __forceinline__ Pieces bucket_pieces(const uint32_t *offsets, uint32_t b, uint32_t k1)
{
    const uint32_t lo = offsets[b], hi = offsets[b + 1];
    if (hi == lo) return {0, 0};
    const uint32_t t0 = lo / k1, t1 = (hi - 1) / k1;
    return {t0, t1 - t0 + 1};
}

// Groups of k2 pieces a bucket still has at a fix-up level whose inputs are
// spaced `stride` pieces apart (zero once the bucket is complete).
constexpr unsigned kFixupBlocks = 148 * 8; // grid cap of a fix-up level

// Buckets of at most kSmallPieces pieces are summed where they are consumed
// (k_reduce_first); only larger ones go through the fix-up levels.
constexpr uint32_t kSmallPieces = 16;

struct LoadLeaders {
    const uint32_t *offsets;
    uint32_t k1, stride, k2;
    __device__ __forceinline__ uint32_t operator()(uint64_t i) const
    {
        const Pieces pc = bucket_pieces(offsets, uint32_t(i), k1);
        if (pc.count <= kSmallPieces) return 0u;
        const uint32_t live = (pc.count + stride - 1) / stride;
        return live > 1 ? (live + k2 - 1) / k2 : 0u;
    }
};

// Level-1 accumulators live in shared memory.  Across the out-of-line product
// calls of a mixed addition the four accumulator coordinates were live in
// registers (G1: 40 of the 168 the 3-blocks-per-SM budget allows, with 100 B of
// spills per thread; G2: 64 of 232, 2 blocks per SM); kept in shared memory and
// loaded where a product needs them, G1 runs its 3-block budget without spills
// (1.4% faster at 2^20) and G2 fits 3 blocks per SM in 167 registers without
// spills (6% faster at 2^18).  Layout: structure of arrays, word w of thread i
// at w * BS + i, so a warp's accesses are conflict-free.
//
// G1: Fq52L coordinates (5 x 64-bit words, lazily reduced), R' domain throughout.
template <int BS>
struct SmXyzz52 {
    using point = Affine<Fq52L>;
    uint64_t *s; // the block's area + threadIdx.x; 20 words per thread
    __device__ __forceinline__ Fq52L ld(int f) const
    {
        Fq52L v;
#pragma unroll
        for (int j = 0; j < 5; ++j) v.l[j] = s[(f * 5 + j) * BS];
        return v;
    }
    __device__ __forceinline__ void st(int f, const Fq52L &v) const
    {
#pragma unroll
        for (int j = 0; j < 5; ++j) s[(f * 5 + j) * BS] = v.l[j];
    }
    __device__ __forceinline__ void set(const Xyzz<Fq52L> &a) const
    {
        st(0, a.x);
        st(1, a.y);
        st(2, a.zz);
        st(3, a.zzz);
    }
    __device__ __forceinline__ Xyzz<Fq> out() const { return stx(Xyzz<Fq52L>{ld(0), ld(1), ld(2), ld(3)}); }
    __device__ __forceinline__ static point load(const Affine<Fq> &p) { return lda(p); }
};

// G2: Fq2 coordinates (16 x 32-bit words), the library's Montgomery domain.
template <int BS>
struct SmXyzzFq2 {
    using point = Affine<Fq2>;
    uint32_t *s; // the block's area + threadIdx.x; 64 words per thread
    __device__ __forceinline__ Fq2 ld(int f) const
    {
        Fq2 v;
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            v.c0.v[j] = s[(f * 16 + j) * BS];
            v.c1.v[j] = s[(f * 16 + 8 + j) * BS];
        }
        return v;
    }
    __device__ __forceinline__ void st(int f, const Fq2 &v) const
    {
#pragma unroll
        for (int j = 0; j < 8; ++j) {
            s[(f * 16 + j) * BS] = v.c0.v[j];
            s[(f * 16 + 8 + j) * BS] = v.c1.v[j];
        }
    }
    __device__ __forceinline__ void set(const Xyzz<Fq2> &a) const
    {
        st(0, a.x);
        st(1, a.y);
        st(2, a.zz);
        st(3, a.zzz);
    }
    __device__ __forceinline__ Xyzz<Fq2> out() const { return {ld(0), ld(1), ld(2), ld(3)}; }
    __device__ __forceinline__ static point load(const Affine<Fq2> &p) { return p; }
};

// acc + q (madd-2008-s: 8M + 2S) on a shared-memory accumulator, q may be
// infinity; the products go in the pairs of xyzz_add_affine (G1's paired
// product)
template <class Acc, class C>
__device__ __forceinline__ void sm_add_affine(const Acc &a, const Affine<C> &q)
{
    if (q.is_inf()) return;
    const C zz = a.ld(2);
    if (zz.is_zero()) {
        a.set({q.x, q.y, C::one(), C::one()});
        return;
    }
    C u2, s2;
    mul2(q.x, zz, q.y, a.ld(3), u2, s2);
    const C p = u2 - a.ld(0);
    const C r = s2 - a.ld(1);
    if (p.is_zero()) {
        a.set(r.is_zero() ? xyzz_from_affine_dbl(q) : Xyzz<C>::inf());
        return;
    }
    C pp, rr, ppp, qq, y1ppp, ry, t;
    mul2(p, p, r, r, pp, rr);
    mul2(p, pp, a.ld(0), pp, ppp, qq);
    mul2(a.ld(3), ppp, a.ld(1), ppp, t, y1ppp);
    a.st(3, t);
    const C ox = rr - ppp - dbl(qq);
    a.st(0, ox);
    mul2(r, qq - ox, a.ld(2), pp, ry, t);
    a.st(2, t);
    a.st(1, ry - y1ppp);
}

// The same for G2, whose products are single calls: each product right before
// its first use keeps fewer values live (167 registers and no spills at the
// 3-block budget, against 104 B of spills in the paired order)
template <int BS>
__device__ __forceinline__ void sm_add_affine(const SmXyzzFq2<BS> &a, const Affine<Fq2> &q)
{
    if (q.is_inf()) return;
    const Fq2 zz = a.ld(2);
    if (zz.is_zero()) {
        a.set({q.x, q.y, Fq2::one(), Fq2::one()});
        return;
    }
    const Fq2 p = q.x * zz - a.ld(0);
    const Fq2 r = q.y * a.ld(3) - a.ld(1);
    if (p.is_zero()) {
        a.set(r.is_zero() ? xyzz_from_affine_dbl(q) : Xyzz<Fq2>::inf());
        return;
    }
    const Fq2 pp = sqr(p);
    const Fq2 ppp = p * pp;
    a.st(3, a.ld(3) * ppp);
    const Fq2 qq = a.ld(0) * pp;
    const Fq2 ox = sqr(r) - ppp - dbl(qq);
    a.st(0, ox);
    const Fq2 y1ppp = a.ld(1) * ppp;
    a.st(1, r * (qq - ox) - y1ppp);
    a.st(2, a.ld(2) * pp);
}

// Level 1: thread t sums the fixed segment [t K1, (t+1) K1) of the sorted
// entries, split into runs at bucket boundaries, so every lane of a warp does
// the same number of mixed additions whatever the bucket sizes.  A run that is
// a whole bucket is written to the bucket; the segment's first / last run, when
// its bucket continues outside the segment, goes to partial slot 2t / 2t + 1.
template <class Acc, class F>
__device__ __forceinline__ void acc_l1_body(const uint32_t *__restrict__ offsets,
                                            const uint32_t *__restrict__ entries,
                                            const Affine<F> *__restrict__ pts, uint32_t nb,
                                            uint32_t k1, Xyzz<F> *__restrict__ partials,
                                            Xyzz<F> *__restrict__ buckets, uint32_t t, const Acc &acc)
{
    using C = decltype(acc.ld(0));
    const uint32_t total = offsets[nb];
    const uint64_t beg64 = uint64_t(t) * k1;
    if (beg64 >= total) return;
    const uint32_t beg = uint32_t(beg64);
    const uint32_t end = min(beg + k1, total);
    uint32_t b = upper_bound_u32(offsets, nb + 1, beg) - 1; // offsets[b] <= beg < offsets[b + 1]
    uint32_t bstart = offsets[b], bend = offsets[b + 1];
    bool first = true;
    acc.set(Xyzz<C>::inf());
    // one flat loop with the same trip count in every lane keeps the additions
    // converged; the flush at a bucket boundary is a short divergent branch
    for (uint32_t j = beg; j < end; ++j) {
        if (j == bend) {
            if (bstart >= beg)
                buckets[b] = acc.out(); // the bucket started and ended inside the segment
            else
                partials[2ull * t] = acc.out(); // first run, bucket began in an earlier segment
            first = false;
            acc.set(Xyzz<C>::inf());
            // next nonempty bucket: usually adjacent, else search
            ++b;
            int steps = 0;
            while (offsets[b + 1] <= j && steps < 8) {
                ++b;
                ++steps;
            }
            if (offsets[b + 1] <= j) b = upper_bound_u32(offsets, nb + 1, j) - 1;
            bstart = offsets[b];
            bend = offsets[b + 1];
        }
        const uint32_t e = entries[j];
        typename Acc::point p = Acc::load(pts[e & 0x7fffffffu]);
        if (e >> 31) p = affine_neg(p);
        sm_add_affine(acc, p);
    }
    if (bstart >= beg && bend <= end)
        buckets[b] = acc.out();
    else
        partials[2ull * t + (first ? 0 : 1)] = acc.out();
}

// Level 1 kernels, 3 blocks of 128 threads per SM.  G1 (FP64 field, paired
// products passed by value): measured against the compiler's own register
// choice (184 registers, 2 blocks) and a 4-block budget (128 registers, 124 B of
// spills), the fastest from 2^16 to 2^20 points, uniform and sparse.  G2 (integer
// pipe): 167 registers without spills, against 232 at 2 blocks per SM before the
// accumulator moved to shared memory (a 4-block budget spills 232 B and is no
// faster).
__global__ void __launch_bounds__(128, 3) k_acc_l1_g1(const uint32_t *__restrict__ offsets,
                                                       const uint32_t *__restrict__ entries,
                                                       const Affine<Fq> *__restrict__ pts,
                                                       uint32_t nb, uint32_t k1,
                                                       Xyzz<Fq> *__restrict__ partials,
                                                       Xyzz<Fq> *__restrict__ buckets)
{
    __shared__ uint64_t sm[20 * 128];
    acc_l1_body(offsets, entries, pts, nb, k1, partials, buckets, blockIdx.x * blockDim.x + threadIdx.x,
                SmXyzz52<128>{sm + threadIdx.x});
}

__global__ void __launch_bounds__(128, 3) k_acc_l1_g2(const uint32_t *__restrict__ offsets,
                                                       const uint32_t *__restrict__ entries,
                                                       const Affine<Fq2> *__restrict__ pts,
                                                       uint32_t nb, uint32_t k1,
                                                       Xyzz<Fq2> *__restrict__ partials,
                                                       Xyzz<Fq2> *__restrict__ buckets)
{
    __shared__ uint32_t sm[64 * 128];
    acc_l1_body(offsets, entries, pts, nb, k1, partials, buckets, blockIdx.x * blockDim.x + threadIdx.x,
                SmXyzzFq2<128>{sm + threadIdx.x});
}

// Level 1 of several MSMs of one group in one launch (a batch's MSMs, any sizes):
// item i owns blocks [first_block, next item's first_block) of the grid.
template <class F>
struct AccItem {
    const uint32_t *offsets, *entries;
    const Affine<F> *pts;
    Xyzz<F> *partials, *buckets;
    uint32_t nb, k1, first_block;
};
static_assert(sizeof(AccItem<Fq>) <= kMsmAccItemBytes, "work-list item size");

// the work-list item of this block (binary search over the items' first blocks)
template <class F>
__device__ __forceinline__ AccItem<F> acc_list_item(const AccItem<F> *items, int n_items)
{
    int lo = 0, hi = n_items - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (items[mid].first_block <= blockIdx.x)
            lo = mid;
        else
            hi = mid - 1;
    }
    return items[lo];
}

__global__ void __launch_bounds__(128, 3) k_acc_l1_g1_list(const AccItem<Fq> *items, int n_items)
{
    __shared__ uint64_t sm[20 * 128];
    const AccItem<Fq> it = acc_list_item(items, n_items);
    acc_l1_body(it.offsets, it.entries, it.pts, it.nb, it.k1, it.partials, it.buckets,
                (blockIdx.x - it.first_block) * blockDim.x + threadIdx.x, SmXyzz52<128>{sm + threadIdx.x});
}

__global__ void __launch_bounds__(128, 3) k_acc_l1_g2_list(const AccItem<Fq2> *items, int n_items)
{
    __shared__ uint32_t sm[64 * 128];
    const AccItem<Fq2> it = acc_list_item(items, n_items);
    acc_l1_body(it.offsets, it.entries, it.pts, it.nb, it.k1, it.partials, it.buckets,
                (blockIdx.x - it.first_block) * blockDim.x + threadIdx.x, SmXyzzFq2<128>{sm + threadIdx.x});
}

// One group of k2 pieces (spaced `stride` pieces apart) of one bucket; the
// group's sum goes back into the group's first piece slot, or into the bucket
// when it was the bucket's last group.
template <class F>
__device__ __forceinline__ void acc_up_group(const uint32_t *__restrict__ offsets,
                                             const uint32_t *__restrict__ lead_off, uint32_t nb,
                                             uint32_t k1, Xyzz<F> *__restrict__ partials,
                                             Xyzz<F> *__restrict__ buckets, uint32_t stride,
                                             uint32_t k2, uint32_t q)
{
    const uint32_t b = upper_bound_u32(lead_off, nb + 1, q) - 1;
    const uint32_t j = q - lead_off[b];
    const Pieces pc = bucket_pieces(offsets, b, k1);
    const uint32_t off_b = offsets[b];
    const uint32_t live = (pc.count + stride - 1) / stride;
    const uint64_t r = uint64_t(j) * k2 * stride;
    Xyzz<CF<F>> acc = Xyzz<CF<F>>::inf();
    for (uint32_t m = 0; m < k2; ++m) {
        const uint64_t idx = r + uint64_t(m) * stride;
        if (idx >= pc.count) break;
        acc = xyzz_add(acc, ldx(partials[pc.slot(off_b, k1, uint32_t(idx))]));
    }
    if (live <= k2)
        buckets[b] = stx(acc);
    else
        partials[pc.slot(off_b, k1, uint32_t(r))] = stx(acc);
}

// Fix-up level: a grid-stride loop over the level's groups (often none).
template <class F>
__global__ void __launch_bounds__(128) k_acc_up(const uint32_t *__restrict__ offsets,
                                                 const uint32_t *__restrict__ lead_off, uint32_t nb,
                                                 uint32_t k1, Xyzz<F> *__restrict__ partials,
                                                 Xyzz<F> *__restrict__ buckets, uint32_t stride,
                                                 uint32_t k2)
{
    const uint32_t total = lead_off[nb];
    for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < total; q += gridDim.x * blockDim.x)
        acc_up_group(offsets, lead_off, nb, k1, partials, buckets, stride, k2, q);
}

// --------------------------------------------------------------------------
// bucket reduction: sum_b b * S_b per set, then + sum_b S_b
// --------------------------------------------------------------------------

// Buckets per thread (G2: per lane pair) of the first reduction level (log2).
// The block levels that follow are latency bound (dependent additions), so the
// first level leaves about 128 x BS items: the next level is then one wave of 128
// blocks (at most one 256-thread block per SM fits) and a single final block.
// Measured fastest for G1 (BS 256) at 2^15, 2^16 and 2^19 buckets and G2 (BS 128)
// at 2^15 and 2^16.
// The environment variable NKR_B200_REDUCE_L2 sets it for tuning experiments.
int first_level_log2(uint32_t m, int log2_bs, int bias)
{
    static const int forced = [] {
        const char *e = std::getenv("NKR_B200_REDUCE_L2");
        return e ? std::atoi(e) : -1;
    }();
    int lg = 0;
    while ((uint64_t(1) << (lg + 1)) <= m) ++lg;
    if (forced >= 0) return forced < lg ? forced : lg;
    const int over = lg - (7 + log2_bs);
    int l2 = (over <= 0 ? 0 : over > 4 ? 4 : over) + bias;
    l2 = l2 < 0 ? 0 : l2;
    return l2 < lg ? l2 : lg;
}

// run += S_b for bucket b: S_b is empty, written whole by the level-1 kernel
// (one piece) or by the fix-up levels (more than kSmallPieces pieces), or else
// its few pieces are added straight from the partial slots.
template <class C, class F>
__device__ __forceinline__ Xyzz<C> add_bucket_sum(Xyzz<C> run,
                                                      const uint32_t *__restrict__ offsets,
                                                      const Xyzz<F> *__restrict__ partials,
                                                      const Xyzz<F> *__restrict__ buckets, uint32_t b,
                                                      uint32_t k1)
{
    const uint32_t lo = offsets[b], hi = offsets[b + 1];
    if (hi == lo) return run;
    const Pieces pc{lo / k1, (hi - 1) / k1 - lo / k1 + 1};
    if (pc.count == 1 || pc.count > kSmallPieces) return xyzz_add(run, ldr<C>(buckets[b]));
    for (uint32_t k = 0; k < pc.count; ++k) run = xyzz_add(run, ldr<C>(partials[pc.slot(lo, k1, k)]));
    return run;
}

// Work-efficient first reduction level: a thread (G2: a lane pair) takes L consecutive buckets
// and forms T = sum_i i S_i and R = sum_i S_i by running sums (2 additions per
// bucket), emitting one (A = T, R) item per L buckets with unit L for the block
// levels that follow.  Bucket sums of few pieces are finished here.
template <class F, int LANES>
__global__ void __launch_bounds__(128) k_reduce_first(const uint32_t *__restrict__ offsets,
                                                       const Xyzz<F> *__restrict__ partials,
                                                       const Xyzz<F> *__restrict__ buckets,
                                                       uint64_t items, uint32_t L, uint32_t k1,
                                                       Xyzz<F> *__restrict__ a_out,
                                                       Xyzz<F> *__restrict__ r_out)
{
    using C = typename MsmReduceArith<F, LANES>::type;
    const uint64_t t = (uint64_t(blockIdx.x) * blockDim.x + threadIdx.x) / LANES; // the lanes' item
    if (t * L >= items) return;
    const uint64_t base = t * L;
    Xyzz<C> run = Xyzz<C>::inf(), tri = Xyzz<C>::inf();
    for (int i = int(L) - 1; i >= 0; --i) {
        run = add_bucket_sum<C>(run, offsets, partials, buckets, uint32_t(base + i), k1);
        if (i > 0) tri = xyzz_add(tri, run);
    }
    if (threadIdx.x % LANES) return;
    a_out[t] = stx(tri);
    r_out[t] = stx(run);
}

// One level of the weighted sum: items carry (A_c, R_c) with
// S = sum_c (A_c + c U R_c) (unit U = 2^log2_unit; level 0 is A = 0, R = the
// buckets, U = 1).  A block takes BS consecutive
// items c (padding with infinity), forms the suffix sums Suf_c = sum_{c' >= c} R_c'
// with a Hillis-Steele scan in shared memory (log2 BS dependent additions),
// then sum_c c R_c = sum_{c >= 1} Suf_c and sum_c A_c by two tree sums on
// disjoint threads, so a level costs about 2 log2(BS) dependent additions
// instead of 2 BS.  With lane pairs (G2) item c belongs to lanes (2c, 2c + 1)
// and the even lane stores.
// Output per block: A' = sum A_c + U sum_c c R_c, R' = sum R_c.
template <class F, int BS, int LANES>
__global__ void __launch_bounds__(BS * LANES) k_reduce_block(const Xyzz<F> *__restrict__ a_in,
                                                      const Xyzz<F> *__restrict__ r_in,
                                                      uint32_t m, int log2_unit,
                                                      Xyzz<F> *__restrict__ a_out,
                                                      Xyzz<F> *__restrict__ r_out)
{
    using C = typename MsmReduceArith<F, LANES>::type;
    extern __shared__ uint8_t smem_raw[];
    Xyzz<C> *buf0 = reinterpret_cast<Xyzz<C> *>(smem_raw);
    Xyzz<C> *buf1 = buf0 + BS;
    const uint32_t blocks_per_set = (m + BS - 1) / BS;
    const uint32_t set = blockIdx.x / blocks_per_set;
    const uint32_t blk = blockIdx.x % blocks_per_set;
    const int i = threadIdx.x / LANES;
    const bool lead = threadIdx.x % LANES == 0;
    const uint64_t idx = uint64_t(blk) * BS + i;
    const bool live = idx < m;
    const uint64_t g = uint64_t(set) * m + idx;
    Xyzz<C> v = live ? ldr<C>(r_in[g]) : Xyzz<C>::inf();
    if (lead) buf0[i] = v;
    __syncthreads();
    Xyzz<C> *cur = buf0, *nxt = buf1;
    for (int d = 1; d < BS; d <<= 1) {
        if (i + d < BS) v = xyzz_add(v, cur[i + d]);
        if (lead) nxt[i] = v;
        __syncthreads();
        Xyzz<C> *t = cur;
        cur = nxt;
        nxt = t;
    }
    // v = Suf_i.  R' = Suf_0; weighted part = sum_{i >= 1} Suf_i; A part = sum A_i
    const Xyzz<C> total = cur[0];
    __syncthreads();
    if (lead) {
        buf0[i] = i >= 1 ? v : Xyzz<C>::inf();
        buf1[i] = (a_in && live) ? ldr<C>(a_in[g]) : Xyzz<C>::inf();
    }
    __syncthreads();
    // the two tree sums run side by side on disjoint lane pairs (first s: weighted
    // suffix sums, next s: A items), one addition per pair and step; the pair has
    // read its operands before the even lane overwrites the first (__syncwarp)
    for (int s = BS / 2; s > 0; s >>= 1) {
        if (i < s) {
            const Xyzz<C> r = xyzz_add(buf0[i], buf0[i + s]);
            if constexpr (LANES == 2) __syncwarp(pair_mask());
            if (lead) buf0[i] = r;
        } else if (i < 2 * s) {
            const int j = i - s;
            const Xyzz<C> r = xyzz_add(buf1[j], buf1[j + s]);
            if constexpr (LANES == 2) __syncwarp(pair_mask());
            if (lead) buf1[j] = r;
        }
        __syncthreads();
    }
    if (i == 0) {
        Xyzz<C> w = buf0[0];
        for (int d = 0; d < log2_unit; ++d) w = xyzz_dbl(w);
        const Xyzz<C> a = xyzz_add(w, buf1[0]);
        if (lead) {
            const uint32_t o = set * blocks_per_set + blk;
            a_out[o] = stx(a);
            r_out[o] = stx(total);
        }
    }
}

// XYZZ -> libff Jacobian layout without inversion: with Z = ZZ ZZZ,
// X' = X ZZ ZZZ^2 and Y' = Y ZZ^3 ZZZ^2 represent the same affine point; the
// coordinates leave the R' domain here (back to the library's R = 2^256).
template <class C, class F>
__device__ __forceinline__ void store_jacobian(const Xyzz<C> &p, F *out)
{
    if (p.is_inf()) {
        out[0] = F::zero();
        out[1] = F::one();
        out[2] = F::zero();
        return;
    }
    const C zzz2 = sqr(p.zzz);
    const C zz2 = sqr(p.zz);
    out[0] = msm_out(msm_leave(p.x * (p.zz * zzz2)));
    out[1] = msm_out(msm_leave(p.y * (zz2 * p.zz * zzz2)));
    out[2] = msm_out(msm_leave(p.zz * p.zzz));
}

// one thread (G2: the lane pair 0, 1); lane 0 stores
template <class F, int LANES>
__global__ void k_finalize(const Xyzz<F> *a, const Xyzz<F> *r, int sets, int c, F *out)
{
    if (threadIdx.x >= unsigned(LANES) || blockIdx.x != 0) return;
    using C = typename MsmReduceArith<F, LANES>::type;
    Xyzz<C> acc = Xyzz<C>::inf();
    for (int k = sets - 1; k >= 0; --k) {
        if (k != sets - 1)
            for (int d = 0; d < c; ++d) acc = xyzz_dbl(acc);
        acc = xyzz_add(acc, a ? xyzz_add(ldr<C>(a[k]), ldr<C>(r[k])) : ldr<C>(r[k]));
    }
    if (threadIdx.x == 0) store_jacobian(acc, out);
}

// Resident bases enter the R' domain once they are final (x 2^4 mod p per
// coordinate; the infinity encoding (0, one) maps to (0, one'))
template <class F>
__global__ void k_bases_to_r260(Affine<F> *__restrict__ pts, uint64_t n)
{
    const uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const Affine<CF<F>> a = lda(pts[i]);
    pts[i] = {msm_out(msm_enter(a.x)), msm_out(msm_enter(a.y))};
}

// --------------------------------------------------------------------------
// normalisation and window copies
// --------------------------------------------------------------------------

constexpr int kNormChunk = 16;

// libff Jacobian (X, Y, Z): x = X / Z^2, y = Y / Z^3; batch inversion per chunk
template <class F>
__global__ void k_jac_to_affine(const F *__restrict__ jac, Affine<F> *__restrict__ out, uint64_t n)
{
    const uint64_t t = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    const uint64_t beg = t * kNormChunk;
    if (beg >= n) return;
    const int cnt = int(n - beg < uint64_t(kNormChunk) ? n - beg : uint64_t(kNormChunk));
    F pre[kNormChunk];
    F acc = F::one();
    for (int j = 0; j < cnt; ++j) {
        pre[j] = acc;
        const F z = jac[3 * (beg + j) + 2];
        if (!z.is_zero()) acc = acc * z;
    }
    F inv = inverse(acc);
    for (int j = cnt - 1; j >= 0; --j) {
        const uint64_t i = beg + j;
        const F z = jac[3 * i + 2];
        if (z.is_zero()) {
            out[i] = Affine<F>::inf();
            continue;
        }
        const F zi = inv * pre[j];
        inv = inv * z;
        const F zi2 = sqr(zi);
        out[i] = {jac[3 * i] * zi2, jac[3 * i + 1] * (zi2 * zi)};
    }
}

template <class P>
__global__ void k_bitrev_points(const P *__restrict__ in, P *__restrict__ out, int logn)
{
    const uint64_t j = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (j >= (uint64_t(1) << logn)) return;
    const uint32_t r = logn == 0 ? 0u : (__brev(uint32_t(j)) >> (32 - logn));
    out[r] = in[j];
}

template <class F>
int jac_to_affine_t(const void *jac, void *aff, uint64_t n, cudaStream_t st)
{
    if (n == 0) return NKR_B200_OK;
    const uint64_t chunks = (n + kNormChunk - 1) / kNormChunk;
    k_jac_to_affine<F><<<blocks_for(chunks, 64), 64, 0, st>>>(static_cast<const F *>(jac),
                                                               static_cast<Affine<F> *>(aff), n);
    NKR_CHECK_LAUNCH();
    return NKR_B200_OK;
}

// Window copies k = 1..W-1 of the points [beg, beg + m): thread i runs the whole
// doubling chain of point beg + i (c (W - 1) doublings, in the MSM's compute
// field) and writes copy k to out[(k - 1) m + i] (XYZZ, storage domain).
template <class F>
__global__ void k_window_chain(const Affine<F> *__restrict__ pts, Xyzz<F> *__restrict__ out,
                               uint64_t beg, uint64_t m, int c, int W)
{
    const uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= m) return;
    using C = CF<F>;
    const Affine<F> s = pts[beg + i];
    if (s.is_inf()) {
        for (int k = 1; k < W; ++k) out[uint64_t(k - 1) * m + i] = Xyzz<F>::inf();
        return;
    }
    const Affine<C> a = lda(s);
    Xyzz<C> x = xyzz_from_affine_dbl(Affine<C>{msm_enter(a.x), msm_enter(a.y)});
    for (int k = 1; k < W; ++k) {
        for (int d = (k == 1 ? 1 : 0); d < c; ++d) x = xyzz_dbl(x);
        out[uint64_t(k - 1) * m + i] = {msm_out(msm_leave(x.x)), msm_out(msm_leave(x.y)),
                                        msm_out(msm_leave(x.zz)), msm_out(msm_leave(x.zzz))};
    }
}

// XYZZ copies of k_window_chain -> affine copies k = 1..W-1 in the bases
// (copy k of point beg + i at pts[k n + beg + i]); batch inversion per chunk of
// kNormChunk scratch entries (a chunk may span two copies: the mapping is per entry)
template <class F>
__global__ void k_window_affine(const Xyzz<F> *__restrict__ in, Affine<F> *__restrict__ pts,
                                uint64_t n, uint64_t beg, uint64_t m, uint64_t count)
{
    const uint64_t t = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    const uint64_t first = t * kNormChunk;
    if (first >= count) return;
    const int cnt = int(count - first < uint64_t(kNormChunk) ? count - first : uint64_t(kNormChunk));
    F pre[kNormChunk];
    F acc = F::one();
    for (int j = 0; j < cnt; ++j) {
        pre[j] = acc;
        const Xyzz<F> p = in[first + j];
        if (!p.is_inf()) acc = acc * (p.zz * p.zzz);
    }
    F inv = inverse(acc);
    for (int j = cnt - 1; j >= 0; --j) {
        const uint64_t e = first + j;
        const uint64_t dst = (e / m + 1) * n + beg + e % m;
        const Xyzz<F> p = in[e];
        if (p.is_inf()) {
            pts[dst] = Affine<F>::inf();
            continue;
        }
        const F d = p.zz * p.zzz;
        const F ti = inv * pre[j];
        inv = inv * d;
        pts[dst] = {p.x * (ti * p.zzz), p.y * (ti * p.zz)};
    }
}

// The W - 1 folded window copies 2^(c k) P of every base: per chunk of points one
// launch runs every copy's doublings (so a small key pays one doubling chain and
// one batch inversion, not W - 1 of each) and one launch converts them to affine.
template <class F>
int build_windows_t(MsmBases &b, cudaStream_t st)
{
    const MsmShape &sh = b.shape;
    if (sh.W < 2 || sh.n == 0) return NKR_B200_OK;
    Affine<F> *pts = b.pts.as<Affine<F>>();
    const uint64_t copies = uint64_t(sh.W - 1);
    // scratch of at most ~1 GiB: chunk * copies XYZZ points
    const uint64_t cap = std::max<uint64_t>(1, (uint64_t(1) << 30) / (copies * sizeof(Xyzz<F>)));
    const uint64_t chunk = std::min<uint64_t>(sh.n, cap);
    DevBuf tmp;
    NKR_TRY(tmp.alloc(chunk * copies * sizeof(Xyzz<F>), "window copy scratch"));
    for (uint64_t beg = 0; beg < sh.n; beg += chunk) {
        const uint64_t m = std::min<uint64_t>(chunk, sh.n - beg);
        k_window_chain<F><<<blocks_for(m, 128), 128, 0, st>>>(pts, tmp.as<Xyzz<F>>(), beg, m, sh.c,
                                                              sh.W);
        NKR_CHECK_LAUNCH();
        const uint64_t count = m * copies;
        k_window_affine<F><<<blocks_for((count + kNormChunk - 1) / kNormChunk, 64), 64, 0, st>>>(
            tmp.as<Xyzz<F>>(), pts, sh.n, beg, m, count);
        NKR_CHECK_LAUNCH();
    }
    NKR_CUDA(cudaStreamSynchronize(st));
    return NKR_B200_OK;
}

template <class F>
int acc_level1_t(const MsmBases &bs, const MsmSort &s, MsmAcc &a, cudaStream_t st)
{
    const MsmShape &sh = bs.shape;
    // no bucket clearing: a bucket is read only after the kernel that wrote it
    const uint64_t segs = sh.segments_max();
    const uint32_t *offsets = s.offsets.as<uint32_t>();
    if (a.timing) NKR_CUDA(cudaEventRecord(a.ev_acc[0], st));
    if constexpr (std::is_same<F, Fq>::value)
        k_acc_l1_g1<<<blocks_for(segs, 128), 128, 0, st>>>(
            offsets, s.entries.as<uint32_t>(), bs.pts.as<Affine<F>>(), sh.nb, uint32_t(sh.k1),
            a.partials.as<Xyzz<F>>(), a.buckets.as<Xyzz<F>>());
    else
        k_acc_l1_g2<<<blocks_for(segs, 128), 128, 0, st>>>(
            offsets, s.entries.as<uint32_t>(), bs.pts.as<Affine<F>>(), sh.nb, uint32_t(sh.k1),
            a.partials.as<Xyzz<F>>(), a.buckets.as<Xyzz<F>>());
    NKR_CHECK_LAUNCH();
    if (a.timing) NKR_CUDA(cudaEventRecord(a.ev_acc[1], st));
    return NKR_B200_OK;
}

// Level 1 of n MSMs of one group in one launch; items_dev is device scratch of n
// work-list items.
template <class F>
int acc_level1_list_t(const MsmAccJob *jobs, int n, void *items_host, void *items_dev, cudaStream_t st)
{
    if (n <= 0) return NKR_B200_OK;
    AccItem<F> *items = static_cast<AccItem<F> *>(items_host);
    uint64_t blocks = 0;
    for (int i = 0; i < n; ++i) {
        const MsmShape &sh = jobs[i].bases->shape;
        AccItem<F> &it = items[i];
        it.offsets = jobs[i].sort->offsets.as<uint32_t>();
        it.entries = jobs[i].sort->entries.as<uint32_t>();
        it.pts = jobs[i].bases->pts.as<Affine<F>>();
        it.partials = jobs[i].acc->partials.as<Xyzz<F>>();
        it.buckets = jobs[i].acc->buckets.as<Xyzz<F>>();
        it.nb = sh.nb;
        it.k1 = uint32_t(sh.k1);
        it.first_block = uint32_t(blocks);
        blocks += blocks_for(sh.segments_max(), 128);
        NKR_REQUIRE(blocks < (uint64_t(1) << 31), "batched accumulation too large");
    }
    AccItem<F> *d = static_cast<AccItem<F> *>(items_dev);
    NKR_CUDA(cudaMemcpyAsync(d, items, n * sizeof(AccItem<F>), cudaMemcpyHostToDevice, st));
    if constexpr (std::is_same<F, Fq>::value)
        k_acc_l1_g1_list<<<unsigned(blocks), 128, 0, st>>>(d, n);
    else
        k_acc_l1_g2_list<<<unsigned(blocks), 128, 0, st>>>(d, n);
    NKR_CHECK_LAUNCH();
    return NKR_B200_OK;
}

// The reduction levels of an MSM whose buckets are final: first level, block
// levels, final combination, with LANES lanes per item.
template <class F, int LANES>
int reduce_run(const MsmBases &bs, const MsmSort &s, MsmAcc &a, void *out_dev, cudaStream_t st)
{
    using RA = MsmReduceArith<F, LANES>;
    const MsmShape &sh = bs.shape;
    const uint32_t *offsets = s.offsets.as<uint32_t>();
    const uint32_t sets = sh.folded ? 1u : uint32_t(sh.W);
    uint32_t m = sh.B;
    Xyzz<F> *bufs_a[2] = {a.red_a.as<Xyzz<F>>(), a.red_a2.as<Xyzz<F>>()};
    Xyzz<F> *bufs_r[2] = {a.red_r.as<Xyzz<F>>(), a.red_r2.as<Xyzz<F>>()};
    constexpr int BS = RA::items;
    constexpr int kLog2BS = RA::log2_items;
    const size_t smem = 2 * BS * sizeof(Xyzz<typename RA::type>);
    NKR_CUDA(cudaFuncSetAttribute(k_reduce_block<F, BS, LANES>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  int(smem)));
    // first level: bucket sums (few-piece buckets finished here), L buckets per item
    const int log2_l = first_level_log2(m, kLog2BS, a.first_level_bias);
    const uint32_t L = 1u << log2_l;
    const uint64_t items = uint64_t(sets) * m;
    k_reduce_first<F, LANES><<<blocks_for(LANES * (items / L), 128), 128, 0, st>>>(
        offsets, a.partials.as<Xyzz<F>>(), a.buckets.as<Xyzz<F>>(), items, L, uint32_t(sh.k1), bufs_a[0],
        bufs_r[0]);
    NKR_CHECK_LAUNCH();
    if (a.timing) NKR_CUDA(cudaEventRecord(a.ev_acc[3], st));
    const Xyzz<F> *a_in = bufs_a[0];
    const Xyzz<F> *r_in = bufs_r[0];
    int flip = 1;
    m /= L;
    int log2_unit = log2_l;
    while (m > 1) {
        const uint32_t per_set = (m + BS - 1) / BS;
        k_reduce_block<F, BS, LANES><<<sets * per_set, LANES * BS, smem, st>>>(
            a_in, r_in, m, log2_unit, bufs_a[flip], bufs_r[flip]);
        NKR_CHECK_LAUNCH();
        a_in = bufs_a[flip];
        r_in = bufs_r[flip];
        flip ^= 1;
        m = per_set;
        log2_unit += kLog2BS;
    }
    k_finalize<F, LANES><<<1, 32, 0, st>>>(a_in, r_in, int(sets), sh.c, static_cast<F *>(out_dev));
    NKR_CHECK_LAUNCH();
    if (a.timing) NKR_CUDA(cudaEventRecord(a.ev_acc[4], st));
    return NKR_B200_OK;
}

// Fix-up levels of a level-1 accumulation with shape sh (segments, buckets,
// k1, k2) whose bucket offsets are `offsets`: inputs spaced `stride` pieces
// apart, groups of k2; one bucket has at most segs + 1 pieces, all buckets at
// most 2 segs.
template <class F>
int fixup_levels_t(const MsmShape &sh, const uint32_t *offsets, uint32_t *lead_off, uint32_t *scan_tmp,
                   Xyzz<F> *partials, Xyzz<F> *buckets, cudaStream_t st)
{
    const uint64_t segs = sh.segments_max();
    const uint64_t k2 = uint64_t(sh.k2);
    for (uint64_t stride = 1; stride < segs + 1; stride *= k2) {
        NKR_TRY(scan_exclusive(LoadLeaders{offsets, uint32_t(sh.k1), uint32_t(stride), uint32_t(k2)},
                               sh.nb, lead_off, scan_tmp, st));
        const uint64_t bound = 2 * segs / (stride * k2) + sh.nb + 1;
        const unsigned grid = std::min<unsigned>(blocks_for(bound, 128), kFixupBlocks);
        k_acc_up<F><<<grid, 128, 0, st>>>(offsets, lead_off, sh.nb, uint32_t(sh.k1), partials, buckets,
                                           uint32_t(stride), uint32_t(k2));
        NKR_CHECK_LAUNCH();
    }
    return NKR_B200_OK;
}

template <class F>
int acc_tail_t(const MsmBases &bs, const MsmSort &s, MsmAcc &a, void *out_dev, cudaStream_t st)
{
    NKR_TRY(fixup_levels_t<F>(bs.shape, s.offsets.as<uint32_t>(), a.lead_off.as<uint32_t>(),
                              a.scan_tmp.as<uint32_t>(), a.partials.as<Xyzz<F>>(), a.buckets.as<Xyzz<F>>(),
                              st));
    if (a.timing) NKR_CUDA(cudaEventRecord(a.ev_acc[2], st));
    // bucket reduction levels (G2 alone: on lane pairs)
    if constexpr (std::is_same<F, Fq2>::value)
        if (a.lane_pairs) return reduce_run<F, 2>(bs, s, a, out_dev, st);
    return reduce_run<F, 1>(bs, s, a, out_dev, st);
}

template <class F>
int acc_run_t(const MsmBases &bs, const MsmSort &s, MsmAcc &a, void *out_dev, cudaStream_t st)
{
    NKR_TRY(acc_level1_t<F>(bs, s, a, st));
    return acc_tail_t<F>(bs, s, a, out_dev, st);
}

template <class F>
int acc_alloc_t(MsmAcc &a, const MsmShape &sh)
{
    const uint32_t sets = sh.folded ? 1u : uint32_t(sh.W);
    // first reduction level output: one item per L buckets (L as in acc_run_t)
    // items per block of the reduction levels (the same for one and two lanes per item)
    constexpr int kLog2BS = MsmReduceArith<F, 1>::log2_items;
    static_assert(MsmReduceArith<F, 1>::log2_items == MsmReduceArith<F, 2>::log2_items || sizeof(F) == sizeof(Fq),
                  "G2 reduction buffers are sized for one block shape");
    const uint64_t red = uint64_t(sets) * (sh.B >> first_level_log2(sh.B, kLog2BS, a.first_level_bias)) + 1;
    NKR_TRY(a.partials.alloc(2 * std::max<uint64_t>(sh.segments_max(), 1) * sizeof(Xyzz<F>),
                             "msm partial sums"));
    NKR_TRY(a.buckets.alloc(uint64_t(sh.nb) * sizeof(Xyzz<F>), "msm buckets"));
    NKR_TRY(a.lead_off.alloc((sh.nb + 1) * 4ull, "msm fix-up offsets"));
    NKR_TRY(a.red_a.alloc(red * sizeof(Xyzz<F>), "msm reduction"));
    NKR_TRY(a.red_r.alloc(red * sizeof(Xyzz<F>), "msm reduction"));
    NKR_TRY(a.red_a2.alloc(red * sizeof(Xyzz<F>), "msm reduction"));
    NKR_TRY(a.red_r2.alloc(red * sizeof(Xyzz<F>), "msm reduction"));
    NKR_TRY(a.scan_tmp.alloc(scan_scratch_words(sh.nb) * 4, "msm scan scratch"));
    NKR_TRY(a.result.alloc(192, "msm result"));
    return NKR_B200_OK;
}

// --------------------------------------------------------------------------
// repeated scalars: classes of equal witness values (msm.cuh)
// --------------------------------------------------------------------------

__device__ __forceinline__ uint32_t scalar_hash(const Fr &s)
{
    return s.v[0] ^ (s.v[1] * 0x9e3779b9u) ^ (s.v[6] * 0x85ebca6bu) ^ (s.v[7] * 0xc2b2ae35u);
}

constexpr int kDedupProbes = 64; // a value not placed within this many slots stays a singleton

// rep[i]: the representative variable of z_i's value (kNoClass for zero).  The
// table holds variable indices (kNoClass = empty); a thread claims an empty
// slot with atomicCAS or finds an equal value on its probe path.
__global__ void k_dedup_insert(const Fr *__restrict__ z, uint64_t cols, uint32_t *__restrict__ table,
                               uint64_t mask, uint32_t *__restrict__ rep)
{
    const uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= cols) return;
    const Fr s = z[i];
    if (s.is_zero()) {
        rep[i] = kNoClass;
        return;
    }
    uint64_t h = scalar_hash(s) & mask;
    uint32_t r = uint32_t(i);
    for (int probe = 0; probe < kDedupProbes; ++probe) {
        const uint32_t cur = atomicCAS(&table[h], kNoClass, uint32_t(i));
        if (cur == kNoClass) break; // this variable represents its value
        if (z[cur] == s) {
            r = cur;
            break;
        }
        h = (h + 1) & mask;
    }
    rep[i] = r;
}

// csize[r]: members of representative r (warp-aggregated per equal r)
__global__ void k_dedup_count(const uint32_t *__restrict__ rep, uint64_t cols, uint32_t *__restrict__ csize)
{
    const uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    const uint32_t r = i < cols ? rep[i] : kNoClass;
    const unsigned act = __ballot_sync(0xffffffffu, r != kNoClass);
    if (r == kNoClass) return;
    const unsigned peers = __match_any_sync(act, r);
    if (int(threadIdx.x & 31) == __ffs(peers) - 1) atomicAdd(&csize[r], uint32_t(__popc(peers)));
}

// class ids for representatives of at least kClassMin members, first come first
// served up to kClassMax; values[id] = the class's value
__global__ void k_dedup_ids(const Fr *__restrict__ z, const uint32_t *__restrict__ rep,
                            const uint32_t *__restrict__ csize, uint64_t cols, uint32_t *__restrict__ cid,
                            Fr *__restrict__ values, uint32_t *__restrict__ nclass)
{
    const uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= cols) return;
    uint32_t id = kNoClass;
    if (rep[i] == uint32_t(i) && csize[i] >= kClassMin) {
        const uint32_t k = atomicAdd(nclass, 1u);
        if (k < kClassMax) {
            id = k;
            values[k] = z[i];
        }
    }
    cid[i] = id;
}

__global__ void k_dedup_mark(const uint32_t *__restrict__ rep, const uint32_t *__restrict__ cid,
                             uint64_t cols, uint32_t *__restrict__ class_of)
{
    const uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= cols) return;
    const uint32_t r = rep[i];
    class_of[i] = r == kNoClass ? kNoClass : cid[r];
}

// class members of a support: counts per class, then a scatter in class order
// (warp-aggregated per equal class)
__global__ void k_cls_count(const uint32_t *__restrict__ class_of, const uint32_t *__restrict__ gather,
                            uint64_t n, uint32_t *__restrict__ counts)
{
    const uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    const uint32_t c = i < n ? class_of[gather ? gather[i] : i] : kNoClass;
    const unsigned act = __ballot_sync(0xffffffffu, c != kNoClass);
    if (c == kNoClass) return;
    const unsigned peers = __match_any_sync(act, c);
    if (int(threadIdx.x & 31) == __ffs(peers) - 1) atomicAdd(&counts[c], uint32_t(__popc(peers)));
}

__global__ void k_cls_scatter(const uint32_t *__restrict__ class_of, const uint32_t *__restrict__ gather,
                              uint64_t n, uint32_t *__restrict__ cursor, uint32_t *__restrict__ entries)
{
    const uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    const uint32_t c = i < n ? class_of[gather ? gather[i] : i] : kNoClass;
    const unsigned act = __ballot_sync(0xffffffffu, c != kNoClass);
    if (c == kNoClass) return;
    const unsigned peers = __match_any_sync(act, c);
    const int lane = int(threadIdx.x & 31), leader = __ffs(peers) - 1;
    uint32_t base = 0;
    if (lane == leader) base = atomicAdd(&cursor[c], uint32_t(__popc(peers)));
    base = __shfl_sync(peers, base, leader);
    entries[base + uint32_t(__popc(peers & ((1u << lane) - 1u)))] = uint32_t(i);
}

// a class sum as an affine base of the small MSM (storage form of the group's
// MSM buffers: G1 in the R' domain; infinity as (0, one))
__device__ __forceinline__ Affine<Fq> class_affine(const Xyzz<Fq52L> &s)
{
    if (s.is_inf()) return {from52(Fq52::zero()), from52(Fq52::one())};
    const Affine<Fq52> a = xyzz_to_affine(Xyzz<Fq52>{s.x.canon(), s.y.canon(), s.zz.canon(), s.zzz.canon()});
    return {from52(a.x), from52(a.y)};
}
__device__ __forceinline__ Affine<Fq2> class_affine(const Xyzz<Fq2> &s) { return xyzz_to_affine(s); }

// S_c for every class: its pieces (level-1 runs and fix-up sums) added up and
// normalised with one inversion per class
template <class F>
__global__ void __launch_bounds__(128) k_cls_finish(const uint32_t *__restrict__ offsets,
                                                     const Xyzz<F> *__restrict__ partials,
                                                     const Xyzz<F> *__restrict__ buckets, uint32_t k1,
                                                     uint32_t nb, Affine<F> *__restrict__ sums)
{
    const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= nb) return;
    using C = CF<F>;
    sums[c] = class_affine(add_bucket_sum<C>(Xyzz<C>::inf(), offsets, partials, buckets, c, k1));
}

// acc += add for two libff-Jacobian points (X, Y, Z; Z = 0 is infinity) in the
// library's Montgomery domain
template <class F>
__global__ void k_result_add(F *acc, const F *add)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    auto xyzz = [](const F *p) {
        if (p[2].is_zero()) return Xyzz<F>::inf();
        const F zz = sqr(p[2]);
        return Xyzz<F>{p[0], p[1], zz, zz * p[2]};
    };
    const Xyzz<F> s = xyzz_add(xyzz(acc), xyzz(add));
    if (s.is_inf()) {
        acc[0] = F::zero();
        acc[1] = F::one();
        acc[2] = F::zero();
        return;
    }
    const F zzz2 = sqr(s.zzz), zz2 = sqr(s.zz);
    acc[0] = s.x * (s.zz * zzz2);
    acc[1] = s.y * (zz2 * s.zz * zzz2);
    acc[2] = s.zz * s.zzz;
}

// G2's MSM over its class values uses the twist Frobenius psi(x, y) =
// (conj(x) gx1, conj(y) gy1), which acts on G2 as multiplication by
// lambda = p mod r = 6 u^2 (127 bits): a class value v = k0 + k1 lambda with
// k0 = v mod lambda and k1 = v div lambda (both below 2^128), so the MSM runs over
// the class sums and their images under psi with 128-bit scalars, and its Horner
// chain has half the doublings.
constexpr uint64_t kPsiLambdaLo = 0xf83e9682e87cfd46ull, kPsiLambdaHi = 0x6f4d8248eeb859fbull;
constexpr int kPsiWindows = 13; // 10-bit signed windows over 128-bit scalars (130 bits, no carry out)

__device__ __forceinline__ Fr fr_from_u128(unsigned __int128 x)
{
    Fr r;
#pragma unroll
    for (int i = 0; i < 4; ++i) r.v[i] = uint32_t(x >> (32 * i));
#pragma unroll
    for (int i = 4; i < 8; ++i) r.v[i] = 0;
    return to_mont(r);
}

// values[c] (Montgomery) -> out[c] = k0, out[n + c] = k1 (Montgomery), by binary
// long division of the canonical value by lambda
__global__ void k_cls_split_psi(const Fr *__restrict__ values, uint32_t n, Fr *__restrict__ out)
{
    const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n) return;
    const Fr v = from_mont(values[c]);
    const unsigned __int128 lam = (unsigned __int128)kPsiLambdaHi << 64 | kPsiLambdaLo;
    unsigned __int128 rem = 0, q = 0;
    for (int i = 253; i >= 0; --i) { // v < r < 2^254; rem < lambda, so 2 rem + 1 < 2^128
        rem = (rem << 1) | ((v.v[i >> 5] >> (i & 31)) & 1u);
        q <<= 1;
        if (rem >= lam) {
            rem -= lam;
            q |= 1;
        }
    }
    out[c] = fr_from_u128(rem);
    out[n + c] = fr_from_u128(q);
}

// sums[n + c] = psi(sums[c]) (infinity stays infinity)
__global__ void k_cls_psi(Affine<Fq2> *sums, uint32_t n)
{
    const uint32_t c = blockIdx.x * blockDim.x + threadIdx.x;
    if (c >= n) return;
    const Affine<Fq2> a = sums[c];
    sums[n + c] = a.is_inf() ? a : twist_frobenius(a);
}

template <class F>
int class_acc_alloc_t(MsmClassAcc &a, uint64_t n)
{
    a.seg = MsmShape{};
    a.seg.n = n;
    a.seg.c = 1;
    a.seg.W = 1;
    a.seg.folded = true;
    a.seg.B = kClassMax;
    a.seg.nb = kClassMax;
    const uint64_t segs = std::max<uint64_t>(a.seg.segments_max(), 1);
    NKR_TRY(a.partials.alloc(2 * segs * sizeof(Xyzz<F>), "class partial sums"));
    NKR_TRY(a.buckets.alloc(uint64_t(kClassMax) * sizeof(Xyzz<F>), "class sums"));
    NKR_TRY(a.lead_off.alloc((kClassMax + 1) * 4ull, "class fix-up offsets"));
    NKR_TRY(a.scan_tmp.alloc(scan_scratch_words(kClassMax) * 4, "class scan scratch"));
    return NKR_B200_OK;
}

template <class F>
int class_acc_issue_t(const MsmBases &b, const MsmClassSort &cs, MsmClassAcc &a, cudaStream_t st)
{
    const uint64_t segs = a.seg.segments_max();
    const uint32_t *offsets = cs.offsets.as<uint32_t>();
    if (segs) {
        if constexpr (std::is_same<F, Fq>::value)
            k_acc_l1_g1<<<blocks_for(segs, 128), 128, 0, st>>>(
                offsets, cs.entries.as<uint32_t>(), b.pts.as<Affine<F>>(), kClassMax, uint32_t(a.seg.k1),
                a.partials.as<Xyzz<F>>(), a.buckets.as<Xyzz<F>>());
        else
            k_acc_l1_g2<<<blocks_for(segs, 128), 128, 0, st>>>(
                offsets, cs.entries.as<uint32_t>(), b.pts.as<Affine<F>>(), kClassMax, uint32_t(a.seg.k1),
                a.partials.as<Xyzz<F>>(), a.buckets.as<Xyzz<F>>());
        NKR_CHECK_LAUNCH();
    }
    NKR_TRY(fixup_levels_t<F>(a.seg, offsets, a.lead_off.as<uint32_t>(), a.scan_tmp.as<uint32_t>(),
                              a.partials.as<Xyzz<F>>(), a.buckets.as<Xyzz<F>>(), st));
    k_cls_finish<F><<<blocks_for(kClassMax, 128), 128, 0, st>>>(
        offsets, a.partials.as<Xyzz<F>>(), a.buckets.as<Xyzz<F>>(), uint32_t(a.seg.k1), kClassMax,
        a.small.pts.as<Affine<F>>());
    NKR_CHECK_LAUNCH();
    return NKR_B200_OK;
}

} // namespace

MsmShape msm_shape(uint64_t n, bool folded, int group, int c_override)
{
    MsmShape sh;
    sh.n = n;
    sh.folded = folded;
    int lg = 0;
    while ((uint64_t(1) << lg) < n) ++lg;
    int c;
    (void)group; // G1 and G2 share the shape so MSMs over the same scalars share one sort
    if (c_override > 0) {
        c = c_override;
    } else if (folded) {
        // One bucket set.  Cost model in point additions: n ceil(255 / c) mixed
        // additions (10 products each) for the accumulation against about two
        // full additions (14 products each) per bucket for the reduction.
        double best = 1e300;
        c = 8;
        for (int cc = 8; cc <= 22; ++cc) {
            const double cost = double(n) * ((255 + cc - 1) / cc) * 10.0 +
                                double(uint64_t(1) << (cc - 1)) * 2.0 * 14.0;
            if (cost < best) {
                best = cost;
                c = cc;
            }
        }
    } else {
        c = lg - 5;
    }
    if (c < 4) c = 4;
    if (c > 22) c = 22;
    sh.c = c;
    sh.W = (255 + c - 1) / c;
    sh.B = 1u << (c - 1);
    sh.nb = folded ? sh.B : sh.B * uint32_t(sh.W);
    return sh;
}

int jacobian_to_affine(int group, const void *jac, void *aff, uint64_t n, cudaStream_t st)
{
    return group == 1 ? jac_to_affine_t<Fq>(jac, aff, n, st) : jac_to_affine_t<Fq2>(jac, aff, n, st);
}

int msm_bases_build(MsmBases &b, int group, const void *jac, bool jac_on_device, uint64_t n,
                    bool folded, int c_override, bool bitrev, cudaStream_t st)
{
    NKR_REQUIRE(group == 1 || group == 2, "group must be 1 (G1) or 2 (G2)");
    b.group = group;
    b.shape = msm_shape(n, folded, group, c_override);
    NKR_REQUIRE(!folded || uint64_t(b.shape.W) * n < (uint64_t(1) << 31),
                "folded MSM of %llu points exceeds the 2^31 entry index space",
                (unsigned long long)n);
    const size_t aff_sz = group == 1 ? sizeof(G1Affine) : sizeof(G2Affine);
    const size_t jac_sz = group == 1 ? 96 : 192;
    const uint64_t copies = folded ? uint64_t(b.shape.W) : 1;
    NKR_TRY(b.pts.alloc(std::max<uint64_t>(n, 1) * copies * aff_sz, "msm bases"));
    if (n == 0) return NKR_B200_OK;
    const void *src = jac;
    DevBuf staging;
    if (!jac_on_device) {
        NKR_TRY(staging.alloc(n * jac_sz, "msm base upload"));
        NKR_CUDA(cudaMemcpyAsync(staging.p, jac, n * jac_sz, cudaMemcpyHostToDevice, st));
        src = staging.p;
    }
    NKR_TRY(jacobian_to_affine(group, src, b.pts.p, n, st));
    if (bitrev) {
        const int lg = log2_exact(n);
        NKR_REQUIRE(lg >= 0 && lg <= 31, "bit-reversed bases need a power-of-two count");
        DevBuf tmp;
        NKR_TRY(tmp.alloc(n * aff_sz, "bitrev base scratch"));
        NKR_CUDA(cudaMemcpyAsync(tmp.p, b.pts.p, n * aff_sz, cudaMemcpyDeviceToDevice, st));
        if (group == 1)
            k_bitrev_points<G1Affine><<<blocks_for(n, 256), 256, 0, st>>>(
                tmp.as<G1Affine>(), b.pts.as<G1Affine>(), lg);
        else
            k_bitrev_points<G2Affine><<<blocks_for(n, 256), 256, 0, st>>>(
                tmp.as<G2Affine>(), b.pts.as<G2Affine>(), lg);
        NKR_CHECK_LAUNCH();
        NKR_CUDA(cudaStreamSynchronize(st));
    }
    if (folded) NKR_TRY(group == 1 ? build_windows_t<Fq>(b, st) : build_windows_t<Fq2>(b, st));
    const uint64_t total = n * copies;
    if (group == 1) { // G2 computes in the library's own domain
        k_bases_to_r260<Fq><<<blocks_for(total, 128), 128, 0, st>>>(b.pts.as<G1Affine>(), total);
        NKR_CHECK_LAUNCH();
    }

    NKR_CUDA(cudaStreamSynchronize(st));
    return NKR_B200_OK;
}

std::vector<uint32_t> msm_support(int group, const void *jac_host, uint64_t n)
{
    const size_t jac_sz = group == 1 ? 96 : 192;
    const size_t z_off = jac_sz / 3 * 2, z_sz = jac_sz / 3;
    const uint8_t *src = static_cast<const uint8_t *>(jac_host);
    std::vector<uint32_t> idx;
    idx.reserve(n);
    for (uint64_t i = 0; i < n; ++i) {
        const uint8_t *z = src + i * jac_sz + z_off;
        bool zero = true;
        for (size_t k = 0; k < z_sz && zero; k += 8) {
            uint64_t w;
            std::memcpy(&w, z + k, 8);
            zero = w == 0;
        }
        if (!zero) idx.push_back(uint32_t(i));
    }
    if (idx.empty() && n) idx.push_back(0); // an all-infinity query still has one (zero) term
    return idx;
}

int msm_bases_build_support(MsmBases &b, int group, const void *jac_host, uint64_t n,
                            std::vector<uint32_t> idx, bool folded, int c_override, cudaStream_t st)
{
    NKR_REQUIRE(group == 1 || group == 2, "group must be 1 (G1) or 2 (G2)");
    NKR_REQUIRE(n < (uint64_t(1) << 32), "support indices are 32-bit");
    NKR_REQUIRE(idx.size() <= n && (n == 0 || !idx.empty()), "support index list does not fit the bases");
    const size_t jac_sz = group == 1 ? 96 : 192;
    const uint8_t *src = static_cast<const uint8_t *>(jac_host);
    std::vector<uint8_t> packed(std::max<size_t>(idx.size(), 1) * jac_sz);
    for (size_t j = 0; j < idx.size(); ++j) {
        NKR_REQUIRE(idx[j] < n, "support index out of range");
        std::memcpy(packed.data() + j * jac_sz, src + uint64_t(idx[j]) * jac_sz, jac_sz);
    }
    NKR_TRY(msm_bases_build(b, group, packed.data(), false, idx.size(), folded, c_override, false, st));
    b.n_full = n;
    NKR_TRY(b.support.alloc(std::max<size_t>(idx.size(), 1) * 4, "msm support indices"));
    if (!idx.empty())
        NKR_CUDA(cudaMemcpyAsync(b.support.p, idx.data(), idx.size() * 4, cudaMemcpyHostToDevice, st));
    NKR_CUDA(cudaStreamSynchronize(st));
    b.support_host = std::move(idx);
    return NKR_B200_OK;
}

int msm_sort_alloc(MsmSort &s, const MsmShape &sh)
{
    NKR_TRY(s.canon.alloc(std::max<uint64_t>(sh.n, 1) * sizeof(Fr), "msm canonical scalars"));
    NKR_TRY(s.counts.alloc((sh.nb + 1) * 4ull, "msm bucket counts"));
    NKR_TRY(s.offsets.alloc((sh.nb + 1) * 4ull, "msm bucket offsets"));
    NKR_TRY(s.cursor.alloc((sh.nb + 1) * 4ull, "msm scatter cursor"));
    NKR_TRY(s.entries.alloc(std::max<uint64_t>(sh.entries_max(), 1) * 4, "msm entries"));
    NKR_TRY(s.scan_tmp.alloc(scan_scratch_words(sh.nb) * 4, "msm scan scratch"));
    return NKR_B200_OK;
}

int msm_acc_alloc(MsmAcc &a, int group, const MsmShape &sh)
{
    return group == 1 ? acc_alloc_t<Fq>(a, sh) : acc_alloc_t<Fq2>(a, sh);
}

int msm_scratch_alloc(MsmScratch &s, int group, const MsmShape &shape)
{
    NKR_TRY(msm_sort_alloc(s.sort, shape));
    NKR_TRY(msm_acc_alloc(s.acc, group, shape));
    return NKR_B200_OK;
}

int msm_sort_run(const MsmShape &sh, MsmSort &s, const void *scalars_dev, cudaStream_t st,
                 const uint32_t *gather, const uint32_t *class_of)
{
    const uint64_t n = sh.n;
    NKR_CUDA(cudaMemsetAsync(s.counts.p, 0, (sh.nb + 1) * 4, st));
    if (n) {
        k_digits_count<<<blocks_for(n, 256), 256, 0, st>>>(
            static_cast<const Fr *>(scalars_dev), gather, class_of, n, sh.c, sh.W, sh.folded, sh.B,
            s.canon.as<Fr>(), s.counts.as<uint32_t>());
        NKR_CHECK_LAUNCH();
    }
    NKR_TRY(scan_exclusive(LoadU32{s.counts.as<uint32_t>()}, sh.nb, s.offsets.as<uint32_t>(),
                           s.scan_tmp.as<uint32_t>(), st));
    NKR_CUDA(cudaMemcpyAsync(s.cursor.p, s.offsets.p, uint64_t(sh.nb) * 4, cudaMemcpyDeviceToDevice,
                             st));
    if (n) {
        k_scatter<<<blocks_for(n, 256), 256, 0, st>>>(s.canon.as<Fr>(), n, sh.c, sh.W, sh.folded, sh.B,
                                                      s.cursor.as<uint32_t>(),
                                                      s.entries.as<uint32_t>());
        NKR_CHECK_LAUNCH();
    }
    return NKR_B200_OK;
}

int msm_acc_run(const MsmBases &b, const MsmSort &s, MsmAcc &a, void *out_dev, cudaStream_t st)
{
    return b.group == 1 ? acc_run_t<Fq>(b, s, a, out_dev, st) : acc_run_t<Fq2>(b, s, a, out_dev, st);
}

int msm_acc_level1_list(int group, const MsmAccJob *jobs, int n, void *items_host, void *items_dev,
                        cudaStream_t st)
{
    NKR_REQUIRE(group == 1 || group == 2, "group must be 1 (G1) or 2 (G2)");
    for (int i = 0; i < n; ++i)
        NKR_REQUIRE(jobs[i].bases->group == group, "batched accumulation mixes G1 and G2");
    return group == 1 ? acc_level1_list_t<Fq>(jobs, n, items_host, items_dev, st)
                      : acc_level1_list_t<Fq2>(jobs, n, items_host, items_dev, st);
}

int msm_acc_level1(const MsmBases &b, const MsmSort &s, MsmAcc &a, cudaStream_t st)
{
    return b.group == 1 ? acc_level1_t<Fq>(b, s, a, st) : acc_level1_t<Fq2>(b, s, a, st);
}

int msm_acc_tail(const MsmBases &b, const MsmSort &s, MsmAcc &a, void *out_dev, cudaStream_t st)
{
    return b.group == 1 ? acc_tail_t<Fq>(b, s, a, out_dev, st) : acc_tail_t<Fq2>(b, s, a, out_dev, st);
}

int msm_run(const MsmBases &b, MsmScratch &s, const void *scalars_dev, void *out_dev,
            cudaStream_t st)
{
    NKR_TRY(msm_sort_run(b.shape, s.sort, scalars_dev, st, b.gather()));
    return msm_acc_run(b, s.sort, s.acc, out_dev, st);
}

int msm_dedup_alloc(MsmDedup &d, uint64_t cols)
{
    NKR_REQUIRE(cols < uint64_t(kNoClass), "witness of %llu variables too long for 32-bit indices",
                (unsigned long long)cols);
    d.cols = cols;
    d.slots = 1;
    while (d.slots < 2 * cols) d.slots <<= 1;
    const uint64_t c = std::max<uint64_t>(cols, 1);
    NKR_TRY(d.table.alloc(d.slots * 4, "dedup table"));
    NKR_TRY(d.rep.alloc(c * 4, "dedup representatives"));
    NKR_TRY(d.csize.alloc(c * 4, "dedup class sizes"));
    NKR_TRY(d.cid.alloc(c * 4, "dedup class ids"));
    NKR_TRY(d.class_of.alloc(c * 4, "dedup classes"));
    NKR_TRY(d.values.alloc(uint64_t(kClassMax) * sizeof(Fr), "class values"));
    NKR_TRY(d.nclass.alloc(4, "class count"));
    return NKR_B200_OK;
}

int msm_dedup_run(MsmDedup &d, const void *z, cudaStream_t st)
{
    const uint64_t cols = d.cols;
    NKR_CUDA(cudaMemsetAsync(d.table.p, 0xff, d.table.bytes, st));
    NKR_CUDA(cudaMemsetAsync(d.csize.p, 0, d.csize.bytes, st));
    NKR_CUDA(cudaMemsetAsync(d.values.p, 0, d.values.bytes, st));
    NKR_CUDA(cudaMemsetAsync(d.nclass.p, 0, 4, st));
    if (!cols) return NKR_B200_OK;
    const Fr *zf = static_cast<const Fr *>(z);
    const unsigned g = blocks_for(cols, 256);
    k_dedup_insert<<<g, 256, 0, st>>>(zf, cols, d.table.as<uint32_t>(), d.slots - 1, d.rep.as<uint32_t>());
    NKR_CHECK_LAUNCH();
    k_dedup_count<<<g, 256, 0, st>>>(d.rep.as<uint32_t>(), cols, d.csize.as<uint32_t>());
    NKR_CHECK_LAUNCH();
    k_dedup_ids<<<g, 256, 0, st>>>(zf, d.rep.as<uint32_t>(), d.csize.as<uint32_t>(), cols, d.cid.as<uint32_t>(),
                                   d.values.as<Fr>(), d.nclass.as<uint32_t>());
    NKR_CHECK_LAUNCH();
    k_dedup_mark<<<g, 256, 0, st>>>(d.rep.as<uint32_t>(), d.cid.as<uint32_t>(), cols,
                                    d.class_of.as<uint32_t>());
    NKR_CHECK_LAUNCH();
    return NKR_B200_OK;
}

int msm_class_sort_alloc(MsmClassSort &s, uint64_t n)
{
    s.n = n;
    NKR_TRY(s.counts.alloc((kClassMax + 1) * 4ull, "class counts"));
    NKR_TRY(s.offsets.alloc((kClassMax + 1) * 4ull, "class offsets"));
    NKR_TRY(s.cursor.alloc((kClassMax + 1) * 4ull, "class cursor"));
    NKR_TRY(s.entries.alloc(std::max<uint64_t>(n, 1) * 4, "class members"));
    NKR_TRY(s.scan_tmp.alloc(scan_scratch_words(kClassMax) * 4, "class scan scratch"));
    return NKR_B200_OK;
}

int msm_class_sort_run(MsmClassSort &s, const MsmDedup &d, const uint32_t *gather, cudaStream_t st)
{
    NKR_CUDA(cudaMemsetAsync(s.counts.p, 0, (kClassMax + 1) * 4ull, st));
    if (s.n)
        k_cls_count<<<blocks_for(s.n, 256), 256, 0, st>>>(d.class_of.as<uint32_t>(), gather, s.n,
                                                            s.counts.as<uint32_t>());
    NKR_CHECK_LAUNCH();
    NKR_TRY(scan_exclusive(LoadU32{s.counts.as<uint32_t>()}, kClassMax, s.offsets.as<uint32_t>(),
                           s.scan_tmp.as<uint32_t>(), st));
    NKR_CUDA(cudaMemcpyAsync(s.cursor.p, s.offsets.p, kClassMax * 4ull, cudaMemcpyDeviceToDevice, st));
    if (s.n)
        k_cls_scatter<<<blocks_for(s.n, 256), 256, 0, st>>>(d.class_of.as<uint32_t>(), gather, s.n,
                                                              s.cursor.as<uint32_t>(), s.entries.as<uint32_t>());
    NKR_CHECK_LAUNCH();
    return NKR_B200_OK;
}

int msm_class_acc_alloc(MsmClassAcc &a, int group, uint64_t n)
{
    NKR_REQUIRE(group == 1 || group == 2, "group must be 1 (G1) or 2 (G2)");
    NKR_TRY(group == 1 ? class_acc_alloc_t<Fq>(a, n) : class_acc_alloc_t<Fq2>(a, n));
    a.small.group = group;
    // 10-bit windows: 26 of them, so the Horner chain that ends the MSM has 25
    // additions between its ~250 doublings (37 for the cost model's 7-bit windows);
    // G2: the class sums and their psi images with 128-bit scalars, 13 windows
    const uint64_t pts = group == 1 ? kClassMax : 2ull * kClassMax;
    a.small.shape = msm_shape(pts, false, group, 10);
    if (group == 2) {
        a.small.shape.W = kPsiWindows;
        a.small.shape.nb = a.small.shape.B * uint32_t(kPsiWindows);
        NKR_TRY(a.split.alloc(pts * sizeof(Fr), "class value halves"));
    }
    NKR_TRY(a.small.pts.alloc(pts * (group == 1 ? sizeof(G1Affine) : sizeof(G2Affine)), "class sums (affine)"));
    // the MSM over the class values ends with a Horner chain of ~250 doublings;
    // G2 runs its reduction levels on lane pairs (half the chain's latency)
    a.small_s.acc.lane_pairs = group == 2;
    NKR_TRY(msm_scratch_alloc(a.small_s, group, a.small.shape));
    NKR_TRY(a.out.alloc(group == 1 ? 96 : 192, "class MSM result"));
    return NKR_B200_OK;
}

int msm_class_acc_issue(const MsmBases &b, const MsmClassSort &cs, const MsmDedup &d, MsmClassAcc &a,
                        cudaStream_t st)
{
    NKR_REQUIRE(b.group == a.small.group, "class path and bases of different groups");
    NKR_REQUIRE(cs.n == a.seg.n, "class sort and class sums of different supports");
    NKR_TRY(b.group == 1 ? class_acc_issue_t<Fq>(b, cs, a, st) : class_acc_issue_t<Fq2>(b, cs, a, st));
    if (b.group == 1) return msm_run(a.small, a.small_s, d.values.p, a.out.p, st);
    const unsigned g = blocks_for(kClassMax, 128);
    k_cls_psi<<<g, 128, 0, st>>>(a.small.pts.as<Affine<Fq2>>(), kClassMax);
    NKR_CHECK_LAUNCH();
    k_cls_split_psi<<<g, 128, 0, st>>>(d.values.as<Fr>(), kClassMax, a.split.as<Fr>());
    NKR_CHECK_LAUNCH();
    return msm_run(a.small, a.small_s, a.split.p, a.out.p, st);
}

int msm_result_add(int group, void *out_dev, const void *add_dev, cudaStream_t st)
{
    NKR_REQUIRE(group == 1 || group == 2, "group must be 1 (G1) or 2 (G2)");
    if (group == 1)
        k_result_add<Fq><<<1, 32, 0, st>>>(static_cast<Fq *>(out_dev), static_cast<const Fq *>(add_dev));
    else
        k_result_add<Fq2><<<1, 32, 0, st>>>(static_cast<Fq2 *>(out_dev), static_cast<const Fq2 *>(add_dev));
    NKR_CHECK_LAUNCH();
    return NKR_B200_OK;
}

int msm_class_acc_run(const MsmBases &b, const MsmClassSort &cs, const MsmDedup &d, MsmClassAcc &a,
                      void *out_dev, cudaStream_t st)
{
    NKR_TRY(msm_class_acc_issue(b, cs, d, a, st));
    return msm_result_add(b.group, out_dev, a.out.p, st);
}

} // namespace nkr
