// Groth16 blinding (common/src/protocol.cpp:85-94) with caller-given r, s:
//   A = alpha1 + ar + r delta1
//   B = beta2 + bs2 + s delta2
//   C = qz + zk + s A + r B1 - r s delta1
//     = qz + zk + s alpha1 + s ar + r beta1 + r bs1 + r s delta1
//
// Seven scalar multiplications, all of them latency chains for a single GPU
// thread if done by double-and-add (a 256-bit chain on G2 is milliseconds).
// Here:
//  - the five multiples of proving-key constants (r delta1, s alpha1, r beta1,
//    rs delta1 on G1, s delta2 on G2) are fixed-base: prepare tabulates
//    d 2^(8j) P for every 8-bit window j < 32 and digit d < 256 (affine), and one
//    warp sums the 32 looked-up points in five shuffle levels;
//  - the two multiples of proof points (s ar, r bs1) use the GLV endomorphism of
//    BN254 G1 (Gallant, Lambert and Vanstone, CRYPTO 2001): k = k1 + k2 lambda
//    (mod r) with |k1|, |k2| < 2^127, and k P = k1 P + k2 phi(P) with
//    phi(x, y) = (beta x, y).  A prove through nkr_b200_prove (slot 0) ends by
//    tabulating d 2^(8j) P (j < 16, d < 256) for its own ar and bs1 on a side
//    stream, behind the H MSM (glv_tables_issue); when the raw proof handed to
//    the blinding is that proof, one warp per point looks up the 32 digits of
//    k1 and k2 and sums them like the fixed bases.  Any other raw proof takes
//    the chain: the two 127-bit halves run as 4-bit window chains on two lanes
//    of the point's warp, from a 16-entry table its lanes build in parallel;
//  - curve arithmetic runs on the 52-bit-limb FP64 field (field52.cuh), whose
//    product has a fraction of the 32-bit Montgomery product's latency.
// The kernel returns A, B, C as Jacobian points; the host normalises them, as it
// does the raw proof.  Results are group elements, so they equal the
// reference's bit for bit once affine-normalised, whatever the addition order.
#define NKR_FIELD_MUL_OUTLINE 1
#include <algorithm>
#include <cstring>

#include "../host/fr_host.hpp"
#include "field52.cuh"
#include "prover.cuh"

namespace nkr {

namespace {

constexpr int kWindows = 32;     // 8-bit windows of a fixed-base scalar
constexpr int kDigits = 255;     // nonzero digits per window
constexpr int kFixedG1 = 3;      // alpha1, beta1, delta1
constexpr size_t kTabG1Bytes = size_t(kFixedG1) * kWindows * kDigits * sizeof(G1Affine);
constexpr size_t kTabG2Bytes = size_t(kWindows) * kDigits * sizeof(G2Affine);

// Host-prepared scalars of one blinding.
struct BlindScalars {
    uint32_t fixed[5][8]; // canonical r, s, r, r s, s for r delta1, s alpha1, r beta1, rs delta1, s delta2
    uint32_t glv[4][4];   // |k1|, |k2| of s (for s ar), then of r (for r bs1)
    uint32_t glv_neg;     // bit c: GLV half c is negative
    uint32_t glv_windows; // 4-bit windows of the longest half
    uint32_t pad[2];
};
static_assert(sizeof(BlindScalars) == 240, "BlindScalars layout");

// blind_io (device) and the slot's pinned staging share this layout
constexpr size_t kIoRaw = 0;       // ar, bs1, zk, qz (G1), bs2 (G2): libff, affine-normalised
constexpr size_t kIoScalars = 576; // BlindScalars
constexpr size_t kIoOut = 832;     // A (G1), B (G2), C (G1): libff Jacobian
constexpr size_t kIoBytes = kIoOut + 384;
static_assert(kIoScalars + sizeof(BlindScalars) <= kIoOut && kIoBytes <= kBlindStage, "io layout");

// a slot's GLV tables (Xyzz<Fq52> entries, R'): the bases ar and bs1, their
// powers Q_j = 2^(8j) P (j < 16), then d Q_j for d = 1..255
constexpr int kGlvWin = 16;
constexpr size_t kGlvPow = 2, kGlvTab = kGlvPow + 2 * kGlvWin;
constexpr size_t kGlvEntries = kGlvTab + 2 * kGlvWin * kDigits;

// pk_const layout: alpha1, beta1, delta1 (G1Affine), beta2, delta2 (G2Affine)
constexpr int kPkAlpha1 = 0, kPkBeta1 = 1, kPkDelta1 = 2, kPkBeta2 = 0, kPkDelta2 = 1;

// ---------------------------------------------------------------------------
// GLV constants of BN254 G1, derived from the curve: beta a primitive cube root
// of unity in Fq and lambda the cube root of unity in Fr with
// (beta x, y) = lambda (x, y); (a1, b1), (a2, b2) the short basis of the lattice
// {(a, b) : a + b lambda = 0 mod r} from the extended Euclidean algorithm on
// (r, lambda) (GLV section 4), b1 < 0 < a1, a2, b2, and a1 b2 - a2 b1 = r;
// g1 = round(b2 2^256 / r), g2 = round(-b1 2^256 / r).
// ---------------------------------------------------------------------------

// beta 2^260 mod p in 52-bit limbs (beta = 0x59e26bcea0d48bacd4f263f1acdb5c4f5763473177fffffe)
__device__ __forceinline__ Fq52 glv_beta()
{
    return {{0x917dda1583b6eull, 0xdc45aa1e7dcf6ull, 0x22e6f2c22a573ull, 0xd1f28e9f64523ull,
             0x1e37a68a14ddull}};
}

constexpr uint64_t kLambda[4] = {0x8b17ea66b99c90ddull, 0x5bfc41088d8daaa7ull, 0xb3c4d79d41a91758ull, 0};
constexpr uint64_t kGlvA1 = 0x89d3256894d213e3ull; // = b2
constexpr uint64_t kGlvA2[2] = {0x0be4e1541221250bull, 0x6f4d8248eeb859fdull};
constexpr uint64_t kGlvB1Abs[2] = {0x8211bbeb7d4f1128ull, 0x6f4d8248eeb859fcull};
constexpr uint64_t kGlvG1[3] = {0xd91d232ec7e0b3d7ull, 0x2ull, 0};
constexpr uint64_t kGlvG2[3] = {0x7a7bd9d4391eb18eull, 0x4ccef014a773d2cfull, 0x2ull};

using u128 = unsigned __int128;

// out[0, na + nb) = a b
void mul_limbs(const uint64_t *a, int na, const uint64_t *b, int nb, uint64_t *out)
{
    for (int i = 0; i < na + nb; ++i) out[i] = 0;
    for (int i = 0; i < na; ++i) {
        u128 carry = 0;
        for (int j = 0; j < nb; ++j) {
            const u128 t = u128(a[i]) * b[j] + out[i + j] + carry;
            out[i + j] = uint64_t(t);
            carry = t >> 64;
        }
        out[i + nb] = uint64_t(carry);
    }
}

u128 load128(const uint64_t *p) { return u128(p[0]) | (u128(p[1]) << 64); }

int bits128(u128 v)
{
    int n = 0;
    while (v) {
        ++n;
        v >>= 1;
    }
    return n;
}

// k (canonical, < r) -> k1 + k2 lambda with |k1|, |k2| < 2^127.  c_i = floor(k g_i /
// 2^256) is within (-1/8, 1 + 1/8) of the exact quotient k b2 / r (resp. -k b1 / r),
// so |k1| < 1.125 (a1 + a2) < 2^126 and |k2| < 1.125 (|b1| + b2) < 2^126: the
// halves are exact in 128-bit two's complement.  Returns false if the identity
// k = k1 + k2 lambda (mod r) fails (it cannot with these constants; checked
// because the result feeds a proof).
bool glv_split(const uint64_t k[4], uint32_t mag1[4], uint32_t mag2[4], bool &neg1, bool &neg2,
               int &bits)
{
    uint64_t p1[7], p2[7];
    mul_limbs(k, 4, kGlvG1, 3, p1);
    mul_limbs(k, 4, kGlvG2, 3, p2);
    const u128 c1 = load128(p1 + 4), c2 = load128(p2 + 4);
    const u128 k1 = load128(k) - c1 * kGlvA1 - c2 * load128(kGlvA2); // mod 2^128
    const u128 k2 = c1 * load128(kGlvB1Abs) - c2 * kGlvA1;
    neg1 = (k1 >> 127) != 0;
    neg2 = (k2 >> 127) != 0;
    const u128 m1 = neg1 ? u128(0) - k1 : k1, m2 = neg2 ? u128(0) - k2 : k2;
    bits = std::max(bits128(m1), bits128(m2));
    for (int i = 0; i < 4; ++i) {
        mag1[i] = uint32_t(m1 >> (32 * i));
        mag2[i] = uint32_t(m2 >> (32 * i));
    }
    const uint64_t w1[4] = {uint64_t(m1), uint64_t(m1 >> 64), 0, 0};
    const uint64_t w2[4] = {uint64_t(m2), uint64_t(m2 >> 64), 0, 0};
    host::Fr f1 = host::from_canonical(w1), f2 = host::from_canonical(w2);
    if (neg1) f1 = -f1;
    if (neg2) f2 = -f2;
    return f1 + f2 * host::from_canonical(kLambda) == host::from_canonical(k);
}

int blind_scalars(const void *r_mont, const void *s_mont, BlindScalars *o)
{
    host::Fr r, s;
    std::memcpy(r.v, r_mont, 32);
    std::memcpy(s.v, s_mont, 32);
    uint64_t rc[4], sc[4], rsc[4];
    host::to_canonical(r, rc);
    host::to_canonical(s, sc);
    host::to_canonical(r * s, rsc);
    std::memset(o, 0, sizeof(*o));
    const uint64_t *fixed[5] = {rc, sc, rc, rsc, sc};
    for (int t = 0; t < 5; ++t)
        std::memcpy(o->fixed[t], fixed[t], 32);
    bool n[4];
    int b_s = 0, b_r = 0;
    if (!glv_split(sc, o->glv[0], o->glv[1], n[0], n[1], b_s) ||
        !glv_split(rc, o->glv[2], o->glv[3], n[2], n[3], b_r)) {
        set_error("blind: GLV decomposition check failed");
        return NKR_B200_EINVAL;
    }
    for (int c = 0; c < 4; ++c) o->glv_neg |= uint32_t(n[c]) << c;
    o->glv_windows = uint32_t((std::max(b_s, b_r) + 3) / 4);
    return NKR_B200_OK;
}

// ---------------------------------------------------------------------------
// device helpers
// ---------------------------------------------------------------------------

__device__ __forceinline__ Fq52 shfl_down(const Fq52 &a, int off)
{
    Fq52 r;
#pragma unroll
    for (int i = 0; i < 5; ++i) r.l[i] = __shfl_down_sync(0xffffffffu, a.l[i], off);
    return r;
}
__device__ __forceinline__ Fq2x52 shfl_down(const Fq2x52 &a, int off)
{
    return {shfl_down(a.c0, off), shfl_down(a.c1, off)};
}
template <class C>
__device__ __forceinline__ Affine<C> shfl_down(const Affine<C> &p, int off)
{
    return {shfl_down(p.x, off), shfl_down(p.y, off)};
}
template <class C>
__device__ __forceinline__ Xyzz<C> shfl_down(const Xyzz<C> &p, int off)
{
    return {shfl_down(p.x, off), shfl_down(p.y, off), shfl_down(p.zz, off), shfl_down(p.zzz, off)};
}

// R-domain (2^256) storage -> R' compute form
__device__ __forceinline__ Fq52 to_r260(const Fq &x) { return r256_to_r260(to52(x)); }
__device__ __forceinline__ Fq2x52 to_r260(const Fq2 &x) { return {to_r260(x.c0), to_r260(x.c1)}; }

// an affine point stored in the R domain (pk_const; its infinity is (0, one))
template <class S>
__device__ __forceinline__ Affine<typename Compute<S>::type> affine_r260(const Affine<S> &p)
{
    using C = typename Compute<S>::type;
    if (p.is_inf()) return Affine<C>::inf();
    return {to_r260(p.x), to_r260(p.y)};
}

// a libff point (X, Y, Z) with Z in {0, 1}: Z = 0 is infinity
template <class S>
__device__ __forceinline__ Affine<typename Compute<S>::type> libff_affine_r260(const S *p)
{
    using C = typename Compute<S>::type;
    if (p[2].is_zero()) return Affine<C>::inf();
    return {to_r260(p[0]), to_r260(p[1])};
}

template <class C>
__device__ __forceinline__ Xyzz<C> xyzz_of(const Affine<C> &a)
{
    if (a.is_inf()) return Xyzz<C>::inf();
    return {a.x, a.y, C::one(), C::one()};
}

// Jacobian image of an XYZZ point (ZZ^3 = ZZZ^2): (X ZZ^2, Y ZZZ^2, ZZZ), written in
// libff layout in the R domain; infinity as (0, 1, 0)
template <class S, class C>
__device__ __forceinline__ void store_jacobian(const Xyzz<C> &p, S *out)
{
    if (p.is_inf()) {
        out[0] = S::zero();
        out[1] = S::one();
        out[2] = S::zero();
        return;
    }
    const C zz2 = sqr(p.zz), zzz2 = sqr(p.zzz);
    out[0] = to_storage(r260_to_r256(p.x * zz2));
    out[1] = to_storage(r260_to_r256(p.y * zzz2));
    out[2] = to_storage(r260_to_r256(p.zzz));
}

// k P for the fixed base P tabulated in tab ([32][255] affine, R' storage): lane j
// looks up the digit of window j; the warp sums the 32 points.  Valid in lane 0.
template <class S>
__device__ __forceinline__ Xyzz<typename Compute<S>::type> fixed_base_sum(const Affine<S> *tab,
                                                                           const uint32_t *k, int lane)
{
    using C = typename Compute<S>::type;
    const uint32_t d = (k[lane >> 2] >> (8 * (lane & 3))) & 255u;
    Affine<C> a = Affine<C>::inf();
    if (d) {
        const Affine<S> e = tab[lane * kDigits + d - 1];
        a = {to_compute(e.x), to_compute(e.y)};
    }
    const Affine<C> o = shfl_down(a, 16);
    Xyzz<C> acc = xyzz_add_affine(xyzz_of(a), o);
#pragma unroll 1
    for (int off = 8; off; off >>= 1) acc = xyzz_add(acc, shfl_down(acc, off));
    return acc;
}

// ---------------------------------------------------------------------------
// prepare: fixed-base tables
// ---------------------------------------------------------------------------

// Q_j = 2^(8j) P for the four fixed bases: warp w < 3 takes G1 base w (alpha1,
// beta1, delta1), warp 3 takes delta2; lane 0 runs the doubling chain.
__global__ void __launch_bounds__(128) k_fb_powers(const uint8_t *pk_const, Xyzz<Fq52> *pow1,
                                                   Xyzz<Fq2x52> *pow2)
{
    const int w = threadIdx.x >> 5;
    if (threadIdx.x & 31) return;
    if (w < kFixedG1) {
        const G1Affine *g1 = reinterpret_cast<const G1Affine *>(pk_const);
        Xyzz<Fq52> q = xyzz_of(affine_r260(g1[w]));
        for (int j = 0; j < kWindows; ++j) {
            pow1[w * kWindows + j] = q;
            if (j + 1 < kWindows)
                for (int i = 0; i < 8; ++i) q = xyzz_dbl(q);
        }
    } else {
        const G2Affine *g2 = reinterpret_cast<const G2Affine *>(pk_const + kFixedG1 * sizeof(G1Affine));
        Xyzz<Fq2x52> q = xyzz_of(affine_r260(g2[kPkDelta2]));
        for (int j = 0; j < kWindows; ++j) {
            pow2[j] = q;
            if (j + 1 < kWindows)
                for (int i = 0; i < 8; ++i) q = xyzz_dbl(q);
        }
    }
}

// tab[i] = d Q_{i / 255} with d = i % 255 + 1, affine in R' storage
template <class S>
__global__ void __launch_bounds__(128) k_fb_entries(const Xyzz<typename Compute<S>::type> *pow,
                                                    Affine<S> *tab, uint32_t count)
{
    using C = typename Compute<S>::type;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const Xyzz<C> q = pow[i / kDigits];
    const uint32_t d = i % kDigits + 1;
    Xyzz<C> acc = Xyzz<C>::inf();
    for (int b = 7; b >= 0; --b) {
        acc = xyzz_dbl(acc);
        if ((d >> b) & 1) acc = xyzz_add(acc, q);
    }
    const Affine<C> a = xyzz_to_affine(acc);
    tab[i] = {to_storage(a.x), to_storage(a.y)};
}

// ---------------------------------------------------------------------------
// prove side: GLV tables of the slot's ar and bs1
// ---------------------------------------------------------------------------

// out: the slot's results (libff Jacobian, R domain), ar at 0 and bs1 at 96.
// Lane pt < 2 converts its point to XYZZ (ZZ = Z^2, ZZZ = Z^3) and runs the
// doubling chain.
__global__ void __launch_bounds__(32) k_glv_pow(const uint8_t *out, Xyzz<Fq52> *t)
{
    const int pt = threadIdx.x;
    if (pt >= 2) return;
    const Fq *p = reinterpret_cast<const Fq *>(out + 96 * pt);
    Xyzz<Fq52> q = Xyzz<Fq52>::inf();
    if (!p[2].is_zero()) {
        const Fq52 z = to_r260(p[2]);
        const Fq52 zz = sqr(z);
        q = {to_r260(p[0]), to_r260(p[1]), zz, zz * z};
    }
    t[pt] = q;
    for (int j = 0; j < kGlvWin; ++j) {
        t[kGlvPow + pt * kGlvWin + j] = q;
        if (j + 1 < kGlvWin)
            for (int i = 0; i < 8; ++i) q = xyzz_dbl(q);
    }
}

__global__ void __launch_bounds__(256) k_glv_entries(Xyzz<Fq52> *t)
{
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= 2 * kGlvWin * kDigits) return;
    const Xyzz<Fq52> q = t[kGlvPow + i / kDigits];
    const uint32_t d = i % kDigits + 1;
    Xyzz<Fq52> acc = Xyzz<Fq52>::inf();
    for (int b = 7; b >= 0; --b) {
        acc = xyzz_dbl(acc);
        if ((d >> b) & 1) acc = xyzz_add(acc, q);
    }
    t[kGlvTab + i] = acc;
}

// ---------------------------------------------------------------------------
// the blinding kernel: warps 0-3 G1 fixed-base sums (r delta1, s alpha1,
// r beta1, rs delta1), warp 4 the G2 one (s delta2), warps 5 and 6 s ar and
// r bs1; then warps 0, 1, 2 assemble A, B, C.
// ---------------------------------------------------------------------------

__global__ void __launch_bounds__(224) k_blind(const G1Affine *g1tab, const G2Affine *g2tab,
                                               const uint8_t *pk_const, const Xyzz<Fq52> *glv,
                                               uint8_t *io)
{
    __shared__ Xyzz<Fq52> fix1[4];
    __shared__ Xyzz<Fq2x52> fix2;
    __shared__ Xyzz<Fq52> var[2];       // s ar, r bs1
    __shared__ Xyzz<Fq52> vtab[4][16];  // chain tables: d ar, d phi(ar), d bs1, d phi(bs1)
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const BlindScalars &sc = *reinterpret_cast<const BlindScalars *>(io + kIoScalars);
    const Fq *raw = reinterpret_cast<const Fq *>(io + kIoRaw);
    const G1Affine *pk1 = reinterpret_cast<const G1Affine *>(pk_const);
    const G2Affine *pk2 = reinterpret_cast<const G2Affine *>(pk_const + kFixedG1 * sizeof(G1Affine));

    if (warp < 4) {
        const int base = warp == 0 ? kPkDelta1 : warp == 1 ? kPkAlpha1 : warp == 2 ? kPkBeta1 : kPkDelta1;
        const Xyzz<Fq52> f = fixed_base_sum(g1tab + size_t(base) * kWindows * kDigits, sc.fixed[warp], lane);
        if (lane == 0) fix1[warp] = f;
    } else if (warp == 4) {
        const Xyzz<Fq2x52> f = fixed_base_sum(g2tab, sc.fixed[4], lane);
        if (lane == 0) fix2 = f;
    } else {
        // point pt (ar with s, bs1 with r); GLV halves c0 = 2 pt (k1), c0 + 1 (k2)
        const int pt = warp - 5, c0 = 2 * pt;
        const Affine<Fq52> p = libff_affine_r260(raw + 3 * pt);
        // is p the base the slot's last prove tabulated (x ZZ = X, y ZZZ = Y)?
        const Xyzz<Fq52> b = glv[pt];
        bool cached;
        if (b.is_inf() || p.is_inf()) {
            cached = b.is_inf() && p.is_inf();
        } else {
            Fq52 u, v;
            mul2(p.x, b.zz, p.y, b.zzz, u, v);
            cached = u == b.x && v == b.y;
        }
        Xyzz<Fq52> acc = Xyzz<Fq52>::inf();
        if (cached) {
            // lane h * 16 + j: digit j (8 bits) of half h over 2^(8j) P, or phi of it
            const int h = lane >> 4, j = lane & 15;
            const uint32_t d = (sc.glv[c0 + h][j >> 2] >> (8 * (j & 3))) & 255u;
            if (d) {
                acc = glv[kGlvTab + (pt * kGlvWin + j) * kDigits + d - 1];
                if (h) acc.x = acc.x * glv_beta();
                if ((sc.glv_neg >> (c0 + h)) & 1u) acc.y = neg(acc.y);
            }
#pragma unroll 1
            for (int off = 16; off; off >>= 1) acc = xyzz_add(acc, shfl_down(acc, off));
        } else {
            // lanes 0-15 tabulate d P and d phi(P) (d < 16); lanes 0, 1 run the halves
            const int d = lane & 15;
            Xyzz<Fq52> t = Xyzz<Fq52>::inf();
#pragma unroll 1
            for (int bit = 3; bit >= 0; --bit) {
                t = xyzz_dbl(t);
                if ((d >> bit) & 1) t = xyzz_add_affine(t, p);
            }
            if (lane < 16) {
                vtab[c0][d] = t;
                t.x = t.x * glv_beta();
                vtab[c0 + 1][d] = t;
            }
            __syncwarp();
            if (lane < 2) {
                const int c = c0 + lane;
                const uint32_t *m = sc.glv[c];
                const bool ng = (sc.glv_neg >> c) & 1u;
#pragma unroll 1
                for (int w = int(sc.glv_windows) - 1; w >= 0; --w) {
#pragma unroll 1
                    for (int i = 0; i < 4; ++i) acc = xyzz_dbl(acc);
                    const uint32_t dig = (m[w >> 3] >> (4 * (w & 7))) & 15u;
                    if (dig) {
                        Xyzz<Fq52> e = vtab[c][dig];
                        if (ng) e.y = neg(e.y);
                        acc = xyzz_add(acc, e);
                    }
                }
            }
            acc = xyzz_add(acc, shfl_down(acc, 1));
        }
        if (lane == 0) var[pt] = acc;
    }
    __syncthreads();

    if (warp == 0 && lane == 0) { // A = alpha1 + ar + r delta1
        Xyzz<Fq52> a = xyzz_add_affine(fix1[0], affine_r260(pk1[kPkAlpha1]));
        a = xyzz_add_affine(a, libff_affine_r260(raw));
        store_jacobian(a, reinterpret_cast<Fq *>(io + kIoOut));
    } else if (warp == 1 && lane == 0) { // B = beta2 + bs2 + s delta2
        Xyzz<Fq2x52> b = xyzz_add_affine(fix2, affine_r260(pk2[kPkBeta2]));
        b = xyzz_add_affine(b, libff_affine_r260(reinterpret_cast<const Fq2 *>(io + kIoRaw + 384)));
        store_jacobian(b, reinterpret_cast<Fq2 *>(io + kIoOut + 96));
    } else if (warp == 2) { // C = (s alpha1 + qz) + (s ar + zk) + (r beta1 + r bs1) + rs delta1
        Xyzz<Fq52> c = Xyzz<Fq52>::inf();
        if (lane == 0) c = xyzz_add_affine(fix1[1], libff_affine_r260(raw + 9));
        if (lane == 1) c = xyzz_add_affine(var[0], libff_affine_r260(raw + 6));
        if (lane == 2) c = xyzz_add(fix1[2], var[1]);
        if (lane == 3) c = fix1[3];
        c = xyzz_add(c, shfl_down(c, 2));
        c = xyzz_add(c, shfl_down(c, 1));
        if (lane == 0) store_jacobian(c, reinterpret_cast<Fq *>(io + kIoOut + 288));
    }
}

bool is_one(const host::Fq &z) { return z == host::Fq::one(); }

// Affine-normalise a libff point held as Z = 1, Z = 0 (infinity) or anything else.
void normalize_g1_if_needed(uint8_t *p)
{
    host::Fq z;
    std::memcpy(z.v, p + 64, 32);
    if (!z.is_zero() && !is_one(z)) host::normalize_g1(p);
}

void normalize_g2_if_needed(uint8_t *p)
{
    host::Fq z0, z1;
    std::memcpy(z0.v, p + 128, 32);
    std::memcpy(z1.v, p + 160, 32);
    const bool inf = z0.is_zero() && z1.is_zero();
    if (!inf && !(is_one(z0) && z1.is_zero())) host::normalize_g2(p);
}

} // namespace

int blind_tables_build(nkr_b200_key *key, cudaStream_t st)
{
    NKR_TRY(key->blind_io.alloc(kIoBytes, "blinding io"));
    NKR_TRY(key->blind_tab.alloc(kTabG1Bytes + kTabG2Bytes, "fixed-base blinding tables"));
    DevBuf pow;
    NKR_TRY(pow.alloc(kFixedG1 * kWindows * sizeof(Xyzz<Fq52>) + kWindows * sizeof(Xyzz<Fq2x52>),
                      "fixed-base powers"));
    Xyzz<Fq52> *pow1 = pow.as<Xyzz<Fq52>>();
    Xyzz<Fq2x52> *pow2 = reinterpret_cast<Xyzz<Fq2x52> *>(pow1 + kFixedG1 * kWindows);
    k_fb_powers<<<1, 128, 0, st>>>(key->pk_const.as<uint8_t>(), pow1, pow2);
    NKR_CHECK_LAUNCH();
    const uint32_t n1 = kFixedG1 * kWindows * kDigits, n2 = kWindows * kDigits;
    G1Affine *t1 = key->blind_tab.as<G1Affine>();
    G2Affine *t2 = reinterpret_cast<G2Affine *>(key->blind_tab.as<uint8_t>() + kTabG1Bytes);
    k_fb_entries<Fq><<<blocks_for(n1, 128), 128, 0, st>>>(pow1, t1, n1);
    NKR_CHECK_LAUNCH();
    k_fb_entries<Fq2><<<blocks_for(n2, 128), 128, 0, st>>>(pow2, t2, n2);
    NKR_CHECK_LAUNCH();
    NKR_CUDA(cudaStreamSynchronize(st)); // pow is released on return
    return NKR_B200_OK;
}

size_t glv_tables_bytes() { return kGlvEntries * sizeof(Xyzz<Fq52>); }

int glv_tables_issue(ProveSlot *sl, cudaStream_t st)
{
    Xyzz<Fq52> *t = sl->glv_tab.as<Xyzz<Fq52>>();
    k_glv_pow<<<1, 32, 0, st>>>(sl->out.as<uint8_t>(), t);
    NKR_CHECK_LAUNCH();
    k_glv_entries<<<blocks_for(2 * kGlvWin * kDigits, 256), 256, 0, st>>>(t);
    NKR_CHECK_LAUNCH();
    return NKR_B200_OK;
}

int key_blind(nkr_b200_key *key, const nkr_b200_raw_proof *raw, const void *r, const void *s,
              nkr_b200_proof *res)
{
    NKR_REQUIRE(key && raw && r && s && res, "null argument");
    NKR_CUDA(cudaSetDevice(key->ctx->device));
    ProveSlot *sl = key->slots[0].get();
    cudaStream_t s0 = sl->main();
    uint8_t *host = static_cast<uint8_t *>(sl->pinned_out) + kOutBytes;
    // the staging area is free once slot 0's queued work (an earlier blind) is done
    NKR_CUDA(cudaStreamSynchronize(s0));
    std::memcpy(host + kIoRaw + 0, raw->ar, 96);
    std::memcpy(host + kIoRaw + 96, raw->bs1, 96);
    std::memcpy(host + kIoRaw + 192, raw->zk, 96);
    std::memcpy(host + kIoRaw + 288, raw->qz, 96);
    std::memcpy(host + kIoRaw + 384, raw->bs2, 192);
    for (int i = 0; i < 4; ++i) normalize_g1_if_needed(host + kIoRaw + 96 * i);
    normalize_g2_if_needed(host + kIoRaw + 384);
    NKR_TRY(blind_scalars(r, s, reinterpret_cast<BlindScalars *>(host + kIoScalars)));
    uint8_t *io = key->blind_io.as<uint8_t>();
    NKR_CUDA(cudaMemcpyAsync(io, host, kIoScalars + sizeof(BlindScalars), cudaMemcpyHostToDevice, s0));
    const G1Affine *t1 = key->blind_tab.as<G1Affine>();
    const G2Affine *t2 = reinterpret_cast<const G2Affine *>(key->blind_tab.as<uint8_t>() + kTabG1Bytes);
    k_blind<<<1, 224, 0, s0>>>(t1, t2, key->pk_const.as<uint8_t>(), sl->glv_tab.as<Xyzz<Fq52>>(), io);
    NKR_CHECK_LAUNCH();
    NKR_CUDA(cudaMemcpyAsync(host + kIoOut, io + kIoOut, 384, cudaMemcpyDeviceToHost, s0));
    NKR_CUDA(cudaStreamSynchronize(s0));
    uint8_t *o = host + kIoOut;
    host::normalize_g1(o);
    host::normalize_g2(o + 96);
    host::normalize_g1(o + 288);
    std::memcpy(res->a, o, 96);
    std::memcpy(res->b, o + 96, 192);
    std::memcpy(res->c, o + 288, 96);
    return NKR_B200_OK;
}

} // namespace nkr
