// Pippenger MSM kernels (design notes in msm.cuh).
#include "msm.cuh"
#include "scan.cuh"

namespace nkr {

namespace {

template <int G>
struct GroupField;
template <>
struct GroupField<1> {
    using F = Fq;
};
template <>
struct GroupField<2> {
    using F = Fq2;
};

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

// Walks the signed digits of one scalar; calls f(k, bucket_in_set, negative)
// for every nonzero digit.  Digits: v = bits + carry; v > 2^(c-1) -> v - 2^c.
template <class Fn>
__device__ __forceinline__ void for_each_digit(const Fr &s, int c, int W, Fn &&f)
{
    uint32_t carry = 0;
    const uint32_t half = 1u << (c - 1), full = 1u << c;
    for (int k = 0; k < W; ++k) {
        uint32_t v = window_bits(s, k * c, c) + carry;
        bool has = false, negd = false;
        uint32_t mag = 0;
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

__global__ void k_digits_count(const Fr *__restrict__ scalars, uint64_t n, int c, int W,
                               bool folded, uint32_t B, Fr *__restrict__ canon,
                               uint32_t *__restrict__ counts)
{
    const uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    const bool live = i < n;
    Fr s = Fr::zero();
    if (live) {
        s = from_mont(scalars[i]);
        canon[i] = s;
    }
    const int lane = threadIdx.x & 31;
    for_each_digit(s, c, W, [&](int k, bool has, uint32_t b, bool) {
        has = has && live;
        const unsigned act = __ballot_sync(0xffffffffu, has);
        if (has) {
            const uint32_t bucket = (folded ? 0u : uint32_t(k) * B) + b;
            const unsigned peers = __match_any_sync(act, bucket);
            if (lane == __ffs(peers) - 1) atomicAdd(&counts[bucket], uint32_t(__popc(peers)));
        }
    });
}

__global__ void k_scatter(const Fr *__restrict__ canon, uint64_t n, int c, int W, bool folded,
                          uint32_t B, uint32_t *__restrict__ cursor, uint32_t *__restrict__ entries)
{
    const uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    const bool live = i < n;
    const Fr s = live ? canon[i] : Fr::zero();
    const int lane = threadIdx.x & 31;
    for_each_digit(s, c, W, [&](int k, bool has, uint32_t b, bool negd) {
        has = has && live;
        const unsigned act = __ballot_sync(0xffffffffu, has);
        if (has) {
            const uint32_t bucket = (folded ? 0u : uint32_t(k) * B) + b;
            const unsigned peers = __match_any_sync(act, bucket);
            const int leader = __ffs(peers) - 1;
            uint32_t base = 0;
            if (lane == leader) base = atomicAdd(&cursor[bucket], uint32_t(__popc(peers)));
            base = __shfl_sync(peers, base, leader);
            const uint32_t rank = __popc(peers & ((1u << lane) - 1u));
            const uint32_t point = folded ? uint32_t(uint64_t(k) * n + i) : uint32_t(i);
            entries[base + rank] = point | (negd ? 0x80000000u : 0u);
        }
    });
}

struct LoadTasks {
    const uint32_t *counts;
    uint32_t k1;
    __device__ __forceinline__ uint32_t operator()(uint64_t i) const
    {
        return (counts[i] + k1 - 1) / k1;
    }
};

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

template <class F>
__global__ void __launch_bounds__(128) k_acc_l1(const uint32_t *__restrict__ task_off,
                                                 const uint32_t *__restrict__ offsets,
                                                 const uint32_t *__restrict__ entries,
                                                 const Affine<F> *__restrict__ pts, uint32_t nb,
                                                 int k1, uint32_t *__restrict__ task_bucket,
                                                 Xyzz<F> *__restrict__ partials,
                                                 Xyzz<F> *__restrict__ buckets)
{
    const uint32_t T1 = task_off[nb];
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= T1) return;
    const uint32_t b = upper_bound_u32(task_off, nb + 1, t) - 1;
    const uint32_t ts = task_off[b], te = task_off[b + 1];
    const uint32_t beg = offsets[b] + (t - ts) * uint32_t(k1);
    const uint32_t end = min(beg + uint32_t(k1), offsets[b + 1]);
    Xyzz<F> acc = Xyzz<F>::inf();
    for (uint32_t j = beg; j < end; ++j) {
        const uint32_t e = entries[j];
        Affine<F> p = pts[e & 0x7fffffffu];
        if (e >> 31) p = affine_neg(p);
        acc = xyzz_add_affine(acc, p);
    }
    task_bucket[t] = b;
    if (te - ts == 1)
        buckets[b] = acc;
    else
        partials[t] = acc;
}

template <class F>
__global__ void __launch_bounds__(128) k_acc_up(const uint32_t *__restrict__ task_off, uint32_t nb,
                                                 const uint32_t *__restrict__ task_bucket,
                                                 Xyzz<F> *__restrict__ partials,
                                                 Xyzz<F> *__restrict__ buckets, uint32_t stride,
                                                 uint32_t k2)
{
    const uint32_t T1 = task_off[nb];
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= T1) return;
    const uint32_t b = task_bucket[t];
    const uint32_t ts = task_off[b], te = task_off[b + 1];
    const uint32_t cnt = te - ts;
    if (cnt == 1) return;
    const uint32_t r = t - ts;
    const uint64_t group = uint64_t(stride) * k2;
    if (r % group) return;
    const uint32_t live = (cnt + stride - 1) / stride; // partials left from the previous level
    if (live <= 1) return;
    Xyzz<F> acc = Xyzz<F>::inf();
    for (uint32_t m = 0; m < k2; ++m) {
        const uint64_t idx = uint64_t(r) + uint64_t(m) * stride;
        if (idx >= cnt) break;
        acc = xyzz_add(acc, partials[ts + idx]);
    }
    if (live <= k2)
        buckets[b] = acc;
    else
        partials[t] = acc;
}

// --------------------------------------------------------------------------
// bucket reduction: sum_b b * S_b per set, then + sum_b S_b
// --------------------------------------------------------------------------

template <class F>
__global__ void __launch_bounds__(128) k_reduce_level(const Xyzz<F> *__restrict__ a_in,
                                                       const Xyzz<F> *__restrict__ r_in,
                                                       uint32_t sets, uint32_t m, uint32_t L,
                                                       int log2_unit, Xyzz<F> *__restrict__ a_out,
                                                       Xyzz<F> *__restrict__ r_out)
{
    const uint32_t cps = m / L;
    const uint64_t t = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (t >= uint64_t(sets) * cps) return;
    const uint64_t base = (t / cps) * m + (t % cps) * L;
    Xyzz<F> run = Xyzz<F>::inf(), tri = Xyzz<F>::inf(), asum = Xyzz<F>::inf();
    for (int i = int(L) - 1; i >= 0; --i) {
        run = xyzz_add(run, r_in[base + i]);
        if (i > 0) tri = xyzz_add(tri, run);
        if (a_in) asum = xyzz_add(asum, a_in[base + i]);
    }
    for (int d = 0; d < log2_unit; ++d) tri = xyzz_dbl(tri);
    a_out[t] = xyzz_add(tri, asum);
    r_out[t] = run;
}

template <class F>
__device__ __forceinline__ void store_jacobian_layout(const Affine<F> &a, F *out)
{
    if (a.is_inf()) {
        out[0] = F::zero();
        out[1] = F::one();
        out[2] = F::zero();
    } else {
        out[0] = a.x;
        out[1] = a.y;
        out[2] = F::one();
    }
}

template <class F>
__global__ void k_finalize(const Xyzz<F> *a, const Xyzz<F> *r, int sets, int c, F *out)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    Xyzz<F> acc = Xyzz<F>::inf();
    for (int k = sets - 1; k >= 0; --k) {
        if (k != sets - 1)
            for (int d = 0; d < c; ++d) acc = xyzz_dbl(acc);
        acc = xyzz_add(acc, xyzz_add(a[k], r[k]));
    }
    store_jacobian_layout(xyzz_to_affine(acc), out);
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

// XYZZ -> affine: 1/ZZ = t ZZZ, 1/ZZZ = t ZZ with t = 1/(ZZ ZZZ)
template <class F>
__global__ void k_xyzz_to_affine(const Xyzz<F> *__restrict__ in, Affine<F> *__restrict__ out,
                                 uint64_t n)
{
    const uint64_t t = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    const uint64_t beg = t * kNormChunk;
    if (beg >= n) return;
    const int cnt = int(n - beg < uint64_t(kNormChunk) ? n - beg : uint64_t(kNormChunk));
    F pre[kNormChunk];
    F acc = F::one();
    for (int j = 0; j < cnt; ++j) {
        pre[j] = acc;
        const Xyzz<F> p = in[beg + j];
        if (!p.is_inf()) acc = acc * (p.zz * p.zzz);
    }
    F inv = inverse(acc);
    for (int j = cnt - 1; j >= 0; --j) {
        const Xyzz<F> p = in[beg + j];
        if (p.is_inf()) {
            out[beg + j] = Affine<F>::inf();
            continue;
        }
        const F d = p.zz * p.zzz;
        const F ti = inv * pre[j];
        inv = inv * d;
        out[beg + j] = {p.x * (ti * p.zzz), p.y * (ti * p.zz)};
    }
}

// out[i] = 2^c * in[i]
template <class F>
__global__ void k_dbl_c(const Affine<F> *__restrict__ in, Xyzz<F> *__restrict__ out, uint64_t n,
                        int c)
{
    const uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const Affine<F> p = in[i];
    if (p.is_inf()) {
        out[i] = Xyzz<F>::inf();
        return;
    }
    Xyzz<F> x = xyzz_from_affine_dbl(p);
    for (int d = 1; d < c; ++d) x = xyzz_dbl(x);
    out[i] = x;
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

template <class F>
int build_windows_t(MsmBases &b, cudaStream_t st)
{
    const MsmShape &sh = b.shape;
    Affine<F> *pts = b.pts.as<Affine<F>>();
    DevBuf tmp;
    NKR_TRY(tmp.alloc(sh.n * sizeof(Xyzz<F>), "window copy scratch"));
    const uint64_t chunks = (sh.n + kNormChunk - 1) / kNormChunk;
    for (int k = 1; k < sh.W; ++k) {
        k_dbl_c<F><<<blocks_for(sh.n, 128), 128, 0, st>>>(pts + uint64_t(k - 1) * sh.n,
                                                          tmp.as<Xyzz<F>>(), sh.n, sh.c);
        NKR_CHECK_LAUNCH();
        k_xyzz_to_affine<F><<<blocks_for(chunks, 64), 64, 0, st>>>(tmp.as<Xyzz<F>>(),
                                                                   pts + uint64_t(k) * sh.n, sh.n);
        NKR_CHECK_LAUNCH();
    }
    NKR_CUDA(cudaStreamSynchronize(st));
    return NKR_B200_OK;
}

template <class F>
int msm_run_t(const MsmBases &bs, MsmScratch &s, const void *scalars_dev, void *out_dev,
              cudaStream_t st)
{
    const MsmShape &sh = bs.shape;
    const uint64_t n = sh.n;
    NKR_CUDA(cudaMemsetAsync(s.counts.p, 0, (sh.nb + 1) * 4, st));
    NKR_CUDA(cudaMemsetAsync(s.buckets.p, 0, uint64_t(sh.nb) * sizeof(Xyzz<F>), st));
    if (n) {
        k_digits_count<<<blocks_for(n, 256), 256, 0, st>>>(
            static_cast<const Fr *>(scalars_dev), n, sh.c, sh.W, sh.folded, sh.B, s.canon.as<Fr>(),
            s.counts.as<uint32_t>());
        NKR_CHECK_LAUNCH();
    }
    NKR_TRY(scan_exclusive(LoadU32{s.counts.as<uint32_t>()}, sh.nb, s.offsets.as<uint32_t>(),
                           s.scan_tmp.as<uint32_t>(), st));
    NKR_TRY(scan_exclusive(LoadTasks{s.counts.as<uint32_t>(), uint32_t(sh.k1)}, sh.nb,
                           s.task_off.as<uint32_t>(), s.scan_tmp.as<uint32_t>(), st));
    NKR_CUDA(cudaMemcpyAsync(s.cursor.p, s.offsets.p, uint64_t(sh.nb) * 4,
                             cudaMemcpyDeviceToDevice, st));
    if (n) {
        k_scatter<<<blocks_for(n, 256), 256, 0, st>>>(s.canon.as<Fr>(), n, sh.c, sh.W, sh.folded,
                                                      sh.B, s.cursor.as<uint32_t>(),
                                                      s.entries.as<uint32_t>());
        NKR_CHECK_LAUNCH();
    }
    const uint64_t tmax = sh.tasks_max();
    const unsigned tb = blocks_for(tmax, 128);
    if (s.timing) NKR_CUDA(cudaEventRecord(s.ev_acc[0], st));
    k_acc_l1<F><<<tb, 128, 0, st>>>(s.task_off.as<uint32_t>(), s.offsets.as<uint32_t>(),
                                    s.entries.as<uint32_t>(), bs.pts.as<Affine<F>>(), sh.nb, sh.k1,
                                    s.task_bucket.as<uint32_t>(), s.partials.as<Xyzz<F>>(),
                                    s.buckets.as<Xyzz<F>>());
    NKR_CHECK_LAUNCH();
    if (s.timing) NKR_CUDA(cudaEventRecord(s.ev_acc[1], st));
    // fix-up levels until one task's fan-in covers the largest possible bucket
    for (uint64_t stride = 1; stride < tmax; stride *= uint64_t(sh.k2)) {
        k_acc_up<F><<<tb, 128, 0, st>>>(s.task_off.as<uint32_t>(), sh.nb,
                                        s.task_bucket.as<uint32_t>(), s.partials.as<Xyzz<F>>(),
                                        s.buckets.as<Xyzz<F>>(), uint32_t(stride), uint32_t(sh.k2));
        NKR_CHECK_LAUNCH();
    }
    // bucket reduction levels
    const uint32_t sets = sh.folded ? 1u : uint32_t(sh.W);
    uint32_t m = sh.B;
    const Xyzz<F> *a_in = nullptr;
    const Xyzz<F> *r_in = s.buckets.as<Xyzz<F>>();
    Xyzz<F> *bufs_a[2] = {s.red_a.as<Xyzz<F>>(), s.red_a2.as<Xyzz<F>>()};
    Xyzz<F> *bufs_r[2] = {s.red_r.as<Xyzz<F>>(), s.red_r2.as<Xyzz<F>>()};
    int flip = 0, log2_unit = 0;
    while (m > 1) {
        const uint32_t L = m >= 8 ? 8u : m;
        const uint64_t threads = uint64_t(sets) * (m / L);
        k_reduce_level<F><<<blocks_for(threads, 128), 128, 0, st>>>(
            a_in, r_in, sets, m, L, log2_unit, bufs_a[flip], bufs_r[flip]);
        NKR_CHECK_LAUNCH();
        a_in = bufs_a[flip];
        r_in = bufs_r[flip];
        flip ^= 1;
        m /= L;
        log2_unit += (L == 8 ? 3 : (L == 4 ? 2 : (L == 2 ? 1 : 0)));
    }
    if (a_in == nullptr) {
        // a single bucket per set: weight 1 each
        NKR_CUDA(cudaMemsetAsync(s.red_a.p, 0, uint64_t(sets) * sizeof(Xyzz<F>), st));
        a_in = s.red_a.as<Xyzz<F>>();
    }
    k_finalize<F><<<1, 32, 0, st>>>(a_in, r_in, int(sets), sh.c, static_cast<F *>(out_dev));
    NKR_CHECK_LAUNCH();
    return NKR_B200_OK;
}

template <class F>
int scratch_alloc_t(MsmScratch &s, const MsmShape &sh)
{
    const uint64_t tmax = sh.tasks_max();
    const uint32_t sets = sh.folded ? 1u : uint32_t(sh.W);
    const uint64_t red = uint64_t(sets) * (sh.B / 8 + 1);
    NKR_TRY(s.canon.alloc(std::max<uint64_t>(sh.n, 1) * sizeof(Fr), "msm canonical scalars"));
    NKR_TRY(s.counts.alloc((sh.nb + 1) * 4ull, "msm bucket counts"));
    NKR_TRY(s.offsets.alloc((sh.nb + 1) * 4ull, "msm bucket offsets"));
    NKR_TRY(s.cursor.alloc((sh.nb + 1) * 4ull, "msm scatter cursor"));
    NKR_TRY(s.task_off.alloc((sh.nb + 1) * 4ull, "msm task offsets"));
    NKR_TRY(s.entries.alloc(std::max<uint64_t>(sh.entries_max(), 1) * 4, "msm entries"));
    NKR_TRY(s.task_bucket.alloc(tmax * 4, "msm task buckets"));
    NKR_TRY(s.partials.alloc(tmax * sizeof(Xyzz<F>), "msm partial sums"));
    NKR_TRY(s.buckets.alloc(uint64_t(sh.nb) * sizeof(Xyzz<F>), "msm buckets"));
    NKR_TRY(s.red_a.alloc(red * sizeof(Xyzz<F>), "msm reduction"));
    NKR_TRY(s.red_r.alloc(red * sizeof(Xyzz<F>), "msm reduction"));
    NKR_TRY(s.red_a2.alloc(red * sizeof(Xyzz<F>), "msm reduction"));
    NKR_TRY(s.red_r2.alloc(red * sizeof(Xyzz<F>), "msm reduction"));
    NKR_TRY(s.scan_tmp.alloc(scan_scratch_words(sh.nb) * 4, "msm scan scratch"));
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
    if (c_override > 0) {
        c = c_override;
    } else if (folded) {
        c = lg - 4; // one bucket set: larger windows pay off
        if (group == 2) c -= 1;
    } else {
        c = lg - 5;
    }
    if (c < 4) c = 4;
    if (c > 20) c = 20;
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
    NKR_CUDA(cudaStreamSynchronize(st));
    return NKR_B200_OK;
}

int msm_scratch_alloc(MsmScratch &s, int group, const MsmShape &shape)
{
    NKR_TRY(group == 1 ? scratch_alloc_t<Fq>(s, shape) : scratch_alloc_t<Fq2>(s, shape));
    NKR_TRY(s.result.alloc(192, "msm result"));
    return NKR_B200_OK;
}

int msm_run(const MsmBases &b, MsmScratch &s, const void *scalars_dev, void *out_dev,
            cudaStream_t st)
{
    return b.group == 1 ? msm_run_t<Fq>(b, s, scalars_dev, out_dev, st)
                        : msm_run_t<Fq2>(b, s, scalars_dev, out_dev, st);
}

} // namespace nkr
