// Elementwise field / group kernels behind nkr_b200_field_op and
// nkr_b200_group_op (used by the parity tests against the oracle), and the
// Montgomery-product throughput microbenchmark that gives the integer roofline.
#include "field52.cuh"
#include "curve.cuh"
#include "ops.cuh"

namespace nkr {

namespace {

template <class F>
__device__ __forceinline__ F field_apply(int op, const F &a, const F &b)
{
    switch (op) {
    case 0: return a * b;
    case 1: return a + b;
    case 2: return a - b;
    case 3: return sqr(a);
    case 4: return inverse(a);
    default: return a;
    }
}

template <class P>
__global__ void k_field_op(int op, const Fp<P> *a, const Fp<P> *b, Fp<P> *out, uint64_t n)
{
    const uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    if (op == 5)
        out[i] = to_mont(a[i]);
    else if (op == 6)
        out[i] = from_mont(a[i]);
    else
        out[i] = field_apply(op, a[i], b ? b[i] : a[i]);
}

__global__ void k_fq2_op(int op, const Fq2 *a, const Fq2 *b, Fq2 *out, uint64_t n)
{
    const uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const Fq2 x = a[i], y = b ? b[i] : a[i];
    Fq2 r;
    switch (op) {
    case 0: r = x * y; break;
    case 1: r = x + y; break;
    case 2: r = x - y; break;
    case 3: r = sqr(x); break;
    case 4: r = inverse(x); break;
    default: r = x;
    }
    out[i] = r;
}

// The same ops in the FP64-limb arithmetic (R' = 2^260): inputs and outputs in
// the library's R = 2^256 Montgomery form, converted at both ends.
template <class S>
__global__ void k_field52_op(int op, const S *a, const S *b, S *out, uint64_t n)
{
    using C = typename Compute<S>::type;
    const uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const C x = r256_to_r260(to_compute(a[i]));
    const C y = r256_to_r260(to_compute(b ? b[i] : a[i]));
    C r;
    switch (op) {
    case 0: r = x * y; break;
    case 1: r = x + y; break;
    case 2: r = x - y; break;
    case 3: r = sqr(x); break;
    default: r = neg(x);
    }
    out[i] = to_storage(r260_to_r256(r));
}

// points in libff layout (X, Y, Z) with Z in {0, 1}
template <class F>
__global__ void k_group_op(int op, const F *a, const F *b, F *out, uint64_t n)
{
    const uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const F *pa = a + 3 * i;
    const Affine<F> pa_aff = pa[2].is_zero() ? Affine<F>::inf() : Affine<F>{pa[0], pa[1]};
    Xyzz<F> r;
    if (op == 0) {
        const F *pb = b + 3 * i;
        const Affine<F> pb_aff = pb[2].is_zero() ? Affine<F>::inf() : Affine<F>{pb[0], pb[1]};
        // exercise both the mixed and the XYZZ + XYZZ additions
        const Xyzz<F> xa = xyzz_add_affine(Xyzz<F>::inf(), pa_aff);
        const Xyzz<F> xb = xyzz_add_affine(Xyzz<F>::inf(), pb_aff);
        r = (i & 1) ? xyzz_add(xa, xb) : xyzz_add_affine(xa, pb_aff);
    } else if (op == 1) {
        r = xyzz_dbl(xyzz_add_affine(Xyzz<F>::inf(), pa_aff));
    } else {
        const Fr k = from_mont(reinterpret_cast<const Fr *>(b)[i]);
        r = xyzz_mul_canon(pa_aff, k.v);
    }
    const Affine<F> o = xyzz_to_affine(r);
    F *po = out + 3 * i;
    if (o.is_inf()) {
        po[0] = F::zero();
        po[1] = F::one();
        po[2] = F::zero();
    } else {
        po[0] = o.x;
        po[1] = o.y;
        po[2] = F::one();
    }
}

// Each thread runs 4 independent product chains; the result is stored so the
// work cannot be eliminated.  variant 0: operator* (64-bit accumulation CIOS),
// 1: mont_mul_cc (PTX carry-chain CIOS), 2: squaring; k_bench_mul52 below is
// variant 3 (the 52-bit-limb FP64 product, canonical) and 4 (lazily reduced).
constexpr int kBenchIters = 256;
template <class P, int V>
__global__ void __launch_bounds__(256) k_bench_mul(const Fp<P> *seed, Fp<P> *sink)
{
    const uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    Fp<P> a = seed[i & 255], b = seed[(i + 1) & 255], c = seed[(i + 2) & 255], d = seed[(i + 3) & 255];
    const Fp<P> m = seed[(i + 7) & 255];
    for (int k = 0; k < kBenchIters; ++k) {
        if (V == 1) {
            a = mont_mul_cc(a, m);
            b = mont_mul_cc(b, m);
            c = mont_mul_cc(c, m);
            d = mont_mul_cc(d, m);
        } else if (V == 2) {
            a = sqr(a);
            b = sqr(b);
            c = sqr(c);
            d = sqr(d);
        } else {
            a = a * m;
            b = b * m;
            c = c * m;
            d = d * m;
        }
    }
    const Fp<P> r = a + b + c + d;
    if (r.v[0] == 0x12345678u) sink[i] = r;
}

template <class P>
__global__ void k_check_wide(const Fp<P> *a, const Fp<P> *b, uint32_t *bad, int n)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n && mont_mul_cc(a[i], b[i]) != a[i] * b[i]) atomicAdd(bad, 1u);
}

// The 52-bit-limb product (R = 2^260) times 2^4 equals the library product (R = 2^256).
__global__ void k_check_52(const Fq *a, const Fq *b, uint32_t *bad, int n)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    Fq r = from52(mul52(to52(a[i]), to52(b[i])));
    for (int k = 0; k < 4; ++k) r = dbl(r);
    if (r != a[i] * b[i]) atomicAdd(bad, 1u);
}

// The lazily reduced product (values in [0, 2p)) agrees with the canonical one
// once canonicalised, also when an input is in [p, 2p).
__global__ void k_check_52l(const Fq *a, const Fq *b, uint32_t *bad, int n)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const Fq52 x = to52(a[i]), y = to52(b[i]);
    Fq52L xl = x, yl = y;
    const Fq52 want = mul52(x, y);
    if ((xl * yl).canon() != want) atomicAdd(bad, 1u);
    xl = xl + Fq52L(Fq52{{f52::p_limb(0), f52::p_limb(1), f52::p_limb(2), f52::p_limb(3), f52::p_limb(4)}});
    if ((xl * yl).canon() != want) atomicAdd(bad, 1u);
}

template <class T>
__device__ __forceinline__ Fq bench52_out(const T &x)
{
    if constexpr (T::kCanonical)
        return from52(x);
    else
        return from52(x.canon());
}

template <class T>
__global__ void __launch_bounds__(256) k_bench_mul52(const Fq *seed, Fq *sink)
{
    const uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    T a = Fq52(to52(seed[i & 255])), b = Fq52(to52(seed[(i + 1) & 255])),
      c = Fq52(to52(seed[(i + 2) & 255])), d = Fq52(to52(seed[(i + 3) & 255]));
    const T m = Fq52(to52(seed[(i + 7) & 255]));
    for (int k = 0; k < kBenchIters; ++k) {
        a = a * m;
        b = b * m;
        c = c * m;
        d = d * m;
    }
    const Fq r = bench52_out(a) + bench52_out(b) + bench52_out(c) + bench52_out(d);
    if (r.v[0] == 0x12345678u) sink[i] = r;
}

} // namespace

int field_op_device(int field, int op, const void *a, const void *b, void *out, uint64_t n,
                    cudaStream_t st)
{
    NKR_REQUIRE(op >= 0 && op <= 6, "field op %d unknown", op);
    const unsigned g = blocks_for(n, 128);
    if (n == 0) return NKR_B200_OK;
    if (field == 0)
        k_field_op<FrParams><<<g, 128, 0, st>>>(op, static_cast<const Fr *>(a),
                                                static_cast<const Fr *>(b), static_cast<Fr *>(out), n);
    else if (field == 1)
        k_field_op<FqParams><<<g, 128, 0, st>>>(op, static_cast<const Fq *>(a),
                                                static_cast<const Fq *>(b), static_cast<Fq *>(out), n);
    else if (field == 2) {
        NKR_REQUIRE(op <= 4, "Fq2 supports ops 0..4");
        k_fq2_op<<<g, 128, 0, st>>>(op, static_cast<const Fq2 *>(a), static_cast<const Fq2 *>(b),
                                    static_cast<Fq2 *>(out), n);
    } else if (field == 3 || field == 4) {
        NKR_REQUIRE(op <= 4, "52-bit-limb field ops are 0..3 and 4 (negation)");
        if (field == 3)
            k_field52_op<Fq><<<g, 128, 0, st>>>(op, static_cast<const Fq *>(a), static_cast<const Fq *>(b),
                                                static_cast<Fq *>(out), n);
        else
            k_field52_op<Fq2><<<g, 128, 0, st>>>(op, static_cast<const Fq2 *>(a),
                                                 static_cast<const Fq2 *>(b), static_cast<Fq2 *>(out), n);
    } else {
        NKR_REQUIRE(false, "field %d unknown", field);
    }
    NKR_CHECK_LAUNCH();
    return NKR_B200_OK;
}

int group_op_device(int group, int op, const void *a, const void *b, void *out, uint64_t n,
                    cudaStream_t st)
{
    NKR_REQUIRE(op >= 0 && op <= 2, "group op %d unknown", op);
    NKR_REQUIRE(group == 1 || group == 2, "group %d unknown", group);
    if (n == 0) return NKR_B200_OK;
    const unsigned g = blocks_for(n, 64);
    if (group == 1)
        k_group_op<Fq><<<g, 64, 0, st>>>(op, static_cast<const Fq *>(a), static_cast<const Fq *>(b),
                                          static_cast<Fq *>(out), n);
    else
        k_group_op<Fq2><<<g, 64, 0, st>>>(op, static_cast<const Fq2 *>(a),
                                           static_cast<const Fq2 *>(b), static_cast<Fq2 *>(out), n);
    NKR_CHECK_LAUNCH();
    return NKR_B200_OK;
}

int bench_mul_device(int field, int sm_count, double *muls_per_s, double *ms, cudaStream_t st)
{
    const unsigned blocks = unsigned(sm_count) * 16;
    const uint64_t threads = uint64_t(blocks) * 256;
    DevBuf seed, sink;
    NKR_TRY(seed.alloc(256 * 32, "bench seed"));
    NKR_TRY(sink.alloc(threads * 32, "bench sink"));
    // seeds: small canonical integers are valid field elements
    std::vector<uint32_t> h(256 * 8, 0);
    for (int i = 0; i < 256; ++i) {
        h[8 * i] = 0x9e3779b9u * (i + 1);
        h[8 * i + 1] = 0x7f4a7c15u * (i + 3);
        h[8 * i + 5] = 0x01234567u * (i + 5);
    }
    NKR_CUDA(cudaMemcpyAsync(seed.p, h.data(), 256 * 32, cudaMemcpyHostToDevice, st));
    cudaEvent_t e0, e1;
    NKR_CUDA(cudaEventCreate(&e0));
    NKR_CUDA(cudaEventCreate(&e1));
    float best = 1e30f;
    const int variant = field >> 8;
    field &= 0xff;
    if (variant == 1 || variant == 3 || variant == 4) {
        // the alternative product must agree with operator* before it is timed
        DevBuf bad;
        NKR_TRY(bad.alloc(4, "bench check"));
        NKR_CUDA(cudaMemsetAsync(bad.p, 0, 4, st));
        if (variant == 1)
            k_check_wide<FqParams><<<1, 256, 0, st>>>(seed.as<Fq>(), seed.as<Fq>() + 1,
                                                       bad.as<uint32_t>(), 255);
        else if (variant == 3)
            k_check_52<<<1, 256, 0, st>>>(seed.as<Fq>(), seed.as<Fq>() + 1, bad.as<uint32_t>(), 255);
        else
            k_check_52l<<<1, 256, 0, st>>>(seed.as<Fq>(), seed.as<Fq>() + 1, bad.as<uint32_t>(), 255);
        NKR_CHECK_LAUNCH();
        uint32_t nbad = 0;
        NKR_CUDA(cudaMemcpyAsync(&nbad, bad.p, 4, cudaMemcpyDeviceToHost, st));
        NKR_CUDA(cudaStreamSynchronize(st));
        NKR_REQUIRE(nbad == 0, "alternative product (variant %d) disagrees on %u inputs", variant, nbad);
    }
    for (int rep = 0; rep < 4; ++rep) {
        NKR_CUDA(cudaEventRecord(e0, st));
        if (field == 0 && variant == 0)
            k_bench_mul<FrParams, 0><<<blocks, 256, 0, st>>>(seed.as<Fr>(), sink.as<Fr>());
        else if (variant == 0)
            k_bench_mul<FqParams, 0><<<blocks, 256, 0, st>>>(seed.as<Fq>(), sink.as<Fq>());
        else if (variant == 1)
            k_bench_mul<FqParams, 1><<<blocks, 256, 0, st>>>(seed.as<Fq>(), sink.as<Fq>());
        else if (variant == 3)
            k_bench_mul52<Fq52><<<blocks, 256, 0, st>>>(seed.as<Fq>(), sink.as<Fq>());
        else if (variant == 4)
            k_bench_mul52<Fq52L><<<blocks, 256, 0, st>>>(seed.as<Fq>(), sink.as<Fq>());
        else
            k_bench_mul<FqParams, 2><<<blocks, 256, 0, st>>>(seed.as<Fq>(), sink.as<Fq>());
        NKR_CHECK_LAUNCH();
        NKR_CUDA(cudaEventRecord(e1, st));
        NKR_CUDA(cudaEventSynchronize(e1));
        float t;
        NKR_CUDA(cudaEventElapsedTime(&t, e0, e1));
        if (rep > 0 && t < best) best = t; // rep 0 is warm-up
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    NKR_CHECK_LAUNCH();
    *ms = best;
    *muls_per_s = double(threads) * kBenchIters * 4 / (best * 1e-3);
    return NKR_B200_OK;
}

} // namespace nkr
