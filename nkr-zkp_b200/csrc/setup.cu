// Groth16 setup with caller-given toxic waste: the scalar part on the host,
// the fixed-base scalar multiplications on the GPU.
//
// Reference: CpuBackend::setup (protocols/groth16/backends/cpu/src/backend.cpp:
// 41-154) -- Lagrange values at t (libfqfft basic_radix2_domain_aux.tcc:182-237),
// A/B/C column sums, l / ic / h query scalars, then fixed-base MSMs with libff
// window tables (operators/include/nkr/operators/fixed_base_msm.hpp:14-39); and
// the CUDA setup (backends/cuda/src/groth16_backend.cu:105-212).  The reference
// draws t, alpha, beta, gamma, delta unseeded (backend.cpp:49-53); here they are
// inputs, so a seeded setup is reproducible.  The VK's pairing value
// e(alpha, beta) is not computed here (no pairing on this path): callers get
// alpha_g1 and beta_g2 and form it with their verifier.
#include <cstring>
#include <vector>

#include "../host/fr_host.hpp"
#include "common.cuh"
#include "curve.cuh"
#include "prover.cuh"

namespace nkr {

namespace {

constexpr int kFbWindows = 32; // 8-bit windows over 256-bit scalars
constexpr int kFbChunk = 16;

__device__ __forceinline__ G1Affine g1_generator()
{
    // (1, 2) in Montgomery form
    Fq one = Fq::one();
    return {one, one + one};
}

// alt_bn128 G2 generator (alt_bn128_init.cpp), Montgomery limbs
__device__ __forceinline__ G2Affine g2_generator()
{
    const uint32_t x0[8] = {0x02bc2026u, 0x8e83b5d1u, 0x497b0172u, 0xdceb1935u,
                            0x97811adfu, 0xfbb82647u, 0xaf96503bu, 0x19573841u};
    const uint32_t x1[8] = {0xa84c6140u, 0xafb4737du, 0x5802d8c4u, 0x6043dd5au,
                            0x52a02f86u, 0x09e950fcu, 0x3aea7b6bu, 0x14fef083u};
    const uint32_t y0[8] = {0x886be9f6u, 0x619dfa9du, 0xf59e9b78u, 0xfe7fd297u,
                            0x231b7dfeu, 0xff9e1a62u, 0xae9e4206u, 0x28fd7eebu};
    const uint32_t y1[8] = {0xc71856eeu, 0x64095b56u, 0x327d3cbbu, 0xdc57f922u,
                            0x33351076u, 0x55f935beu, 0x93fd6482u, 0x0da4a0e6u};
    G2Affine g;
    for (int i = 0; i < 8; ++i) {
        g.x.c0.v[i] = x0[i];
        g.x.c1.v[i] = x1[i];
        g.y.c0.v[i] = y0[i];
        g.y.c1.v[i] = y1[i];
    }
    return g;
}

template <class F>
__device__ __forceinline__ Affine<F> generator();
template <>
__device__ __forceinline__ G1Affine generator<Fq>()
{
    return g1_generator();
}
template <>
__device__ __forceinline__ G2Affine generator<Fq2>()
{
    return g2_generator();
}

// table[w * 256 + j] = j * 2^(8 w) * G (XYZZ; j = 0 is infinity)
template <class F>
__global__ void k_fb_table(const Affine<F> *gen_override, Xyzz<F> *table)
{
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= kFbWindows * 256) return;
    const int w = idx >> 8, j = idx & 255;
    uint32_t k[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    // j << (8 w) as a 256-bit integer
    const int bit = 8 * w;
    k[bit >> 5] = uint32_t(j) << (bit & 31);
    if ((bit & 31) && (bit >> 5) + 1 < 8) k[(bit >> 5) + 1] = uint32_t(j) >> (32 - (bit & 31));
    const Affine<F> g = gen_override ? *gen_override : generator<F>();
    table[idx] = xyzz_mul_canon(g, k);
}

template <class F>
__global__ void k_fixed_base(const Affine<F> *__restrict__ table, const Fr *__restrict__ scalars,
                             Xyzz<F> *__restrict__ out, uint64_t n)
{
    const uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const Fr s = from_mont(scalars[i]);
    Xyzz<F> acc = Xyzz<F>::inf();
    for (int w = 0; w < kFbWindows; ++w) {
        const uint32_t byte = (s.v[w >> 2] >> (8 * (w & 3))) & 255u;
        if (byte) acc = xyzz_add_affine(acc, table[w * 256 + byte]);
    }
    out[i] = acc;
}

// XYZZ -> libff layout (X, Y, Z = 1) / (0, 1, 0); chunked batch inversion
template <class F>
__global__ void k_xyzz_to_libff(const Xyzz<F> *__restrict__ in, F *__restrict__ out, uint64_t n)
{
    const uint64_t t = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    const uint64_t beg = t * kFbChunk;
    if (beg >= n) return;
    const int cnt = int(n - beg < uint64_t(kFbChunk) ? n - beg : uint64_t(kFbChunk));
    F pre[kFbChunk];
    F acc = F::one();
    for (int j = 0; j < cnt; ++j) {
        pre[j] = acc;
        const Xyzz<F> p = in[beg + j];
        if (!p.is_inf()) acc = acc * (p.zz * p.zzz);
    }
    F inv = inverse(acc);
    for (int j = cnt - 1; j >= 0; --j) {
        const Xyzz<F> p = in[beg + j];
        F *o = out + 3 * (beg + j);
        if (p.is_inf()) {
            o[0] = F::zero();
            o[1] = F::one();
            o[2] = F::zero();
            continue;
        }
        const F d = p.zz * p.zzz;
        const F ti = inv * pre[j];
        inv = inv * d;
        o[0] = p.x * (ti * p.zzz);
        o[1] = p.y * (ti * p.zz);
        o[2] = F::one();
    }
}

// Fixed-base multiples k_i * G for a list of Fr scalars (host in, host out in
// libff layout), batched through device memory.
template <class F>
int fixed_base_t(const host::Fr *scalars, uint64_t n, void *out_host, DevBuf &table_aff,
                 cudaStream_t st)
{
    if (n == 0) return NKR_B200_OK;
    const size_t psz = 3 * sizeof(F);
    DevBuf ds, dx, dout;
    NKR_TRY(ds.alloc(n * 32, "setup scalars"));
    NKR_TRY(dx.alloc(n * sizeof(Xyzz<F>), "setup points"));
    NKR_TRY(dout.alloc(n * psz, "setup output"));
    NKR_CUDA(cudaMemcpyAsync(ds.p, scalars, n * 32, cudaMemcpyHostToDevice, st));
    k_fixed_base<F><<<blocks_for(n, 128), 128, 0, st>>>(table_aff.as<Affine<F>>(), ds.as<Fr>(),
                                                       dx.as<Xyzz<F>>(), n);
    NKR_CHECK_LAUNCH();
    k_xyzz_to_libff<F><<<blocks_for((n + kFbChunk - 1) / kFbChunk, 64), 64, 0, st>>>(
        dx.as<Xyzz<F>>(), dout.as<F>(), n);
    NKR_CHECK_LAUNCH();
    NKR_CUDA(cudaMemcpyAsync(out_host, dout.p, n * psz, cudaMemcpyDeviceToHost, st));
    NKR_CUDA(cudaStreamSynchronize(st));
    return NKR_B200_OK;
}

template <class F>
int build_table_t(DevBuf &table_aff, cudaStream_t st)
{
    const int entries = kFbWindows * 256;
    DevBuf tx;
    NKR_TRY(tx.alloc(entries * sizeof(Xyzz<F>), "fixed-base table"));
    NKR_TRY(table_aff.alloc(entries * sizeof(Affine<F>), "fixed-base table"));
    k_fb_table<F><<<blocks_for(entries, 64), 64, 0, st>>>(nullptr, tx.as<Xyzz<F>>());
    NKR_CHECK_LAUNCH();
    // reuse the libff converter, then drop Z (table entries are affine X, Y)
    DevBuf lib;
    NKR_TRY(lib.alloc(entries * 3 * sizeof(F), "fixed-base table"));
    k_xyzz_to_libff<F><<<blocks_for((entries + kFbChunk - 1) / kFbChunk, 64), 64, 0, st>>>(
        tx.as<Xyzz<F>>(), lib.as<F>(), entries);
    NKR_CHECK_LAUNCH();
    NKR_CUDA(cudaMemcpy2DAsync(table_aff.p, sizeof(Affine<F>), lib.p, 3 * sizeof(F),
                               sizeof(Affine<F>), entries, cudaMemcpyDeviceToDevice, st));
    NKR_CUDA(cudaStreamSynchronize(st));
    return NKR_B200_OK;
}

} // namespace

int setup_run(nkr_b200_ctx *ctx, const nkr_b200_circuit *c, const void *toxic_raw,
              const nkr_b200_setup_out *out)
{
    using host::Fr;
    NKR_REQUIRE(ctx && c && toxic_raw && out, "null argument");
    const uint64_t m = c->rows, cols = c->cols;
    const int logm = log2_exact(m);
    NKR_REQUIRE(logm >= 1 && logm <= 28, "constraint count must be a power of two in [2, 2^28]");
    NKR_REQUIRE(c->public_inputs + 1 <= cols, "public input count exceeds the variable count");
    Fr tox[5];
    std::memcpy(tox, toxic_raw, sizeof(tox));
    const Fr &t = tox[0], &alpha = tox[1], &beta = tox[2], &gamma = tox[3], &delta = tox[4];
    NKR_REQUIRE(!gamma.is_zero() && !delta.is_zero(), "gamma and delta must be nonzero");
    // domain generator w = 5^((r-1)/2^28) squared down to 2^logm; (r - 1) >> 28 from the modulus
    uint64_t q[4] = {host::kR[0] - 1, host::kR[1], host::kR[2], host::kR[3]};
    for (int k = 0; k < 28; ++k) {
        for (int i = 0; i < 3; ++i) q[i] = (q[i] >> 1) | (q[i + 1] << 63);
        q[3] >>= 1;
    }
    Fr w = host::pow(host::from_u64(5), q);
    for (int i = 28; i > logm; --i) w = w * w;
    // Z(t) = t^m - 1 and Lagrange values L_i(t) = Z(t)/m * w^i / (t - w^i)
    Fr tm = t;
    for (int i = 0; i < logm; ++i) tm = tm * tm;
    const Fr zt = tm - host::one();
    NKR_REQUIRE(!zt.is_zero(), "toxic t lies in the evaluation domain");
    std::vector<Fr> L(m), diff(m), pref(m);
    {
        Fr r = host::one();
        for (uint64_t i = 0; i < m; ++i) {
            diff[i] = t - r;
            r = r * w;
        }
        Fr acc = host::one();
        for (uint64_t i = 0; i < m; ++i) {
            pref[i] = acc;
            acc = acc * diff[i];
        }
        Fr inv = host::inverse(acc);
        for (uint64_t i = m; i-- > 0;) {
            L[i] = inv * pref[i]; // 1 / (t - w^i)
            inv = inv * diff[i];
        }
        Fr l = zt * host::inverse(host::from_u64(m));
        for (uint64_t i = 0; i < m; ++i) {
            L[i] = l * L[i];
            l = l * w;
        }
    }
    std::vector<Fr> at(cols, host::zero()), bt(cols, host::zero()), ct(cols, host::zero());
    std::vector<Fr> *acc3[3] = {&at, &bt, &ct};
    for (int k = 0; k < 3; ++k) {
        const Fr *vals = static_cast<const Fr *>(c->values[k]);
        for (uint64_t row = 0; row < m; ++row)
            for (uint32_t j = c->row_ptr[k][row]; j < c->row_ptr[k][row + 1]; ++j) {
                NKR_REQUIRE(c->col_idx[k][j] < cols, "column out of range");
                (*acc3[k])[c->col_idx[k][j]] += vals[j] * L[row];
            }
    }
    const Fr gi = host::inverse(gamma), di = host::inverse(delta);
    std::vector<Fr> lt(cols, host::zero()), ic(c->public_inputs + 1);
    for (uint64_t i = 0; i < cols; ++i) {
        const Fr s = beta * at[i] + alpha * bt[i] + ct[i];
        if (i > c->public_inputs)
            lt[i] = s * di;
        else
            ic[i] = s * gi;
    }
    std::vector<Fr> ht(m, host::zero());
    {
        Fr power = host::one();
        const Fr zd = zt * di;
        for (uint64_t i = 0; i + 1 < m; ++i) {
            ht[i] = power * zd;
            power = power * t;
        }
    }
    NKR_CUDA(cudaSetDevice(ctx->device));
    cudaStream_t st = ctx->stream;
    DevBuf t1, t2;
    NKR_TRY(build_table_t<Fq>(t1, st));
    NKR_TRY(build_table_t<Fq2>(t2, st));
    NKR_TRY(fixed_base_t<Fq>(at.data(), cols, out->a_query, t1, st));
    NKR_TRY(fixed_base_t<Fq>(bt.data(), cols, out->b_g1_query, t1, st));
    NKR_TRY(fixed_base_t<Fq2>(bt.data(), cols, out->b_g2_query, t2, st));
    NKR_TRY(fixed_base_t<Fq>(lt.data(), cols, out->l_query, t1, st));
    NKR_TRY(fixed_base_t<Fq>(ht.data(), m, out->h_query, t1, st));
    NKR_TRY(fixed_base_t<Fq>(ic.data(), ic.size(), out->ic, t1, st));
    const Fr g1s[3] = {alpha, beta, delta};
    uint8_t g1o[3 * 96];
    NKR_TRY(fixed_base_t<Fq>(g1s, 3, g1o, t1, st));
    std::memcpy(out->alpha_g1, g1o, 96);
    std::memcpy(out->beta_g1, g1o + 96, 96);
    std::memcpy(out->delta_g1, g1o + 192, 96);
    const Fr g2s[3] = {beta, delta, gamma};
    uint8_t g2o[3 * 192];
    NKR_TRY(fixed_base_t<Fq2>(g2s, 3, g2o, t2, st));
    std::memcpy(out->beta_g2, g2o, 192);
    std::memcpy(out->delta_g2, g2o + 192, 192);
    std::memcpy(out->gamma_g2, g2o + 384, 192);
    return NKR_B200_OK;
}

} // namespace nkr

extern "C" int nkr_b200_setup(nkr_b200_ctx *ctx, const nkr_b200_circuit *circuit,
                              const void *toxic, const nkr_b200_setup_out *out)
{
    return nkr::setup_run(ctx, circuit, toxic, out);
}
