// Radix-2 NTT over Fr for the Groth16 quotient chain.
//
// The reference computes H with libfqfft on the CPU (basic_radix2_domain.tcc:
// iFFT x3, cosetFFT x3, pointwise, divide_by_Z_on_coset, icosetFFT; CPU backend
// backends/cpu/src/backend.cpp:171-179) and with log2(N) global radix-2 passes
// or a three-pass on-chip variant on CUDA (operators/cuda/include/ntt/ntt.cuh:
// 110-207).  Outputs are unique field vectors, so any correct transform order
// is bit-exact against libfqfft.
//
// Layout: transforms are done in place in HBM.  A pass fuses up to 10 radix-2
// stages for one group of 2^t elements (stride 2^s_lo apart) in shared memory.
// Decimation in frequency (DIF) takes natural order to bit-reversed order,
// decimation in time (DIT) takes bit-reversed order back to natural, so the
// prover's chain never runs a separate bit-reversal pass:
//   evals --DIF(w^-1)--> coeffs (bitrev) --x T1, DIT(w)--> coset evals (natural)
//   pointwise (a b - c) / Z(g) --DIF(w^-1), x T2--> H coefficients (bitrev)
// with T1[j] = N^-1 g^bitrev(j) and T2[j] = N^-1 g^-bitrev(j) resident tables;
// the H MSM uses h_query stored in the same bit-reversed order.
#pragma once

#include <cstdint>
#include <memory>

#include "common.cuh"
#include "field.cuh"

namespace nkr {

// Resident twiddle and scale tables for one domain size N = 2^logn.
struct NttTables {
    int logn = 0;
    uint64_t n = 0;
    DevBuf tw_fwd;  // Fr[N]: entry 2^s + k = w_{2^(s+1)}^k (stage s twiddles)
    DevBuf tw_inv;  // same for w^-1
    DevBuf gpow;    // Fr[N]: g^i, natural order
    DevBuf t1;      // Fr[N]: N^-1 g^bitrev(j)
    DevBuf t2;      // Fr[N]: N^-1 g^-bitrev(j)
    DevBuf consts;  // Fr[8]: w, w^-1, N^-1, (g^N - 1)^-1, g, g^-1
    // tile shape of the passes, chosen on this device when the tables are built
    // (ntt_tables_build): at most max_stages radix-2 stages per pass, each thread
    // doing bfly_per_thread butterflies per stage
    int max_stages = 10;
    int bfly_per_thread = 1;
    size_t device_bytes() const
    {
        return tw_fwd.bytes + tw_inv.bytes + gpow.bytes + t1.bytes + t2.bytes + consts.bytes;
    }
};

enum { kConstOmega = 0, kConstOmegaInv = 1, kConstNinv = 2, kConstZinv = 3, kConstG = 4, kConstGinv = 5 };

int ntt_tables_build(NttTables &t, int logn, cudaStream_t st);

// In-place DIF (natural -> bitrev) or DIT (bitrev -> natural) transform.
// pre (indexed by position, applied on load of the first pass) and post
// (applied on store of the last pass) are optional Fr tables; post_const is an
// optional single Fr multiplier used when post is null.
int ntt_dif(const NttTables &t, Fr *data, bool inverse, const Fr *pre, const Fr *post,
            const Fr *post_const, cudaStream_t st);
int ntt_dit(const NttTables &t, Fr *data, bool inverse, const Fr *pre, const Fr *post,
            const Fr *post_const, cudaStream_t st);

// out[bitrev(j)] = in[j] * (scale ? scale[j] : scale_const ? *scale_const : 1)
int ntt_bitrev_permute(const Fr *in, Fr *out, uint64_t n, const Fr *scale, const Fr *scale_const,
                       cudaStream_t st);
// data[i] *= *c
int fr_scale_const(Fr *data, uint64_t n, const Fr *c, cudaStream_t st);
// h[i] = (a[i] * b[i] - c[i]) * *zinv
int fr_quotient_pointwise(const Fr *a, const Fr *b, const Fr *c, Fr *h, uint64_t n,
                          const Fr *zinv, cudaStream_t st);

// Transforms of several vectors (of any sizes, each with its own tables) run pass
// by pass, every pass of all of them in one launch (a batch of proofs' quotient
// chains).  The transforms in one call are independent; each item's passes are
// those ntt_dif / ntt_dit would run for it.
struct NttPassItem {
    Fr *data;
    const Fr *tw, *pre, *post, *post_const;
    uint32_t first_block; // prefix over items of the blocks of this pass
    int s_lo, t;
};
struct NttJob {
    const NttTables *tables;
    Fr *data;
    const Fr *pre, *post, *post_const;
};
// items_host (pinned) and items_dev: 8 n_jobs items each (up to 8 passes); the
// host items are read by the stream's copy, so they must stay untouched until the
// stream has passed this call
int ntt_run_list(const NttJob *jobs, int n_jobs, bool dif, bool inverse, NttPassItem *items_host,
                 NttPassItem *items_dev, cudaStream_t st);

// (a b - c) / Z(g) for several vectors in one launch
struct QuotientItem {
    const Fr *a, *b, *c;
    Fr *h;
    const Fr *zinv;
    uint64_t first; // the caller passes each item's length; replaced by the prefix
};
// items_host: pinned, rewritten in place (lengths -> prefixes) and read by the copy
int fr_quotient_list(QuotientItem *items_host, int n_items, QuotientItem *items_dev, cudaStream_t st);

// Table pieces and the DIT transform over caller-owned device memory (nothing is
// allocated; used by the allocation-free entry point).  The stage twiddle table
// tw[2^s + k] = w_{2^(s+1)}^k does not depend on N, so one table built for 2^L
// serves every domain 2^logn with logn <= L.
int ntt_constants_into(int logn, Fr *consts /* Fr[8], layout of NttTables::consts */,
                       cudaStream_t st);
int fr_powers_into(const Fr *base, Fr *out, uint64_t m, cudaStream_t st); // out[i] = base^i
int ntt_stage_twiddles_into(const Fr *pw /* w_N^i, i < N/2 */, Fr *tw, int logn, cudaStream_t st);
int ntt_dit_raw(int logn, const Fr *tw, Fr *data, const Fr *pre, const Fr *post,
                const Fr *post_const, cudaStream_t st);

} // namespace nkr
