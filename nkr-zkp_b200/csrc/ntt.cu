// Radix-2 NTT kernels and resident tables (see ntt.cuh for the design).
#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <vector>
#include "ntt.cuh"

namespace nkr {

namespace {

// 2^28-th root of unity of Fr in Montgomery form: 5^((r - 1) / 2^28), the root
// libff uses (alt_bn128_init.cpp:56-61 with multiplicative_generator = 5 and
// s = 28; field_utils.tcc:38-51 squares it down to smaller domains).
__device__ __forceinline__ Fr fr_root_2_28()
{
    Fr r;
    const uint32_t v[8] = {0x80d13d9cu, 0x636e7355u, 0x2445ffd6u, 0xa22bf374u,
                           0x1eb203d8u, 0x56452ac0u, 0x2963f9e7u, 0x1860ef94u};
#pragma unroll
    for (int i = 0; i < 8; ++i) r.v[i] = v[i];
    return r;
}

// multiplicative generator g = 5 (Montgomery), the coset shift of cosetFFT
__device__ __forceinline__ Fr fr_gen5()
{
    Fr r;
    const uint32_t v[8] = {0x9fffffe6u, 0x1b0d0ef9u, 0xa32a913fu, 0xeaba68a3u,
                           0xd8dd0689u, 0x47d8eb76u, 0x20f5bbc3u, 0x15d00855u};
#pragma unroll
    for (int i = 0; i < 8; ++i) r.v[i] = v[i];
    return r;
}

__global__ void k_ntt_constants(int logn, Fr *c)
{
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    Fr w = fr_root_2_28();
    for (int i = 28; i > logn; --i) w = sqr(w);
    Fr nn = Fr::zero();
    nn.v[0] = uint32_t(1u << logn);
    nn = to_mont(nn);
    const Fr g = fr_gen5();
    Fr gn = g;
    for (int i = 0; i < logn; ++i) gn = sqr(gn);
    c[kConstOmega] = w;
    c[kConstOmegaInv] = inverse(w);
    c[kConstNinv] = inverse(nn);
    c[kConstZinv] = inverse(gn - Fr::one());
    c[kConstG] = g;
    c[kConstGinv] = inverse(g);
    c[6] = Fr::one();
    c[7] = Fr::zero();
}

// out[i] = base^i, i < m; each thread fills a run of 32 consecutive powers
constexpr int kPowRun = 32;
__global__ void k_powers(const Fr *base_ptr, Fr *out, uint64_t m)
{
    const uint64_t t = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    const uint64_t first = t * kPowRun;
    if (first >= m) return;
    const Fr base = *base_ptr;
    Fr acc = Fr::one();
    // base^first by square-and-multiply over the bits of first
    for (int b = 63; b >= 0; --b) {
        acc = sqr(acc);
        if ((first >> b) & 1) acc = acc * base;
    }
    for (int i = 0; i < kPowRun && first + i < m; ++i) {
        out[first + i] = acc;
        acc = acc * base;
    }
}

// tw[2^s + k] = pw[k << (logn - 1 - s)]  (w_{2^(s+1)}^k from powers of w_N)
__global__ void k_stage_twiddles(const Fr *pw, Fr *tw, int logn)
{
    const uint64_t n = uint64_t(1) << logn;
    const uint64_t j = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (j >= n) return;
    if (j == 0) {
        tw[0] = Fr::one();
        return;
    }
    const int s = 63 - __clzll((long long)j);
    const uint64_t k = j - (uint64_t(1) << s);
    tw[j] = pw[k << (logn - 1 - s)];
}

__device__ __forceinline__ uint32_t brev_n(uint32_t j, int logn)
{
    return logn == 0 ? 0u : (__brev(j) >> (32 - logn));
}

// dst[j] = c * src[bitrev(j)]
__global__ void k_bitrev_scaled(const Fr *src, const Fr *c, Fr *dst, int logn)
{
    const uint64_t n = uint64_t(1) << logn;
    const uint64_t j = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (j >= n) return;
    dst[j] = *c * src[brev_n(uint32_t(j), logn)];
}

// One tile of a pass: the group gid of 2^t elements spaced 2^s_lo apart, staged
// through shared memory sm for t radix-2 stages.
template <bool DIF>
__device__ __forceinline__ void ntt_pass_tile(Fr *sm, Fr *data, int s_lo, int t, const Fr *tw,
                                              const Fr *pre, const Fr *post, const Fr *post_const,
                                              uint64_t gid)
{
    const int G = 1 << t;
    const int half = G >> 1;
    const uint64_t low = gid & ((uint64_t(1) << s_lo) - 1);
    const uint64_t high = gid >> s_lo;
    const uint64_t base = low | (high << (s_lo + t));

    for (int m = threadIdx.x; m < G; m += blockDim.x) {
        const uint64_t j = base + (uint64_t(m) << s_lo);
        Fr x = data[j];
        if (pre) x = x * pre[j];
        sm[m] = x;
    }
    __syncthreads();
    for (int st = 0; st < t; ++st) {
        const int s = DIF ? (s_lo + t - 1 - st) : (s_lo + st);
        const int dl = s - s_lo;
        const int d = 1 << dl;
        for (int b = threadIdx.x; b < half; b += blockDim.x) {
            const int m0 = ((b >> dl) << (dl + 1)) | (b & (d - 1));
            const int m1 = m0 + d;
            const uint64_t k = (uint64_t(m0 & (d - 1)) << s_lo) | low;
            const Fr w = tw[(uint64_t(1) << s) + k];
            const Fr u = sm[m0];
            const Fr v = sm[m1];
            if (DIF) {
                sm[m0] = u + v;
                sm[m1] = (u - v) * w;
            } else {
                const Fr tv = v * w;
                sm[m0] = u + tv;
                sm[m1] = u - tv;
            }
        }
        __syncthreads();
    }
    for (int m = threadIdx.x; m < G; m += blockDim.x) {
        const uint64_t j = base + (uint64_t(m) << s_lo);
        Fr x = sm[m];
        if (post)
            x = x * post[j];
        else if (post_const)
            x = x * *post_const;
        data[j] = x;
    }
}

template <bool DIF>
__global__ void __launch_bounds__(512) k_ntt_pass(Fr *data, int s_lo, int t, const Fr *tw,
                                                   const Fr *pre, const Fr *post,
                                                   const Fr *post_const)
{
    extern __shared__ Fr sm[];
    ntt_pass_tile<DIF>(sm, data, s_lo, t, tw, pre, post, post_const, blockIdx.x);
}

// One pass of many transforms (of any sizes) in one launch: item i owns blocks
// [first_block, first_block + n >> t) of the grid.  Items are few (a batch's
// transforms), so a block finds its item by binary search.
template <bool DIF>
__global__ void __launch_bounds__(512) k_ntt_pass_list(const NttPassItem *items, int n_items)
{
    extern __shared__ Fr sm[];
    int lo = 0, hi = n_items - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (items[mid].first_block <= blockIdx.x)
            lo = mid;
        else
            hi = mid - 1;
    }
    const NttPassItem it = items[lo];
    ntt_pass_tile<DIF>(sm, it.data, it.s_lo, it.t, it.tw, it.pre, it.post, it.post_const,
                       blockIdx.x - it.first_block);
}

// h = (a b - c) (g^n - 1)^-1 for many vectors in one launch (item i owns the
// elements [first, first + n) of the grid-wide index space)
__global__ void k_quotient_list(const QuotientItem *items, int n_items, uint64_t total)
{
    const uint64_t g = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (g >= total) return;
    int lo = 0, hi = n_items - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (items[mid].first <= g)
            lo = mid;
        else
            hi = mid - 1;
    }
    const QuotientItem &it = items[lo];
    const uint64_t i = g - it.first;
    it.h[i] = (it.a[i] * it.b[i] - it.c[i]) * *it.zinv;
}

__global__ void k_bitrev_permute(const Fr *in, Fr *out, int logn, const Fr *scale,
                                 const Fr *scale_const)
{
    const uint64_t n = uint64_t(1) << logn;
    const uint64_t j = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (j >= n) return;
    Fr x = in[j];
    if (scale)
        x = x * scale[j];
    else if (scale_const)
        x = x * *scale_const;
    out[brev_n(uint32_t(j), logn)] = x;
}

__global__ void k_scale_const(Fr *d, uint64_t n, const Fr *c)
{
    const uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < n) d[i] = d[i] * *c;
}

__global__ void k_quotient(const Fr *a, const Fr *b, const Fr *c, Fr *h, uint64_t n,
                           const Fr *zinv)
{
    const uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i < n) h[i] = (a[i] * b[i] - c[i]) * *zinv;
}

// pass split: at most max_stages radix-2 stages per pass, spread evenly
// (ts holds up to 8 passes: max_stages >= 4 for logn <= 28)
int pass_plan(int logn, int max_stages, int *ts)
{
    const int np = (logn + max_stages - 1) / max_stages;
    for (int i = 0; i < np; ++i) ts[i] = logn / np + (i < logn % np ? 1 : 0);
    return np;
}

unsigned pass_threads(int t, int bfly_per_thread)
{
    const unsigned half = 1u << (t - 1);
    const unsigned th = half / unsigned(bfly_per_thread);
    return (t >= 6 && th >= 32) ? th : 32u;
}

int run_passes(const NttTables &tb, Fr *data, bool dif, bool inverse, const Fr *pre,
               const Fr *post, const Fr *post_const, cudaStream_t st)
{
    const int logn = tb.logn;
    int ts[8];
    const int np = pass_plan(logn, tb.max_stages, ts);
    const Fr *tw = inverse ? tb.tw_inv.as<Fr>() : tb.tw_fwd.as<Fr>();
    int s_lo = dif ? logn : 0;
    for (int p = 0; p < np; ++p) {
        const int t = ts[p];
        if (dif) s_lo -= t;
        const int G = 1 << t;
        const unsigned threads = pass_threads(t, tb.bfly_per_thread);
        const unsigned blocks = unsigned(tb.n >> t);
        const Fr *pr = p == 0 ? pre : nullptr;
        const Fr *po = p == np - 1 ? post : nullptr;
        const Fr *pc = p == np - 1 ? post_const : nullptr;
        if (dif)
            k_ntt_pass<true><<<blocks, threads, G * sizeof(Fr), st>>>(data, s_lo, t, tw, pr, po, pc);
        else
            k_ntt_pass<false><<<blocks, threads, G * sizeof(Fr), st>>>(data, s_lo, t, tw, pr, po, pc);
        NKR_CHECK_LAUNCH();
        if (!dif) s_lo += t;
    }
    return NKR_B200_OK;
}

// The passes of several transforms, pass q of all of them in one launch.
int run_list(const NttJob *jobs, int n_jobs, bool dif, bool inverse, NttPassItem *items_host,
             NttPassItem *items_dev, cudaStream_t st)
{
    if (n_jobs <= 0) return NKR_B200_OK;
    struct Plan {
        int np, ts[8], s_lo;
    };
    std::vector<Plan> plans(n_jobs);
    int max_np = 0;
    for (int j = 0; j < n_jobs; ++j) {
        const NttTables &tb = *jobs[j].tables;
        plans[j].np = pass_plan(tb.logn, tb.max_stages, plans[j].ts);
        plans[j].s_lo = dif ? tb.logn : 0;
        max_np = std::max(max_np, plans[j].np);
    }
    NttPassItem *items = items_host;
    std::vector<int> count(max_np, 0);
    std::vector<uint32_t> blocks(max_np, 0), threads(max_np, 32), smem(max_np, 0);
    for (int q = 0; q < max_np; ++q) {
        for (int j = 0; j < n_jobs; ++j) {
            Plan &pl = plans[j];
            if (q >= pl.np) continue;
            const NttTables &tb = *jobs[j].tables;
            const int t = pl.ts[q];
            if (dif) pl.s_lo -= t;
            NttPassItem &it = items[size_t(q) * n_jobs + count[q]++];
            it.data = jobs[j].data;
            it.tw = inverse ? tb.tw_inv.as<Fr>() : tb.tw_fwd.as<Fr>();
            it.pre = q == 0 ? jobs[j].pre : nullptr;
            it.post = q == pl.np - 1 ? jobs[j].post : nullptr;
            it.post_const = q == pl.np - 1 ? jobs[j].post_const : nullptr;
            it.first_block = blocks[q];
            it.s_lo = pl.s_lo;
            it.t = t;
            const uint64_t nb = tb.n >> t;
            NKR_REQUIRE(uint64_t(blocks[q]) + nb < (uint64_t(1) << 31), "batched NTT pass too large");
            blocks[q] += uint32_t(nb);
            threads[q] = std::max(threads[q], pass_threads(t, tb.bfly_per_thread));
            smem[q] = std::max<uint32_t>(smem[q], (1u << t) * uint32_t(sizeof(Fr)));
            if (!dif) pl.s_lo += t;
        }
    }
    NKR_CUDA(cudaMemcpyAsync(items_dev, items, size_t(max_np) * n_jobs * sizeof(NttPassItem),
                             cudaMemcpyHostToDevice, st));
    for (int q = 0; q < max_np; ++q) {
        const NttPassItem *d = items_dev + size_t(q) * n_jobs;
        if (dif)
            k_ntt_pass_list<true><<<blocks[q], threads[q], smem[q], st>>>(d, count[q]);
        else
            k_ntt_pass_list<false><<<blocks[q], threads[q], smem[q], st>>>(d, count[q]);
        NKR_CHECK_LAUNCH();
    }
    return NKR_B200_OK;
}

// NTT tile-shape autotuner: times a forward transform of the table's size for
// every pass split with 7..10 stages per pass and 1, 2 or 4 butterflies per
// thread and stage, and keeps the fastest (every shape gives the same output).
// Sizes below 2^14 keep the default; NKR_B200_AUTOTUNE=0 turns it off.
int ntt_tune(NttTables &t, Fr *work, cudaStream_t st)
{
    const char *e = std::getenv("NKR_B200_AUTOTUNE");
    if (t.logn < 14 || (e && std::strcmp(e, "0") == 0)) return NKR_B200_OK;
    cudaEvent_t e0, e1;
    NKR_CUDA(cudaEventCreate(&e0));
    NKR_CUDA(cudaEventCreate(&e1));
    float best = 0.f;
    int best_s = t.max_stages, best_b = t.bfly_per_thread;
    int prev_ts[8] = {}, prev_np = 0;
    int status = NKR_B200_OK;
    for (int ms = 10; ms >= 7 && status == NKR_B200_OK; --ms) {
        int ts[8];
        const int np = pass_plan(t.logn, ms, ts);
        if (np == prev_np && std::equal(ts, ts + np, prev_ts)) continue; // same split
        std::copy(ts, ts + np, prev_ts);
        prev_np = np;
        for (int bpt = 1; bpt <= 4 && status == NKR_B200_OK; bpt *= 2) {
            t.max_stages = ms;
            t.bfly_per_thread = bpt;
            status = run_passes(t, work, true, false, nullptr, nullptr, nullptr, st); // warm-up
            if (status != NKR_B200_OK) break;
            if (cudaEventRecord(e0, st) != cudaSuccess) status = NKR_B200_ECUDA;
            for (int r = 0; r < 3 && status == NKR_B200_OK; ++r)
                status = run_passes(t, work, true, false, nullptr, nullptr, nullptr, st);
            float ms_run = 0.f;
            if (status == NKR_B200_OK && (cudaEventRecord(e1, st) != cudaSuccess ||
                                          cudaEventSynchronize(e1) != cudaSuccess ||
                                          cudaEventElapsedTime(&ms_run, e0, e1) != cudaSuccess))
                status = NKR_B200_ECUDA;
            if (status == NKR_B200_OK && (best == 0.f || ms_run < best)) {
                best = ms_run;
                best_s = ms;
                best_b = bpt;
            }
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    t.max_stages = best_s;
    t.bfly_per_thread = best_b;
    if (status != NKR_B200_OK) set_error("NTT tile tuning failed: %s", cudaGetErrorString(cudaGetLastError()));
    return status;
}

} // namespace

int ntt_tables_build(NttTables &t, int logn, cudaStream_t st)
{
    NKR_REQUIRE(logn >= 1 && logn <= 28, "NTT domain 2^%d outside [2, 2^28]", logn);
    t.logn = logn;
    t.n = uint64_t(1) << logn;
    const size_t bytes = t.n * sizeof(Fr);
    NKR_TRY(t.consts.alloc(8 * sizeof(Fr), "ntt constants"));
    NKR_TRY(t.tw_fwd.alloc(bytes, "ntt twiddles"));
    NKR_TRY(t.tw_inv.alloc(bytes, "ntt inverse twiddles"));
    NKR_TRY(t.gpow.alloc(bytes, "coset powers"));
    NKR_TRY(t.t1.alloc(bytes, "coset scale table"));
    NKR_TRY(t.t2.alloc(bytes, "inverse coset scale table"));
    DevBuf tmp;
    NKR_TRY(tmp.alloc(bytes, "ntt table scratch"));
    Fr *c = t.consts.as<Fr>();
    k_ntt_constants<<<1, 32, 0, st>>>(logn, c);
    NKR_CHECK_LAUNCH();
    const unsigned pb = blocks_for((t.n + kPowRun - 1) / kPowRun, 128);
    const unsigned nb = blocks_for(t.n, 256);
    // forward stage twiddles from powers of w (tmp holds w^i, i < N/2)
    k_powers<<<pb, 128, 0, st>>>(c + kConstOmega, tmp.as<Fr>(), t.n / 2);
    NKR_CHECK_LAUNCH();
    k_stage_twiddles<<<nb, 256, 0, st>>>(tmp.as<Fr>(), t.tw_fwd.as<Fr>(), logn);
    NKR_CHECK_LAUNCH();
    k_powers<<<pb, 128, 0, st>>>(c + kConstOmegaInv, tmp.as<Fr>(), t.n / 2);
    NKR_CHECK_LAUNCH();
    k_stage_twiddles<<<nb, 256, 0, st>>>(tmp.as<Fr>(), t.tw_inv.as<Fr>(), logn);
    NKR_CHECK_LAUNCH();
    // g^i natural, then the bit-reversed scale tables
    k_powers<<<pb, 128, 0, st>>>(c + kConstG, t.gpow.as<Fr>(), t.n);
    NKR_CHECK_LAUNCH();
    k_bitrev_scaled<<<nb, 256, 0, st>>>(t.gpow.as<Fr>(), c + kConstNinv, t.t1.as<Fr>(), logn);
    NKR_CHECK_LAUNCH();
    k_powers<<<pb, 128, 0, st>>>(c + kConstGinv, tmp.as<Fr>(), t.n);
    NKR_CHECK_LAUNCH();
    k_bitrev_scaled<<<nb, 256, 0, st>>>(tmp.as<Fr>(), c + kConstNinv, t.t2.as<Fr>(), logn);
    NKR_CHECK_LAUNCH();
    NKR_CUDA(cudaStreamSynchronize(st));
    NKR_TRY(ntt_tune(t, tmp.as<Fr>(), st));
    return NKR_B200_OK;
}

int ntt_dif(const NttTables &t, Fr *data, bool inverse, const Fr *pre, const Fr *post,
            const Fr *post_const, cudaStream_t st)
{
    return run_passes(t, data, true, inverse, pre, post, post_const, st);
}

int ntt_dit(const NttTables &t, Fr *data, bool inverse, const Fr *pre, const Fr *post,
            const Fr *post_const, cudaStream_t st)
{
    return run_passes(t, data, false, inverse, pre, post, post_const, st);
}

int ntt_run_list(const NttJob *jobs, int n_jobs, bool dif, bool inverse, NttPassItem *items_host,
                 NttPassItem *items_dev, cudaStream_t st)
{
    return run_list(jobs, n_jobs, dif, inverse, items_host, items_dev, st);
}

int fr_quotient_list(QuotientItem *items, int n_items, QuotientItem *items_dev, cudaStream_t st)
{
    if (n_items <= 0) return NKR_B200_OK;
    uint64_t total = 0;
    for (int i = 0; i < n_items; ++i) {
        const uint64_t n = items[i].first; // on input: the item's length
        items[i].first = total;
        total += n;
    }
    NKR_CUDA(cudaMemcpyAsync(items_dev, items, n_items * sizeof(QuotientItem), cudaMemcpyHostToDevice, st));
    k_quotient_list<<<blocks_for(total, 256), 256, 0, st>>>(items_dev, n_items, total);
    NKR_CHECK_LAUNCH();
    return NKR_B200_OK;
}

int ntt_bitrev_permute(const Fr *in, Fr *out, uint64_t n, const Fr *scale, const Fr *scale_const,
                       cudaStream_t st)
{
    const int logn = log2_exact(n);
    NKR_REQUIRE(logn >= 0 && logn <= 31, "bit reversal needs a power-of-two size");
    k_bitrev_permute<<<blocks_for(n, 256), 256, 0, st>>>(in, out, logn, scale, scale_const);
    NKR_CHECK_LAUNCH();
    return NKR_B200_OK;
}

int fr_scale_const(Fr *data, uint64_t n, const Fr *c, cudaStream_t st)
{
    k_scale_const<<<blocks_for(n, 256), 256, 0, st>>>(data, n, c);
    NKR_CHECK_LAUNCH();
    return NKR_B200_OK;
}

int fr_quotient_pointwise(const Fr *a, const Fr *b, const Fr *c, Fr *h, uint64_t n,
                          const Fr *zinv, cudaStream_t st)
{
    k_quotient<<<blocks_for(n, 256), 256, 0, st>>>(a, b, c, h, n, zinv);
    NKR_CHECK_LAUNCH();
    return NKR_B200_OK;
}

int ntt_constants_into(int logn, Fr *consts, cudaStream_t st)
{
    NKR_REQUIRE(logn >= 1 && logn <= 28, "NTT domain 2^%d outside [2, 2^28]", logn);
    k_ntt_constants<<<1, 32, 0, st>>>(logn, consts);
    NKR_CHECK_LAUNCH();
    return NKR_B200_OK;
}

int fr_powers_into(const Fr *base, Fr *out, uint64_t m, cudaStream_t st)
{
    k_powers<<<blocks_for((m + kPowRun - 1) / kPowRun, 128), 128, 0, st>>>(base, out, m);
    NKR_CHECK_LAUNCH();
    return NKR_B200_OK;
}

int ntt_stage_twiddles_into(const Fr *pw, Fr *tw, int logn, cudaStream_t st)
{
    NKR_REQUIRE(logn >= 1 && logn <= 28, "NTT domain 2^%d outside [2, 2^28]", logn);
    k_stage_twiddles<<<blocks_for(uint64_t(1) << logn, 256), 256, 0, st>>>(pw, tw, logn);
    NKR_CHECK_LAUNCH();
    return NKR_B200_OK;
}

int ntt_dit_raw(int logn, const Fr *tw, Fr *data, const Fr *pre, const Fr *post,
                const Fr *post_const, cudaStream_t st)
{
    NKR_REQUIRE(logn >= 1 && logn <= 28, "NTT domain 2^%d outside [2, 2^28]", logn);
    int ts[8];
    const int np = pass_plan(logn, 10, ts);
    const uint64_t n = uint64_t(1) << logn;
    int s_lo = 0;
    for (int p = 0; p < np; ++p) {
        const int t = ts[p];
        const int G = 1 << t;
        const unsigned threads = pass_threads(t, 1);
        k_ntt_pass<false><<<unsigned(n >> t), threads, G * sizeof(Fr), st>>>(
            data, s_lo, t, tw, p == 0 ? pre : nullptr, p == np - 1 ? post : nullptr,
            p == np - 1 ? post_const : nullptr);
        NKR_CHECK_LAUNCH();
        s_lo += t;
    }
    return NKR_B200_OK;
}

} // namespace nkr
