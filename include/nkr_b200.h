/*
 * nkr_b200.h -- C ABI of the B200 (sm_100a) Groth16 prove backend for BN254.
 *
 * This is the drop-in boundary for NKR-ZKP's `groth16-prove --backend b200`.
 * Every entry point takes plain pointers and sizes; device state lives behind
 * opaque handles.  Each declaration names the reference interface it replaces
 * (paths inside the reference project, file:line).
 *
 * Byte layouts are the reference's in-memory libff layouts (x86-64):
 *   Fr / Fq element   32 B: 4 x u64 little-endian, Montgomery form (R = 2^256)
 *   G1 Jacobian       96 B: {X, Y, Z} Fq, infinity <=> Z = 0      (libff alt_bn128_G1)
 *   G2 Jacobian      192 B: {X, Y, Z} Fq2, Fq2 = {c0, c1}           (libff alt_bn128_G2)
 *   CSR matrix        row_ptr u32[rows + 1], col_idx u32[nnz], values Fr[nnz]
 *                     (protocols/groth16/common/include/r1cs/spmat.hpp:206-215)
 * Points returned by this library are affine-normalised in that same Jacobian
 * layout: Z = 1 (Montgomery), or (0, 1, 0) for infinity, exactly what libff's
 * to_affine_coordinates() produces (libff alt_bn128_g1.cpp to_affine_coordinates).
 *
 * Errors: every call returns NKR_B200_OK (0) or a nonzero status; the message
 * is available from nkr_b200_last_error() on the same thread.  The library
 * never calls exit() (the reference CUDA path does: operators/cuda/include/
 * utils/cuda_check.cuh:6-12).  There is no CPU fallback: without a usable
 * sm_100 device every compute entry point fails with NKR_B200_ENODEV.
 */
#ifndef NKR_B200_H
#define NKR_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum {
    NKR_B200_OK = 0,
    NKR_B200_EINVAL = 1,   /* bad argument / shape / size */
    NKR_B200_ECUDA = 2,    /* CUDA runtime error */
    NKR_B200_ENOMEM = 3,   /* device memory admission refused */
    NKR_B200_ENODEV = 4,   /* no usable sm_100 device */
    NKR_B200_ETIMEOUT = 5, /* bounded device wait expired */
    NKR_B200_EBUSY = 6     /* server queue full / handle in use */
};

typedef struct nkr_b200_ctx nkr_b200_ctx;   /* one GPU: streams, scratch arena */
typedef struct nkr_b200_key nkr_b200_key;   /* a prepared (circuit, proving key) */
typedef struct nkr_b200_vk nkr_b200_vk;     /* a prepared verification key */
typedef struct nkr_b200_msm_bases nkr_b200_msm_bases; /* resident MSM bases */

/* Circuit in the reference's CSR layout: matrices A, B, C share the shape
 * rows x cols (protocols/groth16/common/include/groth16/types.hpp:17-27). */
typedef struct {
    uint64_t rows;          /* constraints, a power of two >= 2 */
    uint64_t cols;          /* variables incl. the constant-one column */
    uint64_t public_inputs; /* number of public inputs (columns 1..public_inputs) */
    const uint32_t *row_ptr[3];
    const uint32_t *col_idx[3];
    const void *values[3]; /* Fr[nnz] Montgomery */
} nkr_b200_circuit;

/* Proving key queries in libff Jacobian layout, as BinaryArchive stores them
 * (types.hpp:29-40, io.cpp:54-61).  Points need not be normalised. */
typedef struct {
    const void *a_query;    /* G1[cols] */
    const void *b_g1_query; /* G1[cols] */
    const void *b_g2_query; /* G2[cols] */
    const void *l_query;    /* G1[cols] */
    const void *h_query;    /* G1[rows] */
    const void *alpha_g1, *beta_g1, *delta_g1; /* G1 */
    const void *beta_g2, *delta_g2;            /* G2 */
} nkr_b200_proving_key;

/* RawProof (types.hpp:47-53), affine-normalised libff Jacobian layout */
typedef struct {
    uint8_t ar[96], bs1[96], zk[96], qz[96];
    uint8_t bs2[192];
} nkr_b200_raw_proof;

/* Proof (types.hpp:55-59) */
typedef struct {
    uint8_t a[96];
    uint8_t b[192];
    uint8_t c[96];
} nkr_b200_proof;

/* VerificationKey (types.hpp:40-45) in libff layout: e(alpha, beta) as
 * alt_bn128_Fq12 (384 B), gamma and delta as G2 (192 B, any Z), ic as n_ic G1
 * points (96 B each, any Z). */
typedef struct {
    const void *alpha_g1_beta_g2;
    const void *gamma_g2;
    const void *delta_g2;
    const void *ic;
    uint64_t n_ic;
} nkr_b200_verification_key;

/* Per-stage device times of the last prove on a key, milliseconds (CUDA events):
 * the reference's profile labels groth16.cuda.prove.{r1cs_matrix_vector,
 * quotient_polynomial, witness_msms, quotient_msm} (groth16_backend.cu:249-274).
 * The stages overlap on the device (the witness MSMs run on their own streams
 * beside the quotient chain), so each MSM's end is also given, measured from the
 * start of the prove: the labels groth16.cpu.prove.msm_{a, b_g1, b_g2, l, h} of
 * the CPU backend (backends/cpu/src/backend.cpp:181-200). */
typedef struct {
    float spmv_ms, quotient_ms, witness_msms_ms, quotient_msm_ms, total_ms;
    float msm_a_end_ms, msm_b_g1_end_ms, msm_b_g2_end_ms, msm_l_end_ms, msm_h_end_ms;
    /* per MSM (A, B_G1, B_G2, L, H), ms from the start of the prove: start and end
     * of the level-1 bucket accumulation, end of the fix-up levels, end of the
     * first reduction level (the MSM ends at msm_*_end_ms) */
    float msm_phase_ms[5][4];
} nkr_b200_stage_times;

/* ---- context -------------------------------------------------------------- */

/* Replaces make_cuda_backend() (backends/cuda/src/groth16_backend.cu:284,
 * registry common/src/backend_registry.cpp:18-27).  device = CUDA ordinal. */
int nkr_b200_open(int device, nkr_b200_ctx **out);
void nkr_b200_close(nkr_b200_ctx *ctx);
const char *nkr_b200_last_error(void);
/* "b200" -- Backend::name() (common/include/groth16/backend.hpp:14) */
const char *nkr_b200_backend_name(void);

/* ---- prove path ----------------------------------------------------------- */

/* Replaces Backend::prepare (backend.hpp:20; CUDA: groth16_backend.cu:214-240):
 * uploads CSR A/B/C, batch-normalises the PK to affine, builds twiddle tables and
 * the per-window MSM base copies; all stay resident until nkr_b200_key_free. */
int nkr_b200_prepare(nkr_b200_ctx *ctx, const nkr_b200_circuit *circuit,
                     const nkr_b200_proving_key *pk, nkr_b200_key **out);
void nkr_b200_key_free(nkr_b200_key *key);
/* device bytes the key holds */
uint64_t nkr_b200_key_device_bytes(const nkr_b200_key *key);

/* Proving-key artifacts in the reference's BinaryArchive format ("LKZ1" v1; the
 * layout of read_proving_key / write_proving_key, common/src/io.cpp:54-61), with
 * no limit on vector size: the reference's BinaryArchive refuses vectors above
 * 1 GiB (common/include/binary_archive.hpp:19, 76-77, 89-90), i.e. every key from
 * 2^24 constraints up.  nkr_b200_prepare_file memory-maps the file and prepares
 * the key from the mapped queries (no host copy; the same checks as
 * nkr_b200_prepare, plus the file's structure and each query's length against the
 * circuit).  nkr_b200_pk_file_info returns the point counts a file holds (rows =
 * h_query, cols = the other queries) without touching a GPU.
 * nkr_b200_write_proving_key writes the same format (queries G1/G2 Jacobian:
 * a, b_g1, b_g2, l with cols points, h with rows points). */
int nkr_b200_prepare_file(nkr_b200_ctx *ctx, const nkr_b200_circuit *circuit, const char *pk_path,
                          nkr_b200_key **out);
int nkr_b200_pk_file_info(const char *path, uint64_t *rows, uint64_t *cols);
int nkr_b200_write_proving_key(const char *path, const nkr_b200_proving_key *pk, uint64_t rows,
                               uint64_t cols);

/* Replaces Backend::prove (backend.hpp:24-28; CPU backends/cpu/src/backend.cpp:156-201,
 * CUDA groth16_backend.cu:242-279).  witness: Fr[cols] host memory. */
int nkr_b200_prove(nkr_b200_key *key, const void *witness, uint64_t n,
                   nkr_b200_raw_proof *out);

/* Replaces blind_proof (common/src/protocol.cpp:85-94) with caller-given r, s
 * (Fr Montgomery, 32 B each); the reference draws them unseeded (:87-88).
 * raw: libff Jacobian points with any Z (as the reference's RawProof allows).
 * The blinding of the last proof of this key's nkr_b200_prove reads tables that
 * prove left on the device; any other raw proof gives the same result by a
 * slower path (about 1 ms).  out: affine-normalised (Z = 1, or (0, 1, 0)). */
int nkr_b200_blind(nkr_b200_key *key, const nkr_b200_raw_proof *raw, const void *r,
                   const void *s, nkr_b200_proof *out);

/* ---- verification -------------------------------------------------------- */

/* Prepares a verification key on the device (ic normalised, the Miller-loop
 * lines of gamma and delta computed once, and signed 5-bit window tables of the
 * ic points: 52 KB of device memory per public input).  A prepared key serves one
 * nkr_b200_verify_batch call at a time (its batch staging is per key). */
int nkr_b200_vk_prepare(nkr_b200_ctx *ctx, const nkr_b200_verification_key *vk,
                        nkr_b200_vk **out);

/* Replaces verify (common/src/protocol.cpp:96-108) for a batch of count proofs
 * of one key, one proof per GPU thread.  proofs: count nkr_b200_proof records
 * (A, B, C in libff layout, any Z) in host memory; public_inputs: count rows of
 * n_public Fr (Montgomery, 32 B each).  accept[i] = 1 when proof i satisfies
 * e(A, B) = e(alpha, beta) e(vk_x, gamma) e(C, delta), else 0; as in the
 * reference, every proof is rejected when n_public + 1 != n_ic.  The GT values
 * are libff's (its reduced pairing, bit for bit), so the verdicts are the
 * reference's. */
int nkr_b200_verify_batch(nkr_b200_vk *vk, const void *public_inputs, uint64_t n_public,
                          const void *proofs, uint64_t count, uint8_t *accept);
void nkr_b200_vk_free(nkr_b200_vk *vk);

/* Replaces Curve::reduced_pairing (libff alt_bn128_reduced_pairing) for count
 * pairs: p_g1 G1[count] (96 B), q_g2 G2[count] (192 B), out_gt Fq12[count]
 * (384 B, libff alt_bn128_Fq12 layout, Montgomery). */
int nkr_b200_reduced_pairing(nkr_b200_ctx *ctx, const void *p_g1, const void *q_g2,
                             uint64_t count, void *out_gt);

/* Intermediates of the last prove on this key, copied to host (for parity
 * checks): az, bz, cz (Fr[rows]) and H (Fr[rows]); any pointer may be NULL. */
int nkr_b200_key_intermediates(nkr_b200_key *key, void *az, void *bz, void *cz, void *h);
int nkr_b200_key_stage_times(const nkr_b200_key *key, nkr_b200_stage_times *out);

/* Batched prove: count proofs over possibly different keys in one call; the
 * per-proof stages are issued across streams and replayed from captured CUDA
 * graphs.  witnesses[i] has keys[i]'s cols elements. */
int nkr_b200_prove_batch(nkr_b200_key *const *keys, const void *const *witnesses, int count,
                         nkr_b200_raw_proof *out);
/* The same batch with cross-proof launches: the proofs run in waves of at most
 * one proof per prove slot, and within a wave every NTT pass of every proof's
 * quotient chain (transforms of any sizes), the pointwise quotient step of all
 * proofs, and the level-1 bucket accumulation of all G1 witness MSMs, of all G2
 * MSMs and of all H MSMs each run as ONE launch over a device work list; the
 * per-proof steps (SpMV, digit sorts, fix-up and reduction levels) run on the
 * proofs' own slot streams beside them.  Results equal nkr_b200_prove_batch's
 * bit for bit.  No counterpart in the reference, which batches by running
 * separate processes (scripts/bench/runner.py:260-354). */
int nkr_b200_prove_batch_lists(nkr_b200_key *const *keys, const void *const *witnesses, int count,
                               nkr_b200_raw_proof *out);

/* ---- request server (continuous batching over resident keys) -------------
 * No counterpart in the reference, which proves one request per process
 * (app/prove.cpp:70-88).  A scheduler thread admits waiting requests, oldest
 * first, onto free prove slots of their key (adding slots while free HBM allows,
 * up to max_slots_per_key per key -- one for keys of 2^19 rows or more, which
 * fill the GPU alone -- and max_inflight in total) and replays each slot's
 * captured prove graph, so requests of different circuits overlap on the GPU.
 * Slot streams take a priority by circuit size, so the GPU's block scheduler
 * serves the smaller proofs in flight first (low median latency).  Requests
 * age: one that waited longer than age_factor (default 0.5) times its key's
 * recent service time is launched at the device's highest stream priority, so
 * the largest circuit's requests do not absorb all of the small ones' priority.
 * The witness memory of a request must stay valid until its wait returns.
 * A key added to a server is proved only through that server while it runs. */
typedef struct nkr_b200_server nkr_b200_server;
int nkr_b200_server_create(nkr_b200_ctx *ctx, int max_inflight, int max_slots_per_key,
                           nkr_b200_server **out);
int nkr_b200_server_add_key(nkr_b200_server *server, nkr_b200_key *key, int *key_id);
int nkr_b200_server_submit(nkr_b200_server *server, int key_id, const void *witness,
                           uint64_t *request_id);
/* Blocks until the request is done; latency = submit to result on the host, queue =
 * submit to start on the GPU (milliseconds; either pointer may be NULL). */
int nkr_b200_server_wait(nkr_b200_server *server, uint64_t request_id, nkr_b200_raw_proof *out,
                         double *latency_ms, double *queue_ms);
int nkr_b200_server_slots(nkr_b200_server *server, int key_id, int *slots);
/* Ageing threshold as a multiple of a key's recent service time (0 turns ageing
 * off); applies to requests started after the call. */
int nkr_b200_server_set_ageing(nkr_b200_server *server, double age_factor);
/* Requests completed, failed, and launched aged (at the highest priority) so far. */
int nkr_b200_server_stats(nkr_b200_server *server, uint64_t *completed, uint64_t *failed,
                          uint64_t *aged);
void nkr_b200_server_destroy(nkr_b200_server *server);

/* ---- operator-level entry points (operators/cuda/include/nkr/operators/cuda.hpp) */

/* libfqfft radix-2 domain ops on n = 2^k Fr values (host buffer, in place):
 * op 0 FFT, 1 iFFT, 2 cosetFFT(g = 5), 3 icosetFFT(g = 5), 4 divide_by_Z_on_coset.
 * Replaces NTTContext::{ntt,intt,coset_ntt,coset_intt} (ntt/ntt.cuh:110-185) and
 * libfqfft basic_radix2_domain.tcc:40-112. */
int nkr_b200_ntt(nkr_b200_ctx *ctx, int op, void *data, uint64_t n);

/* The same five domain ops on device-resident vectors, as NTTContext runs them on
 * its device arrays (ntt/ntt.cuh:110-185).  in and out are n Fr values each on the
 * context's device and must not overlap; the result is written to out and in is
 * overwritten (it is the transform's workspace).  stream is a cudaStream_t; NULL
 * is CUDA's legacy default stream.  Work that produced `in` must be ordered before
 * it on that stream.  The first call for a size builds that size's resident
 * tables (allocation, synchronous); later calls only enqueue work unless device_ms
 * is non-NULL, in which case the call waits and returns the ops' device time. */
int nkr_b200_ntt_device(nkr_b200_ctx *ctx, int op, void *in, void *out, uint64_t n, void *stream,
                        float *device_ms);

/* The constants that define this library's domain of size n (a power of two):
 * omega, the n-th root of unity libfqfft's radix-2 domain uses
 * (get_root_of_unity, libfqfft field_utils.tcc:38-51), and coset, the
 * multiplicative generator 5 (alt_bn128_init.cpp:59), both Fr Montgomery
 * (32 B).  NTTContext is constructed with these two values
 * (backends/cuda/src/groth16_backend.cu:87, ntt/ntt.cuh:52); the operator
 * layer in nkr_b200_operators.hpp checks what its caller passes against them. */
int nkr_b200_domain_constants(nkr_b200_ctx *ctx, uint64_t n, void *omega, void *coset);

/* The pointwise step of the quotient on device vectors of the domain's size n:
 * out[i] = (a[i] b[i] - c[i]) (g^n - 1)^-1 with the coset generator g = 5, what
 * NTTContext::A_times_B_minus_C_divided_by_Z (ntt/ntt.cuh:187-207) computes into
 * its first argument (with one field inverse for the whole call instead of one
 * per element).  Element-wise, so out may be a, b or c.  Enqueued on stream
 * (NULL = the legacy default stream); the first call for a size builds that
 * size's tables. */
int nkr_b200_quotient_device(nkr_b200_ctx *ctx, const void *a, const void *b, const void *c,
                             void *out, uint64_t n, void *stream);

/* The same five domain ops on DEVICE buffers, allocating no device memory.  No
 * counterpart in the reference: it serves callers that cannot allocate (their own
 * pool already holds the device's memory, or cudaFree's device-wide wait would
 * stall their other streams).  in and out (may be equal) hold n Fr values on
 * `device`; stream is a cudaStream_t (NULL = the default stream).  The call only
 * enqueues work: synchronise the stream before reading out.  Scratch is one fixed
 * array inside the library, shared by all calls on a device: n is limited to
 * 2^16 (larger n returns NKR_B200_EINVAL), and two calls in flight at once on
 * different streams or threads race.  The first call on a device builds the
 * array's tables and waits for `stream`; make it before capturing any stream.
 * The set-up belongs to the device's context and runs again after a
 * cudaDeviceReset.  The array takes 10 MiB of each device the library's kernels
 * are used on (of every device context it is loaded into when CUDA loads modules
 * eagerly, CUDA_MODULE_LOADING=EAGER), whether or not this entry point is called. */
int nkr_b200_ntt_noalloc(int device, int op, const void *in, void *out, uint64_t n,
                         void *stream);

/* CSR SpMV over Fr: y = M z (host buffers).  Replaces
 * sparse_matrix_vector_multiplication (backends/cuda/include/spmvm/spmvm.cuh:12-30). */
int nkr_b200_spmv(nkr_b200_ctx *ctx, uint64_t rows, uint64_t cols, const uint32_t *row_ptr,
                  const uint32_t *col_idx, const void *values, const void *z, void *y);

/* Variable-base MSM, bases in libff Jacobian layout (need not be normalised),
 * scalars Fr Montgomery, result affine-normalised.  Replaces MSMContext::msm
 * (msm/msm.cuh:82-122) and libff multi_exp BDLO12 (multiexp.tcc:165-282). */
int nkr_b200_msm_g1(nkr_b200_ctx *ctx, const void *bases, const void *scalars, uint64_t n,
                    void *out);
int nkr_b200_msm_g2(nkr_b200_ctx *ctx, const void *bases, const void *scalars, uint64_t n,
                    void *out);

/* MSM window autotuner (on by default; environment NKR_B200_AUTOTUNE=0 turns it
 * off).  The window width of every resident MSM (prepare, msm_bases_create) is
 * measured once per power-of-two size class on this device: the cost model's
 * width and its neighbours are timed on synthetic bases and the fastest kept.
 * nkr_b200_tune_msm returns (and, if needed, measures) the width for n points and
 * the measured MSM time at that size class (0 when the size is not measured).
 * Replaces choose_window_bits (backends/cuda/src/groth16_backend.cu:17-25: 8, 11
 * or 13 bits by size), which has no tuner. */
/* NTT tile shape for n = 2^k points, chosen on this device when the size's tables
 * are built (the first NTT of that size, or prepare): every pass split with 7..10
 * radix-2 stages per pass and 1, 2 or 4 butterflies per thread and stage is timed
 * and the fastest kept (sizes below 2^14 and NKR_B200_AUTOTUNE=0 keep 10 and 1).
 * The reference's NTT has fixed launch shapes (ntt/ntt.cuh:126-158). */
int nkr_b200_tune_ntt(nkr_b200_ctx *ctx, uint64_t n, int *max_stages, int *bfly_per_thread);
int nkr_b200_set_autotune(nkr_b200_ctx *ctx, int enable);
int nkr_b200_tune_msm(nkr_b200_ctx *ctx, uint64_t n, int *window_bits, float *ms);
/* Measured MSM window widths persist across processes (the reference's CLI proves
 * once per process and would otherwise re-measure on every run):
 * nkr_b200_tune_save writes this context's measured size classes to a text file;
 * nkr_b200_tune_load takes them back (loaded = size classes read), refusing a file
 * written on a different device model or SM count. */
int nkr_b200_tune_save(nkr_b200_ctx *ctx, const char *path);
int nkr_b200_tune_load(nkr_b200_ctx *ctx, const char *path, int *loaded);

/* Resident-bases MSM (the prove path's form): bases uploaded and expanded once
 * into per-window copies, then any number of MSMs with new scalars. */
int nkr_b200_msm_bases_create(nkr_b200_ctx *ctx, int group, const void *bases, uint64_t n,
                              nkr_b200_msm_bases **out);
int nkr_b200_msm_bases_run(nkr_b200_msm_bases *b, const void *scalars, uint64_t n, void *out,
                           float *device_ms);
void nkr_b200_msm_bases_free(nkr_b200_msm_bases *b);

/* Statistics of the last nkr_b200_msm_bases_run: device time of the whole MSM
 * and of the bucket-accumulation kernel (CUDA events on its stream), the number
 * of (point, nonzero digit) entries it accumulated, accumulation tasks, window
 * shape and bucket count; then the other phases' device times: the digit sort,
 * the fix-up levels of buckets spread over many segments, the first bucket
 * reduction level, and the remaining reduction levels with the final combination. */
typedef struct {
    float total_ms, acc_ms;
    uint64_t entries, tasks;
    uint32_t window_bits, windows, buckets;
    float sort_ms, fixup_ms, reduce_first_ms, reduce_levels_ms;
} nkr_b200_msm_stats;
int nkr_b200_msm_bases_stats(const nkr_b200_msm_bases *b, nkr_b200_msm_stats *out);

/* Kernels this library has launched in this process (for launch accounting). */
uint64_t nkr_b200_launch_count(void);

/* ---- field / group primitives (tests and microbenchmarks) ------------------ */

/* Elementwise field op over n pairs (host buffers): field 0 Fr, 1 Fq, 2 Fq2;
 * op 0 mul, 1 add, 2 sub, 3 sqr, 4 inverse, 5 to_mont, 6 from_mont.  Fields 3
 * (Fq) and 4 (Fq2) run ops 0..3 and 4 = negation in the MSM's FP64-limb
 * arithmetic (same inputs and outputs as fields 1 and 2). */
int nkr_b200_field_op(nkr_b200_ctx *ctx, int field, int op, const void *a, const void *b,
                      void *out, uint64_t n);
/* Elementwise group op: group 1 G1, 2 G2; inputs affine-normalised Jacobian layout.
 * op 0 add, 1 double (b ignored), 2 scalar multiple by Fr b (Montgomery). */
int nkr_b200_group_op(nkr_b200_ctx *ctx, int group, int op, const void *a, const void *b,
                      void *out, uint64_t n);
/* Throughput microbenchmark of the Montgomery product: field 0 Fr, 1 Fq; bits
 * 8.. select the formulation (0 the library's product, 1 a 64-bit-accumulation
 * variant, 2 squaring, 3 the 52-bit-limb FP64 product, 4 the same lazily
 * reduced to [0, 2p)).  Returns products per second and the best kernel ms. */
int nkr_b200_bench_mul(nkr_b200_ctx *ctx, int field, double *muls_per_s, double *ms);

/* ---- setup ------------------------------------------------------------------ */

/* Caller-allocated outputs of nkr_b200_setup, libff Jacobian layout (Z = 1). */
typedef struct {
    void *a_query, *b_g1_query, *l_query; /* G1[cols] */
    void *b_g2_query;                     /* G2[cols] */
    void *h_query;                        /* G1[rows] */
    void *ic;                             /* G1[public_inputs + 1] (verification key) */
    void *alpha_g1, *beta_g1, *delta_g1;  /* G1 */
    void *beta_g2, *delta_g2, *gamma_g2;  /* G2 */
} nkr_b200_setup_out;

/* Groth16 setup with given toxic waste Fr[5] = {t, alpha, beta, gamma, delta}
 * (Montgomery): query scalars on the host, fixed-base multiples on the GPU.
 * Replaces Backend::setup (backends/cpu/src/backend.cpp:41-154; CUDA
 * groth16_backend.cu:105-212) except the VK pairing e(alpha, beta), which the
 * verifier side forms from alpha_g1 and beta_g2. */
int nkr_b200_setup(nkr_b200_ctx *ctx, const nkr_b200_circuit *circuit, const void *toxic,
                   const nkr_b200_setup_out *out);

/* ---- seeded circuit + witness generators --------------------------------- */

typedef struct nkr_b200_r1cs nkr_b200_r1cs;

/* Builds one of the reference's benchmark circuits with a satisfying witness,
 * entry for entry as groth16-gen does (protocols/groth16/app/gen.cpp:42-197,
 * r1cs/r1cs.hpp:64-98), from a seed instead of random_device.
 * kind: "matmul" (param = size), "poseidon" (param = hash count),
 * "sql-aggregate" (param = rows, a power of two), "fibonacci" (param = steps).
 * density: 0 full, 1 hybrid (50%), 2 sparse (10%) (common/include/density.hpp). */
int nkr_b200_r1cs_generate(const char *kind, uint64_t param, int density, uint64_t seed,
                           nkr_b200_r1cs **out);
/* sizes[8] = rows, cols, public_inputs, constraints, variables, nnz A, nnz B, nnz C */
int nkr_b200_r1cs_info(const nkr_b200_r1cs *r, uint64_t *sizes);
/* Points a circuit view (and the witness, Fr[cols]) at the generator's arrays;
 * valid until nkr_b200_r1cs_free. */
int nkr_b200_r1cs_view(const nkr_b200_r1cs *r, nkr_b200_circuit *view, const void **witness);
void nkr_b200_r1cs_free(nkr_b200_r1cs *r);
/* Poseidon hash2 over Fr (Montgomery) -- common/include/crypto/poseidon.hpp:114-119 */
int nkr_b200_poseidon_hash2(const void *left, const void *right, void *out);
/* The 195 round constants and 3x3 MDS (Montgomery) -- crypto/poseidon_constants.inc */
int nkr_b200_poseidon_parameters(void *round_constants, void *mds);

#ifdef __cplusplus
}
#endif

#endif /* NKR_B200_H */
