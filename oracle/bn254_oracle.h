/*
 * bn254_oracle.h -- CPU restatement of the reference's Groth16 prove path
 * (BN254 / alt_bn128), used ONLY as test infrastructure: the parity checker for
 * the CUDA path and the CPU-baseline leg of the benchmark.  Nothing in the
 * product library links or calls this code.
 *
 * Parity of this restatement is pinned against the reference's own CPU code
 * compiled from its sources into oracle/_ref (libff + libfqfft + the groth16
 * CPU backend) and against the reference's Poseidon known-answer vector; see
 * tests/test_oracle.py.
 *
 * Layouts (identical to libff's in-memory layout on x86-64):
 *   fe  = 4 x u64 little-endian, Montgomery form (R = 2^256), value < modulus
 *   G1 affine = {x, y} (64 B);  G1 Jacobian = {X, Y, Z} (96 B), infinity <=> Z = 0
 *   Fq2 = {c0, c1};  G2 affine = 128 B;  G2 Jacobian = 192 B
 *   Affine infinity is encoded the libff way after to_affine_coordinates():
 *   X = 0, Y = 1 (Montgomery one), i.e. the 64/128 bytes of (0, 1).
 */
#ifndef NKR_BN254_ORACLE_H
#define NKR_BN254_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* field element ops, Montgomery in/out; which = 0 -> Fr, 1 -> Fq */
void orc_fe_mul(int which, const uint64_t a[4], const uint64_t b[4], uint64_t out[4]);
void orc_fe_add(int which, const uint64_t a[4], const uint64_t b[4], uint64_t out[4]);
void orc_fe_sub(int which, const uint64_t a[4], const uint64_t b[4], uint64_t out[4]);
void orc_fe_inv(int which, const uint64_t a[4], uint64_t out[4]);
void orc_fe_to_mont(int which, const uint64_t canon[4], uint64_t out[4]);
void orc_fe_from_mont(int which, const uint64_t mont[4], uint64_t out[4]);
/* Fr constants (Montgomery): 0 one, 1 multiplicative generator 5, 2 2^28-th root of unity */
void orc_fr_constant(int which, uint64_t out[4]);

/* libfqfft radix-2 domain operations on n = 2^k Fr values, in place.
 * op: 0 FFT, 1 iFFT, 2 cosetFFT(g=5), 3 icosetFFT(g=5), 4 divide_by_Z_on_coset */
int orc_domain_op(int op, uint64_t *data, uint64_t n);

/* CSR sparse matrix-vector product over Fr: y[r] = sum_j values[j] * z[col_idx[j]] */
void orc_spmv(uint64_t rows, const uint32_t *row_ptr, const uint32_t *col_idx,
              const uint64_t *values, const uint64_t *z, uint64_t *y);

/* G1 / G2 group ops on Jacobian points; results affine (libff encoding) */
void orc_g1_to_affine(const uint64_t *jac, uint64_t *aff);
void orc_g2_to_affine(const uint64_t *jac, uint64_t *aff);
void orc_g1_add_affine(const uint64_t *a, const uint64_t *b, uint64_t *out);   /* affine in/out */
void orc_g2_add_affine(const uint64_t *a, const uint64_t *b, uint64_t *out);
void orc_g1_mul_affine(const uint64_t *p, const uint64_t k[4], uint64_t *out); /* k Montgomery Fr */
void orc_g2_mul_affine(const uint64_t *p, const uint64_t k[4], uint64_t *out);
void orc_g1_generator(uint64_t *aff);
void orc_g2_generator(uint64_t *aff);
int orc_g1_on_curve(const uint64_t *aff);
int orc_g2_on_curve(const uint64_t *aff);
/* k_i P for n scalars (Fr Montgomery) and one affine base P of group 1 or 2;
 * results affine (64 / 128 B each).  threads <= 0 -> all cores. */
void orc_fixed_base(int group, const uint64_t *base_aff, const uint64_t *scalars, uint64_t n,
                    int threads, uint64_t *out_aff);

/* Multi-scalar multiplication: bases are AFFINE (64 / 128 B) in libff encoding,
 * scalars Fr Montgomery; result affine.  threads <= 0 -> all cores. */
void orc_msm_g1(const uint64_t *bases_aff, const uint64_t *scalars, uint64_t n, int threads,
                uint64_t *out_aff);
void orc_msm_g2(const uint64_t *bases_aff, const uint64_t *scalars, uint64_t n, int threads,
                uint64_t *out_aff);

/* Quotient polynomial H of the reference CPU prove (backend.cpp:171-179):
 * inputs az, bz, cz (evaluations, n values each) are consumed; H written to h. */
int orc_quotient(uint64_t n, uint64_t *az, uint64_t *bz, uint64_t *cz, uint64_t *h);

/* Full raw prove (backend.cpp:156-201).  Proving key queries are affine.
 * g1_out = {ar, bs1, zk, qz} affine (4 x 64 B); g2_out = bs2 affine (128 B). */
typedef struct {
    uint64_t rows, cols, public_inputs;
    const uint32_t *row_ptr[3];
    const uint32_t *col_idx[3];
    const uint64_t *values[3];
} orc_circuit;

typedef struct {
    const uint64_t *a_query, *b_g1_query, *b_g2_query, *l_query, *h_query; /* affine */
    const uint64_t *alpha_g1, *beta_g1, *beta_g2, *delta_g1, *delta_g2;     /* affine */
} orc_pk;

int orc_prove(const orc_circuit *c, const orc_pk *pk, const uint64_t *witness, int threads,
              uint64_t *g1_out, uint64_t *g2_out);

/* Blinding (protocol.cpp:85-94) with given r, s (Fr Montgomery).
 * raw_g1 = {ar, bs1, zk, qz}, raw_g2 = bs2 (affine).  Output proof {A (G1), B (G2), C (G1)}
 * affine: out_a 64 B, out_b 128 B, out_c 64 B. */
void orc_blind(const orc_pk *pk, const uint64_t *raw_g1, const uint64_t *raw_g2,
               const uint64_t r[4], const uint64_t s[4], uint64_t *out_a, uint64_t *out_b,
               uint64_t *out_c);

/* Seeded restatement of the CPU setup's scalar part (backend.cpp:41-107):
 * given toxic waste t, alpha, beta, gamma, delta (Fr Montgomery), computes the
 * query scalars at[cols], bt[cols], lt[cols] (zero for public columns),
 * ic[public+1] and ht[rows] (last entry zero). */
int orc_setup_scalars(const orc_circuit *c, const uint64_t toxic[5][4], uint64_t *at,
                      uint64_t *bt, uint64_t *lt, uint64_t *ic, uint64_t *ht);

/* Poseidon (width 3, x^5, 8 full + 57 partial rounds) hash2 given the round
 * constants (195) and MDS (9) in Montgomery form. */
void orc_poseidon_hash2(const uint64_t *rc, const uint64_t *mds, const uint64_t l[4],
                        const uint64_t r[4], uint64_t out[4]);

#ifdef __cplusplus
}
#endif

#endif
