/*
 * bn254_oracle.c -- CPU restatement of the reference's Groth16 prove path over
 * BN254 (alt_bn128).  TEST INFRASTRUCTURE ONLY: the parity checker for the CUDA
 * path and the timed CPU baseline; the product library never links it.
 *
 * What each part restates (paths inside the reference project):
 *   field arithmetic   libff Fp_model Montgomery (libff/algebra/fields/fp.tcc),
 *                      constants libff/algebra/curves/alt_bn128/alt_bn128_init.cpp:20-61
 *   Fq2                libff/algebra/fields/fp2.tcc (u^2 = -1, alt_bn128_init.cpp)
 *   G1/G2 group law    libff alt_bn128_g1.cpp / alt_bn128_g2.cpp (Jacobian, Z=0 is
 *                      infinity, to_affine_coordinates: infinity -> (0, 1))
 *   radix-2 FFT        libfqfft basic_radix2_domain_aux.tcc:44-79 (_basic_serial_radix2_FFT),
 *                      basic_radix2_domain.tcc:40-112 (iFFT, cosetFFT, icosetFFT,
 *                      divide_by_Z_on_coset), _multiply_by_coset aux.tcc:171-180,
 *                      root of unity libff field_utils.tcc:38-51
 *   SpMV               protocols/groth16/backends/cpu/src/backend.cpp:25-35
 *   quotient H         backend.cpp:171-179
 *   MSM                any correct algorithm gives the same canonical point; this is a
 *                      windowed bucket method in the spirit of libff BDLO12
 *                      (libff/algebra/scalar_multiplication/multiexp.tcc:165-282)
 *   prove              backend.cpp:156-201
 *   blind              protocols/groth16/common/src/protocol.cpp:85-94 (r, s given)
 *   setup scalars      backend.cpp:41-107, Lagrange values basic_radix2_domain_aux.tcc:182-237
 *   Poseidon hash2     common/include/crypto/poseidon.hpp:86-119
 */
#include "bn254_oracle.h"

#include <pthread.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

typedef unsigned __int128 u128;

/* ------------------------------------------------------------------------- */
/* prime fields                                                              */
/* ------------------------------------------------------------------------- */

typedef struct {
    uint64_t p[4];
    uint64_t inv;   /* -p^{-1} mod 2^64 */
    uint64_t r2[4]; /* 2^512 mod p */
    uint64_t one[4];
} field_t;

static field_t FQ, FR;
static uint64_t FR_GEN[4], FR_ROOT[4]; /* Montgomery: 5 and 5^((r-1)/2^28) */
static uint64_t G1_GEN[8], G2_GEN[16], G2_B[8], G1_B[4];
static pthread_once_t g_once = PTHREAD_ONCE_INIT;

static int geq4(const uint64_t *a, const uint64_t *b)
{
    for (int i = 3; i >= 0; --i) {
        if (a[i] > b[i]) return 1;
        if (a[i] < b[i]) return 0;
    }
    return 1;
}

static uint64_t sub4(uint64_t *out, const uint64_t *a, const uint64_t *b)
{
    uint64_t borrow = 0;
    for (int i = 0; i < 4; ++i) {
        u128 d = (u128)a[i] - b[i] - borrow;
        out[i] = (uint64_t)d;
        borrow = (uint64_t)(d >> 64) ? 1 : 0;
    }
    return borrow;
}

static uint64_t add4(uint64_t *out, const uint64_t *a, const uint64_t *b)
{
    u128 c = 0;
    for (int i = 0; i < 4; ++i) {
        c = (u128)a[i] + b[i] + (uint64_t)(c >> 64);
        out[i] = (uint64_t)c;
    }
    return (uint64_t)(c >> 64);
}

static int is_zero4(const uint64_t *a) { return !(a[0] | a[1] | a[2] | a[3]); }
static int eq4(const uint64_t *a, const uint64_t *b)
{
    return a[0] == b[0] && a[1] == b[1] && a[2] == b[2] && a[3] == b[3];
}

/* CIOS Montgomery product: out = a*b/2^256 mod p, inputs < p */
static void fmul(const field_t *F, const uint64_t *a, const uint64_t *b, uint64_t *out)
{
    uint64_t t[6] = {0, 0, 0, 0, 0, 0};
    for (int i = 0; i < 4; ++i) {
        u128 c = 0;
        for (int j = 0; j < 4; ++j) {
            c = (u128)a[j] * b[i] + t[j] + (uint64_t)(c >> 64);
            t[j] = (uint64_t)c;
        }
        c = (u128)t[4] + (uint64_t)(c >> 64);
        t[4] = (uint64_t)c;
        t[5] = (uint64_t)(c >> 64);
        const uint64_t m = t[0] * F->inv;
        c = (u128)m * F->p[0] + t[0];
        for (int j = 1; j < 4; ++j) {
            c = (u128)m * F->p[j] + t[j] + (uint64_t)(c >> 64);
            t[j - 1] = (uint64_t)c;
        }
        c = (u128)t[4] + (uint64_t)(c >> 64);
        t[3] = (uint64_t)c;
        t[4] = t[5] + (uint64_t)(c >> 64);
    }
    uint64_t r[4];
    if (t[4] || geq4(t, F->p)) {
        sub4(r, t, F->p);
        memcpy(out, r, 32);
    } else {
        memcpy(out, t, 32);
    }
}

static void fadd(const field_t *F, const uint64_t *a, const uint64_t *b, uint64_t *out)
{
    uint64_t t[4];
    uint64_t c = add4(t, a, b);
    if (c || geq4(t, F->p)) sub4(t, t, F->p);
    memcpy(out, t, 32);
}

static void fsub(const field_t *F, const uint64_t *a, const uint64_t *b, uint64_t *out)
{
    uint64_t t[4];
    if (sub4(t, a, b)) add4(t, t, F->p);
    memcpy(out, t, 32);
}

static void fneg(const field_t *F, const uint64_t *a, uint64_t *out)
{
    if (is_zero4(a)) {
        memset(out, 0, 32);
        return;
    }
    sub4(out, F->p, a);
}

/* out = a^e (e canonical, 4 limbs) in Montgomery form */
static void fpow(const field_t *F, const uint64_t *a, const uint64_t *e, uint64_t *out)
{
    uint64_t acc[4], base[4];
    memcpy(acc, F->one, 32);
    memcpy(base, a, 32);
    for (int i = 255; i >= 0; --i) {
        fmul(F, acc, acc, acc);
        if ((e[i / 64] >> (i % 64)) & 1) fmul(F, acc, base, acc);
    }
    memcpy(out, acc, 32);
}

static void finv(const field_t *F, const uint64_t *a, uint64_t *out)
{
    uint64_t e[4], two[4] = {2, 0, 0, 0};
    sub4(e, F->p, two);
    fpow(F, a, e, out);
}

static void to_mont(const field_t *F, const uint64_t *a, uint64_t *out) { fmul(F, a, F->r2, out); }
static void from_mont(const field_t *F, const uint64_t *a, uint64_t *out)
{
    uint64_t one[4] = {1, 0, 0, 0};
    fmul(F, a, one, out);
}

/* parse a decimal string into 4 limbs (value must fit) */
static void dec4(const char *s, uint64_t *out)
{
    memset(out, 0, 32);
    for (; *s; ++s) {
        u128 c = (uint64_t)(*s - '0');
        for (int i = 0; i < 4; ++i) {
            c += (u128)out[i] * 10;
            out[i] = (uint64_t)c;
            c >>= 64;
        }
    }
}

static void init_field(field_t *F, const char *modulus)
{
    dec4(modulus, F->p);
    /* Newton iteration for p^{-1} mod 2^64 */
    uint64_t x = 1;
    for (int i = 0; i < 7; ++i) x *= 2 - F->p[0] * x;
    F->inv = (uint64_t)0 - x;
    /* r2 = 2^512 mod p by doubling 1 */
    uint64_t t[4] = {1, 0, 0, 0};
    for (int i = 0; i < 512; ++i) {
        uint64_t c = add4(t, t, t);
        if (c || geq4(t, F->p)) sub4(t, t, F->p);
    }
    memcpy(F->r2, t, 32);
    uint64_t one[4] = {1, 0, 0, 0};
    to_mont(F, one, F->one);
}

static void fq_from_dec(const char *s, uint64_t *out)
{
    uint64_t c[4];
    dec4(s, c);
    to_mont(&FQ, c, out);
}

static void init_all(void)
{
    /* alt_bn128_init.cpp: Fq and Fr moduli */
    init_field(&FQ, "21888242871839275222246405745257275088696311157297823662689037894645226208583");
    init_field(&FR, "21888242871839275222246405745257275088548364400416034343698204186575808495617");
    uint64_t five[4] = {5, 0, 0, 0}, e[4], one[4] = {1, 0, 0, 0};
    to_mont(&FR, five, FR_GEN);
    /* root of unity: g^((r-1)/2^28), s = 28 */
    sub4(e, FR.p, one);
    for (int k = 0; k < 28; ++k) {
        for (int i = 0; i < 3; ++i) e[i] = (e[i] >> 1) | (e[i + 1] << 63);
        e[3] >>= 1;
    }
    fpow(&FR, FR_GEN, e, FR_ROOT);
    /* G1: y^2 = x^3 + 3, generator (1, 2) */
    uint64_t three[4] = {3, 0, 0, 0}, two[4] = {2, 0, 0, 0};
    to_mont(&FQ, three, G1_B);
    to_mont(&FQ, one, G1_GEN);
    to_mont(&FQ, two, G1_GEN + 4);
    /* G2 generator (alt_bn128_init.cpp G2_one), coordinates c0 + c1*u */
    fq_from_dec("10857046999023057135944570762232829481370756359578518086990519993285655852781", G2_GEN);
    fq_from_dec("11559732032986387107991004021392285783925812861821192530917403151452391805634", G2_GEN + 4);
    fq_from_dec("8495653923123431417604973247489272438418190587263600148770280649306958101930", G2_GEN + 8);
    fq_from_dec("4082367875863433681332203403145435568316851327593401208105741076214120093531", G2_GEN + 12);
}

static void init(void) { pthread_once(&g_once, init_all); }

/* ------------------------------------------------------------------------- */
/* extension field ops, generic over degree d = 1 (Fq) or 2 (Fq2, u^2 = -1)  */
/* ------------------------------------------------------------------------- */

static void emul(int d, const uint64_t *a, const uint64_t *b, uint64_t *out)
{
    if (d == 1) {
        fmul(&FQ, a, b, out);
        return;
    }
    uint64_t t0[4], t1[4], t2[4], t3[4];
    fmul(&FQ, a, b, t0);         /* a0 b0 */
    fmul(&FQ, a + 4, b + 4, t1); /* a1 b1 */
    fmul(&FQ, a, b + 4, t2);     /* a0 b1 */
    fmul(&FQ, a + 4, b, t3);     /* a1 b0 */
    fsub(&FQ, t0, t1, out);
    fadd(&FQ, t2, t3, out + 4);
}
static void eadd(int d, const uint64_t *a, const uint64_t *b, uint64_t *o)
{
    for (int i = 0; i < d; ++i) fadd(&FQ, a + 4 * i, b + 4 * i, o + 4 * i);
}
static void esub(int d, const uint64_t *a, const uint64_t *b, uint64_t *o)
{
    for (int i = 0; i < d; ++i) fsub(&FQ, a + 4 * i, b + 4 * i, o + 4 * i);
}
static int eis_zero(int d, const uint64_t *a)
{
    for (int i = 0; i < d; ++i)
        if (!is_zero4(a + 4 * i)) return 0;
    return 1;
}
static int eeq(int d, const uint64_t *a, const uint64_t *b)
{
    for (int i = 0; i < d; ++i)
        if (!eq4(a + 4 * i, b + 4 * i)) return 0;
    return 1;
}
static void eone(int d, uint64_t *o)
{
    memcpy(o, FQ.one, 32);
    if (d == 2) memset(o + 4, 0, 32);
}
static void einv(int d, const uint64_t *a, uint64_t *o)
{
    if (d == 1) {
        finv(&FQ, a, o);
        return;
    }
    /* 1/(a0 + a1 u) = (a0 - a1 u) / (a0^2 + a1^2) */
    uint64_t t0[4], t1[4], n[4], ni[4];
    fmul(&FQ, a, a, t0);
    fmul(&FQ, a + 4, a + 4, t1);
    fadd(&FQ, t0, t1, n);
    finv(&FQ, n, ni);
    uint64_t neg1[4];
    fneg(&FQ, a + 4, neg1);
    fmul(&FQ, a, ni, o);
    fmul(&FQ, neg1, ni, o + 4);
}

/* ------------------------------------------------------------------------- */
/* curve points: Jacobian (X, Y, Z), infinity <=> Z == 0; a = 0 curves       */
/* ------------------------------------------------------------------------- */

#define EMAX 8 /* max limbs of one coordinate (Fq2) */
typedef struct {
    uint64_t x[EMAX], y[EMAX], z[EMAX];
} jac_t;

static void jac_set_inf(int d, jac_t *P)
{
    memset(P, 0, sizeof(*P));
    eone(d, P->y);
    (void)d;
}

static void jac_dbl(int d, const jac_t *P, jac_t *R)
{
    if (eis_zero(d, P->z)) {
        *R = *P;
        return;
    }
    /* dbl-2009-l */
    uint64_t A[EMAX], B[EMAX], C[EMAX], D[EMAX], E[EMAX], F[EMAX], t[EMAX];
    emul(d, P->x, P->x, A);
    emul(d, P->y, P->y, B);
    emul(d, B, B, C);
    eadd(d, P->x, B, t);
    emul(d, t, t, t);
    esub(d, t, A, t);
    esub(d, t, C, t);
    eadd(d, t, t, D);
    eadd(d, A, A, E);
    eadd(d, E, A, E);
    emul(d, E, E, F);
    jac_t out;
    uint64_t D2[EMAX];
    eadd(d, D, D, D2);
    esub(d, F, D2, out.x);
    esub(d, D, out.x, t);
    emul(d, E, t, t);
    uint64_t C8[EMAX];
    eadd(d, C, C, C8);
    eadd(d, C8, C8, C8);
    eadd(d, C8, C8, C8);
    esub(d, t, C8, out.y);
    emul(d, P->y, P->z, t);
    eadd(d, t, t, out.z);
    *R = out;
}

static void jac_add(int d, const jac_t *P, const jac_t *Q, jac_t *R)
{
    if (eis_zero(d, P->z)) {
        *R = *Q;
        return;
    }
    if (eis_zero(d, Q->z)) {
        *R = *P;
        return;
    }
    /* add-2007-bl with the equal-x branch */
    uint64_t Z1Z1[EMAX], Z2Z2[EMAX], U1[EMAX], U2[EMAX], S1[EMAX], S2[EMAX], t[EMAX];
    emul(d, P->z, P->z, Z1Z1);
    emul(d, Q->z, Q->z, Z2Z2);
    emul(d, P->x, Z2Z2, U1);
    emul(d, Q->x, Z1Z1, U2);
    emul(d, P->y, Q->z, t);
    emul(d, t, Z2Z2, S1);
    emul(d, Q->y, P->z, t);
    emul(d, t, Z1Z1, S2);
    if (eeq(d, U1, U2)) {
        if (eeq(d, S1, S2)) {
            jac_dbl(d, P, R);
        } else {
            jac_set_inf(d, R);
        }
        return;
    }
    uint64_t H[EMAX], I[EMAX], J[EMAX], r[EMAX], V[EMAX];
    esub(d, U2, U1, H);
    eadd(d, H, H, I);
    emul(d, I, I, I);
    emul(d, H, I, J);
    esub(d, S2, S1, r);
    eadd(d, r, r, r);
    emul(d, U1, I, V);
    jac_t out;
    emul(d, r, r, t);
    esub(d, t, J, t);
    esub(d, t, V, t);
    esub(d, t, V, out.x);
    esub(d, V, out.x, t);
    emul(d, r, t, t);
    uint64_t s1j[EMAX];
    emul(d, S1, J, s1j);
    eadd(d, s1j, s1j, s1j);
    esub(d, t, s1j, out.y);
    eadd(d, P->z, Q->z, t);
    emul(d, t, t, t);
    esub(d, t, Z1Z1, t);
    esub(d, t, Z2Z2, t);
    emul(d, t, H, out.z);
    *R = out;
}

/* affine (libff encoding, infinity = (0, 1)) <-> Jacobian */
static int aff_is_inf(int d, const uint64_t *a)
{
    uint64_t one[EMAX];
    eone(d, one);
    return eis_zero(d, a) && eeq(d, a + 4 * d, one);
}

static void aff_to_jac(int d, const uint64_t *a, jac_t *P)
{
    if (aff_is_inf(d, a)) {
        jac_set_inf(d, P);
        return;
    }
    memset(P, 0, sizeof(*P));
    memcpy(P->x, a, 32 * d);
    memcpy(P->y, a + 4 * d, 32 * d);
    eone(d, P->z);
}

static void jac_to_aff(int d, const jac_t *P, uint64_t *a)
{
    if (eis_zero(d, P->z)) {
        memset(a, 0, 64 * d);
        eone(d, a + 4 * d);
        return;
    }
    uint64_t zi[EMAX], zi2[EMAX], zi3[EMAX];
    einv(d, P->z, zi);
    emul(d, zi, zi, zi2);
    emul(d, zi2, zi, zi3);
    emul(d, P->x, zi2, a);
    emul(d, P->y, zi3, a + 4 * d);
}

static void jac_from_raw(int d, const uint64_t *raw, jac_t *P)
{
    memset(P, 0, sizeof(*P));
    memcpy(P->x, raw, 32 * d);
    memcpy(P->y, raw + 4 * d, 32 * d);
    memcpy(P->z, raw + 8 * d, 32 * d);
}

/* scalar multiple by a canonical 256-bit integer, double-and-add */
static void jac_mul_canon(int d, const jac_t *P, const uint64_t *k, jac_t *R)
{
    jac_t acc;
    jac_set_inf(d, &acc);
    for (int i = 255; i >= 0; --i) {
        jac_dbl(d, &acc, &acc);
        if ((k[i / 64] >> (i % 64)) & 1) jac_add(d, &acc, P, &acc);
    }
    *R = acc;
}

static int on_curve(int d, const uint64_t *a)
{
    if (aff_is_inf(d, a)) return 1;
    uint64_t y2[EMAX], x3[EMAX];
    emul(d, a + 4 * d, a + 4 * d, y2);
    emul(d, a, a, x3);
    emul(d, x3, a, x3);
    eadd(d, x3, d == 1 ? G1_B : G2_B, x3);
    return eeq(d, y2, x3);
}

/* ------------------------------------------------------------------------- */
/* exported field / point helpers                                             */
/* ------------------------------------------------------------------------- */

static const field_t *pick(int which) { return which == 0 ? &FR : &FQ; }

void orc_fe_mul(int which, const uint64_t a[4], const uint64_t b[4], uint64_t out[4])
{
    init();
    fmul(pick(which), a, b, out);
}
void orc_fe_add(int which, const uint64_t a[4], const uint64_t b[4], uint64_t out[4])
{
    init();
    fadd(pick(which), a, b, out);
}
void orc_fe_sub(int which, const uint64_t a[4], const uint64_t b[4], uint64_t out[4])
{
    init();
    fsub(pick(which), a, b, out);
}
void orc_fe_inv(int which, const uint64_t a[4], uint64_t out[4])
{
    init();
    finv(pick(which), a, out);
}
void orc_fe_to_mont(int which, const uint64_t c[4], uint64_t out[4])
{
    init();
    to_mont(pick(which), c, out);
}
void orc_fe_from_mont(int which, const uint64_t m[4], uint64_t out[4])
{
    init();
    from_mont(pick(which), m, out);
}
void orc_fr_constant(int which, uint64_t out[4])
{
    init();
    memcpy(out, which == 0 ? FR.one : which == 1 ? FR_GEN : FR_ROOT, 32);
}

static void g2_init_b(void)
{
    /* twist coefficient b' = 3 / (9 + u) */
    static int done = 0;
    if (done) return;
    uint64_t nine[4] = {9, 0, 0, 0}, one[4] = {1, 0, 0, 0}, xi[8], xii[8], three[8];
    to_mont(&FQ, nine, xi);
    to_mont(&FQ, one, xi + 4);
    einv(2, xi, xii);
    memcpy(three, G1_B, 32);
    memset(three + 4, 0, 32);
    emul(2, three, xii, G2_B);
    done = 1;
}

void orc_g1_to_affine(const uint64_t *jac, uint64_t *aff)
{
    init();
    jac_t P;
    jac_from_raw(1, jac, &P);
    jac_to_aff(1, &P, aff);
}
void orc_g2_to_affine(const uint64_t *jac, uint64_t *aff)
{
    init();
    jac_t P;
    jac_from_raw(2, jac, &P);
    jac_to_aff(2, &P, aff);
}
static void add_affine(int d, const uint64_t *a, const uint64_t *b, uint64_t *out)
{
    jac_t P, Q, R;
    aff_to_jac(d, a, &P);
    aff_to_jac(d, b, &Q);
    jac_add(d, &P, &Q, &R);
    jac_to_aff(d, &R, out);
}
void orc_g1_add_affine(const uint64_t *a, const uint64_t *b, uint64_t *out)
{
    init();
    add_affine(1, a, b, out);
}
void orc_g2_add_affine(const uint64_t *a, const uint64_t *b, uint64_t *out)
{
    init();
    add_affine(2, a, b, out);
}
static void mul_affine(int d, const uint64_t *p, const uint64_t *k, uint64_t *out)
{
    uint64_t kc[4];
    from_mont(&FR, k, kc);
    jac_t P, R;
    aff_to_jac(d, p, &P);
    jac_mul_canon(d, &P, kc, &R);
    jac_to_aff(d, &R, out);
}
void orc_g1_mul_affine(const uint64_t *p, const uint64_t k[4], uint64_t *out)
{
    init();
    mul_affine(1, p, k, out);
}
void orc_g2_mul_affine(const uint64_t *p, const uint64_t k[4], uint64_t *out)
{
    init();
    mul_affine(2, p, k, out);
}
void orc_g1_generator(uint64_t *aff)
{
    init();
    memcpy(aff, G1_GEN, 64);
}
void orc_g2_generator(uint64_t *aff)
{
    init();
    memcpy(aff, G2_GEN, 128);
}
int orc_g1_on_curve(const uint64_t *aff)
{
    init();
    return on_curve(1, aff);
}
int orc_g2_on_curve(const uint64_t *aff)
{
    init();
    g2_init_b();
    return on_curve(2, aff);
}

/* Fixed-base multiples k_i P of one point (the setup's query points k_i G,
 * backend.cpp:124-145, where libff uses windowed_exp; any correct method gives
 * the same canonical affine points): a table T[j][d] = d 2^(8j) P for the 32
 * byte windows j and digits d, then k_i P = sum_j T[j][byte_j(k_i)]. */
typedef struct {
    int d;
    uint64_t i0, i1;
    const jac_t *table; /* 32 x 256 */
    const uint64_t *scalars;
    uint64_t *out;
} fixed_job;

static void *fixed_worker(void *arg)
{
    fixed_job *J = (fixed_job *)arg;
    const int d = J->d;
    for (uint64_t i = J->i0; i < J->i1; ++i) {
        uint64_t kc[4];
        from_mont(&FR, J->scalars + 4 * i, kc);
        jac_t acc;
        jac_set_inf(d, &acc);
        for (int j = 0; j < 32; ++j) {
            const unsigned byte = (unsigned)(kc[j / 8] >> (8 * (j % 8))) & 0xff;
            if (byte) jac_add(d, &acc, &J->table[256 * j + byte], &acc);
        }
        jac_to_aff(d, &acc, J->out + 8 * (uint64_t)d * i);
    }
    return NULL;
}

void orc_fixed_base(int group, const uint64_t *base_aff, const uint64_t *scalars, uint64_t n,
                    int threads, uint64_t *out_aff)
{
    init();
    const int d = group == 2 ? 2 : 1;
    if (d == 2) g2_init_b();
    jac_t *table = (jac_t *)malloc(sizeof(jac_t) * 32 * 256);
    jac_t step;
    aff_to_jac(d, base_aff, &step); /* 2^(8j) P */
    for (int j = 0; j < 32; ++j) {
        jac_t *row = table + 256 * j;
        jac_set_inf(d, &row[0]);
        for (int v = 1; v < 256; ++v) jac_add(d, &row[v - 1], &step, &row[v]);
        for (int b = 0; b < 8; ++b) jac_dbl(d, &step, &step);
    }
    if (threads <= 0) threads = (int)sysconf(_SC_NPROCESSORS_ONLN);
    if (threads > 64) threads = 64;
    if ((uint64_t)threads > n) threads = n ? (int)n : 1;
    pthread_t tid[64];
    fixed_job jobs[64];
    for (int t = 0; t < threads; ++t) {
        jobs[t] = (fixed_job){d, n * t / threads, n * (t + 1) / threads, table, scalars, out_aff};
        if (threads == 1)
            fixed_worker(&jobs[t]);
        else
            pthread_create(&tid[t], NULL, fixed_worker, &jobs[t]);
    }
    if (threads > 1)
        for (int t = 0; t < threads; ++t) pthread_join(tid[t], NULL);
    free(table);
}

/* ------------------------------------------------------------------------- */
/* radix-2 domain (libfqfft basic_radix2_domain)                              */
/* ------------------------------------------------------------------------- */

static int log2_exact(uint64_t n)
{
    int k = 0;
    while (((uint64_t)1 << k) < n) ++k;
    return ((uint64_t)1 << k) == n ? k : -1;
}

static uint64_t bitrev(uint64_t x, int bits)
{
    uint64_t r = 0;
    for (int i = 0; i < bits; ++i) r |= ((x >> i) & 1) << (bits - 1 - i);
    return r;
}

/* omega_n = root^(2^(28 - log n)) (field_utils.tcc get_root_of_unity) */
static void root_of_unity(int logn, uint64_t *w)
{
    memcpy(w, FR_ROOT, 32);
    for (int i = 28; i > logn; --i) fmul(&FR, w, w, w);
}

/* _basic_serial_radix2_FFT: bit-reversal permutation then iterative DIT */
static void serial_fft(uint64_t *a, uint64_t n, const uint64_t *omega)
{
    const int logn = log2_exact(n);
    for (uint64_t k = 0; k < n; ++k) {
        const uint64_t rk = bitrev(k, logn);
        if (k < rk) {
            uint64_t t[4];
            memcpy(t, a + 4 * k, 32);
            memcpy(a + 4 * k, a + 4 * rk, 32);
            memcpy(a + 4 * rk, t, 32);
        }
    }
    uint64_t m = 1;
    for (int s = 1; s <= logn; ++s) {
        uint64_t wm[4], e[4] = {n / (2 * m), 0, 0, 0};
        fpow(&FR, omega, e, wm);
        for (uint64_t k = 0; k < n; k += 2 * m) {
            uint64_t w[4];
            memcpy(w, FR.one, 32);
            for (uint64_t j = 0; j < m; ++j) {
                uint64_t t[4];
                uint64_t *x = a + 4 * (k + j), *y = a + 4 * (k + j + m);
                fmul(&FR, w, y, t);
                fsub(&FR, x, t, y);
                fadd(&FR, x, t, x);
                fmul(&FR, w, wm, w);
            }
        }
        m *= 2;
    }
}

static void multiply_by_coset(uint64_t *a, uint64_t n, const uint64_t *g)
{
    uint64_t u[4];
    memcpy(u, g, 32);
    for (uint64_t i = 1; i < n; ++i) {
        fmul(&FR, a + 4 * i, u, a + 4 * i);
        fmul(&FR, u, g, u);
    }
}

static void domain_ifft(uint64_t *a, uint64_t n, int logn)
{
    uint64_t w[4], wi[4], nn[4] = {n, 0, 0, 0}, nm[4], ninv[4];
    root_of_unity(logn, w);
    finv(&FR, w, wi);
    serial_fft(a, n, wi);
    to_mont(&FR, nn, nm);
    finv(&FR, nm, ninv);
    for (uint64_t i = 0; i < n; ++i) fmul(&FR, a + 4 * i, ninv, a + 4 * i);
}

int orc_domain_op(int op, uint64_t *a, uint64_t n)
{
    init();
    const int logn = log2_exact(n);
    if (logn < 1 || logn > 28) return 1;
    uint64_t w[4];
    root_of_unity(logn, w);
    switch (op) {
    case 0:
        serial_fft(a, n, w);
        return 0;
    case 1:
        domain_ifft(a, n, logn);
        return 0;
    case 2:
        multiply_by_coset(a, n, FR_GEN);
        serial_fft(a, n, w);
        return 0;
    case 3: {
        uint64_t gi[4];
        domain_ifft(a, n, logn);
        finv(&FR, FR_GEN, gi);
        multiply_by_coset(a, n, gi);
        return 0;
    }
    case 4: {
        /* Z(g) = g^n - 1, multiply by its inverse */
        uint64_t e[4] = {n, 0, 0, 0}, z[4], zi[4];
        fpow(&FR, FR_GEN, e, z);
        fsub(&FR, z, FR.one, z);
        finv(&FR, z, zi);
        for (uint64_t i = 0; i < n; ++i) fmul(&FR, a + 4 * i, zi, a + 4 * i);
        return 0;
    }
    default:
        return 1;
    }
}

/* ------------------------------------------------------------------------- */
/* SpMV and quotient polynomial                                              */
/* ------------------------------------------------------------------------- */

void orc_spmv(uint64_t rows, const uint32_t *row_ptr, const uint32_t *col_idx,
              const uint64_t *values, const uint64_t *z, uint64_t *y)
{
    init();
    for (uint64_t r = 0; r < rows; ++r) {
        uint64_t acc[4] = {0, 0, 0, 0}, t[4];
        for (uint32_t j = row_ptr[r]; j < row_ptr[r + 1]; ++j) {
            fmul(&FR, values + 4 * (uint64_t)j, z + 4 * (uint64_t)col_idx[j], t);
            fadd(&FR, acc, t, acc);
        }
        memcpy(y + 4 * r, acc, 32);
    }
}

int orc_quotient(uint64_t n, uint64_t *az, uint64_t *bz, uint64_t *cz, uint64_t *h)
{
    init();
    if (orc_domain_op(1, az, n) || orc_domain_op(1, bz, n) || orc_domain_op(1, cz, n)) return 1;
    orc_domain_op(2, az, n);
    orc_domain_op(2, bz, n);
    orc_domain_op(2, cz, n);
    for (uint64_t i = 0; i < n; ++i) {
        uint64_t t[4];
        fmul(&FR, az + 4 * i, bz + 4 * i, t);
        fsub(&FR, t, cz + 4 * i, h + 4 * i);
    }
    orc_domain_op(4, h, n);
    orc_domain_op(3, h, n);
    return 0;
}

/* ------------------------------------------------------------------------- */
/* multi-scalar multiplication: bucket method, windows split over threads     */
/* ------------------------------------------------------------------------- */

typedef struct {
    int d, c, w0, w1;
    uint64_t n;
    const uint64_t *bases;
    const uint64_t *canon; /* canonical scalars */
    jac_t *window_sums;    /* one per window */
} msm_job;

static void *msm_worker(void *arg)
{
    msm_job *J = (msm_job *)arg;
    const int d = J->d, c = J->c;
    const uint64_t nb = ((uint64_t)1 << c);
    jac_t *buckets = (jac_t *)malloc(sizeof(jac_t) * nb);
    const size_t stride = 8 * (size_t)d;
    for (int w = J->w0; w < J->w1; ++w) {
        for (uint64_t b = 0; b < nb; ++b) jac_set_inf(d, &buckets[b]);
        for (uint64_t i = 0; i < J->n; ++i) {
            const uint64_t *k = J->canon + 4 * i;
            /* extract bits [w*c, w*c + c) */
            uint64_t id = 0;
            for (int b = 0; b < c; ++b) {
                const int bit = w * c + b;
                if (bit < 256 && ((k[bit / 64] >> (bit % 64)) & 1)) id |= (uint64_t)1 << b;
            }
            if (!id) continue;
            jac_t P;
            aff_to_jac(d, J->bases + stride * i, &P);
            jac_add(d, &buckets[id], &P, &buckets[id]);
        }
        jac_t running, total;
        jac_set_inf(d, &running);
        jac_set_inf(d, &total);
        for (uint64_t b = nb - 1; b > 0; --b) {
            jac_add(d, &running, &buckets[b], &running);
            jac_add(d, &total, &running, &total);
        }
        J->window_sums[w] = total;
    }
    free(buckets);
    return NULL;
}

static void msm(int d, const uint64_t *bases, const uint64_t *scalars, uint64_t n, int threads,
                uint64_t *out)
{
    init();
    if (d == 2) g2_init_b();
    uint64_t *canon = (uint64_t *)malloc(32 * (n ? n : 1));
    for (uint64_t i = 0; i < n; ++i) from_mont(&FR, scalars + 4 * i, canon + 4 * i);
    int logn = 0;
    while (((uint64_t)1 << logn) < n) ++logn;
    int c = logn < 4 ? 2 : logn - 2;
    if (c > 16) c = 16;
    const int W = (254 + c - 1) / c;
    jac_t *ws = (jac_t *)malloc(sizeof(jac_t) * W);
    if (threads <= 0) threads = (int)sysconf(_SC_NPROCESSORS_ONLN);
    if (threads > W) threads = W;
    if (threads < 1) threads = 1;
    pthread_t tid[64];
    msm_job jobs[64];
    if (threads > 64) threads = 64;
    for (int t = 0; t < threads; ++t) {
        jobs[t] = (msm_job){d, c, W * t / threads, W * (t + 1) / threads, n, bases, canon, ws};
        if (threads == 1)
            msm_worker(&jobs[t]);
        else
            pthread_create(&tid[t], NULL, msm_worker, &jobs[t]);
    }
    if (threads > 1)
        for (int t = 0; t < threads; ++t) pthread_join(tid[t], NULL);
    jac_t acc;
    jac_set_inf(d, &acc);
    for (int w = W - 1; w >= 0; --w) {
        for (int i = 0; i < c; ++i) jac_dbl(d, &acc, &acc);
        jac_add(d, &acc, &ws[w], &acc);
    }
    jac_to_aff(d, &acc, out);
    free(ws);
    free(canon);
}

void orc_msm_g1(const uint64_t *bases_aff, const uint64_t *scalars, uint64_t n, int threads,
                uint64_t *out_aff)
{
    msm(1, bases_aff, scalars, n, threads, out_aff);
}

void orc_msm_g2(const uint64_t *bases_aff, const uint64_t *scalars, uint64_t n, int threads,
                uint64_t *out_aff)
{
    msm(2, bases_aff, scalars, n, threads, out_aff);
}

/* ------------------------------------------------------------------------- */
/* prove / blind / setup scalars                                             */
/* ------------------------------------------------------------------------- */

int orc_prove(const orc_circuit *c, const orc_pk *pk, const uint64_t *z, int threads,
              uint64_t *g1_out, uint64_t *g2_out)
{
    init();
    const uint64_t n = c->rows;
    if (log2_exact(n) < 1) return 1;
    uint64_t *az = (uint64_t *)malloc(32 * n), *bz = (uint64_t *)malloc(32 * n),
             *cz = (uint64_t *)malloc(32 * n), *h = (uint64_t *)malloc(32 * n);
    orc_spmv(n, c->row_ptr[0], c->col_idx[0], c->values[0], z, az);
    orc_spmv(n, c->row_ptr[1], c->col_idx[1], c->values[1], z, bz);
    orc_spmv(n, c->row_ptr[2], c->col_idx[2], c->values[2], z, cz);
    orc_quotient(n, az, bz, cz, h);
    orc_msm_g1(pk->a_query, z, c->cols, threads, g1_out);
    orc_msm_g1(pk->b_g1_query, z, c->cols, threads, g1_out + 8);
    orc_msm_g2(pk->b_g2_query, z, c->cols, threads, g2_out);
    orc_msm_g1(pk->l_query, z, c->cols, threads, g1_out + 16);
    orc_msm_g1(pk->h_query, h, n, threads, g1_out + 24);
    free(az);
    free(bz);
    free(cz);
    free(h);
    return 0;
}

void orc_blind(const orc_pk *pk, const uint64_t *raw_g1, const uint64_t *raw_g2, const uint64_t r[4],
               const uint64_t s[4], uint64_t *out_a, uint64_t *out_b, uint64_t *out_c)
{
    init();
    g2_init_b();
    uint64_t t[8], u[8], A[8], B1[8], rs[4], v[16], w[16];
    /* A = alpha + ar + r delta */
    orc_g1_mul_affine(pk->delta_g1, r, t);
    orc_g1_add_affine(pk->alpha_g1, raw_g1, u);
    orc_g1_add_affine(u, t, A);
    /* B2 = beta2 + bs2 + s delta2 */
    orc_g2_mul_affine(pk->delta_g2, s, v);
    orc_g2_add_affine(pk->beta_g2, raw_g2, w);
    orc_g2_add_affine(w, v, out_b);
    /* B1 = beta1 + bs1 + s delta1 */
    orc_g1_mul_affine(pk->delta_g1, s, t);
    orc_g1_add_affine(pk->beta_g1, raw_g1 + 8, u);
    orc_g1_add_affine(u, t, B1);
    /* C = qz + zk + s A + r B1 - (r s) delta1 */
    uint64_t acc[8];
    orc_g1_add_affine(raw_g1 + 24, raw_g1 + 16, acc);
    orc_g1_mul_affine(A, s, t);
    orc_g1_add_affine(acc, t, acc);
    orc_g1_mul_affine(B1, r, t);
    orc_g1_add_affine(acc, t, acc);
    fmul(&FR, r, s, rs);
    fneg(&FR, rs, rs);
    orc_g1_mul_affine(pk->delta_g1, rs, t);
    orc_g1_add_affine(acc, t, out_c);
    memcpy(out_a, A, 64);
}

int orc_setup_scalars(const orc_circuit *c, const uint64_t toxic[5][4], uint64_t *at, uint64_t *bt,
                      uint64_t *lt, uint64_t *ic, uint64_t *ht)
{
    init();
    const uint64_t m = c->rows, cols = c->cols;
    const int logm = log2_exact(m);
    if (logm < 1) return 1;
    const uint64_t *t = toxic[0], *alpha = toxic[1], *beta = toxic[2], *gamma = toxic[3],
                   *delta = toxic[4];
    uint64_t gi[4], di[4], tm[4], e[4] = {m, 0, 0, 0}, zt[4], omega[4];
    finv(&FR, gamma, gi);
    finv(&FR, delta, di);
    fpow(&FR, t, e, tm);
    fsub(&FR, tm, FR.one, zt);
    root_of_unity(logm, omega);
    /* Lagrange values L_i(t) (basic_radix2_domain_aux.tcc:182-237) */
    uint64_t *L = (uint64_t *)calloc(m, 32);
    if (eq4(tm, FR.one)) {
        uint64_t oi[4];
        memcpy(oi, FR.one, 32);
        for (uint64_t i = 0; i < m; ++i) {
            if (eq4(oi, t)) {
                memcpy(L + 4 * i, FR.one, 32);
                break;
            }
            fmul(&FR, oi, omega, oi);
        }
    } else {
        uint64_t mm[4] = {m, 0, 0, 0}, mmont[4], minv[4], l[4], r[4];
        to_mont(&FR, mm, mmont);
        finv(&FR, mmont, minv);
        fmul(&FR, zt, minv, l);
        memcpy(r, FR.one, 32);
        for (uint64_t i = 0; i < m; ++i) {
            uint64_t diff[4], inv[4];
            fsub(&FR, t, r, diff);
            finv(&FR, diff, inv);
            fmul(&FR, l, inv, L + 4 * i);
            fmul(&FR, l, omega, l);
            fmul(&FR, r, omega, r);
        }
    }
    uint64_t *q[3] = {at, bt, (uint64_t *)calloc(cols, 32)};
    memset(at, 0, 32 * cols);
    memset(bt, 0, 32 * cols);
    for (int k = 0; k < 3; ++k)
        for (uint64_t row = 0; row < m; ++row)
            for (uint32_t j = c->row_ptr[k][row]; j < c->row_ptr[k][row + 1]; ++j) {
                uint64_t p[4];
                fmul(&FR, c->values[k] + 4 * (uint64_t)j, L + 4 * row, p);
                uint64_t *dst = q[k] + 4 * (uint64_t)c->col_idx[k][j];
                fadd(&FR, dst, p, dst);
            }
    const uint64_t *ct = q[2];
    for (uint64_t i = 0; i < cols; ++i) {
        uint64_t x[4], y[4], s[4];
        fmul(&FR, beta, at + 4 * i, x);
        fmul(&FR, alpha, bt + 4 * i, y);
        fadd(&FR, x, y, s);
        fadd(&FR, s, ct + 4 * i, s);
        if (i > c->public_inputs) {
            fmul(&FR, s, di, lt + 4 * i);
        } else {
            memset(lt + 4 * i, 0, 32);
            fmul(&FR, s, gi, ic + 4 * i);
        }
    }
    uint64_t power[4], zd[4];
    memcpy(power, FR.one, 32);
    fmul(&FR, zt, di, zd);
    for (uint64_t i = 0; i + 1 < m; ++i) {
        fmul(&FR, power, zd, ht + 4 * i);
        fmul(&FR, power, t, power);
    }
    memset(ht + 4 * (m - 1), 0, 32);
    free(q[2]);
    free(L);
    return 0;
}

/* ------------------------------------------------------------------------- */
/* Poseidon                                                                   */
/* ------------------------------------------------------------------------- */

void orc_poseidon_hash2(const uint64_t *rc, const uint64_t *mds, const uint64_t l[4],
                        const uint64_t r[4], uint64_t out[4])
{
    init();
    uint64_t st[3][4];
    memset(st[0], 0, 32);
    memcpy(st[1], l, 32);
    memcpy(st[2], r, 32);
    int k = 0;
    for (int round = 0; round < 65; ++round) {
        for (int i = 0; i < 3; ++i) fadd(&FR, st[i], rc + 4 * (k++), st[i]);
        const int full = round < 4 || round >= 61;
        for (int i = 0; i < (full ? 3 : 1); ++i) {
            uint64_t sq[4], q4[4];
            fmul(&FR, st[i], st[i], sq);
            fmul(&FR, sq, sq, q4);
            fmul(&FR, q4, st[i], st[i]);
        }
        uint64_t mixed[3][4];
        for (int row = 0; row < 3; ++row) {
            memset(mixed[row], 0, 32);
            for (int col = 0; col < 3; ++col) {
                uint64_t p[4];
                fmul(&FR, mds + 4 * (3 * row + col), st[col], p);
                fadd(&FR, mixed[row], p, mixed[row]);
            }
        }
        memcpy(st, mixed, sizeof(st));
    }
    memcpy(out, st[0], 32);
}
