/*
 * Declarations-only stand-in for <gmp.h>, used solely to compile the reference's
 * vendored libff/libfqfft CPU path into oracle/_ref (test infrastructure).
 *
 * The image ships the GMP runtime (libgmp.so.10) but not its development header.
 * This file declares only the entry points libff, libfqfft and the reference's
 * Poseidon helper call, written from the GMP manual's documented interface
 * (types mp_limb_t / mp_size_t / mpz_t, the mpn_* low-level functions and the
 * mpz_* integer functions).  The public names are macros over the exported
 * "__gmpn_" / "__gmpz_" symbols, as the manual documents for the ABI.
 * x86-64 only: 64-bit limbs, no nail bits.
 */
#ifndef NKR_ORACLE_GMP_COMPAT_H
#define NKR_ORACLE_GMP_COMPAT_H

#include <stddef.h>
#include <stdio.h>

#if !defined(__x86_64__)
#error "gmp compat header supports x86-64 (64-bit limbs) only"
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef unsigned long int mp_limb_t;
typedef long int mp_size_t;
typedef unsigned long int mp_bitcnt_t;
typedef long int mp_exp_t;
typedef mp_limb_t *mp_ptr;
typedef const mp_limb_t *mp_srcptr;

#define GMP_LIMB_BITS 64
#define GMP_NAIL_BITS 0
#define GMP_NUMB_BITS (GMP_LIMB_BITS - GMP_NAIL_BITS)
#define GMP_NUMB_MAX (~(mp_limb_t)0)

typedef struct {
    int _mp_alloc;
    int _mp_size;
    mp_limb_t *_mp_d;
} __mpz_struct;
typedef __mpz_struct mpz_t[1];
typedef __mpz_struct *mpz_ptr;
typedef const __mpz_struct *mpz_srcptr;

/* low-level natural-number functions */
#define mpn_add_n __gmpn_add_n
mp_limb_t __gmpn_add_n(mp_ptr rp, mp_srcptr s1p, mp_srcptr s2p, mp_size_t n);
#define mpn_sub_n __gmpn_sub_n
mp_limb_t __gmpn_sub_n(mp_ptr rp, mp_srcptr s1p, mp_srcptr s2p, mp_size_t n);
#define mpn_add_1 __gmpn_add_1
mp_limb_t __gmpn_add_1(mp_ptr rp, mp_srcptr s1p, mp_size_t n, mp_limb_t s2);
#define mpn_sub_1 __gmpn_sub_1
mp_limb_t __gmpn_sub_1(mp_ptr rp, mp_srcptr s1p, mp_size_t n, mp_limb_t s2);
#define mpn_add __gmpn_add
mp_limb_t __gmpn_add(mp_ptr rp, mp_srcptr s1p, mp_size_t s1n, mp_srcptr s2p, mp_size_t s2n);
#define mpn_sub __gmpn_sub
mp_limb_t __gmpn_sub(mp_ptr rp, mp_srcptr s1p, mp_size_t s1n, mp_srcptr s2p, mp_size_t s2n);
#define mpn_mul __gmpn_mul
mp_limb_t __gmpn_mul(mp_ptr rp, mp_srcptr s1p, mp_size_t s1n, mp_srcptr s2p, mp_size_t s2n);
#define mpn_mul_n __gmpn_mul_n
void __gmpn_mul_n(mp_ptr rp, mp_srcptr s1p, mp_srcptr s2p, mp_size_t n);
#define mpn_addmul_1 __gmpn_addmul_1
mp_limb_t __gmpn_addmul_1(mp_ptr rp, mp_srcptr s1p, mp_size_t n, mp_limb_t s2);
#define mpn_cmp __gmpn_cmp
int __gmpn_cmp(mp_srcptr s1p, mp_srcptr s2p, mp_size_t n);
#define mpn_copyi __gmpn_copyi
void __gmpn_copyi(mp_ptr rp, mp_srcptr s1p, mp_size_t n);
#define mpn_zero __gmpn_zero
void __gmpn_zero(mp_ptr rp, mp_size_t n);
#define mpn_rshift __gmpn_rshift
mp_limb_t __gmpn_rshift(mp_ptr rp, mp_srcptr sp, mp_size_t n, unsigned int count);
#define mpn_tdiv_qr __gmpn_tdiv_qr
void __gmpn_tdiv_qr(mp_ptr qp, mp_ptr rp, mp_size_t qxn, mp_srcptr np, mp_size_t nn,
                    mp_srcptr dp, mp_size_t dn);
#define mpn_gcdext __gmpn_gcdext
mp_size_t __gmpn_gcdext(mp_ptr gp, mp_ptr sp, mp_size_t *sn, mp_ptr up, mp_size_t un,
                        mp_ptr vp, mp_size_t vn);
#define mpn_set_str __gmpn_set_str
mp_size_t __gmpn_set_str(mp_ptr rp, const unsigned char *str, size_t strsize, int base);

/* integer functions */
#define mpz_init __gmpz_init
void __gmpz_init(mpz_ptr x);
#define mpz_init_set __gmpz_init_set
void __gmpz_init_set(mpz_ptr rop, mpz_srcptr op);
#define mpz_init_set_str __gmpz_init_set_str
int __gmpz_init_set_str(mpz_ptr rop, const char *str, int base);
#define mpz_clear __gmpz_clear
void __gmpz_clear(mpz_ptr x);
#define mpz_set_ui __gmpz_set_ui
void __gmpz_set_ui(mpz_ptr rop, unsigned long int op);
#define mpz_get_ui __gmpz_get_ui
unsigned long int __gmpz_get_ui(mpz_srcptr op);
#define mpz_add_ui __gmpz_add_ui
void __gmpz_add_ui(mpz_ptr rop, mpz_srcptr op1, unsigned long int op2);
#define mpz_mul_2exp __gmpz_mul_2exp
void __gmpz_mul_2exp(mpz_ptr rop, mpz_srcptr op1, mp_bitcnt_t op2);
#define mpz_fdiv_q_2exp __gmpz_fdiv_q_2exp
void __gmpz_fdiv_q_2exp(mpz_ptr q, mpz_srcptr n, mp_bitcnt_t b);
#define mpz_sizeinbase __gmpz_sizeinbase
size_t __gmpz_sizeinbase(mpz_srcptr op, int base);
#define mpz_export __gmpz_export
void *__gmpz_export(void *rop, size_t *countp, int order, size_t size, int endian,
                    size_t nails, mpz_srcptr op);
#define mpz_import __gmpz_import
void __gmpz_import(mpz_ptr rop, size_t count, int order, size_t size, int endian,
                   size_t nails, const void *op);
/* documented as a macro: sign of the integer */
#define mpz_sgn(z) ((z)->_mp_size < 0 ? -1 : (z)->_mp_size > 0)

#define gmp_printf __gmp_printf
int __gmp_printf(const char *fmt, ...);

#ifdef __cplusplus
}
#endif

#endif /* NKR_ORACLE_GMP_COMPAT_H */
