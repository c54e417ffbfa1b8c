/*
 * Minimal GMP public-API header for building the CPU oracle.
 *
 * TEST INFRASTRUCTURE ONLY.  This container ships the GMP 6.3 runtime
 * (libgmp.so.10) but not its development header, so this file declares the
 * small part of GMP's documented public interface that the reference's CPU
 * sources (src/lib/*.c, src/include/*.h of alexp616/rforest) and the oracle
 * harness use: the mpz struct layout, limb types, and the exported
 * __gmpz_* / __gmpn_* entry points under their documented mpz_* / mpn_*
 * names.  Nothing here is product code.
 */
#ifndef MPZMM_ORACLE_GMP_SHIM_H
#define MPZMM_ORACLE_GMP_SHIM_H

#include <stddef.h>
#include <stdio.h>

#ifdef __cplusplus
extern "C" {
#endif

#define GMP_LIMB_BITS 64
#define GMP_NAIL_BITS 0
#define GMP_NUMB_BITS 64
#define __GNU_MP_VERSION 6

typedef unsigned long int mp_limb_t;
typedef long int mp_limb_signed_t;
typedef long int mp_size_t;
typedef unsigned long int mp_bitcnt_t;
typedef long int mp_exp_t;
typedef mp_limb_t *mp_ptr;
typedef const mp_limb_t *mp_srcptr;

/* Documented mpz layout (GMP manual, "Integer Internals"). */
typedef struct {
  int _mp_alloc;
  int _mp_size;
  mp_limb_t *_mp_d;
} __mpz_struct;

typedef __mpz_struct mpz_t[1];
typedef __mpz_struct *mpz_ptr;
typedef const __mpz_struct *mpz_srcptr;

/* Random state: only its size matters to callers that declare one. */
typedef struct {
  __mpz_struct _mp_seed;
  int _mp_alg;
  void *_mp_algdata;
} __gmp_randstate_struct;
typedef __gmp_randstate_struct gmp_randstate_t[1];

#define mpz_sgn(Z) ((Z)->_mp_size < 0 ? -1 : (Z)->_mp_size > 0)
#define mpz_size(Z) ((size_t)((Z)->_mp_size < 0 ? -(Z)->_mp_size : (Z)->_mp_size))

/* ---- mpz ---- */
void __gmpz_init(mpz_ptr);
void __gmpz_clear(mpz_ptr);
void *__gmpz_realloc(mpz_ptr, mp_size_t);
void __gmpz_realloc2(mpz_ptr, mp_bitcnt_t);
void __gmpz_set(mpz_ptr, mpz_srcptr);
void __gmpz_set_ui(mpz_ptr, unsigned long);
void __gmpz_mul(mpz_ptr, mpz_srcptr, mpz_srcptr);
void __gmpz_addmul(mpz_ptr, mpz_srcptr, mpz_srcptr);
void __gmpz_add(mpz_ptr, mpz_srcptr, mpz_srcptr);
void __gmpz_sub(mpz_ptr, mpz_srcptr, mpz_srcptr);
void __gmpz_neg(mpz_ptr, mpz_srcptr);
int __gmpz_cmp(mpz_srcptr, mpz_srcptr);
int __gmpz_cmp_ui(mpz_srcptr, unsigned long);
size_t __gmpz_sizeinbase(mpz_srcptr, int);
void __gmpz_fdiv_r(mpz_ptr, mpz_srcptr, mpz_srcptr);
void __gmpz_urandomb(mpz_ptr, gmp_randstate_t, mp_bitcnt_t);
mp_limb_t *__gmpz_limbs_write(mpz_ptr, mp_size_t);
void __gmpz_limbs_finish(mpz_ptr, mp_size_t);
const mp_limb_t *__gmpz_limbs_read(mpz_srcptr);

#define mpz_init __gmpz_init
#define mpz_clear __gmpz_clear
#define mpz_realloc __gmpz_realloc
#define _mpz_realloc __gmpz_realloc
#define mpz_realloc2 __gmpz_realloc2
#define mpz_set __gmpz_set
#define mpz_set_ui __gmpz_set_ui
#define mpz_mul __gmpz_mul
#define mpz_addmul __gmpz_addmul
#define mpz_add __gmpz_add
#define mpz_sub __gmpz_sub
#define mpz_neg __gmpz_neg
#define mpz_cmp __gmpz_cmp
#define mpz_cmp_ui __gmpz_cmp_ui
#define mpz_sizeinbase __gmpz_sizeinbase
#define mpz_fdiv_r __gmpz_fdiv_r
#define mpz_urandomb __gmpz_urandomb
#define mpz_limbs_write __gmpz_limbs_write
#define mpz_limbs_finish __gmpz_limbs_finish
#define mpz_limbs_read __gmpz_limbs_read

/* ---- mpn ---- */
mp_limb_t __gmpn_add_n(mp_ptr, mp_srcptr, mp_srcptr, mp_size_t);
mp_limb_t __gmpn_sub_n(mp_ptr, mp_srcptr, mp_srcptr, mp_size_t);
mp_limb_t __gmpn_add_1(mp_ptr, mp_srcptr, mp_size_t, mp_limb_t);
mp_limb_t __gmpn_sub_1(mp_ptr, mp_srcptr, mp_size_t, mp_limb_t);
mp_limb_t __gmpn_lshift(mp_ptr, mp_srcptr, mp_size_t, unsigned int);
mp_limb_t __gmpn_rshift(mp_ptr, mp_srcptr, mp_size_t, unsigned int);
mp_limb_t __gmpn_mul_1(mp_ptr, mp_srcptr, mp_size_t, mp_limb_t);
mp_limb_t __gmpn_addmul_1(mp_ptr, mp_srcptr, mp_size_t, mp_limb_t);
mp_limb_t __gmpn_mod_1(mp_srcptr, mp_size_t, mp_limb_t);
mp_limb_t __gmpn_neg(mp_ptr, mp_srcptr, mp_size_t);
int __gmpn_cmp(mp_srcptr, mp_srcptr, mp_size_t);
void __gmpn_zero(mp_ptr, mp_size_t);
void __gmpn_copyi(mp_ptr, mp_srcptr, mp_size_t);
mp_limb_t __gmpn_add(mp_ptr, mp_srcptr, mp_size_t, mp_srcptr, mp_size_t);
mp_limb_t __gmpn_sub(mp_ptr, mp_srcptr, mp_size_t, mp_srcptr, mp_size_t);
void __gmpn_tdiv_qr(mp_ptr, mp_ptr, mp_size_t, mp_srcptr, mp_size_t, mp_srcptr, mp_size_t);

#define mpn_add_n __gmpn_add_n
#define mpn_sub_n __gmpn_sub_n
#define mpn_add_1 __gmpn_add_1
#define mpn_sub_1 __gmpn_sub_1
#define mpn_lshift __gmpn_lshift
#define mpn_rshift __gmpn_rshift
#define mpn_mul_1 __gmpn_mul_1
#define mpn_addmul_1 __gmpn_addmul_1
#define mpn_mod_1 __gmpn_mod_1
#define mpn_neg __gmpn_neg
#define mpn_cmp __gmpn_cmp
#define mpn_zero __gmpn_zero
#define mpn_copyi __gmpn_copyi
#define mpn_add __gmpn_add
#define mpn_sub __gmpn_sub
#define mpn_tdiv_qr __gmpn_tdiv_qr

/* ---- misc ---- */
void __gmp_set_memory_functions(void *(*)(size_t),
                                void *(*)(void *, size_t, size_t),
                                void (*)(void *, size_t));
void __gmp_get_memory_functions(void *(**)(size_t),
                                void *(**)(void *, size_t, size_t),
                                void (**)(void *, size_t));
void __gmp_randinit_default(gmp_randstate_t);
void __gmp_randseed_ui(gmp_randstate_t, unsigned long);
void __gmp_randclear(gmp_randstate_t);

#define mp_set_memory_functions __gmp_set_memory_functions
#define mp_get_memory_functions __gmp_get_memory_functions
#define gmp_randinit_default __gmp_randinit_default
#define gmp_randseed_ui __gmp_randseed_ui
#define gmp_randclear __gmp_randclear

#ifdef __cplusplus
}
#endif

#endif
