/*
 * The part of GMP's ABI that libmpzmm_b200 relies on.
 *
 * With <gmp.h> on the include path (an rforest build) this just includes it.
 * Without it (this library's own build: only the GMP 6 runtime,
 * libgmp.so.10, is installed) it declares the documented mpz layout and the
 * GMP routines the library calls, under GMP's exported names:
 * __gmpz_realloc (mpz_realloc), so mpz_t arguments and the caller's GMP
 * allocator are handled exactly as GMP itself would, and the few used once
 * to set up a modular reduction's reciprocal.
 */
#ifndef MPZMM_GMP_ABI_H
#define MPZMM_GMP_ABI_H

#if defined(__has_include)
#if __has_include(<gmp.h>) && !defined(MPZMM_NO_SYSTEM_GMP_H)
#include <gmp.h>
#define MPZMM_HAVE_GMP_H 1
#endif
#endif

#ifndef MPZMM_HAVE_GMP_H
#ifdef __cplusplus
extern "C" {
#endif
typedef unsigned long int mp_limb_t;
typedef long int mp_size_t;
/* GMP manual, "Integer Internals": the mpz_t layout. */
typedef struct {
  int _mp_alloc;
  int _mp_size;
  mp_limb_t *_mp_d;
} __mpz_struct;
typedef __mpz_struct mpz_t[1];
typedef __mpz_struct *mpz_ptr;
void *__gmpz_realloc(mpz_ptr, mp_size_t);
/* set-up of a modular reduction (mpzmm_mod_create): floor(B^L / d) */
void __gmpz_init(mpz_ptr);
void __gmpz_clear(mpz_ptr);
void __gmpz_setbit(mpz_ptr, unsigned long int);
void __gmpz_tdiv_q(mpz_ptr, const __mpz_struct *, const __mpz_struct *);
const __mpz_struct *__gmpz_roinit_n(mpz_ptr, const mp_limb_t *, mp_size_t);
#ifdef __cplusplus
}
#endif
#endif

#endif /* MPZMM_GMP_ABI_H */
