/*
 * Packed-vector front end to the reference's own CPU mpz_rmatrix_mult_fft
 * (alexp616/rforest src/lib/hwmpz.c:65-130), compiled from the reference
 * sources in place.
 *
 * TEST INFRASTRUCTURE ONLY.  Builds mpz_t matrices from packed limb arrays,
 * calls the unmodified reference function and writes the result back in the
 * same packed form.  The reference API multiplies r x d by d x d; a general
 * m x k by k x n product is zero-padded to d = max(k, n) (extra columns of A
 * and extra rows/columns of B are zero), which leaves the m x n block exact.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include "gmp.h"
#include "hwmpz.h"
#include "mpzfft.h"

static int ref_ready;

void ref_setup(void) {
  if (!ref_ready) {
    hw_mpz_setup();
    ref_ready = 1;
  }
}

static void load(mpz_ptr z, const uint64_t *limbs, int64_t off, int32_t size) {
  mp_size_t n = size < 0 ? -size : size;
  if (n == 0) {
    mpz_set_ui(z, 0);
    return;
  }
  mp_limb_t *d = mpz_limbs_write(z, n);
  memcpy(d, limbs + off, (size_t)n * 8);
  mpz_limbs_finish(z, size);
}

/* Returns 0 on success, -1 if an output capacity is too small. */
int ref_matmul(int m, int k, int n, const uint64_t *a_limbs,
               const int64_t *a_offs, const int32_t *a_sizes,
               const uint64_t *b_limbs, const int64_t *b_offs,
               const int32_t *b_sizes, uint64_t *out_limbs,
               const int64_t *out_offs, const int64_t *out_caps,
               int32_t *out_sizes) {
  ref_setup();
  int d = k > n ? k : n;
  mpz_t *A = malloc(sizeof(mpz_t) * (size_t)m * d);
  mpz_t *B = malloc(sizeof(mpz_t) * (size_t)d * d);
  mpz_t *C = malloc(sizeof(mpz_t) * (size_t)m * d);
  for (int i = 0; i < m * d; i++) { mpz_init(A[i]); mpz_init(C[i]); }
  for (int i = 0; i < d * d; i++) mpz_init(B[i]);
  for (int i = 0; i < m; i++)
    for (int l = 0; l < k; l++)
      load(A[i * d + l], a_limbs, a_offs[i * k + l], a_sizes[i * k + l]);
  for (int l = 0; l < k; l++)
    for (int j = 0; j < n; j++)
      load(B[l * d + j], b_limbs, b_offs[l * n + j], b_sizes[l * n + j]);
  mpz_t w;
  mpz_init(w);
  mpz_rmatrix_mult_fft(C, A, m, B, d, w);
  mpz_clear(w);
  int status = 0;
  for (int i = 0; i < m; i++)
    for (int j = 0; j < n; j++) {
      int e = i * n + j;
      mpz_ptr z = C[i * d + j];
      size_t sz = mpz_size(z);
      if ((int64_t)sz > out_caps[e]) {
        status = -1;
        out_sizes[e] = 0;
        continue;
      }
      if (sz) memcpy(out_limbs + out_offs[e], z->_mp_d, sz * 8);
      out_sizes[e] = z->_mp_size;
    }
  for (int i = 0; i < m * d; i++) { mpz_clear(A[i]); mpz_clear(C[i]); }
  for (int i = 0; i < d * d; i++) mpz_clear(B[i]);
  free(A);
  free(B);
  free(C);
  return status;
}

/* x mod d in [0, d) for `count` packed x through the reference's own
 * mpzfft_mod_init / mpzfft_mod_mod (src/lib/mpzfft.c:59-100; Fermat-transform
 * reciprocal, src/lib/mpnfft_mod.c:283-476) with 4 FFT primes, as hwmpz.c
 * uses for the product.  `bits` bounds |x| (and d's bit length).  Returns 0,
 * or -1 if an output capacity is too small. */
static zz_moduli_t mod_moduli;
static int mod_moduli_ready;

int ref_mod(const uint64_t *d_limbs, int32_t d_size, int64_t bits, int count,
            const uint64_t *x_limbs, const int64_t *x_offs, const int32_t *x_sizes,
            uint64_t *r_limbs, const int64_t *r_offs, const int64_t *r_caps,
            int32_t *r_sizes) {
  if (!mod_moduli_ready) {
    zz_moduli_init(&mod_moduli, 4);
    mod_moduli_ready = 1;
  }
  mpz_t d, x, r;
  mpz_init(d);
  mpz_init(x);
  mpz_init(r);
  load(d, d_limbs, 0, d_size);
  mpzfft_mod_t M;
  mpzfft_mod_init(&M, (size_t)bits, d, 4, &mod_moduli, 1);
  int status = 0;
  for (int i = 0; i < count; i++) {
    load(x, x_limbs, x_offs[i], x_sizes[i]);
    mpzfft_mod_mod(&M, r, x, 1);
    size_t sz = mpz_size(r);
    if ((int64_t)sz > r_caps[i]) {
      status = -1;
      r_sizes[i] = 0;
      continue;
    }
    if (sz) memcpy(r_limbs + r_offs[i], r->_mp_d, sz * 8);
    r_sizes[i] = r->_mp_size;
  }
  mpzfft_mod_clear(&M);
  mpz_clear(d);
  mpz_clear(x);
  mpz_clear(r);
  return status;
}
