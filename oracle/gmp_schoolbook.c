/*
 * GMP schoolbook matrix product: the second oracle.
 *
 * TEST INFRASTRUCTURE ONLY (never linked into the product).  Restates
 * mpz_rmatrix_mult_naive (alexp616/rforest src/include/hwmpz.h:117-124) for a
 * general m x k by k x n shape, using GMP's mpz_mul / mpz_addmul, over the
 * same packed-vector convention as mpzmm_oracle.c.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include "gmp.h"

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
int orc_matmul_naive(int m, int k, int n, const uint64_t *a_limbs,
                     const int64_t *a_offs, const int32_t *a_sizes,
                     const uint64_t *b_limbs, const int64_t *b_offs,
                     const int32_t *b_sizes, uint64_t *out_limbs,
                     const int64_t *out_offs, const int64_t *out_caps,
                     int32_t *out_sizes) {
  int status = 0;
  mpz_t w, x, y;
  mpz_init(w);
  mpz_init(x);
  mpz_init(y);
  for (int i = 0; i < m; i++)
    for (int j = 0; j < n; j++) {
      mpz_set_ui(w, 0);
      for (int l = 0; l < k; l++) {
        load(x, a_limbs, a_offs[i * k + l], a_sizes[i * k + l]);
        load(y, b_limbs, b_offs[l * n + j], b_sizes[l * n + j]);
        mpz_addmul(w, x, y);
      }
      int e = i * n + j;
      size_t sz = mpz_size(w);
      if ((int64_t)sz > out_caps[e]) {
        status = -1;
        out_sizes[e] = 0;
        continue;
      }
      if (sz) memcpy(out_limbs + out_offs[e], w->_mp_d, sz * 8);
      out_sizes[e] = w->_mp_size;
    }
  mpz_clear(w);
  mpz_clear(x);
  mpz_clear(y);
  return status;
}
