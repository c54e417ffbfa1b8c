/*
 * Host-side stand-ins for the reference's GPU hooks, so that its CPU path
 * (src/lib/hwmpz.c, mpnfft.c) links without CUDA or the GPU-NTT library.
 *
 * TEST INFRASTRUCTURE ONLY.  hw_mpz_setup() (src/lib/hwmpz.c:24-40) calls
 * create_cu_zz_moduli_t / cu_zz_moduli_init / cu_crt_constants_create: those
 * become no-ops.  Every other hook belongs to cu_mpz_rmatrix_mult_fft, which
 * the oracle never calls; they abort loudly if reached.
 */
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>

typedef struct cu_zz_moduli_t cu_zz_moduli_t;
typedef struct cu_crt_constants_t cu_crt_constants_t;

cu_zz_moduli_t *cu_zz_moduli = NULL;

cu_zz_moduli_t *create_cu_zz_moduli_t(void) { return NULL; }
void cu_zz_moduli_init(cu_zz_moduli_t *m, int n) { (void)m; (void)n; }
void cu_zz_moduli_clear(cu_zz_moduli_t *m) { (void)m; }
cu_crt_constants_t *cu_crt_constants_create(const void *m, unsigned n) {
  (void)m; (void)n;
  return NULL;
}
void cu_crt_constants_destroy(cu_crt_constants_t *c) { (void)c; }

static void gpu_hook_unavailable(const char *name) {
  fprintf(stderr, "oracle: reference GPU hook %s is not available\n", name);
  abort();
}
#define ABORT_STUB(ret, name, args) \
  ret name args { gpu_hook_unavailable(#name); return (ret)0; }

ABORT_STUB(void *, cu_malloc_pinned, (size_t n))
ABORT_STUB(void *, cu_device_malloc, (size_t n))
ABORT_STUB(uint64_t *, cu_fft62_fft_batch, (uint64_t *d, int np, unsigned lg, cu_zz_moduli_t *m, int sz))
void cu_free_pinned(void *p) { (void)p; gpu_hook_unavailable("cu_free_pinned"); }
void cu_device_free(void *p) { (void)p; gpu_hook_unavailable("cu_device_free"); }
void cu_memcpy_d2h(void *d, const void *s, size_t n) { (void)d; (void)s; (void)n; gpu_hook_unavailable("cu_memcpy_d2h"); }
void cu_fft62_ifft_batch(uint64_t *h, uint64_t *d, int np, unsigned lg, cu_zz_moduli_t *m, int sz) {
  (void)h; (void)d; (void)np; (void)lg; (void)m; (void)sz;
  gpu_hook_unavailable("cu_fft62_ifft_batch");
}
void cu_intt_batch_only(uint64_t *d, int np, unsigned lg, int sz) {
  (void)d; (void)np; (void)lg; (void)sz;
  gpu_hook_unavailable("cu_intt_batch_only");
}
void cu_mpzfft_matrix_mul(uint64_t *C, uint64_t *A, uint64_t *B, int d1, int d2, int d3, int np, int n, cu_zz_moduli_t *m) {
  (void)C; (void)A; (void)B; (void)d1; (void)d2; (void)d3; (void)np; (void)n; (void)m;
  gpu_hook_unavailable("cu_mpzfft_matrix_mul");
}
void cu_zz_crt_batch(uint64_t *o, const uint64_t *d, size_t sz, const cu_crt_constants_t *c) {
  (void)o; (void)d; (void)sz; (void)c;
  gpu_hook_unavailable("cu_zz_crt_batch");
}
