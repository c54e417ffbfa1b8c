/*
 * CPU restatement of the reference exact big-integer matrix product
 * mpz_rmatrix_mult_fft() (alexp616/rforest, src/lib/hwmpz.c:65-130).
 *
 * TEST INFRASTRUCTURE ONLY.  This is the oracle: tests, the smoke check and
 * the benchmark's CPU-baseline leg call it to check or time the product path;
 * the product library never links, loads or calls it.
 *
 * It follows the reference pipeline stage by stage, with the reference's own
 * parameters (the eight 62-bit primes of src/include/fft62.h:24-31, four of
 * them used as in src/lib/hwmpz.c:13, r / lgN / points from
 * src/lib/mpnfft.c:18-78), written plainly with unsigned __int128 arithmetic:
 *
 *   split + reduce   src/lib/split.c:10-81, src/lib/reduce.c:10-28,
 *                    src/lib/split_reduce.c:15-66  (sign folded into residues)
 *   forward NTT      src/lib/mpnfft.c:354-383 (any correct cyclic NTT of
 *                    length N evaluates the same polynomial product; the
 *                    reference's truncated bit-reversed fft62 layout is an
 *                    implementation detail that does not reach the output)
 *   contraction      src/lib/mpnfft.c:559-651
 *   inverse NTT      src/lib/mpnfft.c:386-432 with scale = 1 (times 1/N)
 *   Garner CRT       src/lib/crt.c:11-94 (symmetric residue, 2's complement)
 *   recompose        src/lib/recompose.c:11-107, src/lib/crt_recompose.c
 *   sign/normalise   src/lib/hwmpz.c:108-126
 *
 * Integers are passed as "packed vectors": entry e has |sizes[e]| 64-bit limbs
 * starting at limbs[offs[e]] (least significant first) and the sign of
 * sizes[e], i.e. GMP's own (_mp_size, _mp_d) convention.
 */
#include <assert.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef unsigned __int128 u128;

#define ORC_MAX_PRIMES 8
#define ORC_NUM_PRIMES 4 /* HW_ZZ_PRIMES, src/lib/hwmpz.c:13 */

/* src/include/fft62.h:24-31: primes p = 1 mod 2^44, 2^61 < p < 2^62. */
static const uint64_t orc_primes[ORC_MAX_PRIMES] = {
    0x3fffc00000000001ULL, 0x3ffdf00000000001ULL, 0x3ffd900000000001ULL,
    0x3ffd500000000001ULL, 0x3ffc100000000001ULL, 0x3ffbb00000000001ULL,
    0x3ffaf00000000001ULL, 0x3ffac00000000001ULL};

static uint64_t mulmod(uint64_t a, uint64_t b, uint64_t p) {
  return (uint64_t)(((u128)a * b) % p);
}
static uint64_t addmod(uint64_t a, uint64_t b, uint64_t p) {
  uint64_t s = a + b; /* p < 2^62, no overflow */
  return s >= p ? s - p : s;
}
static uint64_t submod(uint64_t a, uint64_t b, uint64_t p) {
  return a >= b ? a - b : a + p - b;
}
static uint64_t powmod(uint64_t a, uint64_t e, uint64_t p) {
  uint64_t r = 1 % p;
  a %= p;
  while (e) {
    if (e & 1) r = mulmod(r, a, p);
    a = mulmod(a, a, p);
    e >>= 1;
  }
  return r;
}
static uint64_t invmod(uint64_t a, uint64_t p) { return powmod(a, p - 2, p); }

/* src/lib/fft62.c:40-50: smallest u >= 2 whose power u^((p-1)/2^44) has
   order exactly 2^44. */
static uint64_t primitive_root_2_44(uint64_t p) {
  const uint64_t N = (uint64_t)1 << 44;
  for (uint64_t u = 2;; u++) {
    uint64_t w = powmod(u, (p - 1) / N, p);
    if (powmod(w, N / 2, p) != 1) return w;
  }
}

/* src/lib/fft62.c:26-35 */
unsigned orc_log2(size_t n) {
  if (n == 0) return 0;
  unsigned b = 0;
  n--;
  while (n) {
    b++;
    n >>= 1;
  }
  return b;
}

/* src/lib/fft62.c:156-168 with fft62_fft_array_params (fft62.c:146-150):
   admissible sizes are arbitrary up to 2^16, then rounded to multiples of
   2^lgM where lgM = lgN - lgN/2, recursively. */
static size_t orc_next_size(size_t n, unsigned lgN) {
  if (n == 0) n = 1;
  if (lgN <= 16) return n;
  unsigned lgK = lgN / 2, lgM = lgN - lgK;
  size_t k = ((n - 1) >> lgM) + 1;
  return orc_next_size(k, lgK) << lgM;
}

/* src/lib/mpnfft.c:18-78 (CPU parameter choice; double/frexp as in the
   reference, so the oracle picks the identical r, lgN, points). */
void orc_params(size_t bits, size_t terms, unsigned num_primes, unsigned *r_out,
                unsigned *lgN_out, size_t *points_out) {
  double bound = 0.4999;
  for (unsigned i = 0; i < num_primes; i++) bound *= (double)orc_primes[i];
  double bound2 = bound / (double)terms;
  unsigned r = 62 * num_primes / 2;
  for (;;) {
    size_t points = (bits - 1) / r + 2;
    double thing = bound2 / (double)((points + 1) / 2);
    int e;
    frexp(thing, &e);
    unsigned rr = ((unsigned)e - 1) / 2;
    if (rr == r) {
      unsigned lgN = orc_log2(points);
      *r_out = r;
      *lgN_out = lgN;
      *points_out = orc_next_size(points, lgN);
      return;
    }
    r = rr;
  }
}

/* Bits [i*r, (i+1)*r) of the magnitude {up,un}: coefficient i of the split
   (src/lib/split.c:10-81), returned as up to 4 limbs (r <= 124 here). */
static void split_coeff(uint64_t *out, unsigned t, const uint64_t *up,
                        size_t un, size_t i, unsigned r) {
  size_t bit = (size_t)i * r;
  for (unsigned w = 0; w < t; w++) {
    size_t b = bit + 64 * (size_t)w;
    size_t li = b / 64;
    unsigned sh = b % 64;
    uint64_t lo = li < un ? up[li] : 0;
    uint64_t hi = (li + 1) < un ? up[li + 1] : 0;
    out[w] = sh ? (lo >> sh) | (hi << (64 - sh)) : lo;
  }
  unsigned top = r - 64 * (t - 1); /* bits kept in the last word */
  if (top < 64) out[t - 1] &= ((uint64_t)1 << top) - 1;
}

/* Cyclic NTT of length N = 2^lgN in natural order (radix-2 DIT with an
   explicit bit-reversal), w a primitive N-th root of unity mod p. */
static void ntt(uint64_t *a, unsigned lgN, uint64_t w, uint64_t p) {
  size_t N = (size_t)1 << lgN;
  for (size_t i = 1, j = 0; i < N; i++) {
    size_t bit = N >> 1;
    for (; j & bit; bit >>= 1) j ^= bit;
    j ^= bit;
    if (i < j) {
      uint64_t t = a[i];
      a[i] = a[j];
      a[j] = t;
    }
  }
  for (size_t len = 2; len <= N; len <<= 1) {
    uint64_t wl = powmod(w, N / len, p);
    for (size_t s = 0; s < N; s += len) {
      uint64_t x = 1;
      for (size_t j = 0; j < len / 2; j++) {
        uint64_t u = a[s + j], v = mulmod(a[s + j + len / 2], x, p);
        a[s + j] = addmod(u, v, p);
        a[s + j + len / 2] = submod(u, v, p);
        x = mulmod(x, wl, p);
      }
    }
  }
}

/* ---- small fixed-width multi-limb helpers for the CRT ---- */
#define ML 9
typedef struct {
  uint64_t d[ML];
} mlimb;

static void ml_addmul1(mlimb *x, const mlimb *u, unsigned n, uint64_t v) {
  u128 cy = 0;
  for (unsigned i = 0; i < n + 1 && i < ML; i++) {
    u128 t = (u128)x->d[i] + (i < n ? (u128)u->d[i] * v : 0) + cy;
    x->d[i] = (uint64_t)t;
    cy = t >> 64;
  }
}
static int ml_cmp(const mlimb *a, const mlimb *b, unsigned n) {
  for (int i = (int)n - 1; i >= 0; i--) {
    if (a->d[i] != b->d[i]) return a->d[i] > b->d[i] ? 1 : -1;
  }
  return 0;
}
static void ml_sub(mlimb *a, const mlimb *b, unsigned n) {
  uint64_t br = 0;
  for (unsigned i = 0; i < n; i++) {
    u128 t = (u128)a->d[i] - b->d[i] - br;
    a->d[i] = (uint64_t)t;
    br = (uint64_t)(t >> 64) & 1;
  }
}
static uint64_t ml_mod1(const mlimb *a, unsigned n, uint64_t p) {
  u128 r = 0;
  for (int i = (int)n - 1; i >= 0; i--) r = ((r << 64) | a->d[i]) % p;
  return (uint64_t)r;
}

/* Adds the signed P-limb two's complement value c, shifted left by `shift`
   bits, into the 2's complement accumulator {acc, rn} modulo B^rn. */
static void add_shifted_signed(uint64_t *acc, size_t rn, const uint64_t *c,
                               unsigned P, size_t shift) {
  size_t l0 = shift / 64;
  unsigned sh = shift % 64;
  if (l0 >= rn) return;
  uint64_t ext = (c[P - 1] >> 63) ? ~(uint64_t)0 : 0;
  /* shifted value occupies limbs l0 .. l0+P, then sign extension */
  uint64_t carry = 0;
  size_t i;
  for (i = 0; l0 + i < rn; i++) {
    uint64_t lo = i < P ? c[i] : ext;
    uint64_t prev = (i == 0) ? 0 : ((i - 1) < P ? c[i - 1] : ext);
    uint64_t w = sh ? (lo << sh) | (prev >> (64 - sh)) : lo;
    if (i > P + 1) {
      /* beyond the value only sign-extension limbs remain: add ext + carry */
      if (ext == 0 && carry == 0) break;
    }
    u128 t = (u128)acc[l0 + i] + w + carry;
    acc[l0 + i] = (uint64_t)t;
    carry = (uint64_t)(t >> 64);
    if (i > P + 1 && ext == ~(uint64_t)0 && carry == 1) {
      /* adding all-ones with carry-in 1 leaves the limb unchanged and carries
         on: the rest of the sign extension is a no-op. */
      break;
    }
  }
}

/*
 * Exact product C = A*B for A of m x k and B of k x n (row-major packed
 * vectors).  The reference API is A: r x d, B: d x d; it is the special case
 * k == n.  The general shape runs the same pipeline with terms = k.
 *
 * Output entry e is written at out_limbs[out_offs[e]], with capacity
 * out_caps[e] limbs; out_sizes[e] receives the signed GMP-style size.
 * Returns 0 on success, -1 if some output capacity is too small.
 */
int orc_matmul(int m, int k, int n, const uint64_t *a_limbs,
               const int64_t *a_offs, const int32_t *a_sizes,
               const uint64_t *b_limbs, const int64_t *b_offs,
               const int32_t *b_sizes, uint64_t *out_limbs,
               const int64_t *out_offs, const int64_t *out_caps,
               int32_t *out_sizes) {
  const unsigned P = ORC_NUM_PRIMES;
  if (m <= 0 || n <= 0) return 0;
  if (k <= 0) {
    for (int e = 0; e < m * n; e++) out_sizes[e] = 0;
    return 0;
  }
  /* src/lib/hwmpz.c:54-63 */
  size_t maxl = 0;
  for (int e = 0; e < m * k; e++) {
    size_t s = (size_t)llabs(a_sizes[e]);
    if (s > maxl) maxl = s;
  }
  for (int e = 0; e < k * n; e++) {
    size_t s = (size_t)llabs(b_sizes[e]);
    if (s > maxl) maxl = s;
  }
  size_t bits = 64 * (2 * maxl + 1);
  unsigned r, lgN;
  size_t points;
  orc_params(bits, (size_t)k, P, &r, &lgN, &points);
  size_t N = (size_t)1 << lgN;
  unsigned t = (r + 63) / 64;

  uint64_t *resA = calloc((size_t)m * k * P * N, 8);
  uint64_t *resB = calloc((size_t)k * n * P * N, 8);
  uint64_t *resC = calloc((size_t)m * n * P * N, 8);
  if (!resA || !resB || !resC) abort();

  uint64_t w[ORC_MAX_PRIMES], winv[ORC_MAX_PRIMES];
  for (unsigned j = 0; j < P; j++) {
    uint64_t p = orc_primes[j];
    uint64_t g = primitive_root_2_44(p);
    w[j] = powmod(g, ((uint64_t)1 << 44) >> lgN, p);
    winv[j] = invmod(w[j], p);
  }

  /* split + reduce + forward NTT (src/lib/mpnfft.c:119-145, 354-383) */
  for (int side = 0; side < 2; side++) {
    int cnt = side ? k * n : m * k;
    const uint64_t *lim = side ? b_limbs : a_limbs;
    const int64_t *offs = side ? b_offs : a_offs;
    const int32_t *sz = side ? b_sizes : a_sizes;
    uint64_t *res = side ? resB : resA;
    for (int e = 0; e < cnt; e++) {
      int s = sz[e];
      size_t un = (size_t)llabs(s);
      if (s == 0) continue; /* zero polynomial (mpnfft.c:122-126) */
      const uint64_t *up = lim + offs[e];
      size_t size = (64 * un + r - 1) / r;
      if (size > points) size = points;
      for (unsigned j = 0; j < P; j++) {
        uint64_t p = orc_primes[j];
        uint64_t *dst = res + ((size_t)e * P + j) * N;
        uint64_t B = (uint64_t)(((u128)1 << 64) % p);
        for (size_t i = 0; i < size; i++) {
          uint64_t c[4];
          split_coeff(c, t, up, un, i, r);
          uint64_t v = 0; /* Horner, most significant limb first */
          for (int q = (int)t - 1; q >= 0; q--)
            v = addmod(mulmod(v, B, p), c[q] % p, p);
          dst[i] = s < 0 ? submod(0, v, p) : v; /* split_reduce.c:27-38 */
        }
        ntt(dst, lgN, w[j], p);
      }
    }
  }

  /* contraction per frequency (src/lib/mpnfft.c:559-651) */
  for (unsigned j = 0; j < P; j++) {
    uint64_t p = orc_primes[j];
    for (int i = 0; i < m; i++)
      for (int q = 0; q < n; q++) {
        uint64_t *dst = resC + ((size_t)(i * n + q) * P + j) * N;
        for (size_t h = 0; h < N; h++) {
          uint64_t acc = 0;
          for (int l = 0; l < k; l++) {
            uint64_t x = resA[((size_t)(i * k + l) * P + j) * N + h];
            uint64_t y = resB[((size_t)(l * n + q) * P + j) * N + h];
            acc = addmod(acc, mulmod(x, y, p), p);
          }
          dst[h] = acc;
        }
      }
  }

  /* CRT moduli (src/lib/moduli.c:42-58): u[i] = p0...p(i-1) */
  mlimb u[ORC_MAX_PRIMES + 1];
  memset(u, 0, sizeof(u));
  u[0].d[0] = 1;
  for (unsigned i = 1; i <= P; i++) {
    memset(&u[i], 0, sizeof(mlimb));
    ml_addmul1(&u[i], &u[i - 1], i - 1 + 1, orc_primes[i - 1]);
  }
  mlimb uhalf = u[P]; /* floor(M/2) */
  for (unsigned i = 0; i < P; i++)
    uhalf.d[i] = (uhalf.d[i] >> 1) | (i + 1 < P ? uhalf.d[i + 1] << 63 : 0);

  int status = 0;
  uint64_t *coef = malloc(points * P * 8);
  for (int e = 0; e < m * n; e++) {
    uint64_t *res = resC + (size_t)e * P * N;
    /* inverse NTT, times 1/N (src/lib/mpnfft.c:386-432, scale = 1) */
    for (unsigned j = 0; j < P; j++) {
      uint64_t p = orc_primes[j];
      uint64_t *x = res + (size_t)j * N;
      ntt(x, lgN, winv[j], p);
      uint64_t ninv = invmod(N % p, p);
      for (size_t h = 0; h < N; h++) x[h] = mulmod(x[h], ninv, p);
    }
    /* Garner CRT to a symmetric residue (src/lib/crt.c:11-94) */
    for (size_t h = 0; h < points; h++) {
      mlimb X;
      memset(&X, 0, sizeof(X));
      X.d[0] = res[h];
      for (unsigned i = 1; i < P; i++) {
        uint64_t p = orc_primes[i];
        uint64_t xm = ml_mod1(&X, i, p);
        uint64_t um = ml_mod1(&u[i], i, p);
        uint64_t v = mulmod(submod(res[(size_t)i * N + h], xm, p),
                            invmod(um, p), p);
        ml_addmul1(&X, &u[i], i, v);
      }
      if (ml_cmp(&X, &uhalf, P) > 0) ml_sub(&X, &u[P], P);
      memcpy(coef + h * P, X.d, P * 8);
    }
    /* recompose: sum c_h 2^(h r) mod B^rn (src/lib/recompose.c:11-107) with
       rn from src/lib/hwmpz.c:112 */
    size_t rn = ((points - 1) * r + 62 * P + 2) / 64 + 1;
    uint64_t *acc = calloc(rn + 1, 8);
    for (size_t h = 0; h < points; h++)
      add_shifted_signed(acc, rn, coef + h * P, P, (size_t)h * r);
    /* sign and normalise (src/lib/hwmpz.c:116-122) */
    int neg = 0;
    if (acc[rn - 1] >> 63) {
      uint64_t cy = 1;
      for (size_t i = 0; i < rn; i++) {
        u128 tt = (u128)(~acc[i]) + cy;
        acc[i] = (uint64_t)tt;
        cy = (uint64_t)(tt >> 64);
      }
      neg = 1;
    }
    size_t nn = rn;
    while (nn > 0 && acc[nn - 1] == 0) nn--;
    if ((int64_t)nn > out_caps[e]) {
      status = -1;
      out_sizes[e] = 0;
    } else {
      memcpy(out_limbs + out_offs[e], acc, nn * 8);
      out_sizes[e] = neg ? -(int32_t)nn : (int32_t)nn;
    }
    free(acc);
  }
  free(coef);
  free(resA);
  free(resB);
  free(resC);
  return status;
}

/* Parameters the reference would pick for this call (for tests/reporting). */
void orc_query_params(size_t maxlimbs, size_t terms, unsigned *r,
                      unsigned *lgN, size_t *points) {
  orc_params(64 * (2 * maxlimbs + 1), terms, ORC_NUM_PRIMES, r, lgN, points);
}
