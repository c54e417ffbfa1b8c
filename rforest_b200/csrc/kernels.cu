// sm_100a kernels of the exact matrix-product pipeline.
//
//   k_fwd2           limbs -> r-bit coefficients -> 30-bit digits ->
//                    residues mod p -> forward NTT, register-blocked passes
//                    (several small transforms or one large one per CTA)
//   k_split_fwd      the same, radix 2, one CTA per (entry, prime): tiny
//                    transforms and digit counts above 7
//   k_contract       per frequency h and prime: C[h] = A[h] B[h] mod p on
//                    CUDA cores (64-bit lazy accumulation, Montgomery fold)
//   k_contract_tc    the same on tensor cores (tcgen05 kind::i8, exact
//                    byte split; contract_tc.cuh)
//   k_inv2           inverse NTT, register-blocked; k_inv_ntt radix 2
//   k_crt_mixed      explicit CRT to signed multi-word coefficients, then
//                    sum_i c_i 2^(i r) with carries resolved by a
//                    carry-lookahead prefix scan over 32-bit output words,
//                    sign + negation + normalisation (one warp per entry,
//                    every prime count of a range in one launch);
//                    k_crt_warp the same for one prime count
//
// Reference counterparts: split/reduce src/lib/split_reduce.c:15-66,
// NTTs src/lib/mpnfft.c:354-432, contraction src/lib/mpnfft.c:559-651,
// CRT src/lib/crt.c:11-94, recompose src/lib/recompose.c:11-107 and
// src/lib/crt_recompose.c:15-156, sign/normalise src/lib/hwmpz.c:116-122.

#include <cuda_runtime.h>

#include <cstdint>

#include "kernels.h"
#include "modarith.cuh"
#include "mpzmm_internal.h"
#include "ntt_fast.cuh"
#include "contract_tc.cuh"

namespace mpzmm {

__constant__ PrimeConst c_primes[kMaxPrimes];
__constant__ CrtConst c_crt;

constexpr int kTwStride = 1 << kTwiddleLg;  // twiddle entries per prime

// ---------------------------------------------------------------------------
// NTT building blocks (shared memory, radix-2)
//
// Forward (Cooley-Tukey, natural order in, bit-reversed order out): for
// m = 1, 2, ..., N/2 and t = N/(2m), block i of 2t values is split with the
// twiddle T[m + i] = w_{2m}^{brev(i)}, a primitive-root power that does not
// depend on N, so one table of 2^kTwiddleLg entries per prime serves every N.
// Inverse (Gentleman-Sande) runs the same (m, i) pairs in reverse order with
// T^{-1}; it returns N times the input, the factor is removed before CRT.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void ntt_fwd_smem(uint32_t* a, int lgN, const uint2* tw,
                                             uint32_t p) {
  const int half = 1 << (lgN - 1);
  for (int lgm = 0; lgm < lgN; ++lgm) {
    const int lgt = lgN - 1 - lgm;
    const int t = 1 << lgt;
    const int m = 1 << lgm;
    for (int b = threadIdx.x; b < half; b += blockDim.x) {
      const int i = b >> lgt;
      const int j = (i << (lgt + 1)) + (b & (t - 1));
      const uint2 S = tw[m + i];
      const uint32_t U = a[j];
      const uint32_t V = mul_shoup(a[j + t], S.x, S.y, p);
      a[j] = add_mod(U, V, p);
      a[j + t] = sub_mod(U, V, p);
    }
    __syncthreads();
  }
}

__device__ __forceinline__ void ntt_inv_smem(uint32_t* a, int lgN, const uint2* tw,
                                             uint32_t p) {
  const int half = 1 << (lgN - 1);
  for (int lgm = lgN - 1; lgm >= 0; --lgm) {
    const int lgt = lgN - 1 - lgm;
    const int t = 1 << lgt;
    const int m = 1 << lgm;
    for (int b = threadIdx.x; b < half; b += blockDim.x) {
      const int i = b >> lgt;
      const int j = (i << (lgt + 1)) + (b & (t - 1));
      const uint2 S = tw[m + i];
      const uint32_t X = a[j];
      const uint32_t Y = a[j + t];
      a[j] = add_mod(X, Y, p);
      a[j + t] = mul_shoup(sub_mod(X, Y, p), S.x, S.y, p);
    }
    __syncthreads();
  }
}

// ---------------------------------------------------------------------------
// Split + reduce + forward NTT.  grid = (entries of this class, P).
// Coefficient i of an entry is bits [i r, (i+1) r) of its magnitude; its
// residue is taken by Horner over 32-bit words (Shoup multiply by 2^32 mod p)
// and negated for a negative entry, which is how the reference folds the
// sign into the split (src/lib/split_reduce.c:27-38).
// ---------------------------------------------------------------------------
__global__ void k_split_fwd(const FwdDesc* __restrict__ descs,
                            const uint32_t* __restrict__ idx,
                            const uint64_t* __restrict__ limbs,
                            uint32_t* __restrict__ res,
                            const uint2* __restrict__ twf) {
  extern __shared__ uint32_t sm[];
  const FwdDesc d = descs[idx[blockIdx.x]];
  const int j = blockIdx.y;
  const uint32_t p = c_primes[j].p;
  const uint32_t mu = c_primes[j].mu;
  const uint32_t b32 = c_primes[j].b32;
  const uint32_t b32q = c_primes[j].b32q;
  const int N = 1 << d.lgN;
  const uint32_t nl = (uint32_t)(d.size < 0 ? -d.size : d.size);
  const uint32_t nw = 2 * nl;
  const uint32_t* __restrict__ w32 = reinterpret_cast<const uint32_t*>(limbs + d.limb_off);
  const uint32_t r = d.r;
  const int ncw = (int)((r + 31) >> 5);
  const uint32_t topbits = r - 32u * (uint32_t)(ncw - 1);
  const uint32_t topmask = topbits >= 32 ? 0xffffffffu : ((1u << topbits) - 1u);
  const bool neg = d.size < 0;

  for (int i = threadIdx.x; i < N; i += blockDim.x) {
    uint32_t v = 0;
    if ((uint32_t)i < d.ncoef) {
      const uint64_t bit = (uint64_t)i * r;
      const uint64_t wi = bit >> 5;
      const uint32_t sh = (uint32_t)(bit & 31);
      uint32_t acc = 0;
      for (int q = ncw - 1; q >= 0; --q) {
        const uint64_t a0 = wi + (uint64_t)q;
        const uint32_t lo = a0 < nw ? w32[a0] : 0u;
        const uint32_t hi = a0 + 1 < nw ? w32[a0 + 1] : 0u;
        uint32_t c = __funnelshift_r(lo, hi, sh);
        if (q == ncw - 1) c &= topmask;
        acc = add_mod(mul_shoup(acc, b32, b32q, p), mod32(c, p, mu), p);
      }
      v = (neg && acc) ? p - acc : acc;
    }
    sm[i] = v;
  }
  __syncthreads();
  ntt_fwd_smem(sm, d.lgN, twf + (size_t)j * kTwStride, p);
  uint32_t* out = res + d.res_off + (uint64_t)j * (uint64_t)N;
  for (int i = threadIdx.x; i < N; i += blockDim.x) out[i] = sm[i];
}

// ---------------------------------------------------------------------------
// Inverse NTT.  grid = (entries of this class, P).
// ---------------------------------------------------------------------------
__global__ void k_inv_ntt(const InvDesc* __restrict__ descs,
                          const uint32_t* __restrict__ idx, uint32_t* __restrict__ res,
                          const uint2* __restrict__ twi) {
  extern __shared__ uint32_t sm[];
  const InvDesc d = descs[idx[blockIdx.x]];
  const int j = blockIdx.y;
  const uint32_t p = c_primes[j].p;
  const int N = 1 << d.lgN;
  uint32_t* io = res + d.res_off + (uint64_t)j * (uint64_t)N;
  for (int i = threadIdx.x; i < N; i += blockDim.x) sm[i] = io[i];
  __syncthreads();
  ntt_inv_smem(sm, d.lgN, twi + (size_t)j * kTwStride, p);
  for (int i = threadIdx.x; i < N; i += blockDim.x) io[i] = sm[i];
}

// ---------------------------------------------------------------------------
// Contraction on CUDA cores.  One thread per frequency h; it walks the m x n
// outputs in register tiles of TI x TJ (2 or 4 each, chosen per product and
// stored in ProdDesc::pad), loading TI + TJ residues per TI * TJ products.
// Edge tiles clamp their row/column to the last one (in-bounds duplicate
// work, results discarded).  Products of residues < p < 2^30 are < 2^60, so
// sixteen of them accumulate exactly in 64 bits before a Montgomery fold (the
// reference reduces every 16 terms for the same reason with 128-bit
// accumulators, src/lib/mpnfft.c:621-627).  Outputs carry a factor 2^-32
// that the CRT stage removes.
// ---------------------------------------------------------------------------
constexpr int kContractThreads = 128;

// x mod p for any 64-bit x (Barrett on the high word, then REDC of the
// reduced value times 2^32): keeps the accumulator's value, not its
// Montgomery image, so folds can be repeated.
__device__ __forceinline__ uint64_t fold64(uint64_t x, uint32_t p, uint32_t pinv, uint32_t mu,
                                           uint32_t r2) {
  // x = hi 2^32 + lo;  x mod p = REDC((x 2^-32 mod p) * 2^64 mod p)
  const uint32_t t = redc64(x, p, pinv, mu);           // x 2^-32 mod p
  return redc((uint64_t)t * r2, p, pinv);              // x mod p
}

template <int TI, int TJ>
__device__ __forceinline__ void contract_tiles(const ProdDesc& d, int j, uint32_t h,
                                               uint32_t* __restrict__ res) {
  const int N = 1 << d.lgN;
  const uint32_t p = c_primes[j].p;
  const uint32_t pinv = c_primes[j].pinv;
  const uint32_t mu = c_primes[j].mu;
  const uint32_t r2 = c_primes[j].r2;
  const uint32_t stride = (uint32_t)d.P * (uint32_t)N;  // words between polynomials
  const uint64_t base = (uint64_t)j * (uint64_t)N + h;
  const uint32_t* __restrict__ A = res + d.a_res + base;
  const uint32_t* __restrict__ B = res + d.b_res + base;
  uint32_t* C = res + d.c_res + base;
  const int m = d.m, k = d.k, n = d.n;
  const uint32_t bstep = (uint32_t)n * stride;
  for (int i0 = 0; i0 < m; i0 += TI) {
    for (int l0 = 0; l0 < n; l0 += TJ) {
      uint32_t ao[TI], bo[TJ];  // word offsets of the tile's rows / columns
#pragma unroll
      for (int x = 0; x < TI; ++x) {
        const int ii = (i0 + x) < m ? (i0 + x) : (m - 1);
        ao[x] = (uint32_t)ii * (uint32_t)k * stride;
      }
#pragma unroll
      for (int y = 0; y < TJ; ++y) {
        const int ll = (l0 + y) < n ? (l0 + y) : (n - 1);
        bo[y] = (uint32_t)ll * stride;
      }
      uint64_t acc[TI][TJ];
#pragma unroll
      for (int x = 0; x < TI; ++x)
#pragma unroll
        for (int y = 0; y < TJ; ++y) acc[x][y] = 0;
      // acc < p + 15 p^2 < 2^64 between folds
      int since = 0;
      int q = 0;
      for (; q + 4 <= k; q += 4) {
        uint32_t av[4][TI], bv[4][TJ];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
#pragma unroll
          for (int x = 0; x < TI; ++x) av[u][x] = __ldg(A + ao[x] + (uint32_t)(q + u) * stride);
#pragma unroll
          for (int y = 0; y < TJ; ++y) bv[u][y] = __ldg(B + bo[y] + (uint32_t)(q + u) * bstep);
        }
        if (since + 4 > 15) {
#pragma unroll
          for (int x = 0; x < TI; ++x)
#pragma unroll
            for (int y = 0; y < TJ; ++y) acc[x][y] = fold64(acc[x][y], p, pinv, mu, r2);
          since = 0;
        }
#pragma unroll
        for (int u = 0; u < 4; ++u)
#pragma unroll
          for (int x = 0; x < TI; ++x)
#pragma unroll
            for (int y = 0; y < TJ; ++y) acc[x][y] += (uint64_t)av[u][x] * bv[u][y];
        since += 4;
      }
      for (; q < k; ++q) {
        if (since + 1 > 15) {
#pragma unroll
          for (int x = 0; x < TI; ++x)
#pragma unroll
            for (int y = 0; y < TJ; ++y) acc[x][y] = fold64(acc[x][y], p, pinv, mu, r2);
          since = 0;
        }
        uint32_t av[TI], bv[TJ];
#pragma unroll
        for (int x = 0; x < TI; ++x) av[x] = __ldg(A + ao[x] + (uint32_t)q * stride);
#pragma unroll
        for (int y = 0; y < TJ; ++y) bv[y] = __ldg(B + bo[y] + (uint32_t)q * bstep);
#pragma unroll
        for (int x = 0; x < TI; ++x)
#pragma unroll
          for (int y = 0; y < TJ; ++y) acc[x][y] += (uint64_t)av[x] * bv[y];
        ++since;
      }
#pragma unroll
      for (int x = 0; x < TI; ++x) {
        if (i0 + x >= m) continue;
#pragma unroll
        for (int y = 0; y < TJ; ++y) {
          if (l0 + y >= n) continue;
          // the value times 2^-32 (the Montgomery factor the CRT removes)
          C[(uint32_t)((i0 + x) * n + (l0 + y)) * stride] = redc64(acc[x][y], p, pinv, mu);
        }
      }
    }
  }
}

__global__ void __launch_bounds__(kContractThreads)
k_contract(const ProdDesc* __restrict__ prods, const ContractItem* __restrict__ items,
           uint32_t* __restrict__ res) {
  const ContractItem it = items[blockIdx.x];
  const ProdDesc d = prods[it.prod];
  const int N = 1 << d.lgN;
  const uint32_t h = it.h0 + threadIdx.x;
  if (h >= (uint32_t)N) return;
  switch (d.pad) {  // tile shape, uniform over the CTA
    case 3: contract_tiles<4, 4>(d, it.prime, h, res); break;
    case 2: contract_tiles<4, 2>(d, it.prime, h, res); break;
    case 1: contract_tiles<2, 4>(d, it.prime, h, res); break;
    default: contract_tiles<2, 2>(d, it.prime, h, res); break;
  }
}

// ---------------------------------------------------------------------------
// CRT + recompose + sign + normalise: shared pieces.
//
// Coefficient i of an output entry is recovered as the symmetric residue
// X_i in (-M/4, M/4), M = p_0...p_{P-1}, written as X_i = U_i - s_i 2^(32P)
// with U_i the P-word two's complement and s_i its sign bit.  The entry is
// sum_i X_i 2^(i r) mod 2^(32 W).  Output word w gathers its local sum
//      s_w = sum_i slice_w(U_i 2^(i r)) - sum_i s_i [borrow of i lands in w]
// (a small signed 64-bit value), then s_w = lo_w + 2^32 hi_w is rewritten as
// words y_w with carries g_w in {-1,0,1}; the remaining carry ripple is a
// prefix scan whose element is the word's transfer function
// {-1,0,1} -> {-1,0,1}, composed associatively.  This is the parallel form
// of the reference's serial borrow chain (src/lib/recompose.c:43-87) and of
// its chunk fix-up (src/lib/crt_recompose.c:101-153); the reference's CRT is
// Garner's (src/lib/crt.c:11-94), the explicit form here needs O(P) modular
// products instead of O(P^2).
// ---------------------------------------------------------------------------

__device__ __forceinline__ int apply_tf(uint32_t f, int c) {
  return (int)((f >> (2 * (c + 1))) & 3u) - 1;
}
// g after f
__device__ __forceinline__ uint32_t compose_tf(uint32_t g, uint32_t f) {
  uint32_t out = 0;
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    const uint32_t fc = (f >> (2 * c)) & 3u;
    out |= ((g >> (2 * fc)) & 3u) << (2 * c);
  }
  return out;
}
constexpr uint32_t kTfIdentity = (0u) | (1u << 2) | (2u << 4);

__device__ __forceinline__ uint32_t word_tf(uint32_t y, int g) {
  uint32_t f = 0;
#pragma unroll
  for (int c = -1; c <= 1; ++c) {
    int delta = 0;
    if (c == 1 && y == 0xffffffffu) delta = 1;
    if (c == -1 && y == 0u) delta = -1;
    f |= (uint32_t)(g + delta + 1) << (2 * (c + 1));
  }
  return f;
}

// ---------------------------------------------------------------------------
// Split + forward NTT, register-blocked (lgN >= 3).
//
// 256 threads per CTA.  Small transforms (N <= 2048) are packed several per
// CTA: a team of N/8 threads owns one entry and each thread the 8 points
// x = q N/8 + t of the first pass, whose 30-bit coefficient digits it
// extracts once and keeps in registers for all P primes.  A residue is
//     c mod p = REDC( sum_q d_q * (2^(30 q + 32) mod p) )
// (D products of 30-bit by 30-bit numbers, exact in 64 bits for D <= 8), so
// each prime costs D wide multiply-adds and one Montgomery reduction instead
// of a Horner chain.  Larger transforms take a whole CTA; their digits are
// extracted once into shared memory when it has room (else per prime).  Then
// passes of 3 stages in registers (ntt_fast.cuh).
// ---------------------------------------------------------------------------
constexpr int kFwdThreads = 256;
// dynamic shared memory of a whole-CTA forward launch up to which its
// digits are cached (three CTAs still fit an SM)
constexpr int kFwdCacheBytes = 72 * 1024;

// Digits of the coefficient starting at bit bit0 (r bits of the entry's nw
// 32-bit words; bits past the entry read as 0).  Bit positions fit 32 bits:
// a transform has at most 2^15 coefficients of at most 210 bits.
template <int D>
__device__ __forceinline__ void coeff_digits(const uint32_t* __restrict__ w32, uint32_t nw,
                                             uint32_t bit0, uint32_t r, bool live,
                                             uint32_t (&dg)[D]) {
  // every word the D digits touch lies inside the entry (the usual case)
  const bool inside = live && ((bit0 + 30u * (D - 1)) >> 5) + 2u <= nw;
#pragma unroll
  for (int q = 0; q < D; ++q) {
    const uint32_t b = bit0 + 30u * q;
    const uint32_t wi = b >> 5;
    uint32_t lo, hi;
    if (inside) {
      lo = __ldg(w32 + wi);
      hi = __ldg(w32 + wi + 1);
    } else {
      lo = (live && wi < nw) ? __ldg(w32 + wi) : 0u;
      hi = (live && wi + 1 < nw) ? __ldg(w32 + wi + 1) : 0u;
    }
    uint32_t v = __funnelshift_r(lo, hi, b & 31u) & 0x3fffffffu;
    const int rem = (int)r - 30 * q;  // bits of the coefficient left for this digit
    if (rem < 30) v = rem <= 0 ? 0u : (v & ((1u << rem) - 1u));
    dg[q] = v;
  }
}

// The residue of a coefficient from its digits, lazily reduced: the REDC
// of S = sum_q d_q (2^(30q+32) mod p) < D 2^30 p is below (D/4 + 1) p < 3p
// for D <= 7, and a negative entry's residue is taken as 3p - v, in (0, 3p]:
// both below 4p, the forward transform's input range.
template <int D>
__device__ __forceinline__ uint32_t digits_residue(const uint32_t (&dg)[D], int j, bool neg) {
  const uint32_t p = c_primes[j].p;
  uint64_t S = 0;
#pragma unroll
  for (int q = 0; q < D; ++q) S += (uint64_t)dg[q] * c_primes[j].dig[q];
  const uint32_t m = (uint32_t)S * c_primes[j].pinv;
  const uint32_t v = (uint32_t)((S + (uint64_t)m * p) >> 32);
  return neg ? 3u * p - v : v;
}

// 2^L consecutive points reduced from [0, 4p) to [0, p), vector stores
template <int L>
__device__ __forceinline__ void store_points(uint32_t* dst, uint32_t* a, uint32_t p) {
  const uint32_t p2 = 2 * p;
#pragma unroll
  for (int q = 0; q < (1 << L); ++q) {
    const uint32_t v = reduce_2p(a[q], p2);
    a[q] = v >= p ? v - p : v;
  }
  if (L == 3) {
    reinterpret_cast<uint4*>(dst)[0] = make_uint4(a[0], a[1], a[2], a[3]);
    reinterpret_cast<uint4*>(dst)[1] = make_uint4(a[4], a[5], a[6], a[7]);
  } else if (L == 2) {
    reinterpret_cast<uint4*>(dst)[0] = make_uint4(a[0], a[1], a[2], a[3]);
  } else {
    reinterpret_cast<uint2*>(dst)[0] = make_uint2(a[0], a[1]);
  }
}

template <int LP>
__device__ __forceinline__ void fwd_last_pass(const uint32_t* s, uint32_t* out, bool valid,
                                              int lgN, int last_s0, int tt, int TS,
                                              const uint2* __restrict__ tw, uint32_t p) {
  for (int g = tt; g < ((1 << lgN) >> LP); g += TS) {
    uint32_t a[1 << LP];
#pragma unroll
    for (int q = 0; q < (1 << LP); ++q) a[q] = s[smi((g << LP) + q)];
    fwd_group<LP>(a, last_s0, g, tw, p);
    if (valid) store_points<LP>(out + (g << LP), a, p);
  }
}

// The body of k_fwd2.  HZ: every polynomial of the CTA has at most N/2
// coefficients (the usual case: both factors of a product fit in N
// together), so the first pass's upper four points are zero: their digits
// and residues are skipped and stage 0 only copies.  dig (whole-CTA HZ
// transforms, NULL otherwise): shared memory for the entry's digits, digit q
// of coefficient x at dig[q N/2 + x], extracted once for all P primes.
template <int D, bool TEAM, bool HZ>
__device__ __forceinline__ void fwd_body(const FwdDesc& d, uint32_t* s, uint32_t* dig,
                                         bool valid, int lgN, int P, int tt, int TS,
                                         const uint64_t* __restrict__ limbs,
                                         uint32_t* __restrict__ res,
                                         const uint2* __restrict__ twf) {
  const int N = 1 << lgN;
  const uint32_t nl = (uint32_t)(d.size < 0 ? -d.size : d.size);
  const uint32_t nw = nl < 0x40000000u ? 2u * nl : 0x80000000u;
  const uint32_t* __restrict__ w32 = reinterpret_cast<const uint32_t*>(limbs + d.limb_off);
  const bool neg = d.size < 0;
  const int ng0 = N >> 3;  // groups (and the point stride) of the first pass
  constexpr int QN = HZ ? 4 : 8;  // points of a first-pass group that can be nonzero
  const bool cached = !TEAM && HZ && dig != nullptr;

  uint32_t dg[QN][D];
  if (TEAM) {
#pragma unroll
    for (int q = 0; q < QN; ++q) {
      const int x = q * ng0 + tt;
      coeff_digits<D>(w32, nw, (uint32_t)x * d.r, d.r, (uint32_t)x < d.ncoef, dg[q]);
    }
  } else if (cached) {
    const int half = N >> 1;
    for (int x = tt; x < half; x += TS) {
      uint32_t t[D];
      coeff_digits<D>(w32, nw, (uint32_t)x * d.r, d.r, (uint32_t)x < d.ncoef, t);
#pragma unroll
      for (int q = 0; q < D; ++q) dig[q * half + x] = t[q];
    }
    __syncthreads();
  }
  for (int j = 0; j < P; ++j) {
    const uint32_t p = c_primes[j].p;
    const uint2* tw = twf + (size_t)j * kTwStride;
    uint32_t* out = res + d.res_off + (uint64_t)j * (uint64_t)N;
    for (int g = tt; g < ng0; g += TS) {
      uint32_t a[8];
#pragma unroll
      for (int q = 0; q < QN; ++q) {
        const int x = q * ng0 + g;
        if (!TEAM) {
          if (cached) {
#pragma unroll
            for (int u = 0; u < D; ++u) dg[q][u] = dig[u * (N >> 1) + x];
          } else {
            coeff_digits<D>(w32, nw, (uint32_t)x * d.r, d.r, (uint32_t)x < d.ncoef, dg[q]);
          }
        }
        a[q] = digits_residue<D>(dg[q], j, neg);
      }
      if (HZ) {
        fwd_stage0_upper_zero<3>(a, p);
        fwd_group<3, 1>(a, 0, 0, tw, p);
      } else {
        fwd_group<3>(a, 0, 0, tw, p);
      }
      if (lgN == 3) {  // the only pass: eight consecutive points, straight out
        if (valid) store_points<3>(out, a, p);
      } else {
#pragma unroll
        for (int q = 0; q < 8; ++q) s[smi(q * ng0 + g)] = a[q];
      }
    }
    if (lgN == 3) continue;  // uniform per CTA
    __syncthreads();
    const int last_s0 = ((lgN - 1) / 3) * 3;
    for (int s0 = 3; s0 < last_s0; s0 += 3) {
      smem_pass<3, true>(s, lgN, s0, 3, tt, TS, tw, p);
      __syncthreads();
    }
    // the last pass works on groups of 2^LP consecutive points: reduced and
    // stored straight from registers with vector stores
    switch (lgN - last_s0) {
      case 1: fwd_last_pass<1>(s, out, valid, lgN, last_s0, tt, TS, tw, p); break;
      case 2: fwd_last_pass<2>(s, out, valid, lgN, last_s0, tt, TS, tw, p); break;
      default: fwd_last_pass<3>(s, out, valid, lgN, last_s0, tt, TS, tw, p); break;
    }
    __syncthreads();  // before the next prime's first pass overwrites s
  }
}

// dig_words: shared memory words after the transform reserved for the digit
// cache of a whole-CTA launch (0: none); it holds D N/2 words for the CTA's
// transform size.
template <int D, bool TEAM>
__global__ void __launch_bounds__(kFwdThreads, 3)
k_fwd2(const FwdDesc* __restrict__ descs, const uint32_t* __restrict__ idx,
       const CtaItem* __restrict__ items, const uint64_t* __restrict__ limbs,
       uint32_t* __restrict__ res, const uint2* __restrict__ twf, int dig_words) {
  extern __shared__ uint32_t sm[];
  const CtaItem item = items[blockIdx.x];
  const int lgN = item.lgN;
  const int P = item.P;
  const int N = 1 << lgN;
  const int TS = TEAM ? (N >> 3) : kFwdThreads;  // threads per entry
  const int team = TEAM ? (int)threadIdx.x / TS : 0;
  const int tt = TEAM ? (int)threadIdx.x % TS : (int)threadIdx.x;
  const bool valid = team < (int)item.count;
  uint32_t* s = sm + team * (N + (N >> 5));
  uint32_t* dig = (!TEAM && dig_words >= D * (N >> 1)) ? s + N + (N >> 5) : nullptr;
  FwdDesc d;
  d.limb_off = 0;
  d.res_off = 0;
  d.size = 0;
  d.r = 1;
  d.ncoef = 0;
  if (valid) d = descs[idx[item.first + team]];
  // one variant for the whole CTA (its barriers must be the same code)
  if (__syncthreads_and(d.ncoef <= (uint32_t)(N >> 1)))
    fwd_body<D, TEAM, true>(d, s, dig, valid, lgN, P, tt, TS, limbs, res, twf);
  else
    fwd_body<D, TEAM, false>(d, s, nullptr, valid, lgN, P, tt, TS, limbs, res, twf);
}

// Inverse NTT, register-blocked (lgN >= 3): the forward passes backwards.
//
// The last forward pass (stages last_s0 .. lgN-1, LP = lgN - last_s0 of
// them) works on groups of 2^LP consecutive points, so its inverse reads
// each group straight from global memory with one or two vector loads and
// only then goes to shared memory.  In a team CTA every thread owns exactly
// eight of those points per prime, and the next prime's eight are loaded
// into registers before the current prime's passes run, so the loads
// overlap the arithmetic instead of stalling the warps.

template <int L>
__device__ __forceinline__ void load_points(const uint32_t* src, uint32_t* a) {
  if (L == 3) {
    const uint4 u = *reinterpret_cast<const uint4*>(src);
    const uint4 v = *reinterpret_cast<const uint4*>(src + 4);
    a[0] = u.x; a[1] = u.y; a[2] = u.z; a[3] = u.w;
    a[4] = v.x; a[5] = v.y; a[6] = v.z; a[7] = v.w;
  } else if (L == 2) {
    const uint4 u = *reinterpret_cast<const uint4*>(src);
    a[0] = u.x; a[1] = u.y; a[2] = u.z; a[3] = u.w;
  } else {
    const uint2 u = *reinterpret_cast<const uint2*>(src);
    a[0] = u.x; a[1] = u.y;
  }
}

// the groups of the last forward pass (2^LP points each) in registers:
// inverse stages, then into shared memory
template <int LP>
__device__ __forceinline__ void inv_last_pass(uint32_t* s, const uint32_t* a_in, int g,
                                              int last_s0, const uint2* tw, uint32_t p) {
  uint32_t a[1 << LP];
#pragma unroll
  for (int q = 0; q < (1 << LP); ++q) a[q] = a_in[q];
  inv_group<LP>(a, last_s0, g, tw, p);
#pragma unroll
  for (int q = 0; q < (1 << LP); ++q) s[smi((g << LP) + q)] = a[q];
}

template <int LP, bool TEAM>
__device__ __forceinline__ void inv_run(uint32_t* s, uint32_t* __restrict__ res, uint64_t off,
                                        bool valid, int lgN, int P, int tt, int TS,
                                        const uint2* __restrict__ twi) {
  const int N = 1 << lgN;
  const int last_s0 = lgN - LP;
  constexpr int GT = 8 >> LP;  // groups per thread in a team CTA
  uint32_t nx[8];               // team: the next prime's points
  if (TEAM && valid) {
#pragma unroll
    for (int k = 0; k < GT; ++k) load_points<LP>(res + off + ((tt + k * TS) << LP), nx + (k << LP));
  }
  for (int j = 0; j < P; ++j) {
    const uint32_t p = c_primes[j].p;
    const uint2* tw = twi + (size_t)j * kTwStride;
    uint32_t* io = res + off + (uint64_t)j * (uint64_t)N;
    if (last_s0 == 0) {
      // lgN = 3: one pass, global -> registers -> global
      if (TEAM && valid) {
        uint32_t a[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) a[q] = nx[q];
        if (j + 1 < P) load_points<3>(io + N, nx);
        inv_group<3>(a, 0, 0, tw, p);
        uint4* o = reinterpret_cast<uint4*>(io);
        o[0] = make_uint4(a[0], a[1], a[2], a[3]);
        o[1] = make_uint4(a[4], a[5], a[6], a[7]);
      }
      continue;
    }
    if (TEAM) {
      uint32_t a[8];
#pragma unroll
      for (int q = 0; q < 8; ++q) a[q] = valid ? nx[q] : 0u;
      if (valid && j + 1 < P) {
#pragma unroll
        for (int k = 0; k < GT; ++k)
          load_points<LP>(io + N + ((tt + k * TS) << LP), nx + (k << LP));
      }
#pragma unroll
      for (int k = 0; k < GT; ++k) inv_last_pass<LP>(s, a + (k << LP), tt + k * TS, last_s0, tw, p);
    } else {
      for (int g = tt; g < (N >> LP); g += TS) {
        uint32_t a[1 << LP];
        if (valid) {
          load_points<LP>(io + (g << LP), a);
        } else {
#pragma unroll
          for (int q = 0; q < (1 << LP); ++q) a[q] = 0u;
        }
        inv_last_pass<LP>(s, a, g, last_s0, tw, p);
      }
    }
    __syncthreads();
    for (int s0 = last_s0 - 3; s0 >= 3; s0 -= 3) {
      smem_pass<3, false>(s, lgN, s0, 3, tt, TS, tw, p);
      __syncthreads();
    }
    // first forward pass (stages 0..2) inverted, straight to global memory
    for (int g = tt; g < (N >> 3); g += TS) {
      uint32_t a[8];
#pragma unroll
      for (int q = 0; q < 8; ++q) a[q] = s[smi(q * (N >> 3) + g)];
      inv_group<3>(a, 0, 0, tw, p);
      if (valid) {
#pragma unroll
        for (int q = 0; q < 8; ++q) io[q * (N >> 3) + g] = a[q];  // in [0, 2p)
      }
    }
    __syncthreads();
  }
}

template <bool TEAM>
__global__ void __launch_bounds__(kFwdThreads)
k_inv2(const InvDesc* __restrict__ descs, const uint32_t* __restrict__ idx,
       const CtaItem* __restrict__ items, uint32_t* __restrict__ res,
       const uint2* __restrict__ twi) {
  extern __shared__ uint32_t sm[];
  const CtaItem item = items[blockIdx.x];
  const int lgN = item.lgN;
  const int P = item.P;
  const int N = 1 << lgN;
  const int TS = TEAM ? (N >> 3) : kFwdThreads;
  const int team = TEAM ? (int)threadIdx.x / TS : 0;
  const int tt = TEAM ? (int)threadIdx.x % TS : (int)threadIdx.x;
  const bool valid = team < (int)item.count;
  uint32_t* s = sm + team * (N + (N >> 5));
  const uint64_t off = valid ? descs[idx[item.first + team]].res_off : 0;
  const int last_s0 = ((lgN - 1) / 3) * 3;  // start of the last forward pass
  switch (lgN - last_s0) {
    case 1: inv_run<1, TEAM>(s, res, off, valid, lgN, P, tt, TS, twi); break;
    case 2: inv_run<2, TEAM>(s, res, off, valid, lgN, P, tt, TS, twi); break;
    default: inv_run<3, TEAM>(s, res, off, valid, lgN, P, tt, TS, twi); break;
  }
}


// ---------------------------------------------------------------------------
// CRT + recompose, one warp per output entry (no block barriers).
//
// Explicit CRT (crt_coeff) to the symmetric P-word value U_i - s_i 2^(32P)
// of each coefficient (s_i = top bit of U_i), per-word gathered sums, carries
// normalised into {-1, 0, 1}.  The ripple is resolved per 32-word step: when
// no word of the step is 0 or all-ones (a carry can only pass through such a
// word), word w's incoming carry is just the generated carry g_{w-1}; only
// otherwise does the warp run the prefix scan of transfer functions.
// ---------------------------------------------------------------------------
constexpr int kCrtWarps = 4;       // entries per CTA
constexpr int kCrtSteps = 8;       // 32-word steps per tile
constexpr int kCrtTileWords = 32 * kCrtSteps;

// Explicit CRT of one coefficient (constants in CrtConst): the symmetric
// residue X in (-M_P/4, M_P/4) as P words of two's complement.
template <int P>
__device__ __forceinline__ void crt_coeff(const uint32_t* __restrict__ res, uint64_t res_off,
                                          int lgN, int64_t ic, uint32_t (&X)[P]) {
  const uint64_t N = (uint64_t)1 << lgN;
  uint32_t y[P];
  uint64_t frac = 0;
#pragma unroll
  for (int j = 0; j < P; ++j) {
    const uint32_t p = c_primes[j].p;
    const uint32_t x = __ldg(res + res_off + (uint64_t)j * N + (uint64_t)ic);  // [0, 2p)
    y[j] = redc((uint64_t)x * c_crt.cm[P][lgN][j], p, c_primes[j].pinv);
    frac += (uint64_t)y[j] * c_crt.fq[j];
  }
  const uint32_t q = (uint32_t)((frac + (1ull << 57)) >> 58);  // nearest integer
  // sum_j y_j (M_P / p_j) in base-2^30 columns (M_P / p_j has P - 1 digits):
  // products below 2^60, at most 16 per column, no carries inside the sum
  uint64_t acc[P];
#pragma unroll
  for (int w = 0; w < P; ++w) acc[w] = 0;
#pragma unroll
  for (int j = 0; j < P; ++j)
#pragma unroll
    for (int w = 0; w + 1 < P; ++w) acc[w] += (uint64_t)y[j] * c_crt.mop30[P][j][w];
  // digits: carry-normalise (column + carry < 2^64), then subtract q M_P with
  // a signed borrow; the top digit is 0 for X >= 0 and -1 for X < 0
  uint32_t dg[P];
  uint64_t cy = 0;
#pragma unroll
  for (int w = 0; w < P; ++w) {
    const uint64_t t = acc[w] + cy;
    dg[w] = (uint32_t)t & 0x3fffffffu;
    cy = t >> 30;
  }
  int64_t b = 0;
#pragma unroll
  for (int w = 0; w < P; ++w) {
    const int64_t e = (int64_t)dg[w] - (int64_t)q * (int64_t)c_crt.M30[P][w] + b;
    dg[w] = (uint32_t)e & 0x3fffffffu;
    b = e >> 30;  // arithmetic: floor division
  }
  const bool neg = ((int64_t)cy + b) < 0;
  // repack the 30P bits to P 32-bit words of the two's complement value
  uint64_t buf = 0;
  int bits = 0, wi = 0;
#pragma unroll
  for (int w = 0; w < P; ++w) {
    buf |= (uint64_t)dg[w] << bits;
    bits += 30;
    if (bits >= 32) {
      X[wi++] = (uint32_t)buf;
      buf >>= 32;
      bits -= 32;
    }
  }
  const uint32_t fill = neg ? 0xffffffffu : 0u;
#pragma unroll
  for (int w = 0; w < P; ++w) {
    if (w < wi) continue;
    X[w] = (w == wi) ? ((uint32_t)buf | (fill << bits)) : fill;
  }
}

// floor(x / d) for x < 2^31: a multiply-high by floor((2^32 - 1) / d) is at
// most 2 below the quotient, then at most two corrections
struct FastDiv {
  uint32_t d, m;
  __device__ explicit FastDiv(uint32_t d_) : d(d_), m(0xffffffffu / d_) {}
  __device__ __forceinline__ uint32_t operator()(uint32_t x) const {
    uint32_t q = __umulhi(x, m);
    if ((q + 1) * d <= x) ++q;
    if ((q + 1) * d <= x) ++q;
    return q;
  }
};

// One output entry by one warp: CRT of its coefficients tile by tile into
// the warp's scratch sU (word q of tile coefficient c at [q * cmax + c]),
// the words' sums, the carry ripple, the sign and the size.
template <int P>
__device__ __forceinline__ void crt_entry(const InvDesc& d, const uint32_t* __restrict__ res,
                                          uint32_t* __restrict__ out,
                                          int32_t* __restrict__ out_sizes, uint32_t* sU,
                                          int cmax, int lane) {
  const unsigned FULL = 0xffffffffu;
  // bit positions fit 31 bits (an entry's words times 32 stays below 2^31),
  // so index arithmetic is 32-bit and the divisions by r are multiply-highs
  const int r = (int)d.r;
  const FastDiv divr((uint32_t)r);
  const int W = (int)d.out_words;
  const int ncoef = (int)d.ncoef;
  uint32_t* o = out + d.out_word;

  int hi_prev = 0, carry = 0;
  int first_nz = 0x7fffffff, last_nz = -1, last_no = -1;
  uint32_t topval = 0;
  for (int w0 = 0; w0 < W; w0 += kCrtTileWords) {
    int lo_i = 0;
    if (32 * w0 > 32 * P) lo_i = (int)divr((uint32_t)(32 * w0 - 32 * P + r - 1));
    int hi_i = (int)divr((uint32_t)(32 * (w0 + kCrtTileWords) - 1));
    if (hi_i > ncoef - 1) hi_i = ncoef - 1;
    const int ncf = hi_i >= lo_i ? hi_i - lo_i + 1 : 0;
    for (int c = lane; c < ncf; c += 32) {
      uint32_t X[P];
      crt_coeff<P>(res, d.res_off, d.lgN, lo_i + c, X);
#pragma unroll
      for (int q = 0; q < P; ++q) sU[q * cmax + c] = X[q];
    }
    __syncwarp();
    for (int st = 0; st < kCrtSteps; ++st) {
      const int w = w0 + st * 32 + lane;
      const bool active = w < W;
      int64_t sw = 0;
      if (active) {
        int ia = lo_i;
        if (32 * w > 32 * P) {
          const int t = (int)divr((uint32_t)(32 * w - 32 * P + r - 1));
          if (t > ia) ia = t;
        }
        int ib = (int)divr((uint32_t)(32 * w + 31));
        if (ib > hi_i) ib = hi_i;
        for (int i = ia; i <= ib; ++i) {
          const int c = i - lo_i;
          const int bi = i * r;
          const int dd = 32 * w - bi;
          const uint32_t* U = sU + c;  // word q at U[q * cmax]
          uint32_t slice;
          if (dd < 0) {
            slice = U[0] << (uint32_t)(-dd);
          } else {
            const int q = dd >> 5;
            const uint32_t sh = (uint32_t)(dd & 31);
            const uint32_t lo = q < P ? U[q * cmax] : 0u;
            const uint32_t hi = q + 1 < P ? U[(q + 1) * cmax] : 0u;
            slice = __funnelshift_r(lo, hi, sh);
          }
          sw += slice;
          // the sign of X_i is the top bit of U_i; its borrow lands in word
          // (i r) / 32 + P
          if ((bi >> 5) + P == w && (U[(P - 1) * cmax] >> 31)) sw -= (int64_t)1 << (bi & 31);
        }
      }
      const int hi = active ? (int)(sw >> 32) : 0;
      int hprev = __shfl_up_sync(FULL, hi, 1);
      if (lane == 0) hprev = hi_prev;
      const int64_t z = (int64_t)(uint32_t)sw + hprev;
      const uint32_t y = (uint32_t)z;
      const int g = active ? (int)(z >> 32) : 0;
      const bool prop = active && (y == 0u || y == 0xffffffffu);
      int cin, cout;
      if (__any_sync(FULL, prop)) {
        const uint32_t f = active ? word_tf(y, g) : kTfIdentity;
        uint32_t inc = f;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
          const uint32_t u = __shfl_up_sync(FULL, inc, off);
          if (lane >= off) inc = compose_tf(inc, u);
        }
        uint32_t exc = __shfl_up_sync(FULL, inc, 1);
        if (lane == 0) exc = kTfIdentity;
        cin = apply_tf(exc, carry);
        cout = apply_tf(__shfl_sync(FULL, inc, 31), carry);
      } else {
        cin = __shfl_up_sync(FULL, g, 1);
        if (lane == 0) cin = carry;
        cout = __shfl_sync(FULL, g, 31);
      }
      if (active) {
        const uint32_t F = y + (uint32_t)cin;
        o[w] = F;
        if (F != 0u) {
          if ((int)w < first_nz) first_nz = (int)w;
          last_nz = (int)w;
        }
        if (F != 0xffffffffu) last_no = (int)w;
        if (w == W - 1) topval = F;
      }
      hi_prev = __shfl_sync(FULL, hi, 31);
      carry = cout;
    }
    __syncwarp();
  }
  first_nz = __reduce_min_sync(FULL, first_nz);
  last_nz = __reduce_max_sync(FULL, last_nz);
  last_no = __reduce_max_sync(FULL, last_no);
  topval = __reduce_or_sync(FULL, topval);
  const bool negative = W > 0 && (topval >> 31);
  int top;
  if (negative) {
    const int zf = first_nz;
    for (int64_t w = zf + lane; w < W; w += 32) {
      const uint32_t F = o[w];
      o[w] = (w == zf) ? (0u - F) : ~F;
    }
    top = last_no > zf ? last_no : zf;
  } else {
    top = last_nz;
  }
  if (lane == 0) {
    const int limbs = top >= 0 ? top / 2 + 1 : 0;
    out_sizes[d.entry] = negative ? -limbs : limbs;
  }
}

// One prime count per launch.
template <int P>
__global__ void __launch_bounds__(32 * kCrtWarps)
k_crt_warp(const InvDesc* __restrict__ descs, const uint32_t* __restrict__ idx, int count,
           const uint32_t* __restrict__ res, uint32_t* __restrict__ out,
           int32_t* __restrict__ out_sizes, int cmax) {
  extern __shared__ uint32_t sm[];
  const int warp = threadIdx.x >> 5;
  const int slot = blockIdx.x * kCrtWarps + warp;
  if (slot >= count) return;  // whole warp; no block-wide barrier below
  const InvDesc d = descs[idx[slot]];
  crt_entry<P>(d, res, out, out_sizes, sm + warp * (cmax * P), cmax, threadIdx.x & 31);
}

template <int P, int PHI>
__device__ __forceinline__ void crt_dispatch(const InvDesc& d, const uint32_t* __restrict__ res,
                                             uint32_t* __restrict__ out,
                                             int32_t* __restrict__ out_sizes, uint32_t* sU,
                                             const CrtScratch& cs, int lane) {
  if (d.P == P) {
    crt_entry<P>(d, res, out, out_sizes, sU, cs.cmax[P], lane);
  } else {
    if constexpr (P < PHI) crt_dispatch<P + 1, PHI>(d, res, out, out_sizes, sU, cs, lane);
  }
}

// Prime counts PLO..PHI in one launch (the entries longest first across
// them, so the long entries of every count start together and the launch
// has one tail instead of one per count); each warp's scratch holds
// cs.warp_words words.
template <int PLO, int PHI>
__global__ void __launch_bounds__(32 * kCrtWarps)
k_crt_mixed(const InvDesc* __restrict__ descs, const uint32_t* __restrict__ idx, int count,
            const uint32_t* __restrict__ res, uint32_t* __restrict__ out,
            int32_t* __restrict__ out_sizes, CrtScratch cs) {
  extern __shared__ uint32_t sm[];
  const int warp = threadIdx.x >> 5;
  const int slot = blockIdx.x * kCrtWarps + warp;
  if (slot >= count) return;  // whole warp; no block-wide barrier below
  const InvDesc d = descs[idx[slot]];
  crt_dispatch<PLO, PHI>(d, res, out, out_sizes, sm + warp * cs.warp_words, cs,
                         threadIdx.x & 31);
}


// ---------------------------------------------------------------------------
// Tensor-core contraction (see contract_tc.cuh for the exact-split scheme).
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(tc::kThreads, 1)
k_contract_tc(const ProdDesc* __restrict__ prods, const ContractItem* __restrict__ items,
              uint32_t* __restrict__ res, int fb, int* __restrict__ status, int stall) {
  extern __shared__ __align__(1024) uint8_t tsm[];
  __shared__ __align__(8) uint64_t bar;
  __shared__ uint32_t tmem_slot;
  const int tid = threadIdx.x;
  const int warp = tid >> 5;
  const int lane = tid & 31;
  const ContractItem it = items[blockIdx.x];
  const ProdDesc d = prods[it.prod];
  const int m = d.m, k = d.k, n = d.n;
  const int N = 1 << d.lgN;
  const int j = it.prime;
  const uint32_t p = c_primes[j].p;
  const uint64_t stride = (uint64_t)d.P * (uint64_t)N;
  const uint32_t kprime = (uint32_t)((4 * k + 31) & ~31);
  const uint32_t ncols = (uint32_t)((8 * n + 15) & ~15);  // B' rows = D columns
  uint8_t* As = tsm;
  uint8_t* Bs = tsm + 128u * kprime;
  const uint32_t tile_bytes = (128u + ncols) * kprime;

  // zero both tiles once: padding rows/columns stay zero for every frequency
  for (uint32_t o = 16u * tid; o < tile_bytes; o += 16u * tc::kThreads)
    *reinterpret_cast<uint4*>(tsm + o) = make_uint4(0, 0, 0, 0);
  if (warp == 0) {
    const uint32_t slot = tc::smem_u32(&tmem_slot);
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                 :: "r"(slot), "r"((uint32_t)tc::kTmemCols) : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(tc::smem_u32(&bar)) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_slot;
  const uint32_t barp = tc::smem_u32(&bar);
  uint32_t phase = 0;
  const uint64_t bias = c_primes[j].bias;
  const uint32_t pinv = c_primes[j].pinv;
  const uint32_t mu = c_primes[j].mu;

  for (int f = 0; f < fb; ++f) {
    const uint32_t h = it.h0 + (uint32_t)f;
    if (h >= (uint32_t)N) break;  // uniform over the CTA
    const uint64_t base = (uint64_t)j * (uint64_t)N + h;
    // stage A' (row i, bytes 4kk..4kk+3) and B' (rows 8l+u, same bytes)
    for (int idx = tid; idx < m * k; idx += tc::kThreads) {
      const int i = idx / k, kk = idx - (idx / k) * k;
      const uint32_t x = __ldg(res + d.a_res + (uint64_t)(i * k + kk) * stride + base);
      *reinterpret_cast<uint32_t*>(As + tc::tile_off((uint32_t)i, 4u * kk, kprime)) =
          tc::split_bytes(x, p);
    }
    for (int idx = tid; idx < k * n; idx += tc::kThreads) {
      const int kk = idx / n, l = idx - (idx / n) * n;
      const uint32_t x = __ldg(res + d.b_res + (uint64_t)(kk * n + l) * stride + base);
      const uint32_t rev = __byte_perm(tc::split_bytes(x, p), 0u, 0x0123u);  // d3 d2 d1 d0
      const uint64_t T = (uint64_t)rev << 32;
#pragma unroll
      for (int u = 0; u < 7; ++u)
        *reinterpret_cast<uint32_t*>(Bs + tc::tile_off((uint32_t)(8 * l + u), 4u * kk, kprime)) =
            (uint32_t)(T >> (8 * (7 - u)));
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    // stall (failure-path tests only): no MMA and no commit are issued, so
    // nothing ever arrives on the barrier and the bounded wait below runs out
    // with no tensor operation outstanding
    if (tid == 0 && !stall) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      for (uint32_t t0 = 0; t0 < ncols; t0 += 256) {
        const uint32_t nt = (ncols - t0) < 256u ? (ncols - t0) : 256u;
        const uint32_t idesc = tc::idesc_i8(nt);
        for (uint32_t ks = 0; ks < kprime / 32; ++ks) {
          const uint64_t ad = tc::smem_desc(tc::smem_u32(As) + 256u * ks, kprime);
          const uint64_t bd = tc::smem_desc(tc::smem_u32(Bs) + t0 * kprime + 256u * ks, kprime);
          const uint32_t acc = ks > 0 ? 1u : 0u;
          asm volatile(
              "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
              "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
              :: "r"(tmem + t0), "l"(ad), "l"(bd), "r"(idesc), "r"(acc),
                 "r"(0u), "r"(0u), "r"(0u), "r"(0u)
              : "memory");
        }
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
                   :: "r"(barp) : "memory");
    }
    const bool ok = tc::mbar_wait(barp, phase);
    phase ^= 1u;
    if (__syncthreads_or(!ok)) {  // every thread takes the same branch
      if (tid == 0) atomicExch(status, 1);
      break;
    }
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    // epilogue: warp w owns TMEM lanes 32w..32w+31 = rows i
    const int i = 32 * warp + lane;
    const uint32_t lane_addr = tmem + ((uint32_t)(32 * warp) << 16);
    for (int l0 = 0; l0 < n; l0 += 4) {
      uint32_t v[32];
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x32.b32 "
          "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
          "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
          : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]),
            "=r"(v[6]), "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]),
            "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15]), "=r"(v[16]), "=r"(v[17]),
            "=r"(v[18]), "=r"(v[19]), "=r"(v[20]), "=r"(v[21]), "=r"(v[22]), "=r"(v[23]),
            "=r"(v[24]), "=r"(v[25]), "=r"(v[26]), "=r"(v[27]), "=r"(v[28]), "=r"(v[29]),
            "=r"(v[30]), "=r"(v[31])
          : "r"(lane_addr + 8u * (uint32_t)l0));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      if (i < m) {
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const int l = l0 + q;
          if (l < n) {
            int64_t z = 0;
#pragma unroll
            for (int u = 0; u < 7; ++u) z += (int64_t)(int32_t)v[8 * q + u] * c_primes[j].w8[u];
            const uint32_t out = redc64((uint64_t)(z + (int64_t)bias), p, pinv, mu);
            res[d.c_res + (uint64_t)(i * n + l) * stride + base] = out;
          }
        }
      }
    }
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
  }
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;"
                 :: "r"(tmem), "r"((uint32_t)tc::kTmemCols) : "memory");
}

// ---------------------------------------------------------------------------
// Sizes of operands that live in device memory (results of an earlier plan):
// the planner sized their transforms for a bound; the true signed size and
// coefficient count go into the forward descriptors before the transforms.
// ---------------------------------------------------------------------------
__global__ void k_fix_sizes(FwdDesc* __restrict__ descs, int count,
                            const int32_t* __restrict__ sizes) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  FwdDesc d = descs[i];
  const int32_t sz = sizes[i];
  const uint64_t nl = (uint64_t)(sz < 0 ? -(int64_t)sz : sz);
  const uint64_t nc = (nl * 64 + d.r - 1) / d.r;
  const uint64_t N = (uint64_t)1 << d.lgN;
  descs[i].size = sz;
  descs[i].ncoef = (uint32_t)(nc < N ? nc : N);
}

cudaError_t launch_fix_sizes(FwdDesc* descs, int count, const int32_t* sizes, cudaStream_t st) {
  if (count <= 0) return cudaSuccess;
  k_fix_sizes<<<(count + 255) / 256, 256, 0, st>>>(descs, count, sizes);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Modular reduction r = x mod d (Barrett, HAC 14.42 with B = 2^64): the two
// big products run on the multiplication engine; these kernels shift sizes
// between them and finish each x with one warp.
// ---------------------------------------------------------------------------
// out[i] = max(0, |in[i]| - shift): sizes of operands viewed `shift` limbs up
__global__ void k_shift_sizes(const int32_t* __restrict__ in, int32_t* __restrict__ out,
                              int count, int shift) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= count) return;
  const int32_t s = in[i];
  const int32_t a = s < 0 ? -s : s;
  out[i] = a > shift ? a - shift : 0;
}

cudaError_t launch_shift_sizes(const int32_t* in, int32_t* out, int count, int shift,
                               cudaStream_t st) {
  if (count <= 0) return cudaSuccess;
  k_shift_sizes<<<(count + 255) / 256, 256, 0, st>>>(in, out, count, shift);
  return cudaGetLastError();
}

namespace {
// One 32-limb step of a - b - bin over the warp (limb `lane`): returns the
// difference limb; *bstep carries the borrow into the next step.
__device__ __forceinline__ uint64_t warp_sub_step(uint64_t a, uint64_t b, uint32_t* bstep) {
  const unsigned FULL = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  // borrow transfer per limb: out = g | (p & in)
  uint32_t g = a < b ? 1u : 0u, pp = a == b ? 1u : 0u;
#pragma unroll
  for (int off = 1; off < 32; off <<= 1) {
    const uint32_t gu = __shfl_up_sync(FULL, g, off), pu = __shfl_up_sync(FULL, pp, off);
    if (lane >= off) {
      g = g | (pp & gu);
      pp = pp & pu;
    }
  }
  const uint32_t out = g | (pp & *bstep);  // borrow out of this limb
  uint32_t in = __shfl_up_sync(FULL, out, 1);
  if (lane == 0) in = *bstep;
  *bstep = __shfl_sync(FULL, out, 31);
  return a - b - (uint64_t)in;
}

// r >= d over limbs [0, nl) (d is zero from limb nd on), warp-wide
__device__ __forceinline__ bool warp_geq(const uint64_t* r, const uint64_t* d, int nl, int nd) {
  const unsigned FULL = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  for (int j0 = ((nl - 1) >> 5) << 5; j0 >= 0; j0 -= 32) {
    const int j = j0 + lane;
    const uint64_t a = j < nl ? r[j] : 0, b = j < nd ? d[j] : 0;
    const unsigned diff = __ballot_sync(FULL, a != b);
    if (diff) {
      const int top = 31 - __clz(diff);
      return __shfl_sync(FULL, a > b ? 1 : 0, top) != 0;
    }
  }
  return true;  // equal
}
}  // namespace

// r_i = x_i mod d in [0, d): r = (|x| - s) mod B^(n+1) with s = q d and q at
// most 2 below floor(|x| / d), then up to two subtractions of d, then d - r
// for a negative x with r != 0.  One warp per x; rbuf holds n + 1 limbs per x.
__global__ void __launch_bounds__(128)
k_mod_finish(int count, int n, const uint64_t* __restrict__ xl, const int64_t* __restrict__ xo,
             const int32_t* __restrict__ xs, const uint64_t* __restrict__ sl, int64_t s_stride,
             const int32_t* __restrict__ ss, const uint64_t* __restrict__ d,
             uint64_t* __restrict__ rbuf, int32_t* __restrict__ rs) {
  const unsigned FULL = 0xffffffffu;
  const int lane = threadIdx.x & 31;
  const int i = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (i >= count) return;  // whole warp
  const int nl = n + 1;
  const int32_t xsz = xs[i];
  const bool neg = xsz < 0;
  const int xa = neg ? -xsz : xsz;
  const int sa = ss[i] < 0 ? -ss[i] : ss[i];
  const uint64_t* x = xl + xo[i];
  const uint64_t* s = sl + (int64_t)i * s_stride;
  uint64_t* r = rbuf + (int64_t)i * nl;
  uint32_t b = 0;
  for (int j0 = 0; j0 < nl; j0 += 32) {  // r = |x| - s mod B^(n+1)
    const int j = j0 + lane;
    const uint64_t a = (j < xa && j < nl) ? x[j] : 0, c = (j < sa && j < nl) ? s[j] : 0;
    const uint64_t v = warp_sub_step(a, c, &b);
    if (j < nl) r[j] = v;
  }
  __syncwarp();
  for (int rep = 0; rep < 2; ++rep) {  // r < 3d: at most two subtractions
    if (!warp_geq(r, d, nl, n)) break;
    b = 0;
    for (int j0 = 0; j0 < nl; j0 += 32) {
      const int j = j0 + lane;
      const uint64_t a = j < nl ? r[j] : 0, c = j < n ? d[j] : 0;
      const uint64_t v = warp_sub_step(a, c, &b);
      if (j < nl) r[j] = v;
    }
    __syncwarp();
  }
  // size, and d - r for a negative x with r != 0
  int top = -1;
  for (int j0 = 0; j0 < nl; j0 += 32) {
    const int j = j0 + lane;
    const unsigned nz = __ballot_sync(FULL, j < nl && r[j] != 0);
    if (nz) top = j0 + 31 - __clz(nz);
  }
  if (neg && top >= 0) {
    b = 0;
    top = -1;
    for (int j0 = 0; j0 < nl; j0 += 32) {
      const int j = j0 + lane;
      const uint64_t a = j < n ? d[j] : 0, c = j < nl ? r[j] : 0;
      const uint64_t v = warp_sub_step(a, c, &b);
      if (j < nl) r[j] = v;
      const unsigned nz = __ballot_sync(FULL, j < nl && v != 0);
      if (nz) top = j0 + 31 - __clz(nz);
    }
  }
  if (lane == 0) rs[i] = top + 1;
}

cudaError_t launch_mod_finish(int count, int n, const uint64_t* xl, const int64_t* xo,
                              const int32_t* xs, const uint64_t* sl, int64_t s_stride,
                              const int32_t* ss, const uint64_t* d, uint64_t* rbuf, int32_t* rs,
                              cudaStream_t st) {
  if (count <= 0) return cudaSuccess;
  k_mod_finish<<<(count + 3) / 4, 128, 0, st>>>(count, n, xl, xo, xs, sl, s_stride, ss, d, rbuf,
                                                rs);
  return cudaGetLastError();
}

// ---------------------------------------------------------------------------
// Host launchers
// ---------------------------------------------------------------------------
cudaError_t upload_constants(const PrimeConst* primes, const CrtConst* crt) {
  cudaError_t e = cudaMemcpyToSymbol(c_primes, primes, sizeof(PrimeConst) * kMaxPrimes);
  if (e != cudaSuccess) return e;
  return cudaMemcpyToSymbol(c_crt, crt, sizeof(CrtConst));
}

static int ntt_threads(int lgN) {
  const int half = 1 << (lgN - 1);
  return half < 32 ? 32 : (half > 1024 ? 1024 : half);
}

template <int D>
static cudaError_t launch_fwd2_d(const FwdDesc* descs, const uint32_t* idx,
                                 const CtaItem* items, int nitems, bool team, int max_lgN,
                                 const uint64_t* limbs, uint32_t* res, const uint2* twf,
                                 cudaStream_t st) {
  const int Nmax = 1 << max_lgN;
  if (team) {
    const size_t smem = sizeof(uint32_t) * (size_t)(8 * kFwdThreads + (8 * kFwdThreads >> 5));
    k_fwd2<D, true><<<nitems, kFwdThreads, smem, st>>>(descs, idx, items, limbs, res, twf, 0);
  } else {
    // whole-CTA transforms: the digit cache when the launch still fits
    // three CTAs an SM with it (every CTA's transform is at most Nmax)
    size_t smem = sizeof(uint32_t) * (size_t)(Nmax + (Nmax >> 5));
    const size_t cache = sizeof(uint32_t) * (size_t)D * (size_t)(Nmax >> 1);
    int dig_words = 0;
    if (smem + cache <= (size_t)kFwdCacheBytes) {
      smem += cache;
      dig_words = D * (Nmax >> 1);
    }
    k_fwd2<D, false><<<nitems, kFwdThreads, smem, st>>>(descs, idx, items, limbs, res, twf,
                                                        dig_words);
  }
  return cudaGetLastError();
}

int fwd_team_points() { return 8 * kFwdThreads; }

cudaError_t launch_fwd_items(const FwdDesc* descs, const uint32_t* idx, const CtaItem* items,
                             int nitems, int D, bool team, int max_lgN, const uint64_t* limbs,
                             uint32_t* res, const uint2* twf, cudaStream_t st) {
  if (nitems == 0) return cudaSuccess;
  switch (D) {
    case 1: return launch_fwd2_d<1>(descs, idx, items, nitems, team, max_lgN, limbs, res, twf, st);
    case 2: return launch_fwd2_d<2>(descs, idx, items, nitems, team, max_lgN, limbs, res, twf, st);
    case 3: return launch_fwd2_d<3>(descs, idx, items, nitems, team, max_lgN, limbs, res, twf, st);
    case 4: return launch_fwd2_d<4>(descs, idx, items, nitems, team, max_lgN, limbs, res, twf, st);
    case 5: return launch_fwd2_d<5>(descs, idx, items, nitems, team, max_lgN, limbs, res, twf, st);
    case 6: return launch_fwd2_d<6>(descs, idx, items, nitems, team, max_lgN, limbs, res, twf, st);
    case 7: return launch_fwd2_d<7>(descs, idx, items, nitems, team, max_lgN, limbs, res, twf, st);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t launch_inv_items(const InvDesc* descs, const uint32_t* idx, const CtaItem* items,
                             int nitems, bool team, int max_lgN, uint32_t* res,
                             const uint2* twi, cudaStream_t st) {
  if (nitems == 0) return cudaSuccess;
  const int Nmax = 1 << max_lgN;
  const size_t smem = team ? sizeof(uint32_t) * (size_t)(8 * kFwdThreads + (8 * kFwdThreads >> 5))
                           : sizeof(uint32_t) * (size_t)(Nmax + (Nmax >> 5));
  if (team) {
    k_inv2<true><<<nitems, kFwdThreads, smem, st>>>(descs, idx, items, res, twi);
  } else {
    k_inv2<false><<<nitems, kFwdThreads, smem, st>>>(descs, idx, items, res, twi);
  }
  return cudaGetLastError();
}

cudaError_t launch_split_fwd(const FwdDesc* descs, const uint32_t* idx, int count, int P,
                             int lgN, const uint64_t* limbs, uint32_t* res,
                             const uint2* twf, cudaStream_t st) {
  if (count == 0) return cudaSuccess;
  const size_t smem = sizeof(uint32_t) << lgN;
  dim3 grid(count, P);
  k_split_fwd<<<grid, ntt_threads(lgN), smem, st>>>(descs, idx, limbs, res, twf);
  return cudaGetLastError();
}

cudaError_t launch_inv_ntt(const InvDesc* descs, const uint32_t* idx, int count, int P,
                           int lgN, uint32_t* res, const uint2* twi, cudaStream_t st) {
  if (count == 0) return cudaSuccess;
  const size_t smem = sizeof(uint32_t) << lgN;
  dim3 grid(count, P);
  k_inv_ntt<<<grid, ntt_threads(lgN), smem, st>>>(descs, idx, res, twi);
  return cudaGetLastError();
}

cudaError_t launch_contract(const ProdDesc* prods, const ContractItem* items, int count,
                            uint32_t* res, cudaStream_t st) {
  if (count == 0) return cudaSuccess;
  k_contract<<<count, kContractThreads, 0, st>>>(prods, items, res);
  return cudaGetLastError();
}

int contract_block_freqs() { return kContractThreads; }

bool contract_tc_eligible(int m, int k, int n) {
  return m >= 1 && m <= tc::kMaxM && k >= 1 && k <= tc::kMaxK && n >= 1 && n <= tc::kMaxN;
}

cudaError_t launch_contract_tc(const ProdDesc* prods, const ContractItem* items, int count,
                               uint32_t* res, int fb, int max_k, int max_n, int* status,
                               cudaStream_t st, int stall) {
  if (count == 0) return cudaSuccess;
  const size_t kprime = (size_t)((4 * max_k + 31) & ~31);
  const size_t ncols = (size_t)((8 * max_n + 15) & ~15);
  size_t smem = (128 + ncols) * kprime;
  // at least 120 KB so that one CTA (512 TMEM columns) runs per SM
  if (smem < 120 * 1024) smem = 120 * 1024;
  k_contract_tc<<<count, tc::kThreads, smem, st>>>(prods, items, res, fb, status, stall);
  return cudaGetLastError();
}

// coefficients a CRT tile can touch for coefficient width rmin
static int crt_cmax(int P, int rmin) {
  return (int)((32 * (int64_t)kCrtTileWords + 32 * P) / rmin + 3);
}

cudaError_t launch_crt_mixed(const InvDesc* descs, const uint32_t* idx, int count, bool high,
                             const int* rmin, const uint32_t* res, uint32_t* out, int32_t* sizes,
                             cudaStream_t st) {
  if (count == 0) return cudaSuccess;
  const int plo = high ? kCrtMixedSplit + 1 : 2, phi = high ? kMaxPrimes : kCrtMixedSplit;
  CrtScratch cs;
  cs.warp_words = 0;
  for (int P = 0; P <= kMaxPrimes; ++P) {
    cs.cmax[P] = 0;
    if (P < plo || P > phi || rmin[P] <= 0) continue;
    cs.cmax[P] = crt_cmax(P, rmin[P]);
    if (cs.cmax[P] * P > cs.warp_words) cs.warp_words = cs.cmax[P] * P;
  }
  if (cs.warp_words == 0) return cudaErrorInvalidValue;
  const size_t smem = sizeof(uint32_t) * (size_t)cs.warp_words * kCrtWarps;
  if (smem > 200 * 1024) return cudaErrorInvalidValue;
  const int grid = (count + kCrtWarps - 1) / kCrtWarps;
  if (high)
    k_crt_mixed<kCrtMixedSplit + 1, kMaxPrimes><<<grid, 32 * kCrtWarps, smem, st>>>(
        descs, idx, count, res, out, sizes, cs);
  else
    k_crt_mixed<2, kCrtMixedSplit><<<grid, 32 * kCrtWarps, smem, st>>>(descs, idx, count, res,
                                                                      out, sizes, cs);
  return cudaGetLastError();
}

template <int P>
static cudaError_t launch_crt_t(const InvDesc* descs, const uint32_t* idx, int count,
                                const uint32_t* res, uint32_t* out, int32_t* sizes, int rmin,
                                cudaStream_t st) {
  const int cmax = crt_cmax(P, rmin);
  const size_t per_warp = sizeof(uint32_t) * (size_t)(cmax * P);
  const size_t smem = per_warp * kCrtWarps;
  if (smem > 200 * 1024) return cudaErrorInvalidValue;
  const int grid = (count + kCrtWarps - 1) / kCrtWarps;
  k_crt_warp<P><<<grid, 32 * kCrtWarps, smem, st>>>(descs, idx, count, res, out, sizes, cmax);
  return cudaGetLastError();
}

cudaError_t launch_crt_recompose(const InvDesc* descs, const uint32_t* idx, int count, int P,
                                 const uint32_t* res, uint32_t* out, int32_t* sizes, int rmin,
                                 cudaStream_t st) {
  if (count == 0) return cudaSuccess;
  if (rmin < 1) return cudaErrorInvalidValue;
  switch (P) {
#define MPZMM_CRT_CASE(PP) \
  case PP:                 \
    return launch_crt_t<PP>(descs, idx, count, res, out, sizes, rmin, st);
    MPZMM_CRT_CASE(2)
    MPZMM_CRT_CASE(3)
    MPZMM_CRT_CASE(4)
    MPZMM_CRT_CASE(5)
    MPZMM_CRT_CASE(6)
    MPZMM_CRT_CASE(7)
    MPZMM_CRT_CASE(8)
    MPZMM_CRT_CASE(9)
    MPZMM_CRT_CASE(10)
    MPZMM_CRT_CASE(11)
    MPZMM_CRT_CASE(12)
    MPZMM_CRT_CASE(13)
    MPZMM_CRT_CASE(14)
    MPZMM_CRT_CASE(15)
    MPZMM_CRT_CASE(16)
#undef MPZMM_CRT_CASE
    default:
      return cudaErrorInvalidValue;
  }
}


// Dynamic shared memory limits of every kernel, set once per device at
// set-up (so that launches, including those captured into a CUDA graph,
// issue nothing but stream work).
template <int D>
static cudaError_t set_fwd_attrs() {
  const int big = (int)(sizeof(uint32_t) * ((1 << kMaxLgN) + ((1 << kMaxLgN) >> 5)));
  cudaError_t e = cudaFuncSetAttribute(k_fwd2<D, true>,
                                       cudaFuncAttributeMaxDynamicSharedMemorySize, big);
  if (e != cudaSuccess) return e;
  return cudaFuncSetAttribute(k_fwd2<D, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, big);
}

template <int P>
static cudaError_t set_crt_attr() {
  return cudaFuncSetAttribute(k_crt_warp<P>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              200 * 1024);
}

cudaError_t init_kernel_attributes() {
  cudaError_t e;
  const int big = (int)(sizeof(uint32_t) * ((1 << kMaxLgN) + ((1 << kMaxLgN) >> 5)));
  if ((e = cudaFuncSetAttribute(k_split_fwd, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)(sizeof(uint32_t) << kMaxLgN))) != cudaSuccess)
    return e;
  if ((e = cudaFuncSetAttribute(k_inv_ntt, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)(sizeof(uint32_t) << kMaxLgN))) != cudaSuccess)
    return e;
  if ((e = cudaFuncSetAttribute(k_inv2<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, big)) !=
      cudaSuccess)
    return e;
  if ((e = cudaFuncSetAttribute(k_inv2<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, big)) !=
      cudaSuccess)
    return e;
  if ((e = set_fwd_attrs<1>()) != cudaSuccess || (e = set_fwd_attrs<2>()) != cudaSuccess ||
      (e = set_fwd_attrs<3>()) != cudaSuccess || (e = set_fwd_attrs<4>()) != cudaSuccess ||
      (e = set_fwd_attrs<5>()) != cudaSuccess || (e = set_fwd_attrs<6>()) != cudaSuccess ||
      (e = set_fwd_attrs<7>()) != cudaSuccess)
    return e;
  if ((e = set_crt_attr<2>()) != cudaSuccess || (e = set_crt_attr<3>()) != cudaSuccess ||
      (e = set_crt_attr<4>()) != cudaSuccess || (e = set_crt_attr<5>()) != cudaSuccess ||
      (e = set_crt_attr<6>()) != cudaSuccess || (e = set_crt_attr<7>()) != cudaSuccess ||
      (e = set_crt_attr<8>()) != cudaSuccess || (e = set_crt_attr<9>()) != cudaSuccess ||
      (e = set_crt_attr<10>()) != cudaSuccess || (e = set_crt_attr<11>()) != cudaSuccess ||
      (e = set_crt_attr<12>()) != cudaSuccess || (e = set_crt_attr<13>()) != cudaSuccess ||
      (e = set_crt_attr<14>()) != cudaSuccess || (e = set_crt_attr<15>()) != cudaSuccess ||
      (e = set_crt_attr<16>()) != cudaSuccess)
    return e;
  if ((e = cudaFuncSetAttribute(k_crt_mixed<2, kCrtMixedSplit>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024)) !=
          cudaSuccess ||
      (e = cudaFuncSetAttribute(k_crt_mixed<kCrtMixedSplit + 1, kMaxPrimes>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024)) !=
          cudaSuccess)
    return e;
  return cudaFuncSetAttribute(k_contract_tc, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              (int)((128 + 8 * tc::kMaxN) * 4 * tc::kMaxK));
}

}  // namespace mpzmm
