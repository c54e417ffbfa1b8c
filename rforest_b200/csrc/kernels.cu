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
#include <cstdlib>

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
  switch (d.pad) {  // tile shape 3 (TI - 2) + (TJ - 2), uniform over the CTA
    case 8: contract_tiles<4, 4>(d, it.prime, h, res); break;
    case 7: contract_tiles<4, 3>(d, it.prime, h, res); break;
    case 6: contract_tiles<4, 2>(d, it.prime, h, res); break;
    case 5: contract_tiles<3, 4>(d, it.prime, h, res); break;
    case 4: contract_tiles<3, 3>(d, it.prime, h, res); break;
    case 3: contract_tiles<3, 2>(d, it.prime, h, res); break;
    case 2: contract_tiles<2, 4>(d, it.prime, h, res); break;
    case 1: contract_tiles<2, 3>(d, it.prime, h, res); break;
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

// Where the forward transform leaves point h of prime j of an entry: the
// plain frequency-contiguous layout (base + j N + h), or, for an operand of a
// tensor-core product, blocked by kTcTile = 8 frequencies (a 32-byte sector)
// across the operand's np entries (base + ((j N / 8 + h / 8) np + e) 8 +
// h mod 8).
// TILED is a template flag so that plain launches carry none of the
// blocked layout's state.
template <bool TILED>
struct FwdOut {
  uint32_t* base;
  uint32_t np, e;
  int lgN;
  __device__ __forceinline__ uint32_t* at(int j, uint32_t h) const {
    if (!TILED) return base + ((uint64_t)j << lgN) + h;
    const uint64_t tile = ((uint64_t)j << (lgN - kTcTileLg)) + (h >> kTcTileLg);
    return base + (tile * np + e) * (uint64_t)kTcTile + (h & (kTcTile - 1u));
  }
};

// 2^L consecutive points h0 .. (h0 a multiple of 2^L) reduced from [0, 4p)
// to [0, p), vector stores (a run of up to 8 points never crosses a block)
template <int L, bool TILED>
__device__ __forceinline__ void store_points(const FwdOut<TILED>& fo, int j, uint32_t h0,
                                             uint32_t* a, uint32_t p) {
  static_assert(kTcTile == 8, "vector stores assume 8-frequency blocks");
  const uint32_t p2 = 2 * p;
#pragma unroll
  for (int q = 0; q < (1 << L); ++q) {
    const uint32_t v = reduce_2p(a[q], p2);
    a[q] = v >= p ? v - p : v;
  }
  if (L == 3) {
    *reinterpret_cast<uint4*>(fo.at(j, h0)) = make_uint4(a[0], a[1], a[2], a[3]);
    *reinterpret_cast<uint4*>(fo.at(j, h0 + 4)) = make_uint4(a[4], a[5], a[6], a[7]);
  } else if (L == 2) {
    *reinterpret_cast<uint4*>(fo.at(j, h0)) = make_uint4(a[0], a[1], a[2], a[3]);
  } else {
    *reinterpret_cast<uint2*>(fo.at(j, h0)) = make_uint2(a[0], a[1]);
  }
}

template <int LP, bool TILED>
__device__ __forceinline__ void fwd_last_pass(const uint32_t* s, const FwdOut<TILED>& fo, int j,
                                              bool valid, int lgN, int last_s0, int tt, int TS,
                                              const uint2* __restrict__ tw, uint32_t p) {
  for (int g = tt; g < ((1 << lgN) >> LP); g += TS) {
    uint32_t a[1 << LP];
#pragma unroll
    for (int q = 0; q < (1 << LP); ++q) a[q] = s[smi((g << LP) + q)];
    fwd_group<LP>(a, last_s0, g, tw, p);
    if (valid) store_points<LP, TILED>(fo, j, (uint32_t)(g << LP), a, p);
  }
}

// The body of k_fwd2.  HZ: every polynomial of the CTA has at most N/2
// coefficients (the usual case: both factors of a product fit in N
// together), so the first pass's upper four points are zero: their digits
// and residues are skipped and stage 0 only copies.  dig (whole-CTA HZ
// transforms, NULL otherwise): shared memory for the entry's digits, digit q
// of coefficient x at dig[q N/2 + x], extracted once for all P primes.
template <int D, bool TEAM, bool HZ, bool TILED>
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
  FwdOut<TILED> fo;
  fo.base = res + d.res_off;
  fo.np = d.tile_np;
  fo.e = d.tile_e;
  fo.lgN = lgN;
  for (int j = 0; j < P; ++j) {
    const uint32_t p = c_primes[j].p;
    const uint2* tw = twf + (size_t)j * kTwStride;
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
        if (valid) store_points<3, TILED>(fo, j, 0u, a, p);
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
      case 1: fwd_last_pass<1, TILED>(s, fo, j, valid, lgN, last_s0, tt, TS, tw, p); break;
      case 2: fwd_last_pass<2, TILED>(s, fo, j, valid, lgN, last_s0, tt, TS, tw, p); break;
      default: fwd_last_pass<3, TILED>(s, fo, j, valid, lgN, last_s0, tt, TS, tw, p); break;
    }
    __syncthreads();  // before the next prime's first pass overwrites s
  }
}

// dig_words: shared memory words after the transform reserved for the digit
// cache of a whole-CTA launch (0: none); it holds D N/2 words for the CTA's
// transform size.
template <int D, bool TEAM, bool TILED>
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
    fwd_body<D, TEAM, true, TILED>(d, s, dig, valid, lgN, P, tt, TS, limbs, res, twf);
  else
    fwd_body<D, TEAM, false, TILED>(d, s, nullptr, valid, lgN, P, tt, TS, limbs, res, twf);
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
// Transforms longer than one CTA holds (2^16 .. 2^20 points): four steps on
// the same tree.
//
// The forward tree's first lgR stages only combine points x = q C + lo with
// the same lo (C = 2^kLargeLgC, R = N / C), and their twiddles T[m + i] do
// not depend on N: for each of the C columns they are an ordinary R-point
// forward transform.  Afterwards block b = [b C, (b + 1) C) (b = the row
// position, already bit-reversed) holds a(X) mod (X^C - psi_b^C) with
// psi_b = w_N^brev(b), and the remaining stages on the block equal the
// twist y -> psi_b^y a_y followed by an ordinary C-point transform.  So:
//   k_fwd_cols           split + column transforms + twist, on tiles of
//                        R rows x W columns (R W = 2048 points: one group of
//                        eight a thread, its digits kept in registers for all
//                        P primes)
//   k_ntt_blocks<true>   C-point transforms of the blocks (vector loads)
// and the inverse the other way round:
//   k_ntt_blocks<false>  inverse C-point transforms, untwist by psi_b^-y
//   k_inv_cols           inverse column transforms, natural order out
// The result is the same canonical evaluation at the same position as the
// one-CTA transform, and the inverse again returns N times its input.
// Twist factors W^E, W a primitive 2^20-th root with W^32 the 2^15 table's
// root and E = brev(b) y 2^(20 - lgN), take one Shoup product of two table
// entries (TwistTab) and one Montgomery product.
// ---------------------------------------------------------------------------
constexpr int kColPoints = 2048;  // points of a column tile (R x W)
constexpr int kLgColPoints = 11;

// x W^E mod p in [0, p) for x < 4p, E < 2^20 (tables of one prime)
__device__ __forceinline__ uint32_t twist_mul(uint32_t x, uint32_t E,
                                              const uint2* __restrict__ hi,
                                              const uint32_t* __restrict__ lo, uint32_t p,
                                              uint32_t pinv) {
  const uint2 h = __ldg(hi + (E >> 10));
  const uint32_t f = mul_shoup(__ldg(lo + (E & 1023u)), h.x, h.y, p);  // W^E 2^32 mod p
  return redc((uint64_t)x * f, p, pinv);  // x f < 4 p^2 < p 2^32
}

// element (row q, column c) of a column tile with 2^lgW columns
__device__ __forceinline__ int cti(int q, int c, int lgW) { return smi((q << lgW) + c); }

// one pass of three stages (s0 .. s0 + 2) over every column of the tile
template <bool FWD>
__device__ __forceinline__ void col_pass3(uint32_t* s, int lgR, int lgW, int s0,
                                          const uint2* __restrict__ tw, uint32_t p) {
  const int lg_tmin = lgR - s0 - 3;
  const int groups = (1 << (lgR - 3)) << lgW;
  for (int gi = threadIdx.x; gi < groups; gi += blockDim.x) {
    const int c = gi & ((1 << lgW) - 1);
    const int g = gi >> lgW;
    const int lo = g & ((1 << lg_tmin) - 1);
    const int hi = g >> lg_tmin;
    const int base = (hi << (lg_tmin + 3)) + lo;
    uint32_t a[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) a[q] = s[cti(base + (q << lg_tmin), c, lgW)];
    if (FWD)
      fwd_group<3>(a, s0, hi, tw, p);
    else
      inv_group<3>(a, s0, hi, tw, p);
#pragma unroll
    for (int q = 0; q < 8; ++q) s[cti(base + (q << lg_tmin), c, lgW)] = a[q];
  }
}

// the last forward column pass (LP stages from last_s0, groups of 2^LP
// consecutive rows), twisted and stored to the polynomial `out`
template <int LP>
__device__ __forceinline__ void col_last_fwd(const uint32_t* s, uint32_t* __restrict__ out,
                                             int lgR, int lgW, int lgN, int lo0, int last_s0,
                                             const uint2* __restrict__ tw,
                                             const uint2* __restrict__ th,
                                             const uint32_t* __restrict__ tl, uint32_t p,
                                             uint32_t pinv) {
  const int groups = (1 << (lgR - LP)) << lgW;
  for (int gi = threadIdx.x; gi < groups; gi += blockDim.x) {
    const int c = gi & ((1 << lgW) - 1);
    const int hi = gi >> lgW;
    uint32_t a[1 << LP];
#pragma unroll
    for (int q = 0; q < (1 << LP); ++q) a[q] = s[cti((hi << LP) + q, c, lgW)];
    fwd_group<LP>(a, last_s0, hi, tw, p);
    const uint32_t y = (uint32_t)(lo0 + c);
#pragma unroll
    for (int q = 0; q < (1 << LP); ++q) {
      const uint32_t row = (uint32_t)((hi << LP) + q);
      const uint32_t E = ((__brev(row) >> (32 - lgR)) * y) << (20 - lgN);
      out[((uint64_t)row << kLargeLgC) + y] = twist_mul(a[q], E, th, tl, p, pinv);
    }
  }
}

// the last forward column pass inverted: groups of 2^LP consecutive rows
// from the polynomial `in`, into the tile
template <int LP>
__device__ __forceinline__ void col_last_inv(uint32_t* s, const uint32_t* __restrict__ in,
                                             int lgR, int lgW, int lo0, int last_s0,
                                             const uint2* __restrict__ tw, uint32_t p) {
  const int groups = (1 << (lgR - LP)) << lgW;
  for (int gi = threadIdx.x; gi < groups; gi += blockDim.x) {
    const int c = gi & ((1 << lgW) - 1);
    const int hi = gi >> lgW;
    uint32_t a[1 << LP];
#pragma unroll
    for (int q = 0; q < (1 << LP); ++q)
      a[q] = in[((uint64_t)((hi << LP) + q) << kLargeLgC) + (uint32_t)(lo0 + c)];
    inv_group<LP>(a, last_s0, hi, tw, p);
#pragma unroll
    for (int q = 0; q < (1 << LP); ++q) s[cti((hi << LP) + q, c, lgW)] = a[q];
  }
}

// Split + column transforms + twist.  grid = entries x tiles (2 R tiles of
// W = 2048 / R columns per entry); every entry of a launch has 2^lgN points.
template <int D>
__global__ void __launch_bounds__(kFwdThreads, 3)
k_fwd_cols(const FwdDesc* __restrict__ descs, const uint32_t* __restrict__ idx, int tiles,
           const uint64_t* __restrict__ limbs, uint32_t* __restrict__ res,
           const uint2* __restrict__ twf, TwistTab tt) {
  extern __shared__ uint32_t sm[];
  const int e = blockIdx.x / tiles;
  const int tile = blockIdx.x - e * tiles;
  const FwdDesc d = descs[idx[e]];
  const int lgN = d.lgN;
  const int lgR = lgN - kLargeLgC;
  const int lgW = kLgColPoints - lgR;
  const int lo0 = tile << lgW;
  const uint64_t N = (uint64_t)1 << lgN;
  const uint32_t nl = (uint32_t)(d.size < 0 ? -d.size : d.size);
  const uint32_t nw = nl < 0x40000000u ? 2u * nl : 0x80000000u;
  const uint32_t* __restrict__ w32 = reinterpret_cast<const uint32_t*>(limbs + d.limb_off);
  const bool neg = d.size < 0;
  // first-pass group of this thread: rows k R/8 + g of column c
  const int c = (int)threadIdx.x & ((1 << lgW) - 1);
  const int g = (int)threadIdx.x >> lgW;
  const int lgR8 = lgR - 3;
  // no coefficient in the upper half of the transform: rows k >= 4 of every
  // first-pass group are zero (uniform: one entry per CTA)
  const bool hz = d.ncoef <= (uint32_t)(N >> 1);
  uint32_t dg[8][D];
#pragma unroll
  for (int k = 0; k < 8; ++k) {
    const uint32_t x = ((uint32_t)((k << lgR8) + g) << kLargeLgC) + (uint32_t)(lo0 + c);
    coeff_digits<D>(w32, nw, x * d.r, d.r, x < d.ncoef && !(hz && k >= 4), dg[k]);
  }
  const int last_s0 = ((lgR - 1) / 3) * 3;
  for (int j = 0; j < (int)d.P; ++j) {
    const uint32_t p = c_primes[j].p;
    const uint2* tw = twf + (size_t)j * kTwStride;
    uint32_t a[8];
    if (hz) {
#pragma unroll
      for (int k = 0; k < 4; ++k) a[k] = digits_residue<D>(dg[k], j, neg);
      fwd_stage0_upper_zero<3>(a, p);
      fwd_group<3, 1>(a, 0, 0, tw, p);
    } else {
#pragma unroll
      for (int k = 0; k < 8; ++k) a[k] = digits_residue<D>(dg[k], j, neg);
      fwd_group<3>(a, 0, 0, tw, p);
    }
#pragma unroll
    for (int k = 0; k < 8; ++k) sm[cti((k << lgR8) + g, c, lgW)] = a[k];
    __syncthreads();
    for (int s0 = 3; s0 < last_s0; s0 += 3) {
      col_pass3<true>(sm, lgR, lgW, s0, tw, p);
      __syncthreads();
    }
    uint32_t* out = res + d.res_off + (uint64_t)j * N;
    const uint2* th = tt.hi + (size_t)j * kTwistEntries;
    const uint32_t* tl = tt.lo + (size_t)j * kTwistEntries;
    const uint32_t pinv = c_primes[j].pinv;
    switch (lgR - last_s0) {
      case 1: col_last_fwd<1>(sm, out, lgR, lgW, lgN, lo0, last_s0, tw, th, tl, p, pinv); break;
      case 2: col_last_fwd<2>(sm, out, lgR, lgW, lgN, lo0, last_s0, tw, th, tl, p, pinv); break;
      default: col_last_fwd<3>(sm, out, lgR, lgW, lgN, lo0, last_s0, tw, th, tl, p, pinv); break;
    }
    __syncthreads();  // before the next prime overwrites the tile
  }
}

// C-point transforms of the blocks.  grid = entries x R blocks.  Forward:
// ordinary forward transform of each (twisted) block.  Inverse: ordinary
// inverse transform, then the untwist psi_b^-y (tt holds the inverse twist
// tables).  Descriptors: fdescs (forward) or idescs (inverse).
template <bool FWD>
__global__ void __launch_bounds__(kFwdThreads)
k_ntt_blocks(const FwdDesc* __restrict__ fdescs, const InvDesc* __restrict__ idescs,
             const uint32_t* __restrict__ idx, int blocks, uint32_t* __restrict__ res,
             const uint2* __restrict__ tws, TwistTab tt) {
  extern __shared__ uint32_t sm[];
  const int e = blockIdx.x / blocks;
  const int b = blockIdx.x - e * blocks;
  uint64_t off;
  int lgN, P;
  if (FWD) {
    const FwdDesc& d = fdescs[idx[e]];
    off = d.res_off;
    lgN = d.lgN;
    P = d.P;
  } else {
    const InvDesc& d = idescs[idx[e]];
    off = d.res_off;
    lgN = d.lgN;
    P = d.P;
  }
  constexpr int lgC = kLargeLgC;
  constexpr int C = 1 << lgC;
  constexpr int last_s0 = ((lgC - 1) / 3) * 3;
  static_assert(lgC - last_s0 == 3, "the block length must end on a full pass");
  const int lgR = lgN - lgC;
  const uint64_t N = (uint64_t)1 << lgN;
  const int tid = threadIdx.x;
  const uint32_t bb = __brev((uint32_t)b) >> (32 - lgR);
  for (int j = 0; j < P; ++j) {
    const uint32_t p = c_primes[j].p;
    const uint2* tw = tws + (size_t)j * kTwStride;
    uint32_t* io = res + off + (uint64_t)j * N + ((uint64_t)b << lgC);
    if (FWD) {
      for (int v = tid; v < C / 4; v += kFwdThreads) {
        const uint4 u = reinterpret_cast<const uint4*>(io)[v];
        sm[smi(4 * v)] = u.x;
        sm[smi(4 * v + 1)] = u.y;
        sm[smi(4 * v + 2)] = u.z;
        sm[smi(4 * v + 3)] = u.w;
      }
      __syncthreads();
      for (int s0 = 0; s0 < last_s0; s0 += 3) {
        smem_pass<3, true>(sm, lgC, s0, 3, tid, kFwdThreads, tw, p);
        __syncthreads();
      }
      // a four-step block: plain layout, the block's points from b C on
      FwdOut<false> fo;
      fo.base = res + off + ((uint64_t)b << lgC);
      fo.np = 0;
      fo.e = 0;
      fo.lgN = lgN;
      fwd_last_pass<3>(sm, fo, j, true, lgC, last_s0, tid, kFwdThreads, tw, p);
      __syncthreads();
    } else {
      for (int g = tid; g < C / 8; g += kFwdThreads) {
        uint32_t a[8];
        load_points<3>(io + (g << 3), a);
        inv_last_pass<3>(sm, a, g, last_s0, tw, p);
      }
      __syncthreads();
      for (int s0 = last_s0 - 3; s0 >= 3; s0 -= 3) {
        smem_pass<3, false>(sm, lgC, s0, 3, tid, kFwdThreads, tw, p);
        __syncthreads();
      }
      const uint2* th = tt.hi + (size_t)j * kTwistEntries;
      const uint32_t* tl = tt.lo + (size_t)j * kTwistEntries;
      const uint32_t pinv = c_primes[j].pinv;
      for (int g = tid; g < C / 8; g += kFwdThreads) {
        uint32_t a[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) a[q] = sm[smi(q * (C / 8) + g)];
        inv_group<3>(a, 0, 0, tw, p);
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          const uint32_t y = (uint32_t)(q * (C / 8) + g);
          io[y] = twist_mul(a[q], (bb * y) << (20 - lgN), th, tl, p, pinv);
        }
      }
      __syncthreads();
    }
  }
}

// Inverse column transforms, natural coefficient order out (values in
// [0, 2p), as the CRT expects).  grid = entries x tiles, as k_fwd_cols.
__global__ void __launch_bounds__(kFwdThreads)
k_inv_cols(const InvDesc* __restrict__ descs, const uint32_t* __restrict__ idx, int tiles,
           uint32_t* __restrict__ res, const uint2* __restrict__ twi) {
  extern __shared__ uint32_t sm[];
  const int e = blockIdx.x / tiles;
  const int tile = blockIdx.x - e * tiles;
  const InvDesc d = descs[idx[e]];
  const int lgN = d.lgN;
  const int lgR = lgN - kLargeLgC;
  const int lgW = kLgColPoints - lgR;
  const int lo0 = tile << lgW;
  const uint64_t N = (uint64_t)1 << lgN;
  const int c = (int)threadIdx.x & ((1 << lgW) - 1);
  const int g = (int)threadIdx.x >> lgW;
  const int lgR8 = lgR - 3;
  const int last_s0 = ((lgR - 1) / 3) * 3;
  for (int j = 0; j < (int)d.P; ++j) {
    const uint32_t p = c_primes[j].p;
    const uint2* tw = twi + (size_t)j * kTwStride;
    uint32_t* io = res + d.res_off + (uint64_t)j * N;
    switch (lgR - last_s0) {
      case 1: col_last_inv<1>(sm, io, lgR, lgW, lo0, last_s0, tw, p); break;
      case 2: col_last_inv<2>(sm, io, lgR, lgW, lo0, last_s0, tw, p); break;
      default: col_last_inv<3>(sm, io, lgR, lgW, lo0, last_s0, tw, p); break;
    }
    __syncthreads();
    for (int s0 = last_s0 - 3; s0 >= 3; s0 -= 3) {
      col_pass3<false>(sm, lgR, lgW, s0, tw, p);
      __syncthreads();
    }
    uint32_t a[8];
#pragma unroll
    for (int k = 0; k < 8; ++k) a[k] = sm[cti((k << lgR8) + g, c, lgW)];
    inv_group<3>(a, 0, 0, tw, p);
#pragma unroll
    for (int k = 0; k < 8; ++k)
      io[((uint64_t)((k << lgR8) + g) << kLargeLgC) + (uint32_t)(lo0 + c)] = a[k];
    __syncthreads();  // before the next prime overwrites the tile
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
// the warp's scratch sV, each coefficient pre-shifted to its place in the
// output words (P + 1 words of tile coefficient c at [c (P + 1)]), the
// words' sums, the carry ripple, the sign and the size.
template <int P>
__device__ __forceinline__ void crt_entry(const InvDesc& d, const uint32_t* __restrict__ res,
                                          uint32_t* __restrict__ out,
                                          int32_t* __restrict__ out_sizes, uint32_t* sV,
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
    // coefficient i = lo_i + c as X_i 2^(i r mod 32): P + 1 words, the top
    // one signed (it carries the sign's borrow), so output word w adds word
    // w - floor(i r / 32) of every coefficient that reaches it
    for (int c = lane; c < ncf; c += 32) {
      uint32_t X[P];
      crt_coeff<P>(res, d.res_off, d.lgN, lo_i + c, X);
      const uint32_t sh = (uint32_t)((lo_i + c) * r) & 31u;
      uint32_t* v = sV + c * (P + 1);
      uint32_t prev = 0;
#pragma unroll
      for (int q = 0; q < P; ++q) {
        v[q] = sh ? ((X[q] << sh) | (prev >> (32u - sh))) : X[q];
        prev = X[q];
      }
      const uint32_t fill = (uint32_t)((int32_t)X[P - 1] >> 31);
      v[P] = sh ? ((fill << sh) | (prev >> (32u - sh))) : fill;
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
        // 0 <= w - floor(i r / 32) <= P for every i in [ia, ib]
        for (int i = ia; i <= ib; ++i) {
          const int q = w - ((i * r) >> 5);
          const uint32_t x = sV[(i - lo_i) * (P + 1) + q];
          sw += q == P ? (int64_t)(int32_t)x : (int64_t)x;
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
  crt_entry<P>(d, res, out, out_sizes, sm + warp * (cmax * (P + 1)), cmax, threadIdx.x & 31);
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
// Tensor-core contraction (byte-plane scheme: contract_tc.cuh).
// ---------------------------------------------------------------------------
__device__ __forceinline__ void tc_mma(uint32_t d, uint64_t ad, uint64_t bd, uint32_t idesc,
                                       uint32_t acc) {
  asm volatile(
      "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n"
      :: "r"(d), "l"(ad), "l"(bd), "r"(idesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
      : "memory");
}

__device__ __forceinline__ void tc_commit(uint32_t barp) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];"
               :: "r"(barp) : "memory");
}

// The MMAs of group gu / nunits of the staged block, output columns
// npl (gu mod nunits) .., into the accumulator at TMEM column dcol: one M
// tile of 128 A' rows at a time, K' in steps of 32 bytes.
__device__ __forceinline__ void tc_issue_unit(const tc::Shape& sh, uint32_t a_base,
                                              uint32_t b_base, int gu, uint32_t dcol) {
  const int g = gu / sh.nunits;
  const int uu = gu - g * sh.nunits;
  const uint32_t kp = (uint32_t)sh.kp;
  const uint32_t a0 = a_base + (uint32_t)(g * sh.a_bytes);
  // B' row 4 npl uu (a multiple of 8: npl = 32 when there are several units)
  const uint32_t b0 = b_base + (uint32_t)(g * sh.b_bytes) + (uint32_t)(4 * sh.npl * uu) * kp;
  const uint32_t idesc = tc::idesc_u8((uint32_t)sh.ncol);
  for (int q = 0; q < sh.mt; ++q)
    for (uint32_t ks = 0; ks < kp / 32; ++ks)
      tc_mma(dcol + (uint32_t)(q * sh.ncol),
             tc::smem_desc(a0 + 128u * (uint32_t)q * kp + 256u * ks, kp),
             tc::smem_desc(b0 + 256u * ks, kp), idesc, ks > 0 ? 1u : 0u);
}

__device__ __forceinline__ void tmem_ld16(uint32_t addr, uint32_t (&v)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 "
      "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]),
        "=r"(v[7]), "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]),
        "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
      : "r"(addr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}

// F consecutive residues (frequencies hs .. hs + F - 1) of entry e of an
// operand stored in the blocked layout (FwdOut): blk is the operand block, np
// its entries, tile the block of frequency hs (prime j included: j N/8 +
// hs/8) and sub = hs mod 8.  Only nf of them exist when the transform is
// shorter than the CTA's frequencies.  Lanes take consecutive entries, so a
// warp's loads are one contiguous run per block.
template <int F>
__device__ __forceinline__ void load_freqs(const uint32_t* __restrict__ blk, uint64_t np,
                                           uint64_t e, uint64_t tile, uint32_t sub, bool ok,
                                           int nf, uint32_t (&x)[F]) {
  if (ok && nf == F && F >= 4) {  // sub is a multiple of 4: 16-byte pieces of blocks
#pragma unroll
    for (int c = 0; c < F / 4; ++c) {
      const uint32_t h = sub + 4u * (uint32_t)c;
      const uint4 u = __ldg(reinterpret_cast<const uint4*>(
          blk + ((tile + (h >> kTcTileLg)) * np + e) * kTcTile + (h & (kTcTile - 1u))));
      x[4 * c] = u.x;
      x[4 * c + 1] = u.y;
      x[4 * c + 2] = u.z;
      x[4 * c + 3] = u.w;
    }
  } else {
#pragma unroll
    for (int f = 0; f < F; ++f) {
      const uint32_t h = sub + (uint32_t)f;
      x[f] = (ok && f < nf) ? __ldg(blk + ((tile + (h >> kTcTileLg)) * np + e) * kTcTile +
                                    (h & (kTcTile - 1u)))
                            : 0u;
    }
  }
}

// NT threads: 128 where four CTAs share an SM (one warp a TMEM lane
// quadrant), 256 where two do, 512 where one CTA has it to itself.
template <int F, int NT>
__global__ void __launch_bounds__(NT, 512 / NT)
k_contract_tc(const ProdDesc* __restrict__ prods, const ContractItem* __restrict__ items,
              uint32_t* __restrict__ res, int bufcols, int* __restrict__ status, int stall) {
  extern __shared__ __align__(1024) uint8_t tsm[];
  __shared__ __align__(8) uint64_t bars[2];
  __shared__ uint32_t tmem_slot;
  const int tid = threadIdx.x;
  const int warp = tid >> 5;
  const int lane = tid & 31;
  const ContractItem it = items[blockIdx.x];
  const ProdDesc d = prods[it.prod];
  // the item's block of C: rows i_base .. + m, columns l_base .. + n (at
  // most kBlock each); m, n below are the block's, d.m, d.n the product's
  const int i_base = (int)(it.pad >> 8) * tc::kBlock, l_base = (int)(it.pad & 0xffu) * tc::kBlock;
  const int m = d.m - i_base < tc::kBlock ? d.m - i_base : tc::kBlock;
  const int n = d.n - l_base < tc::kBlock ? d.n - l_base : tc::kBlock;
  const int k = d.k;
  const int N = 1 << d.lgN;
  const int j = it.prime;
  const uint32_t p = c_primes[j].p;
  const uint32_t pinv = c_primes[j].pinv;
  const uint32_t mu = c_primes[j].mu;
  const uint64_t stride = (uint64_t)d.P * (uint64_t)N;
  const tc::Shape sh = tc::shape_of(m, k, n, F);
  const int phi = sh.phi;
  const int G = F / phi;  // groups of a staged block
  const bool dbl = tc::double_buffered(bufcols);
  const int tmem_cols = dbl ? 2 * bufcols : bufcols;
  const uint32_t ucols = (uint32_t)tc::unit_cols(sh);
  // groups per unit: products with one column range put several groups'
  // accumulators side by side in a TMEM buffer
  const int gf = tc::group_freqs(sh, F, bufcols);
  uint8_t* As = tsm;
  uint8_t* Bs = As + G * sh.a_bytes;
  // results of the staged frequencies, F + 1 words an output entry (odd
  // stride: the epilogue's scattered stores spread over the banks)
  uint32_t* outs = reinterpret_cast<uint32_t*>(Bs + G * sh.b_bytes);
  // this lane's byte plane s of A (rows 4 i + s) and its four weights
  // 2^(8(s+t)) mod p, t = 0..3
  uint32_t wt[4];
#pragma unroll
  for (int t = 0; t < 4; ++t) wt[t] = (uint32_t)c_primes[j].w8[(lane & 3) + t];
  const uint32_t a_base = tc::smem_u32(As), b_base = tc::smem_u32(Bs);
  const uint32_t barp[2] = {tc::smem_u32(&bars[0]), tc::smem_u32(&bars[1])};

  // packed groups: A' is zero outside each slot's K' bytes; the staging
  // writes only inside the slots, so the zeros stay for the whole CTA
  if (phi > 1)
    for (int x = tid; x < G * sh.a_bytes / 16; x += NT)
      reinterpret_cast<uint4*>(As)[x] = make_uint4(0u, 0u, 0u, 0u);
  if (warp == 0) {
    const uint32_t slot = tc::smem_u32(&tmem_slot);
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                 :: "r"(slot), "r"((uint32_t)tmem_cols) : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(barp[0]) : "memory");
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" :: "r"(barp[1]) : "memory");
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = tmem_slot;
  // commits issued and not yet waited for, and the parity to wait for, per
  // accumulator (the same on every thread)
  uint32_t phase[2] = {0u, 0u};
  int pending[2] = {0, 0};
  bool failed = false;
  const int issue_mma = stall ? 0 : 1;  // stall (failure-path tests only): no MMA, no commit
  // this warp's TMEM lanes 32 qd + lane of every M tile: packed slot fl and
  // first row i (ib0 + 32 q; lane / 4 is added)
  const int qd = warp & 3;
  const int fl = phi > 1 ? (32 * qd) / (4 * sh.mp) : 0;
  const int ib0 = phi > 1 ? ((32 * qd) % (4 * sh.mp)) / 4 : 8 * qd;

  for (int fb0 = 0; fb0 < tc::kFreqs; fb0 += F) {
    const uint32_t hs = it.h0 + (uint32_t)fb0;
    if (hs >= (uint32_t)N) break;  // uniform over the CTA
    const int nf = (int)((uint32_t)N - hs < (uint32_t)F ? (uint32_t)N - hs : (uint32_t)F);
    const uint64_t base = (uint64_t)j * (uint64_t)N + hs;
    // the operands' blocked layout: frequency block of hs, offset inside it
    const uint64_t tile0 = ((uint64_t)j << (d.lgN - kTcTileLg)) + (hs >> kTcTileLg);
    const uint32_t sub0 = hs & (kTcTile - 1u);

    // ---- stage A' and B' of the nf frequencies: a warp task is 8 rows
    // (i of A, l of B) by 16 terms of a slot; a thread gathers four terms'
    // residues of one row for every frequency and writes their byte planes.
    // Small F keeps TU tasks' loads in flight at once.
    const int kbn = (sh.kq + 15) / 16;
    const int a_tasks = ((m + 7) / 8) * kbn;
    const int tasks = a_tasks + ((n + 7) / 8) * kbn;
    constexpr int TU = F <= 4 ? 2 : 1;
    constexpr int kWarps = NT / 32;
    for (int task0 = warp; task0 < tasks; task0 += TU * kWarps) {
      uint32_t x[TU][4][F];
      int rr[TU], kq[TU];
      bool isa[TU];
#pragma unroll
      for (int w2 = 0; w2 < TU; ++w2) {
        const int task = task0 + w2 * kWarps;
        const bool live = task < tasks;
        const bool isA = task < a_tasks;
        const int tt = isA ? task : task - a_tasks;
        const int rb = tt / kbn;
        const int kb = tt - rb * kbn;
        const int kk0 = 16 * kb + 4 * (lane & 3);
        // lane -> (row i of A or column l of B mod 8, term quad)
        const int r = 8 * rb + (lane >> 2);
        rr[w2] = r;
        kq[w2] = kk0;
        isa[w2] = isA;
#pragma unroll
        for (int c = 0; c < 4; ++c) {
          const int kk = kk0 + c;
          const bool ok = live && kk < k && r < (isA ? m : n);
          const uint64_t poly =
              ok ? (isA ? (uint64_t)((i_base + r) * k + kk) : (uint64_t)(kk * d.n + l_base + r))
                 : 0;
          load_freqs<F>(res + (isA ? d.a_res : d.b_res),
                        isA ? (uint64_t)d.m * k : (uint64_t)k * d.n, poly, tile0, sub0, ok, nf,
                        x[w2][c]);
        }
      }
#pragma unroll
      for (int w2 = 0; w2 < TU; ++w2) {
        if (task0 + w2 * kWarps >= tasks) break;  // uniform over the warp
        const int r = rr[w2], kk0 = kq[w2];
        if (kk0 >= sh.kq) continue;  // past the slot (a packed slot of 8 or 24 bytes)
#pragma unroll
        for (int f = 0; f < F; ++f) {
          if (f >= nf) break;
          // frequency f: group f / phi, slot f mod phi
          const int g = f / phi, sl = f - g * phi;
          uint32_t pl[4];
          tc::byte_planes(x[w2][0][f], x[w2][1][f], x[w2][2][f], x[w2][3][f], pl);
          // plane s of row i of A (column l of B): row 4 mp sl + 4 r + s of
          // A' (4 r + s of B'), bytes sl kq + kk; the store order rotates
          // with bits 3-4 of the lane so every store covers all 32 banks
          uint8_t* t = isa[w2] ? As + g * sh.a_bytes : Bs + g * sh.b_bytes;
          const uint32_t row0 = isa[w2] ? (uint32_t)(4 * sh.mp * sl + 4 * r) : (uint32_t)(4 * r);
          const uint32_t kb = (uint32_t)(sl * sh.kq + kk0);
          const int gq = (lane >> 3) & 3;
#pragma unroll
          for (int q = 0; q < 4; ++q) {
            const int tp = (q + gq) & 3;
            const uint32_t v = tp == 0 ? pl[0] : (tp == 1 ? pl[1] : (tp == 2 ? pl[2] : pl[3]));
            *reinterpret_cast<uint32_t*>(t + tc::tile_off(row0 + (uint32_t)tp, kb,
                                                          (uint32_t)sh.kp)) = v;
          }
        }
      }
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();

    // ---- units: MMAs, then the epilogue of each.  A unit is gf groups
    // (products with one column range) or one frequency's column range uu;
    // its accumulators are consecutive in TMEM ----
    const int ng = (nf + phi - 1) / phi;  // groups holding staged frequencies
    const int U = sh.nunits == 1 ? (ng + gf - 1) / gf : nf * sh.nunits;
    auto unit_groups = [&](int u, int* g0, int* ngu, int* uu) {
      if (sh.nunits == 1) {
        *g0 = u * gf;
        *ngu = (ng - *g0) < gf ? (ng - *g0) : gf;
        *uu = 0;
      } else {
        *g0 = u / sh.nunits;
        *ngu = 1;
        *uu = u - *g0 * sh.nunits;
      }
    };
    auto issue = [&](int u, uint32_t dcol) {
      int g0, ngu, uu;
      unit_groups(u, &g0, &ngu, &uu);
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      for (int gi = 0; gi < ngu; ++gi)
        tc_issue_unit(sh, a_base, b_base, (g0 + gi) * sh.nunits + uu,
                      dcol + (uint32_t)gi * ucols);
    };
    // both buffers are free at a block's start (every warp passed the last
    // block's barriers after draining them): units 0 and 1 go at once
    const bool two = dbl && U > 1;
    if (tid == 0 && issue_mma) {
      issue(0, tmem);
      tc_commit(barp[0]);
      if (two) {
        issue(1, tmem + (uint32_t)bufcols);
        tc_commit(barp[1]);
      }
    }
    pending[0] += issue_mma;
    if (two) pending[1] += issue_mma;
    for (int u = 0; u < U; ++u) {
      const int buf = dbl ? (u & 1) : 0;
      // one warp waits for the unit's MMAs; the barrier releases the others
      // and, with two buffers, tells that every warp has drained unit u - 1
      const bool ok = warp == 0 ? tc::mbar_wait(barp[buf], phase[buf]) : true;
      if (__syncthreads_or(!ok)) {  // every thread takes the same branch
        failed = true;
        break;
      }
      phase[buf] ^= 1u;
      pending[buf] -= 1;
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      if (dbl && u >= 1 && u + 1 < U) {  // into unit u - 1's buffer: overlaps this epilogue
        const int nb = (u + 1) & 1;
        if (tid == 0 && issue_mma) {
          issue(u + 1, tmem + (uint32_t)(nb * bufcols));
          tc_commit(barp[nb]);
        }
        pending[nb] += issue_mma;
      }
      int g0, ngu, uu;
      unit_groups(u, &g0, &ngu, &uu);
      const int l0 = uu * sh.npl;
      const int nl = (n - l0) < sh.npl ? (n - l0) : sh.npl;
      const int nch = (nl + 3) / 4;
      const uint32_t laddr = tmem + ((uint32_t)(32 * qd) << 16) + (uint32_t)(buf * bufcols);
      // the warps of quadrant qd share its (group, M tile, 16-column chunk)
      // items; rows i of the quadrant in tile q: ib0 + 32 q + lane / 4
      const int per_g = sh.mt * nch;
      for (int xi = warp >> 2; xi < ngu * per_g; xi += NT / 128) {
        const int gi = xi / per_g;
        const int rem = xi - gi * per_g;
        const int q = rem / nch;
        const int ch = rem - q * nch;
        const int f = (g0 + gi) * phi + fl;  // phi = 1 when nunits > 1
        const int ib = ib0 + 32 * q;
        if (fl >= phi || f >= nf || ib >= m) continue;  // warp-uniform: no row here
        uint32_t v[16];
        tmem_ld16(laddr + (uint32_t)(gi * (int)ucols + q * sh.ncol + 16 * ch), v);
        // columns 4 c + t of the chunk: output l0 + 4 ch + c, B plane t
        uint64_t part[4];
#pragma unroll
        for (int c = 0; c < 4; ++c) {
          uint64_t z = 0;
#pragma unroll
          for (int t = 0; t < 4; ++t) z += (uint64_t)v[4 * c + t] * wt[t];
          part[c] = z;
        }
        // add over the four lanes of row i (planes s), lane s ending with
        // output c = s: swap halves across lane bit 1, then across bit 0
        const bool h1 = (lane & 2) != 0, h0 = (lane & 1) != 0;
        uint64_t k0 = h1 ? part[2] : part[0], k1 = h1 ? part[3] : part[1];
        k0 += __shfl_xor_sync(0xffffffffu, h1 ? part[0] : part[2], 2);
        k1 += __shfl_xor_sync(0xffffffffu, h1 ? part[1] : part[3], 2);
        uint64_t z = h0 ? k1 : k0;
        z += __shfl_xor_sync(0xffffffffu, h0 ? k0 : k1, 1);
        const int i = ib + (lane >> 2);
        const int l = 4 * ch + (lane & 3);
        if (i < m && l < nl) outs[(i * n + l0 + l) * (F + 1) + f] = redc64(z, p, pinv, mu);
      }
      asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
      if (!dbl && u + 1 < U) {  // one buffer: the next MMAs wait for every warp
        __syncthreads();
        if (tid == 0 && issue_mma) {
          issue(u + 1, tmem);
          tc_commit(barp[0]);
        }
        pending[0] += issue_mma;
      }
    }
    if (failed) break;
    __syncthreads();  // every epilogue store of the block is in outs
    // ---- the nf frequencies of every output, F residues a vector store.
    // The next block's staging may start at once: this block's MMAs have
    // all completed, and its epilogue writes outs only after its own barrier.
    for (int e = tid; e < m * n; e += NT) {
      const int ei = e / n, el = e - ei * n;  // the block's row and column
      const uint64_t ge = (uint64_t)(i_base + ei) * (uint64_t)d.n + (uint64_t)(l_base + el);
      uint32_t* dst = res + d.c_res + ge * stride + base;
      const uint32_t* sv = outs + e * (F + 1);
      if (nf == F && F >= 4) {
#pragma unroll
        for (int c = 0; c < F / 4; ++c)
          reinterpret_cast<uint4*>(dst)[c] =
              make_uint4(sv[4 * c], sv[4 * c + 1], sv[4 * c + 2], sv[4 * c + 3]);
      } else {
        for (int f = 0; f < nf; ++f) dst[f] = sv[f];
      }
    }
  }
  if (failed) {
    if (tid == 0) atomicExch(status, 1);
    // MMAs already issued must finish before their TMEM is freed
    for (int b = 0; b < 2; ++b)
      while (pending[b] > 0) {
        if (!tc::mbar_wait(barp[b], phase[b])) break;
        phase[b] ^= 1u;
        pending[b] -= 1;
      }
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;"
                 :: "r"(tmem), "r"((uint32_t)tmem_cols) : "memory");
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

template <int D, bool TILED>
static cudaError_t launch_fwd2_d(const FwdDesc* descs, const uint32_t* idx,
                                 const CtaItem* items, int nitems, bool team, int max_lgN,
                                 const uint64_t* limbs, uint32_t* res, const uint2* twf,
                                 cudaStream_t st) {
  const int Nmax = 1 << max_lgN;
  if (team) {
    const size_t smem = sizeof(uint32_t) * (size_t)(8 * kFwdThreads + (8 * kFwdThreads >> 5));
    k_fwd2<D, true, TILED><<<nitems, kFwdThreads, smem, st>>>(descs, idx, items, limbs, res, twf, 0);
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
    k_fwd2<D, false, TILED><<<nitems, kFwdThreads, smem, st>>>(descs, idx, items, limbs, res, twf,
                                                        dig_words);
  }
  return cudaGetLastError();
}

int fwd_team_points() { return 8 * kFwdThreads; }

template <bool TILED>
static cudaError_t launch_fwd_items_t(const FwdDesc* descs, const uint32_t* idx,
                                      const CtaItem* items, int nitems, int D, bool team,
                                      int max_lgN, const uint64_t* limbs, uint32_t* res,
                                      const uint2* twf, cudaStream_t st) {
  switch (D) {
#define MPZMM_FWD_CASE(DD) \
  case DD:                 \
    return launch_fwd2_d<DD, TILED>(descs, idx, items, nitems, team, max_lgN, limbs, res, twf, st);
    MPZMM_FWD_CASE(1)
    MPZMM_FWD_CASE(2)
    MPZMM_FWD_CASE(3)
    MPZMM_FWD_CASE(4)
    MPZMM_FWD_CASE(5)
    MPZMM_FWD_CASE(6)
    MPZMM_FWD_CASE(7)
#undef MPZMM_FWD_CASE
    default:
      return cudaErrorInvalidValue;
  }
}

cudaError_t launch_fwd_items(const FwdDesc* descs, const uint32_t* idx, const CtaItem* items,
                             int nitems, int D, bool team, int max_lgN, const uint64_t* limbs,
                             uint32_t* res, const uint2* twf, cudaStream_t st, bool tiled) {
  if (nitems == 0) return cudaSuccess;
  return tiled ? launch_fwd_items_t<true>(descs, idx, items, nitems, D, team, max_lgN, limbs, res,
                                         twf, st)
               : launch_fwd_items_t<false>(descs, idx, items, nitems, D, team, max_lgN, limbs,
                                          res, twf, st);
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

// shared memory of the four-step kernels
static size_t col_tile_bytes() { return sizeof(uint32_t) * (size_t)(kColPoints + (kColPoints >> 5)); }
static size_t block_bytes() {
  return sizeof(uint32_t) * (size_t)((1 << kLargeLgC) + ((1 << kLargeLgC) >> 5));
}

template <int D>
static void launch_fwd_cols_d(int grid, cudaStream_t st, const FwdDesc* descs, const uint32_t* idx,
                              int tiles, const uint64_t* limbs, uint32_t* res, const uint2* twf,
                              const TwistTab& tt) {
  k_fwd_cols<D><<<grid, kFwdThreads, col_tile_bytes(), st>>>(descs, idx, tiles, limbs, res, twf,
                                                             tt);
}

int large_tiles(int lgN) { return 1 << (lgN - kLargeLgC + 1); }

cudaError_t launch_large_fwd(const FwdDesc* descs, const uint32_t* idx, int count, int lgN, int D,
                             const uint64_t* limbs, uint32_t* res, const uint2* twf,
                             const TwistTab& tt, cudaStream_t st) {
  if (count == 0) return cudaSuccess;
  if (lgN <= kMaxLgNOneCta || lgN > kMaxLgN) return cudaErrorInvalidValue;
  const int tiles = large_tiles(lgN);
  const int blocks = 1 << (lgN - kLargeLgC);
  const int grid = count * tiles;
  switch (D) {
    case 1: launch_fwd_cols_d<1>(grid, st, descs, idx, tiles, limbs, res, twf, tt); break;
    case 2: launch_fwd_cols_d<2>(grid, st, descs, idx, tiles, limbs, res, twf, tt); break;
    case 3: launch_fwd_cols_d<3>(grid, st, descs, idx, tiles, limbs, res, twf, tt); break;
    case 4: launch_fwd_cols_d<4>(grid, st, descs, idx, tiles, limbs, res, twf, tt); break;
    case 5: launch_fwd_cols_d<5>(grid, st, descs, idx, tiles, limbs, res, twf, tt); break;
    case 6: launch_fwd_cols_d<6>(grid, st, descs, idx, tiles, limbs, res, twf, tt); break;
    case 7: launch_fwd_cols_d<7>(grid, st, descs, idx, tiles, limbs, res, twf, tt); break;
    default: return cudaErrorInvalidValue;
  }
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  k_ntt_blocks<true><<<count * blocks, kFwdThreads, block_bytes(), st>>>(descs, nullptr, idx,
                                                                         blocks, res, twf, tt);
  return cudaGetLastError();
}

cudaError_t launch_large_inv(const InvDesc* descs, const uint32_t* idx, int count, int lgN,
                             uint32_t* res, const uint2* twi, const TwistTab& tt,
                             cudaStream_t st) {
  if (count == 0) return cudaSuccess;
  if (lgN <= kMaxLgNOneCta || lgN > kMaxLgN) return cudaErrorInvalidValue;
  const int tiles = large_tiles(lgN);
  const int blocks = 1 << (lgN - kLargeLgC);
  k_ntt_blocks<false><<<count * blocks, kFwdThreads, block_bytes(), st>>>(nullptr, descs, idx,
                                                                          blocks, res, twi, tt);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  k_inv_cols<<<count * tiles, kFwdThreads, col_tile_bytes(), st>>>(descs, idx, tiles, res, twi);
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

__device__ __forceinline__ bool fwd_in_bounds(const FwdDesc& f, const BoundsCaps& c) {
  if (f.lgN > kMaxLgN || f.P > kMaxPrimes) return false;
  const uint64_t nl = f.size < 0 ? (uint64_t)(-(int64_t)f.size) : (uint64_t)f.size;
  if (f.limb_off + nl > c.limbs) return false;
  if (f.tile_np && f.tile_e >= f.tile_np) return false;
  // the plain layout: P polynomials of N words; blocked: the operand's block
  const uint64_t words = ((uint64_t)f.P << f.lgN) * (f.tile_np ? f.tile_np : 1u);
  return f.res_off + words <= c.res;
}

__device__ __forceinline__ bool inv_in_bounds(const InvDesc& v, const BoundsCaps& c) {
  if (v.lgN > kMaxLgN || v.P > kMaxPrimes) return false;
  return v.res_off + ((uint64_t)v.P << v.lgN) <= c.res &&
         v.out_word + v.out_words <= c.out_words && v.entry < c.sizes;
}

__device__ __forceinline__ bool prod_in_bounds(const ProdDesc& d, const BoundsCaps& c) {
  if (d.lgN > kMaxLgN || d.P > kMaxPrimes) return false;
  const uint64_t poly = (uint64_t)d.P << d.lgN;
  return d.a_res + (uint64_t)d.m * d.k * poly <= c.res &&
         d.b_res + (uint64_t)d.k * d.n * poly <= c.res &&
         d.c_res + (uint64_t)d.m * d.n * poly <= c.res;
}

__global__ void k_check_bounds(const FwdDesc* __restrict__ fwd, int nfwd,
                               const InvDesc* __restrict__ inv, int ninv,
                               const ProdDesc* __restrict__ prods, int nprods, BoundsCaps caps,
                               int* __restrict__ status) {
  const int total = nfwd + ninv + nprods;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
    const bool ok = i < nfwd          ? fwd_in_bounds(fwd[i], caps)
                    : i < nfwd + ninv ? inv_in_bounds(inv[i - nfwd], caps)
                                      : prod_in_bounds(prods[i - nfwd - ninv], caps);
    if (!ok) atomicExch(status, 2);
  }
}

cudaError_t launch_check_bounds(const FwdDesc* fwd, int nfwd, const InvDesc* inv, int ninv,
                                const ProdDesc* prods, int nprods, BoundsCaps caps, int* status,
                                cudaStream_t st) {
  const int total = nfwd + ninv + nprods;
  if (total <= 0) return cudaSuccess;
  const int blocks = (total + 255) / 256 < 1184 ? (total + 255) / 256 : 1184;
  k_check_bounds<<<blocks, 256, 0, st>>>(fwd, nfwd, inv, ninv, prods, nprods, caps, status);
  return cudaGetLastError();
}

bool contract_tc_eligible(int m, int k, int n) {
  return m >= 1 && m <= tc::kMaxM && k >= 1 && k <= tc::kMaxK && n >= 1 && n <= tc::kMaxN;
}

// Dynamic shared memory of one product's CTA with F frequencies staged: the
// byte tiles of A' and B' and the results of the F frequencies.
int tc_smem_bytes(int m, int k, int n, int F) {
  const tc::Shape sh = tc::shape_of(m, k, n, F);
  return (F / sh.phi) * (sh.a_bytes + sh.b_bytes) + ((m * n * (F + 1) * 4 + 15) & ~15);
}

// Accumulator buffer width, frequencies staged at once (F), dynamic shared
// memory and threads of a launch over products of the given shapes.  The
// buffer is the widest accumulator rounded up to a power of two, at least
// the floor below; CTAs share an SM as far as TMEM allows (four of 128
// threads, two of 256, or one of 512), and F is the largest whose shared
// memory lets them, else the launch takes fewer CTAs an SM.
static bool tc_launch_config(const int* shapes, int nshapes, int* bufcols, int* F, int* smem,
                             int* threads) {
  int widest = 0;
  for (int i = 0; i < nshapes; ++i) {
    // the accumulator width does not depend on F
    const int c =
        tc::unit_cols(tc::shape_of(shapes[3 * i], shapes[3 * i + 1], shapes[3 * i + 2], 1));
    if (c > widest) widest = c;
  }
  // The narrowest buffer is 64 columns, so four double-buffered CTAs of
  // 128 threads share an SM and overlap one another's staging, MMA round
  // trips and barriers: 4096 products of 2..16 rows and columns forced onto
  // the tensor cores contracted in 74 ms that way, 107 ms with 128 columns
  // (two CTAs of 256 threads an SM).  MPZMM_TC_BUFCOLS (a power of two from
  // 32 to 256) replaces that floor for tuning.
  static const int b_floor = [] {
    const char* e = std::getenv("MPZMM_TC_BUFCOLS");
    const int v = e ? std::atoi(e) : 0;
    return (v >= 32 && v <= 256 && (v & (v - 1)) == 0) ? v : 64;
  }();
  int b = b_floor;
  while (b < widest) b <<= 1;
  *bufcols = b;
  const int tcols = tc::double_buffered(b) ? 2 * b : b;
  const int per_sm = 512 / tcols >= 4 ? 4 : (512 / tcols >= 2 ? 2 : 1);
  for (int target = per_sm; target >= 1; target >>= 1) {
    const int limit = target == 1 ? tc::kDynSmemLimit
                                  : (tc::kSmemLimit / target) - tc::kStaticSmem - 1024;
    for (int f = 16; f >= 1; f >>= 1) {
      int bytes = 0;
      for (int i = 0; i < nshapes; ++i) {
        const int sb = tc_smem_bytes(shapes[3 * i], shapes[3 * i + 1], shapes[3 * i + 2], f);
        if (sb > bytes) bytes = sb;
      }
      // below four staged frequencies a shared SM is not worth the loss
      if (bytes <= limit && (target == 1 || f >= 4)) {
        *F = f;
        *smem = bytes;
        *threads = 512 / target;  // as many threads an SM either way
        return true;
      }
    }
  }
  return false;
}

template <int F>
static void launch_tc_f(int count, int smem, int threads, cudaStream_t st,
                        const ProdDesc* prods, const ContractItem* items, uint32_t* res,
                        int bufcols, int* status, int stall) {
  if (threads == 512)
    k_contract_tc<F, 512><<<count, 512, smem, st>>>(prods, items, res, bufcols, status, stall);
  else if (threads == 256)
    k_contract_tc<F, 256><<<count, 256, smem, st>>>(prods, items, res, bufcols, status, stall);
  else
    k_contract_tc<F, 128><<<count, 128, smem, st>>>(prods, items, res, bufcols, status, stall);
}

cudaError_t launch_contract_tc(const ProdDesc* prods, const ContractItem* items, int count,
                               uint32_t* res, const int* shapes, int nshapes, int* status,
                               cudaStream_t st, int stall) {
  if (count == 0) return cudaSuccess;
  for (int i = 0; i < nshapes; ++i)
    if (!contract_tc_eligible(shapes[3 * i], shapes[3 * i + 1], shapes[3 * i + 2]))
      return cudaErrorInvalidValue;
  int F = 0, smem = 0, bufcols = 0, threads = 0;
  if (!tc_launch_config(shapes, nshapes, &bufcols, &F, &smem, &threads))
    return cudaErrorInvalidValue;
  switch (F) {
    case 16: launch_tc_f<16>(count, smem, threads, st, prods, items, res, bufcols, status, stall); break;
    case 8: launch_tc_f<8>(count, smem, threads, st, prods, items, res, bufcols, status, stall); break;
    case 4: launch_tc_f<4>(count, smem, threads, st, prods, items, res, bufcols, status, stall); break;
    case 2: launch_tc_f<2>(count, smem, threads, st, prods, items, res, bufcols, status, stall); break;
    default: launch_tc_f<1>(count, smem, threads, st, prods, items, res, bufcols, status, stall); break;
  }
  return cudaGetLastError();
}

int contract_tc_freqs() { return tc::kFreqs; }

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
    if (cs.cmax[P] * (P + 1) > cs.warp_words) cs.warp_words = cs.cmax[P] * (P + 1);
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
  const size_t per_warp = sizeof(uint32_t) * (size_t)(cmax * (P + 1));
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
  const int big =
      (int)(sizeof(uint32_t) * ((1 << kMaxLgNOneCta) + ((1 << kMaxLgNOneCta) >> 5)));
  cudaError_t e;
  for (auto fn : {k_fwd2<D, true, false>, k_fwd2<D, false, false>, k_fwd2<D, true, true>,
                  k_fwd2<D, false, true>})
    if ((e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, big)) !=
        cudaSuccess)
      return e;
  return cudaSuccess;
}

template <int P>
static cudaError_t set_crt_attr() {
  return cudaFuncSetAttribute(k_crt_warp<P>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                              200 * 1024);
}

cudaError_t init_kernel_attributes() {
  cudaError_t e;
  const int big =
      (int)(sizeof(uint32_t) * ((1 << kMaxLgNOneCta) + ((1 << kMaxLgNOneCta) >> 5)));
  if ((e = cudaFuncSetAttribute(k_split_fwd, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)(sizeof(uint32_t) << kMaxLgNOneCta))) != cudaSuccess)
    return e;
  if ((e = cudaFuncSetAttribute(k_inv_ntt, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)(sizeof(uint32_t) << kMaxLgNOneCta))) != cudaSuccess)
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
  for (auto fn : {k_contract_tc<16, 128>, k_contract_tc<8, 128>, k_contract_tc<4, 128>,
                  k_contract_tc<2, 128>, k_contract_tc<1, 128>, k_contract_tc<16, 256>,
                  k_contract_tc<8, 256>, k_contract_tc<4, 256>, k_contract_tc<2, 256>,
                  k_contract_tc<1, 256>, k_contract_tc<16, 512>, k_contract_tc<8, 512>,
                  k_contract_tc<4, 512>, k_contract_tc<2, 512>, k_contract_tc<1, 512>})
    if ((e = cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  tc::kDynSmemLimit)) != cudaSuccess)
      return e;
  return cudaSuccess;
}

}  // namespace mpzmm
