// Register-blocked NTT passes in shared memory (sm_100a, CUDA cores).
//
// A transform of N = 2^lgN points is done in passes of up to L = 3 stages.
// In a pass covering stages s0 .. s0+L-1 a "group" is the 2^L points
//     x = hi * 2 t_max + q * t_min + lo,   q = 0 .. 2^L - 1,
// with t_max = N >> (s0+1), t_min = N >> (s0+L), lo < t_min, hi < 2^s0; all
// butterflies of the pass stay inside a group, so one thread loads its group
// into registers, runs the L stages there and stores it back: one shared
// memory round trip and one barrier per pass instead of per stage.
//
// Forward stages are Cooley-Tukey (natural order in, bit-reversed order out)
// with twiddle T[m + i] = w_{2m}^{brev(i)}, m = 2^s, i = x / (2t); the
// inverse runs the same butterflies backwards (Gentleman-Sande) with T^{-1}.
// Values are lazy (Harvey, "Faster arithmetic for number-theoretic
// transforms", JSC 2014): in [0, 4p) between forward stages, [0, 2p)
// between inverse stages; p < 2^30 keeps 4p below 2^32.
#pragma once

#include <cstdint>

namespace mpzmm {

// shared-memory index with one pad word per 32 (spreads power-of-two strides
// over the banks)
__device__ __forceinline__ int smi(int x) { return x + (x >> 5); }

// x * w mod p in [0, 2p) for any 32-bit x (Shoup, no final correction)
__device__ __forceinline__ uint32_t mul_shoup_lazy(uint32_t x, uint32_t w, uint32_t wq,
                                                   uint32_t p) {
  const uint32_t q = __umulhi(x, wq);
  return x * w - q * p;
}

__device__ __forceinline__ uint32_t reduce_2p(uint32_t x, uint32_t p2) {
  const uint32_t y = x - p2;
  return y < x ? y : x;  // x >= 2p ? x - 2p : x (unsigned min)
}

// Forward: L stages starting at s0 on the 2^L registers a[] of one group.
// hi is the group's high index; twiddles from tw (the prime's table).
template <int L, int LSTART = 0>
__device__ __forceinline__ void fwd_group(uint32_t (&a)[1 << L], int s0, int hi,
                                          const uint2* __restrict__ tw, uint32_t p) {
  const uint32_t p2 = 2 * p;
#pragma unroll
  for (int l = LSTART; l < L; ++l) {
    const int span = 1 << (L - 1 - l);
    const int m = 1 << (s0 + l);
#pragma unroll
    for (int q = 0; q < (1 << L); ++q) {
      if (q & span) continue;
      const int i = (hi << l) + (q >> (L - l));
      const uint2 S = __ldg(tw + m + i);
      const uint32_t U = reduce_2p(a[q], p2);
      const uint32_t V = mul_shoup_lazy(a[q + span], S.x, S.y, p);
      a[q] = U + V;
      a[q + span] = U - V + p2;
    }
  }
}

// First forward stage of a group whose upper half (points a[2^(L-1) ..])
// is zero: every butterfly's product is 0, so it only copies -- the same
// values the general butterfly gives (U and U + 2p).
template <int L>
__device__ __forceinline__ void fwd_stage0_upper_zero(uint32_t (&a)[1 << L], uint32_t p) {
  const uint32_t p2 = 2 * p;
#pragma unroll
  for (int q = 0; q < (1 << (L - 1)); ++q) {
    const uint32_t U = reduce_2p(a[q], p2);
    a[q] = U;
    a[q + (1 << (L - 1))] = U + p2;
  }
}

// Inverse: the same L stages in reverse order (Gentleman-Sande).
template <int L>
__device__ __forceinline__ void inv_group(uint32_t (&a)[1 << L], int s0, int hi,
                                          const uint2* __restrict__ tw, uint32_t p) {
  const uint32_t p2 = 2 * p;
#pragma unroll
  for (int l = L - 1; l >= 0; --l) {
    const int span = 1 << (L - 1 - l);
    const int m = 1 << (s0 + l);
#pragma unroll
    for (int q = 0; q < (1 << L); ++q) {
      if (q & span) continue;
      const int i = (hi << l) + (q >> (L - l));
      const uint2 S = __ldg(tw + m + i);
      const uint32_t X = a[q];
      const uint32_t Y = a[q + span];
      a[q] = reduce_2p(X + Y, p2);
      a[q + span] = mul_shoup_lazy(X - Y + p2, S.x, S.y, p);
    }
  }
}

// One pass with Lp <= L stages over the team's transform in shared memory
// (team of nthr threads, transform base pointer s).  Forward direction.
template <int L, bool FWD>
__device__ __forceinline__ void smem_pass(uint32_t* s, int lgN, int s0, int Lp, int tid,
                                          int nthr, const uint2* __restrict__ tw,
                                          uint32_t p) {
  const int N = 1 << lgN;
  const int groups = N >> Lp;
  const int lg_tmin = lgN - s0 - Lp;
  const int tmin = 1 << lg_tmin;
  for (int g = tid; g < groups; g += nthr) {
    const int lo = g & (tmin - 1);
    const int hi = g >> lg_tmin;
    const int base = (hi << (lg_tmin + Lp)) + lo;
    if (Lp == L) {
      uint32_t a[1 << L];
#pragma unroll
      for (int q = 0; q < (1 << L); ++q) a[q] = s[smi(base + (q << lg_tmin))];
      if (FWD)
        fwd_group<L>(a, s0, hi, tw, p);
      else
        inv_group<L>(a, s0, hi, tw, p);
#pragma unroll
      for (int q = 0; q < (1 << L); ++q) s[smi(base + (q << lg_tmin))] = a[q];
    } else if (Lp == 2) {
      uint32_t a[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) a[q] = s[smi(base + (q << lg_tmin))];
      if (FWD)
        fwd_group<2>(a, s0, hi, tw, p);
      else
        inv_group<2>(a, s0, hi, tw, p);
#pragma unroll
      for (int q = 0; q < 4; ++q) s[smi(base + (q << lg_tmin))] = a[q];
    } else {
      uint32_t a[2];
#pragma unroll
      for (int q = 0; q < 2; ++q) a[q] = s[smi(base + (q << lg_tmin))];
      if (FWD)
        fwd_group<1>(a, s0, hi, tw, p);
      else
        inv_group<1>(a, s0, hi, tw, p);
#pragma unroll
      for (int q = 0; q < 2; ++q) s[smi(base + (q << lg_tmin))] = a[q];
    }
  }
}

}  // namespace mpzmm
