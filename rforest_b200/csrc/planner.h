// Host-side tables and parameter selection (integer arithmetic only).
#pragma once

#include <cstdint>
#include <vector>

#include <cuda_runtime.h>

#include "mpzmm_internal.h"

namespace mpzmm {

struct Moduli {
  uint32_t p[kMaxPrimes];
  PrimeConst pc[kMaxPrimes];
  CrtConst crt;
  int mbits[kMaxPrimes + 1];   // floor(log2(p_0 ... p_{P-1}))
  std::vector<uint2> twf;      // [kMaxPrimes][1 << kTwiddleLg] forward {w, wq}
  std::vector<uint2> twi;      // inverse
  // twist tables of the four-step transforms ([kMaxPrimes][kTwistEntries]
  // each; see TwistTab): forward (W) and inverse (W^-1)
  std::vector<uint2> twh_f, twh_i;
  std::vector<uint32_t> twl_f, twl_i;
};

// The first kMaxPrimes primes p < 2^30 with p = 1 mod 2^kPrimeLgRoot, in
// decreasing order, with all derived constants and twiddle tables.
const Moduli& moduli();

struct Params {
  int P = 0;      // primes (0: the product is identically zero)
  int r = 0;      // coefficient bits
  int lgN = 0;    // transform length 2^lgN
  int64_t lenA = 0, lenB = 0;  // coefficients of the longest A / B entry
  int64_t out_limbs = 0;       // 64-bit limbs of every output entry
};

int ceil_log2(uint64_t x);

// Picks (P, r, lgN) for an m x k by k x n product whose A / B entries have at
// most a_bits / b_bits bits.  Every output coefficient c satisfies
// 4 |c| < p_0...p_{P-1} (proved with the integer bound
// 2 + ceil(log2 k) + ceil(log2 min(lenA, lenB)) + 2r <= floor(log2 M)), so
// the symmetric CRT residue is c itself, with the margin the rounded
// explicit CRT needs.  Returns false if no supported (P, r, lgN) exists.
bool choose_params(int64_t a_bits, int64_t b_bits, int m, int k, int n, Params* out);
// Register tile of the CUDA-core contraction for an m x n product, encoded
// as 3 (TI - 2) + (TJ - 2) with 2 <= TI, TJ <= 4 (ProdDesc::pad).
int contract_tile(int m, int n);

// ceil((a_bits + b_bits + ceil(log2 k) + 1) / 64)
int64_t output_limbs(int k, int64_t a_bits, int64_t b_bits);

}  // namespace mpzmm
