// Internal types shared by the host engine and the sm_100a kernels.
//
// Residue arithmetic runs modulo word-size NTT primes p < 2^30 with
// p = 1 (mod 2^20), so that 4p < 2^32 (lazy 32-bit Montgomery/Shoup
// arithmetic) and p^2 < 2^60 (sixteen products accumulate exactly in 64 bits).
// The reference's 62-bit primes (src/include/fft62.h:24-31) would force
// multi-instruction 64-bit products on CUDA cores; the result is the same
// exact integer either way.
#pragma once

#include <cuda_runtime.h>

#include <cstddef>
#include <cstdint>

namespace mpzmm {

constexpr int kMaxPrimes = 16;      // primes available to a product
constexpr int kPrimeLgRoot = 20;    // every prime is 1 mod 2^20
constexpr int kMaxLgN = 20;         // largest transform (2^20 points: p = 1 mod 2^20)
constexpr int kMaxLgNOneCta = 15;   // largest transform done in one CTA
constexpr int kTwiddleLg = 15;      // twiddle tables cover N <= 2^15; every pass of
                                    // a longer (four-step) transform is shorter
constexpr int kLargeLgC = 12;       // block length of a four-step transform's second pass
constexpr int kTwistEntries = 1024; // entries of each twist table per prime
static_assert(kMaxLgN <= kPrimeLgRoot, "transform longer than the primes' 2-power roots");
static_assert(kMaxLgN - kLargeLgC <= kTwiddleLg, "four-step columns beyond the table");
static_assert(2 * 10 == kPrimeLgRoot, "twist exponents are split 10 + 10 bits");
constexpr int kMaxCoeffBits = 192;  // largest split coefficient (r)
constexpr int kMaxCrtWords = kMaxPrimes + 1;  // 32-bit words of a CRT value

// Per-prime constants, in __constant__ memory on the device.
struct PrimeConst {
  uint32_t p;        // the prime
  uint32_t pinv;     // -p^{-1} mod 2^32 (Montgomery)
  uint32_t r2;       // 2^64 mod p
  uint32_t mu;       // floor(2^32 / p) (Barrett for 32-bit words)
  uint32_t b32;      // 2^32 mod p
  uint32_t b32q;     // Shoup companion of b32
  uint32_t post;     // unused (the CRT scale 2^32 N^{-1} depends on N)
  uint32_t pad;
  uint32_t dig[8];   // 2^(30 q + 32) mod p: weights of the 30-bit digits of a
                     // coefficient, with the Montgomery factor folded in
  uint32_t w8[8];    // 2^(8 u) mod p: weights of the byte convolutions (tensor cores)
  uint64_t bias;     // a multiple of p >= 2^56 (makes signed sums non-negative)
};

// Explicit CRT constants (all exact integers).  For the first P primes with
// product M_P, a coefficient with residues x_j is
//     X = sum_j y_j (M_P / p_j) - q M_P,   y_j = x_j (M_P / p_j)^{-1} mod p_j,
// where q is sum_j y_j / p_j rounded to the nearest integer (computed in
// 2^-58 fixed point; the planner keeps |X| < M_P / 4, so the rounding has a
// margin of 1/4 against a fixed-point error below 2^-24).  The sums run in
// base 2^30: every y_j d product is below 2^60, so a column of up to 16 of
// them fits one 64-bit accumulator without carry handling.
struct CrtConst {
  uint32_t M[kMaxPrimes + 1][kMaxCrtWords];          // M_P, little-endian words
  int Mwords[kMaxPrimes + 1];
  uint32_t M30[kMaxPrimes + 1][kMaxPrimes];          // M_P, base-2^30 digits (P of them)
  uint32_t mop30[kMaxPrimes + 1][kMaxPrimes][kMaxPrimes];  // M_P / p_j, base-2^30 digits
  // Montgomery form (times 2^32) of 2^32 N^{-1} (M_P / p_j)^{-1} mod p_j for
  // N = 2^lgN: removes the contraction's 2^-32 and the inverse transform's N
  uint32_t cm[kMaxPrimes + 1][kMaxLgN + 1][kMaxPrimes];
  uint32_t fq[kMaxPrimes];                           // floor(2^58 / p_j)
};

// Twist tables of the four-step transforms, one direction: per prime,
// hi[u] = {W^(1024 u), its Shoup companion} and lo[v] = W^v 2^32 mod p for
// u, v < 1024, W a primitive 2^20-th root (inverse direction: W^-1).
struct TwistTab {
  const uint2* hi;
  const uint32_t* lo;
};

// One polynomial (one matrix entry) of the forward transform.
struct FwdDesc {
  uint64_t limb_off;   // first limb in the input limb buffer
  uint64_t res_off;    // first residue word (prime 0); prime j at + j*N
  int32_t size;        // signed limb count (GMP convention)
  uint32_t r;          // coefficient width in bits
  uint16_t lgN;
  uint16_t P;
  uint32_t ncoef;      // coefficients to split (<= N)
  // Operand of a tensor-core product: its residues are blocked by
  // kTcTile frequencies across the operand's tile_np entries (res_off is the
  // operand block, tile_e this entry), so one frequency block of every entry
  // is one contiguous run; tile_np == 0: the plain layout above.
  uint32_t tile_np = 0;
  uint32_t tile_e = 0;
};
constexpr int kTcTile = 8;      // frequencies a block of the tensor-core layout (32 bytes)
constexpr int kTcBlock = 32;    // rows and columns of C a tensor-core work item covers
constexpr int kTcTileLg = 3;

// One output polynomial of the inverse transform + CRT + recompose.
struct InvDesc {
  uint64_t res_off;
  uint64_t out_word;   // first 32-bit output word
  uint32_t out_words;  // output words (even: whole 64-bit limbs)
  uint32_t r;
  uint32_t ncoef;      // coefficients that can be nonzero
  uint16_t lgN;
  uint16_t P;
  uint32_t entry;      // output entry index (for the size array)
};

// One product of the contraction (per frequency: C = A B mod p).
struct ProdDesc {
  uint64_t a_res;      // residue offset of A's poly 0 (row-major m x k)
  uint64_t b_res;      // of B's poly 0 (k x n)
  uint64_t c_res;      // of C's poly 0 (m x n)
  uint16_t m, k, n;
  uint16_t lgN;
  uint16_t P;
  uint16_t pad;        // contraction register tile TI x TJ (2..4 each): 3 (TI - 2) + TJ - 2
};

// Work item of the contraction: one product, one prime, one frequency block.
struct ContractItem {
  uint32_t prod;
  uint16_t prime;
  uint16_t pad;        // tensor cores: block of C, (row block << 8) | column block
  uint32_t h0;         // first frequency of the block
};

// Work item of one CTA of the batched transform kernels: `count` entries of
// one size class (all 2^lgN points, P primes), descriptor indices
// idx[first .. first + count).
struct CtaItem {
  uint32_t first;
  uint16_t count;
  uint8_t lgN;
  uint8_t P;
};

}  // namespace mpzmm
