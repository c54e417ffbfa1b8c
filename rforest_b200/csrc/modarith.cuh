// 32-bit modular arithmetic for primes p < 2^30 (device side).
//
// Montgomery reduction (Montgomery, "Modular multiplication without trial
// division", Math. Comp. 1985) for variable x variable products and Shoup's
// precomputed-quotient multiplication (V. Shoup, NTL; see also Harvey,
// "Faster arithmetic for number-theoretic transforms", JSC 2014) for products
// with a fixed operand such as a twiddle factor.  Everything is exact integer
// arithmetic.
#pragma once

#include <cstdint>

namespace mpzmm {

__device__ __forceinline__ uint32_t add_mod(uint32_t a, uint32_t b, uint32_t p) {
  uint32_t s = a + b;  // a, b < p < 2^30: no overflow
  return s >= p ? s - p : s;
}

__device__ __forceinline__ uint32_t sub_mod(uint32_t a, uint32_t b, uint32_t p) {
  uint32_t s = a - b;
  return a < b ? s + p : s;
}

// x * w mod p for any x < 2^32, w < p, wq = floor(w 2^32 / p); result in [0, p).
__device__ __forceinline__ uint32_t mul_shoup(uint32_t x, uint32_t w, uint32_t wq,
                                              uint32_t p) {
  uint32_t q = __umulhi(x, wq);
  uint32_t r = x * w - q * p;  // in [0, 2p)
  return r >= p ? r - p : r;
}

// Montgomery reduction: T < p 2^32  ->  T 2^-32 mod p in [0, p).
__device__ __forceinline__ uint32_t redc(uint64_t T, uint32_t p, uint32_t pinv) {
  uint32_t m = (uint32_t)T * pinv;
  uint64_t t = (T + (uint64_t)m * p) >> 32;  // < 2p
  uint32_t r = (uint32_t)t;
  return r >= p ? r - p : r;
}

// x mod p for a 32-bit x, mu = floor(2^32 / p).
__device__ __forceinline__ uint32_t mod32(uint32_t x, uint32_t p, uint32_t mu) {
  uint32_t q = __umulhi(x, mu);
  uint32_t r = x - q * p;  // in [0, 2p)
  return r >= p ? r - p : r;
}

// Any 64-bit T  ->  T 2^-32 mod p (fold the high word below p, then REDC).
__device__ __forceinline__ uint32_t redc64(uint64_t T, uint32_t p, uint32_t pinv,
                                           uint32_t mu) {
  uint32_t hi = mod32((uint32_t)(T >> 32), p, mu);
  return redc(((uint64_t)hi << 32) | (uint32_t)T, p, pinv);
}

// Shoup companion floor(w 2^32 / p) computed on the device (w < p).
__device__ __forceinline__ uint32_t shoup_of(uint32_t w, uint32_t p) {
  return (uint32_t)(((uint64_t)w << 32) / p);
}

}  // namespace mpzmm
