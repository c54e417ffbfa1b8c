// Tensor-core contraction (tcgen05.mma kind::i8, sm_100a), exact.
//
// Per frequency h and prime p: C = A B mod p with A (m x k), B (k x n)
// residues in [0, p), p < 2^30.  Each residue is centred (v in (-p/2, p/2))
// and split into balanced signed bytes v = d0 + 2^8 d1 + 2^16 d2 + 2^24 d3
// (|d_s| <= 128, |d3| <= 33).  With
//     A'[i, 4kk + s]       = a_s[i, kk]
//     B'[8l + u, 4kk + s]  = b_{u-s}[kk, l]   (0 <= u - s <= 3, else 0)
// the int8 GEMM D = A' B'^T (K' = 4k) gives D[i, 8l + u] =
// sum_kk sum_s a_s b_{u-s}, the u-th digit convolution, so
//     sum_kk a b = sum_{u=0..6} 2^(8u) D[i, 8l + u]
// exactly; |D| <= 4k 2^14 fits the int32 accumulators for k < 2^15.  Column
// 8l + 7 is padding (zero), which keeps each output's 8 columns aligned for
// one tcgen05.ld.32x32b.x8.  The epilogue forms z = sum_u D_u (2^(8u) mod p)
// in 64 bits (|z| < 2^56 for k <= 64), adds a bias that is a multiple of p,
// and Montgomery-reduces, so the result carries the same 2^-32 factor as the
// CUDA-core contraction.
//
// One CTA of 128 threads per (product, prime, block of frequencies): the
// operands of one frequency are staged in shared memory in the canonical
// K-major no-swizzle layout (8-row x 16-byte core matrices), one elected
// thread issues the MMAs (M = 128 rows = TMEM lanes, N <= 256 per MMA,
// K = 32 bytes per MMA), tcgen05.commit arrives on an mbarrier, and warp w
// reads TMEM lanes 32w..32w+31.  Every wait is bounded (one second of wall
// time): on time-out the CTA records an error, stops issuing work, frees its
// TMEM and returns.
#pragma once

#include <cstdint>

namespace mpzmm {
namespace tc {

constexpr int kThreads = 128;
constexpr int kMaxK = 64;        // k <= 64  -> K' <= 256 bytes
constexpr int kMaxN = 64;        // n <= 64  -> 8n <= 512 TMEM columns
constexpr int kMaxM = 128;       // one M = 128 tile
constexpr int kTmemCols = 512;   // allocated per CTA (one CTA per SM by shared memory)
constexpr uint32_t kSpinLimit = 1u << 26;
constexpr uint64_t kWaitLimitNs = 1000000000ull;  // one second of wall time

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}

// K-major, no swizzle: core matrices of 8 rows x 16 bytes; LBO = 128 bytes
// (next 16 bytes of K), SBO = 8 K' bytes (next 8 rows).
__device__ __forceinline__ uint64_t smem_desc(uint32_t addr, uint32_t kprime) {
  uint64_t d = (uint64_t)((addr >> 4) & 0x3FFFu);
  d |= (uint64_t)(128u >> 4) << 16;
  d |= (uint64_t)(((8u * kprime) >> 4) & 0x3FFFu) << 32;
  d |= (uint64_t)1 << 46;  // descriptor version for sm_100
  return d;                // base offset 0, legacy LBO mode, layout type 0
}

// kind::i8 instruction descriptor: D s32, A s8, B s8, both K-major, M = 128.
__host__ __device__ constexpr uint32_t idesc_i8(uint32_t n) {
  return (2u << 4) | (1u << 7) | (1u << 10) | ((n >> 3) << 17) | ((128u >> 4) << 24);
}

// byte offset of (row, kbyte) in a K-major canonical tile with K' bytes/row
__device__ __forceinline__ uint32_t tile_off(uint32_t row, uint32_t kb, uint32_t kprime) {
  return (row >> 3) * (8u * kprime) + (kb >> 4) * 128u + (row & 7u) * 16u + (kb & 15u);
}

// balanced signed bytes of the centred residue, packed byte s = d_s
__device__ __forceinline__ uint32_t split_bytes(uint32_t x, uint32_t p) {
  int32_t v = (int32_t)x - (x > (p >> 1) ? (int32_t)p : 0);
  uint32_t packed = 0;
#pragma unroll
  for (int s = 0; s < 3; ++s) {
    const int32_t d = (int32_t)(int8_t)(v & 0xff);
    packed |= ((uint32_t)(uint8_t)d) << (8 * s);
    v = (v - d) >> 8;
  }
  packed |= ((uint32_t)(uint8_t)v) << 24;  // |d3| <= 33
  return packed;
}

__device__ __forceinline__ uint64_t global_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Waits for the phase with the given parity to complete; gives up (false)
// after kWaitLimitNs of wall time or kSpinLimit polls, whichever comes first.
__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t phase) {
  uint64_t t0 = 0;
  for (uint32_t it = 0; it < kSpinLimit; ++it) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred P1;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 P1, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, P1;\n\t}"
        : "=r"(done)
        : "r"(bar), "r"(phase)
        : "memory");
    if (done) return true;
    if ((it & 63u) == 0) {
      const uint64_t t = global_ns();
      if (it == 0)
        t0 = t;
      else if (t - t0 > kWaitLimitNs)
        return false;
    }
  }
  return false;
}

}  // namespace tc
}  // namespace mpzmm
