// Tensor-core contraction (tcgen05.mma kind::i8, sm_100a), exact.
//
// Per frequency h and prime p: C = A B mod p with A (m x k), B (k x n)
// residues below 2^32.  Each residue is its four unsigned bytes,
// x = sum_s 2^(8s) x_s, so
//     sum_kk A[i,kk] B[kk,l] = sum_{s,t} 2^(8(s+t)) D_st[i,l],
//     D_st[i,l] = sum_kk a_s[i,kk] b_t[kk,l]      (0 <= D < k 2^16, exact in int32),
// sixteen byte-plane products that one u8 x u8 GEMM computes at once:
//   A' rows 4 i + s    (the four byte planes of A interleaved along M, in
//                       tiles of 128 rows = 32 rows i), bytes kk;
//   B' rows 4 l + t    (the planes of B interleaved along N), bytes kk;
//   D = A' B'^T        (M = 4 m in tiles of 128 TMEM lanes, N = 4 n).
// Half the MACs of a Toeplitz-expanded split and no expansion of either
// operand: the split is four byte permutes per four residues.  The four
// planes of row i sit in four adjacent TMEM lanes, so one warp holds them:
// the epilogue weights a lane's sixteen values by 2^(8(s+t)) mod p in 64
// bits, adds the four lanes' sums with three shuffles (z < 2^57 for
// k <= 64) and Montgomery-reduces z, so C carries the same 2^-32 factor as
// the CUDA-core contraction.  Small products pack two or four frequencies
// into one MMA (Shape).
//
// One CTA of 128, 256 or 512 threads (four, two or one an SM, as TMEM and
// shared memory allow) per (product, prime, block of 128 frequencies, block
// of at most 32 rows and 32 columns of C: its rows of A and columns of B),
// processed F frequencies at a time: all warps stage A' and B' of the F
// frequencies straight from global memory (F consecutive residues of a
// polynomial per vector load) into canonical K-major no-swizzle tiles (8-row
// x 16-byte core matrices; every st.shared of a warp hits 32 distinct
// banks); one thread issues the MMAs of a unit (several groups of a
// product with at most 32 output columns, else one frequency's 32 columns),
// tcgen05.commit arrives on the unit's mbarrier, which one warp waits for
// before a block barrier releases the rest; with two TMEM buffers the
// next unit's MMAs run while the warps drain the current one (warp w reads
// TMEM lanes 32 (w mod 4) .. + 31; warps whose lanes hold no row skip the
// unit).  Results of the F
// frequencies are gathered in shared memory and stored F residues per vector
// store.  Every wait is bounded (one second of wall time): on time-out the
// CTA records an error, waits (bounded) for MMAs it has issued, frees its
// TMEM and returns.
#pragma once

#include <cstdint>

namespace mpzmm {
namespace tc {

constexpr int kMaxK = 64;        // k <= 64: K' = k bytes padded to 32, z < 2^57
constexpr int kBlock = kTcBlock;  // rows i and columns l of C a work item covers
constexpr int kMaxN = 1024;      // n, m <= 1024: block indices fit the item's 8-bit fields
constexpr int kMaxM = 1024;
constexpr int kFreqs = 128;      // frequencies per CTA (each polynomial's 512 bytes)
constexpr int kUnitCols = 32;    // output columns l per unit
constexpr uint32_t kSpinLimit = 1u << 26;
constexpr uint64_t kWaitLimitNs = 1000000000ull;  // one second of wall time
constexpr int kSmemLimit = 227 * 1024;  // shared memory of a block, static included
constexpr int kStaticSmem = 1024;       // the kernel's barriers and TMEM slot (aligned)
constexpr int kDynSmemLimit = kSmemLimit - kStaticSmem;

// Shape of one product on the tensor cores (host and device) when F
// frequencies are staged at once.  Products with at most 16 rows and 32
// columns pack phi frequencies into one 128-row M tile (a group): slot fl
// holds rows 4 mp fl + 4 i + s of A' and bytes fl kq .. fl kq + kq of K'
// in both A' and B', and A' is zero outside its slot, so the one MMA gives
// each frequency's sixteen plane products in its own rows; the groups of a
// block then fill all four TMEM lane quadrants instead of the first one or
// two.
struct Shape {
  int phi;     // frequencies a group: 4 (m <= 8), 2 (m <= 16), else 1; at most F
  int mp;      // rows i a packed slot spans: 8 or 16 (32 when phi = 1)
  int mt;      // 128-lane M tiles of a group: 1 when packed, else ceil(m / 32)
  int kq;      // K' bytes of a slot: k rounded up to 8 when packed, to 32 when not
  int kp;      // K' bytes of a group: phi kq rounded up to 32
  int npl;     // output columns per unit: min(n, 32)
  int nunits;  // units per frequency: ceil(n / npl) (1 when packed)
  int ncol;    // MMA N of a unit: 4 npl rounded up to 16
  int a_bytes, b_bytes;  // A' and B' tiles of one group
};

__host__ __device__ inline Shape shape_of(int m, int k, int n, int F) {
  Shape s;
  s.phi = n > kUnitCols ? 1 : (m <= 8 ? 4 : (m <= 16 ? 2 : 1));
  if (s.phi > F) s.phi = F;
  s.mp = s.phi > 1 ? (m <= 8 ? 8 : 16) : 32;
  s.mt = s.phi > 1 ? 1 : (m + 31) / 32;
  s.kq = s.phi > 1 ? (k + 7) & ~7 : (k + 31) & ~31;
  s.kp = (s.phi * s.kq + 31) & ~31;
  s.npl = n < kUnitCols ? n : kUnitCols;
  s.nunits = (n + s.npl - 1) / s.npl;
  s.ncol = (4 * s.npl + 15) & ~15;
  s.a_bytes = 128 * s.mt * s.kp;  // multiple of 4096
  // B' rows: every unit's MMA reads ncol rows from row 4 npl u, and the
  // staging writes rows 4 l + t for l up to n rounded up to 8
  int brows = 4 * s.npl * (s.nunits - 1) + s.ncol;
  if (brows < 4 * ((n + 7) & ~7)) brows = 4 * ((n + 7) & ~7);
  s.b_bytes = ((brows * s.kp) + 1023) & ~1023;
  return s;
}

// TMEM columns of one group's accumulator (one column range).
__host__ __device__ inline int unit_cols(const Shape& s) { return s.mt * s.ncol; }

// A launch keeps two accumulator buffers of `bufcols` TMEM columns (a power
// of two at least as wide as its widest product's accumulator) when both fit
// the 512 columns of an SM, one otherwise.
__host__ __device__ inline bool double_buffered(int bufcols) { return 2 * bufcols <= 512; }

// Groups per unit when F frequencies are staged: products with one column
// range (n <= 32) put that many groups' accumulators side by side in a
// buffer, so one commit and one epilogue pass serve them all.
__host__ __device__ inline int group_freqs(const Shape& s, int F, int bufcols) {
  if (s.nunits != 1) return 1;
  const int groups = F / s.phi;
  int g = bufcols / unit_cols(s);
  return g < 1 ? 1 : (g > groups ? groups : g);
}

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

// kind::i8 instruction descriptor: D s32, A u8, B u8, both K-major, M = 128.
__host__ __device__ constexpr uint32_t idesc_u8(uint32_t n) {
  return (2u << 4) | ((n >> 3) << 17) | ((128u >> 4) << 24);
}

// byte offset of (row, kbyte) in a K-major canonical tile with K' bytes/row
__device__ __forceinline__ uint32_t tile_off(uint32_t row, uint32_t kb, uint32_t kprime) {
  return (row >> 3) * (8u * kprime) + (kb >> 4) * 128u + (row & 7u) * 16u + (kb & 15u);
}

// byte planes of four residues: plane s = (x0_s, x1_s, x2_s, x3_s)
__device__ __forceinline__ void byte_planes(uint32_t x0, uint32_t x1, uint32_t x2, uint32_t x3,
                                            uint32_t (&pl)[4]) {
  const uint32_t lo01 = __byte_perm(x0, x1, 0x5140), hi01 = __byte_perm(x0, x1, 0x7362);
  const uint32_t lo23 = __byte_perm(x2, x3, 0x5140), hi23 = __byte_perm(x2, x3, 0x7362);
  pl[0] = __byte_perm(lo01, lo23, 0x5410);
  pl[1] = __byte_perm(lo01, lo23, 0x7632);
  pl[2] = __byte_perm(hi01, hi23, 0x5410);
  pl[3] = __byte_perm(hi01, hi23, 0x7632);
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
