// Prime tables, twiddle tables, Garner constants and parameter selection.
//
// The reference uses fixed 62-bit primes (src/include/fft62.h:24-31) and
// picks (r, lgN) with a double-precision loop (src/lib/mpnfft.c:18-78).  Here
// the primes are found at set-up (deterministic Miller-Rabin), and the
// parameter choice is integer-only with an explicit exactness bound.
#include "planner.h"

#include <array>
#include <cinttypes>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>

namespace mpzmm {

namespace {

uint64_t powmod(uint64_t a, uint64_t e, uint64_t p) {
  uint64_t r = 1 % p;
  a %= p;
  while (e) {
    if (e & 1) r = r * a % p;
    a = a * a % p;
    e >>= 1;
  }
  return r;
}

// Deterministic for n < 3,215,031,751 with bases 2, 3, 5, 7 (Pomerance,
// Selfridge and Wagstaff); all candidates here are below 2^30.
bool is_prime(uint32_t n) {
  if (n < 2) return false;
  for (uint32_t q : {2u, 3u, 5u, 7u, 11u, 13u}) {
    if (n % q == 0) return n == q;
  }
  uint32_t d = n - 1;
  int s = 0;
  while ((d & 1) == 0) {
    d >>= 1;
    ++s;
  }
  for (uint64_t a : {2ull, 3ull, 5ull, 7ull}) {
    uint64_t x = powmod(a, d, n);
    if (x == 1 || x == n - 1) continue;
    bool comp = true;
    for (int i = 1; i < s; ++i) {
      x = x * x % n;
      if (x == n - 1) {
        comp = false;
        break;
      }
    }
    if (comp) return false;
  }
  return true;
}

uint32_t primitive_root(uint32_t p) {
  // factor p - 1
  std::vector<uint32_t> f;
  uint32_t m = p - 1;
  for (uint32_t q = 2; q * q <= m; ++q) {
    if (m % q == 0) {
      f.push_back(q);
      while (m % q == 0) m /= q;
    }
  }
  if (m > 1) f.push_back(m);
  for (uint32_t g = 2;; ++g) {
    bool ok = true;
    for (uint32_t q : f) {
      if (powmod(g, (p - 1) / q, p) == 1) {
        ok = false;
        break;
      }
    }
    if (ok) return g;
  }
}

uint32_t shoup(uint32_t w, uint32_t p) { return (uint32_t)(((uint64_t)w << 32) / p); }

uint32_t brev(uint32_t x, int bits) {
  uint32_t r = 0;
  for (int i = 0; i < bits; ++i) r |= ((x >> i) & 1u) << (bits - 1 - i);
  return r;
}

// little-endian 32-bit word vectors
void mul_small(std::vector<uint32_t>& x, uint32_t v) {
  uint64_t cy = 0;
  for (auto& w : x) {
    uint64_t t = (uint64_t)w * v + cy;
    w = (uint32_t)t;
    cy = t >> 32;
  }
  if (cy) x.push_back((uint32_t)cy);
}

// base-2^32 little-endian words -> base-2^30 digits (no trailing zero digits)
std::vector<uint32_t> to_base30(const std::vector<uint32_t>& w32) {
  std::vector<uint32_t> out;
  unsigned __int128 buf = 0;
  int bits = 0;
  for (uint32_t w : w32) {
    buf |= (unsigned __int128)w << bits;
    bits += 32;
    while (bits >= 30) {
      out.push_back((uint32_t)(buf & 0x3fffffffu));
      buf >>= 30;
      bits -= 30;
    }
  }
  if (bits > 0) out.push_back((uint32_t)buf);
  while (!out.empty() && out.back() == 0) out.pop_back();
  return out;
}

Moduli* g_moduli = nullptr;
std::once_flag g_once;

void build(Moduli& M) {
  int cnt = 0;
  for (uint32_t c = (1u << (30 - kPrimeLgRoot)) - 1; c > 0 && cnt < kMaxPrimes; --c) {
    uint32_t p = (c << kPrimeLgRoot) + 1;
    if (p < (1u << 30) && is_prime(p)) M.p[cnt++] = p;
  }
  std::memset(M.pc, 0, sizeof(M.pc));
  std::memset(&M.crt, 0, sizeof(M.crt));
  const int TS = 1 << kTwiddleLg;
  M.twf.assign((size_t)kMaxPrimes * TS, make_uint2(0, 0));
  M.twi.assign((size_t)kMaxPrimes * TS, make_uint2(0, 0));
  M.twh_f.assign((size_t)kMaxPrimes * kTwistEntries, make_uint2(0, 0));
  M.twh_i.assign((size_t)kMaxPrimes * kTwistEntries, make_uint2(0, 0));
  M.twl_f.assign((size_t)kMaxPrimes * kTwistEntries, 0);
  M.twl_i.assign((size_t)kMaxPrimes * kTwistEntries, 0);
  for (int j = 0; j < kMaxPrimes; ++j) {
    const uint32_t p = M.p[j];
    PrimeConst& pc = M.pc[j];
    pc.p = p;
    uint32_t inv = p;  // Newton iteration for p^{-1} mod 2^32 (p odd)
    for (int i = 0; i < 5; ++i) inv *= 2 - p * inv;
    pc.pinv = (uint32_t)(0u - inv);
    pc.r2 = (uint32_t)(((unsigned __int128)1 << 64) % p);
    pc.mu = (uint32_t)((((uint64_t)1) << 32) / p);
    pc.b32 = (uint32_t)((((uint64_t)1) << 32) % p);
    pc.b32q = shoup(pc.b32, p);
    for (int q = 0; q < 8; ++q) pc.dig[q] = (uint32_t)powmod(2, (uint64_t)(30 * q + 32), p);
    for (int u = 0; u < 8; ++u) pc.w8[u] = (uint32_t)powmod(2, (uint64_t)(8 * u), p);
    pc.bias = ((((uint64_t)1 << 56) + p - 1) / p) * p;
    const uint32_t g = primitive_root(p);
    const uint64_t wmax = powmod(g, (p - 1) >> kTwiddleLg, p);  // order 2^kTwiddleLg
    {
      // twist tables: W = g^((p-1)/2^20), so W^(2^(20-kTwiddleLg)) = wmax
      const uint64_t W = powmod(g, (p - 1) >> kPrimeLgRoot, p);
      const uint64_t Wi = powmod(W, p - 2, p);
      const uint64_t r32 = (((uint64_t)1) << 32) % p;
      const size_t o = (size_t)j * kTwistEntries;
      uint64_t hf = 1, hi = 1, lf = 1, li = 1;
      const uint64_t Wk = powmod(W, kTwistEntries, p), Wik = powmod(Wi, kTwistEntries, p);
      for (int u = 0; u < kTwistEntries; ++u) {
        M.twh_f[o + u] = make_uint2((uint32_t)hf, shoup((uint32_t)hf, p));
        M.twh_i[o + u] = make_uint2((uint32_t)hi, shoup((uint32_t)hi, p));
        M.twl_f[o + u] = (uint32_t)(lf * r32 % p);
        M.twl_i[o + u] = (uint32_t)(li * r32 % p);
        hf = hf * Wk % p;
        hi = hi * Wik % p;
        lf = lf * W % p;
        li = li * Wi % p;
      }
    }
    for (int lgm = 0; lgm < kTwiddleLg; ++lgm) {
      const uint32_t m = 1u << lgm;
      // w_{2m} = wmax^(TS / (2m))
      const uint64_t w2m = powmod(wmax, (uint64_t)TS >> (lgm + 1), p);
      const uint64_t w2mi = powmod(w2m, p - 2, p);
      for (uint32_t i = 0; i < m; ++i) {
        const uint32_t e = brev(i, lgm);
        const uint32_t w = (uint32_t)powmod(w2m, e, p);
        const uint32_t wi = (uint32_t)powmod(w2mi, e, p);
        M.twf[(size_t)j * TS + m + i] = make_uint2(w, shoup(w, p));
        M.twi[(size_t)j * TS + m + i] = make_uint2(wi, shoup(wi, p));
      }
    }
  }
  std::vector<uint32_t> acc{1};
  for (int P = 1; P <= kMaxPrimes; ++P) {
    mul_small(acc, M.p[P - 1]);
    int words = (int)acc.size();
    M.crt.Mwords[P] = words;
    for (int q = 0; q < words && q < kMaxCrtWords; ++q) M.crt.M[P][q] = acc[q];
    const std::vector<uint32_t> m30 = to_base30(acc);
    for (int w = 0; w < kMaxPrimes; ++w) M.crt.M30[P][w] = w < (int)m30.size() ? m30[w] : 0u;
    int top = 31;
    while (!((acc.back() >> top) & 1u)) --top;
    M.mbits[P] = 32 * (words - 1) + top;  // floor(log2 M)
  }
  // explicit CRT: for P primes, M_P / p_j as P words, and the Montgomery form
  // of 2^32 N^{-1} (M_P / p_j)^{-1} mod p_j for every transform length
  for (int P = 1; P <= kMaxPrimes; ++P)
    for (int j = 0; j < P; ++j) {
      std::vector<uint32_t> mop{1};
      uint64_t mop_mod = 1;  // (M_P / p_j) mod p_j
      const uint32_t pj = M.p[j];
      for (int a = 0; a < P; ++a) {
        if (a == j) continue;
        mul_small(mop, M.p[a]);
        mop_mod = mop_mod * (M.p[a] % pj) % pj;
      }
      const std::vector<uint32_t> m30 = to_base30(mop);
      for (int w = 0; w < kMaxPrimes; ++w)
        M.crt.mop30[P][j][w] = w < (int)m30.size() ? m30[w] : 0u;
      const uint64_t inv = powmod(mop_mod, pj - 2, pj);
      const uint64_t r32 = (((uint64_t)1) << 32) % pj;
      for (int lg = 0; lg <= kMaxLgN; ++lg) {
        const uint64_t ninv = powmod((uint64_t)1 << lg, pj - 2, pj);
        // post = 2^32 N^{-1}; Montgomery form multiplies by 2^32 once more
        const uint64_t post = r32 * ninv % pj;
        M.crt.cm[P][lg][j] = (uint32_t)(post * inv % pj * r32 % pj);
      }
    }
  for (int j = 0; j < kMaxPrimes; ++j)
    M.crt.fq[j] = (uint32_t)((((uint64_t)1) << 58) / M.p[j]);
  M.mbits[0] = 0;
}

}  // namespace

const Moduli& moduli() {
  std::call_once(g_once, [] {
    g_moduli = new Moduli;
    build(*g_moduli);
  });
  return *g_moduli;
}

int ceil_log2(uint64_t x) {
  int b = 0;
  while (((uint64_t)1 << b) < x) ++b;
  return b;
}

int64_t output_limbs(int k, int64_t a_bits, int64_t b_bits) {
  if (k <= 0 || a_bits <= 0 || b_bits <= 0) return 1;
  return (a_bits + b_bits + ceil_log2((uint64_t)k) + 1 + 63) / 64;
}

// Register tile of the CUDA-core contraction, TI x TJ with 2 <= TI, TJ <= 4,
// as 3 (TI - 2) + (TJ - 2): the one with the fewest modelled instructions a
// frequency and term, tiles x (2 per multiply-add + 3 per load), so a
// 5 x 5 product takes 3 x 3 tiles (no row or column computed twice over)
// and a 16 x 16 one 4 x 4 (fewer loads a multiply-add).  On the default
// batch this models 8 % fewer instructions than tiles of 4 or 2 and
// measured 9.77 against 9.87 ms: the contraction waits on its loads more
// than it issues.
int contract_tile(int m, int n) {
  int best = 0, best_cost = -1;
  for (int ti = 2; ti <= 4; ++ti)
    for (int tj = 2; tj <= 4; ++tj) {
      const int tiles = ((m + ti - 1) / ti) * ((n + tj - 1) / tj);
      const int cost = tiles * (2 * ti * tj + 3 * (ti + tj));
      if (best_cost < 0 || cost < best_cost) {
        best_cost = cost;
        best = 3 * (ti - 2) + (tj - 2);
      }
    }
  return best;
}

bool choose_params(int64_t a_bits, int64_t b_bits, int m, int k, int n, Params* out) {
  *out = Params();
  if (a_bits <= 0 || b_bits <= 0 || k <= 0 || m <= 0 || n <= 0) {
    out->out_limbs = 1;
    return true;  // identically zero product: P = 0
  }
  const Moduli& M = moduli();
  const int clk = ceil_log2((uint64_t)k);
  // optional limits on the prime count (tuning experiments)
  static const int pmin_env = [] {
    const char* e = std::getenv("MPZMM_PMIN");
    return e ? std::atoi(e) : 2;
  }();
  static const int pmax_env = [] {
    const char* e = std::getenv("MPZMM_PMAX");
    return e ? std::atoi(e) : kMaxPrimes;
  }();
  // cost-model weights: per point and stage of a transform, per point of a
  // transform, per multiply-add of the contraction, per prime and per point
  // of the CRT (MPZMM_COST="a,b,c,d,e" replaces them for tuning experiments)
  static const std::array<int64_t, 5> wgt = [] {
    std::array<int64_t, 5> w{5, 12, 2, 3, 10};
    if (const char* e = std::getenv("MPZMM_COST")) {
      std::array<int64_t, 5> v{};
      if (std::sscanf(e, "%" SCNd64 ",%" SCNd64 ",%" SCNd64 ",%" SCNd64 ",%" SCNd64, &v[0], &v[1],
                      &v[2], &v[3], &v[4]) == 5)
        w = v;
    }
    return w;
  }();
  const int64_t nfwd = (int64_t)m * k + (int64_t)k * n;
  const int64_t ninv = (int64_t)m * n;
  int64_t best = -1;
  for (int P = 2; P <= kMaxPrimes; ++P) {
    if (P < pmin_env || P > pmax_env) continue;
    const int budget = M.mbits[P] - 2 - clk;  // 2r + ceil(log2 minlen) <= budget
    if (budget < 3) continue;
    int r = budget / 2;
    if (r > kMaxCoeffBits) r = kMaxCoeffBits;
    {
      // lengths only grow as r shrinks, so no r above this one is feasible
      const int64_t mn0 = ((a_bits < b_bits ? a_bits : b_bits) + r - 1) / r;
      const int r1 = (budget - ceil_log2((uint64_t)mn0)) / 2;
      if (r1 < r) r = r1;
    }
    int64_t lenA = 0, lenB = 0;
    for (; r >= 1; --r) {
      lenA = (a_bits + r - 1) / r;
      lenB = (b_bits + r - 1) / r;
      const int64_t mn = lenA < lenB ? lenA : lenB;
      if (2 * r + ceil_log2((uint64_t)mn) <= budget) break;
    }
    if (r < 1) continue;
    const int64_t len = lenA + lenB - 1;
    int lgN = ceil_log2((uint64_t)len);
    if (lgN < 2) lgN = 2;
    if (lgN > kMaxLgN) continue;
    // per (prime, frequency) work: transforms, contraction, CRT/recompose
    const int64_t Nn = (int64_t)1 << lgN;
    const int64_t cost = P * Nn *
                         ((nfwd + ninv) * (wgt[0] * lgN + wgt[1]) + wgt[2] * (int64_t)m * n * k +
                          ninv * (wgt[3] * P + wgt[4]));
    if (best < 0 || cost < best) {
      best = cost;
      out->P = P;
      out->r = r;
      out->lgN = lgN;
      out->lenA = lenA;
      out->lenB = lenB;
    }
  }
  if (best < 0) return false;
  out->out_limbs = output_limbs(k, a_bits, b_bits);
  return true;
}

}  // namespace mpzmm
