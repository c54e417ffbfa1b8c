// Batched modular reduction r = x mod d (mpzmm_mod_* in include/mpzmm_b200.h).
//
// The reference reduces by one modulus d many times with a precomputed
// Fermat-transform reciprocal (src/lib/mpnfft_mod.c:283-476, wrapped by
// src/lib/mpzfft.c:59-100: mpzfft_mod_init / mpzfft_mod_mod).  Here the same
// job is a Barrett reduction (Menezes, van Oorschot, Vanstone, Handbook of
// Applied Cryptography, 14.42, with base B = 2^64) whose two big products run
// on this library's multiplication engine, batched over all the x of a call
// and kept in device memory between the steps:
//   mu = floor(B^L / d)                 (once, GMP, at set-up; L = max x limbs)
//   t  = floor(|x| / B^(n-1)) * mu      (engine: an m x 1 by 1 x 1 product)
//   s  = floor(t / B^(L-n+1)) * d       (engine: device A, the shifted t)
//   r  = (|x| - s) mod B^(n+1), minus d at most twice, d - r for x < 0
// For 0 <= |x| < B^L and d >= B^(n-1) (n limbs, top limb nonzero) the
// quotient estimate is at most 2 below floor(|x| / d), so r < 3d before the
// corrections.
#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/mpzmm_b200.h"
#include "engine.h"
#include "kernels.h"

using namespace mpzmm;

namespace {

int cu(cudaError_t e, const char* what) {
  return e == cudaSuccess ? kOk
                          : set_error(kErrCuda, std::string(what) + ": " + cudaGetErrorString(e));
}

// A grow-only device buffer with an optional pinned host twin.
template <typename T>
struct Buf {
  T* d = nullptr;
  T* h = nullptr;
  size_t cap = 0;
  int grow(size_t want, bool host) {
    if (want <= cap) return kOk;
    free();
    const size_t n = want + want / 2;
    if (cudaMalloc((void**)&d, n * sizeof(T)) != cudaSuccess) {
      cudaGetLastError();
      d = nullptr;
      return set_error(kErrNoMem, "device buffer of " + std::to_string(n * sizeof(T)) + " bytes");
    }
    if (host && cudaMallocHost((void**)&h, n * sizeof(T)) != cudaSuccess) {
      cudaGetLastError();
      h = nullptr;
      return set_error(kErrNoMem, "pinned buffer of " + std::to_string(n * sizeof(T)) + " bytes");
    }
    cap = n;
    return kOk;
  }
  void free() {
    if (d) cudaFree(d);
    if (h) cudaFreeHost(h);
    d = h = nullptr;
    cap = 0;
  }
};

// one product of `count` rows (k = n = 1): A from device memory, B one host
// entry, the results left on the device
ProductSpec column_product(size_t count, std::shared_ptr<DeviceOperand> a, const uint64_t* b,
                           int32_t b_size) {
  ProductSpec ps;
  ps.m = (int)count;
  ps.k = 1;
  ps.n = 1;
  ps.a.assign(count, EntryRef{nullptr, 0});
  ps.dev_a = std::move(a);
  ps.b.push_back(EntryRef{b, b_size});
  ps.c.assign(count, OutRef{nullptr, 0, nullptr, nullptr});
  ps.device_only = true;
  return ps;
}

}  // namespace

struct mpzmm_mod {
  int n = 0;      // limbs of d
  int64_t L = 0;  // limbs of the largest x
  std::vector<uint64_t> d, mu;
  int64_t mu_bits = 0;
  uint64_t* d_d = nullptr;  // device copy of d
  Buf<uint64_t> x, r;       // x limbs back to back; r with n + 1 limbs per x
  Buf<int64_t> xo;          // x offsets
  Buf<int32_t> xs, s1, s2, rs;
  Workspace ws1, ws2;  // the two products
  ~mpzmm_mod() {
    if (d_d) cudaFree(d_d);
    x.free();
    r.free();
    xo.free();
    xs.free();
    s1.free();
    s2.free();
    rs.free();
  }
};

extern "C" {

int mpzmm_mod_create(mpzmm_mod** out, const uint64_t* d_limbs, int32_t d_size,
                     int64_t max_x_limbs) {
  if (!out) return set_error(kErrArg, "null output pointer");
  *out = nullptr;
  if (d_size <= 0 || !d_limbs) return set_error(kErrArg, "the modulus must be positive");
  int n = d_size;
  while (n > 0 && d_limbs[n - 1] == 0) --n;
  if (n == 0) return set_error(kErrArg, "the modulus must be positive");
  int st = ensure_setup(-1);
  if (st) return st;
  std::unique_ptr<mpzmm_mod> m(new mpzmm_mod);
  m->n = n;
  m->L = max_x_limbs > n ? max_x_limbs : n;
  m->d.assign(d_limbs, d_limbs + n);
  // mu = floor(B^L / d), at most B^(L-n+1) (d >= B^(n-1))
  __mpz_struct num, q, dd;
  __gmpz_init(&num);
  __gmpz_init(&q);
  __gmpz_setbit(&num, (unsigned long)(64 * m->L));
  __gmpz_tdiv_q(&q, &num, __gmpz_roinit_n(&dd, m->d.data(), n));
  m->mu.assign(q._mp_d, q._mp_d + q._mp_size);
  __gmpz_clear(&num);
  __gmpz_clear(&q);
  m->mu_bits = bit_length(EntryRef{m->mu.data(), (int32_t)m->mu.size()});
  if ((st = cu(cudaMalloc((void**)&m->d_d, (size_t)n * 8), "cudaMalloc modulus"))) return st;
  if ((st = cu(cudaMemcpy(m->d_d, m->d.data(), (size_t)n * 8, cudaMemcpyHostToDevice),
               "copy modulus")))
    return st;
  *out = m.release();
  return kOk;
}

void mpzmm_mod_destroy(mpzmm_mod* m) { delete m; }

int64_t mpzmm_mod_limbs(const mpzmm_mod* m) { return m ? m->n : -1; }

int mpzmm_mod_batch(mpzmm_mod* m, int count, const uint64_t* x_limbs, const int64_t* x_offs,
                    const int32_t* x_sizes, uint64_t* r_limbs, const int64_t* r_offs,
                    const int64_t* r_caps, int32_t* r_sizes, void* stream) {
  if (!m) return set_error(kErrArg, "null modulus");
  if (count < 0) return set_error(kErrArg, "negative count");
  if (count == 0) return kOk;
  if (!x_offs || !x_sizes || !r_limbs || !r_offs || !r_caps || !r_sizes)
    return set_error(kErrArg, "null array");
  int st = ensure_setup(-1);
  if (st) return st;
  std::lock_guard<std::mutex> lk(workspace_mutex());
  cudaStream_t s = stream ? static_cast<cudaStream_t>(stream) : context().stream;
  const int n = m->n;
  const int64_t L = m->L, sh1 = n - 1, sh2 = L - n + 1;
  for (int i = 0; i < count; ++i) {
    const int64_t a = x_sizes[i] < 0 ? -(int64_t)x_sizes[i] : x_sizes[i];
    if (a > L)
      return set_error(kErrTooLarge, "x " + std::to_string(i) + " has " + std::to_string(a) +
                                         " limbs, the reduction was set up for " +
                                         std::to_string(L));
    if (a && !x_limbs) return set_error(kErrArg, "null limb pointer");
  }
  // rows per pass: the engine addresses a product's residues with 32-bit
  // offsets, so (2 rows + 1) P N words must stay below 2^32
  Params p1, p2;
  if (!choose_params(64 * sh2, m->mu_bits, 1, 1, 1, &p1) ||
      !choose_params(64 * (sh2 + 2), 64 * (int64_t)n, 1, 1, 1, &p2))
    return set_error(kErrTooLarge, "modulus or x too large for a single transform");
  const uint64_t pn = std::max((uint64_t)p1.P << p1.lgN, (uint64_t)p2.P << p2.lgN);
  uint64_t rows = pn ? ((1ull << 31) / pn - 1) / 2 : 65535;
  if (rows > 65535) rows = 65535;
  if (rows < 1) return set_error(kErrTooLarge, "modulus or x too large for a single transform");
  int status = kOk;

  for (int c0 = 0; c0 < count; c0 += (int)rows) {
    const int cnt = (int)std::min<uint64_t>(rows, (uint64_t)(count - c0));
    // x limbs back to back (pinned staging), padded by L limbs so that the
    // views shifted up by n - 1 limbs stay inside the buffer
    size_t tot = 0;
    for (int i = 0; i < cnt; ++i) tot += (size_t)std::llabs((long long)x_sizes[c0 + i]);
    if ((st = m->x.grow(tot + (size_t)L + 1, true)) || (st = m->xo.grow((size_t)cnt, true)) ||
        (st = m->xs.grow((size_t)cnt, true)) || (st = m->s1.grow((size_t)cnt, false)) ||
        (st = m->s2.grow((size_t)cnt, false)) || (st = m->rs.grow((size_t)cnt, true)) ||
        (st = m->r.grow((size_t)cnt * (n + 1), true)))
      return st;
    std::vector<int64_t> offs((size_t)cnt);
    size_t off = 0;
    for (int i = 0; i < cnt; ++i) {
      const int32_t sz = x_sizes[c0 + i];
      const size_t a = (size_t)std::llabs((long long)sz);
      offs[i] = (int64_t)off;
      m->xo.h[i] = (int64_t)off;
      m->xs.h[i] = sz;
      off += a;
    }
    parallel_chunks((size_t)cnt, off * 8, [&](size_t lo, size_t hi) {
      for (size_t i = lo; i < hi; ++i) {
        const size_t a = (size_t)std::llabs((long long)x_sizes[c0 + i]);
        if (a) std::memcpy(m->x.h + offs[i], x_limbs + x_offs[c0 + i], a * 8);
      }
    });
    if ((st = cu(cudaMemcpyAsync(m->x.d, m->x.h, std::max<size_t>(off, 1) * 8,
                                 cudaMemcpyHostToDevice, s), "H2D x")) ||
        (st = cu(cudaMemcpyAsync(m->xo.d, m->xo.h, (size_t)cnt * 8, cudaMemcpyHostToDevice, s),
                 "H2D x offsets")) ||
        (st = cu(cudaMemcpyAsync(m->xs.d, m->xs.h, (size_t)cnt * 4, cudaMemcpyHostToDevice, s),
                 "H2D x sizes")) ||
        (st = cu(launch_shift_sizes(m->xs.d, m->s1.d, cnt, (int)sh1, s), "size shift")))
      return st;
    // t = floor(|x| / B^(n-1)) * mu
    auto a1 = std::make_shared<DeviceOperand>();
    a1->limbs = m->x.d + sh1;
    a1->sizes = m->s1.d;
    a1->offs = offs;
    a1->cap_limbs = sh2;
    a1->span_limbs = (uint64_t)offs.back() + (uint64_t)sh2;
    Plan pl1;
    std::vector<ProductSpec> v1;
    v1.push_back(column_product((size_t)cnt, a1, m->mu.data(), (int32_t)m->mu.size()));
    if ((st = pl1.build(std::move(v1), &m->ws1)) || (st = pl1.upload(s)) ||
        (st = pl1.execute(s)))
      return st;
    const DeviceOperand t = pl1.device_output(0);
    if (!t.limbs || t.cap_limbs <= sh2) return set_error(kErrState, "no quotient product");
    if ((st = cu(launch_shift_sizes(t.sizes, m->s2.d, cnt, (int)sh2, s), "size shift"))) return st;
    // s = floor(t / B^(L-n+1)) * d
    auto a2 = std::make_shared<DeviceOperand>();
    a2->limbs = t.limbs + sh2;
    a2->sizes = m->s2.d;
    a2->offs = t.offs;
    a2->cap_limbs = t.cap_limbs - sh2;
    a2->span_limbs = t.span_limbs - (uint64_t)sh2;
    Plan pl2;
    std::vector<ProductSpec> v2;
    v2.push_back(column_product((size_t)cnt, a2, m->d.data(), (int32_t)n));
    if ((st = pl2.build(std::move(v2), &m->ws2)) || (st = pl2.upload(s)) ||
        (st = pl2.execute(s)))
      return st;
    const DeviceOperand sv = pl2.device_output(0);
    if (!sv.limbs) return set_error(kErrState, "no product by the modulus");
    if ((st = cu(launch_mod_finish(cnt, n, m->x.d, m->xo.d, m->xs.d, sv.limbs, sv.cap_limbs,
                                   sv.sizes, m->d_d, m->r.d, m->rs.d, s),
                 "reduction launch")) ||
        (st = cu(cudaMemcpyAsync(m->r.h, m->r.d, (size_t)cnt * (n + 1) * 8,
                                 cudaMemcpyDeviceToHost, s), "D2H r")) ||
        (st = cu(cudaMemcpyAsync(m->rs.h, m->rs.d, (size_t)cnt * 4, cudaMemcpyDeviceToHost, s),
                 "D2H r sizes")) ||
        (st = cu(cudaStreamSynchronize(s), "reduction")))
      return st;
    for (int i = 0; i < cnt; ++i) {
      const int32_t sz = m->rs.h[i];
      const int e = c0 + i;
      if (sz > r_caps[e]) {
        if (!status)
          status = set_error(kErrCapacity, "remainder " + std::to_string(e) + " needs " +
                                               std::to_string(sz) + " limbs, capacity " +
                                               std::to_string(r_caps[e]));
        r_sizes[e] = 0;
        continue;
      }
      if (sz) std::memcpy(r_limbs + r_offs[e], m->r.h + (size_t)i * (n + 1), (size_t)sz * 8);
      r_sizes[e] = sz;
    }
  }
  return status;
}

// mpz_t front end: rop[i] = op[i] mod d in [0, d), grown with GMP's own
// allocator like the reference's mpzfft_mod_mod (src/lib/mpzfft.c:73-100)
int mpzmm_mod_mpz(mpzmm_mod* m, mpz_t* rop, mpz_t* op, int count, void* stream) {
  if (!m) return set_error(kErrArg, "null modulus");
  if (count < 0 || (count > 0 && (!rop || !op))) return set_error(kErrArg, "bad mpz arrays");
  if (count == 0) return kOk;
  std::vector<int64_t> xo((size_t)count), ro((size_t)count), rc((size_t)count, m->n);
  std::vector<int32_t> xs((size_t)count), rs((size_t)count);
  size_t tot = 0;
  for (int i = 0; i < count; ++i) {
    xo[i] = (int64_t)tot;
    xs[i] = op[i]->_mp_size;
    tot += (size_t)std::llabs((long long)op[i]->_mp_size);
  }
  std::vector<uint64_t> xl(tot ? tot : 1), rl((size_t)count * m->n);
  for (int i = 0; i < count; ++i)
    if (xs[i])
      std::memcpy(xl.data() + xo[i], op[i]->_mp_d, (size_t)std::llabs((long long)xs[i]) * 8);
  for (int i = 0; i < count; ++i) ro[i] = (int64_t)i * m->n;
  int st = mpzmm_mod_batch(m, count, xl.data(), xo.data(), xs.data(), rl.data(), ro.data(),
                           rc.data(), rs.data(), stream);
  if (st) return st;
  for (int i = 0; i < count; ++i) {
    __mpz_struct* z = rop[i];
    if (z->_mp_alloc < rs[i]) __gmpz_realloc(z, (mp_size_t)rs[i]);
    if (rs[i]) std::memcpy(z->_mp_d, rl.data() + ro[i], (size_t)rs[i] * 8);
    z->_mp_size = rs[i];
  }
  return kOk;
}

}  // extern "C"
