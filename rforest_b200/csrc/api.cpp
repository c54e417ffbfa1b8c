// extern "C" entry points of libmpzmm_b200.so (declared in include/mpzmm_b200.h).
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <memory>
#include <mutex>
#include <vector>

#include "../../include/mpzmm_b200.h"
#include "engine.h"

using namespace mpzmm;

namespace {

void default_fatal(int status, const char* msg) {
  std::fprintf(stderr, "mpzmm_b200: fatal error %d: %s\n", status, msg);
  std::abort();
}
mpzmm_fatal_fn g_fatal = default_fatal;
std::mutex g_call_mu;  // the reference API is single-threaded global state

cudaStream_t pick_stream(void* stream) {
  return stream ? static_cast<cudaStream_t>(stream) : context().stream;
}

int check_product_packed(const mpzmm_product& p) {
  if (p.m < 0 || p.k < 0 || p.n < 0) return set_error(kErrArg, "negative dimension");
  const int64_t na = (int64_t)p.m * p.k, nb = (int64_t)p.k * p.n, nc = (int64_t)p.m * p.n;
  if ((na && (!p.a_offs || !p.a_sizes)) || (nb && (!p.b_offs || !p.b_sizes)) ||
      (nc && (!p.c_offs || !p.c_caps || !p.c_sizes || !p.c_limbs)))
    return set_error(kErrArg, "null array");
  return kOk;
}

// the entry references of a checked product
void fill_spec_packed(const mpzmm_product& p, ProductSpec* ps) {
  ps->m = p.m;
  ps->k = p.k;
  ps->n = p.n;
  const int64_t na = (int64_t)p.m * p.k, nb = (int64_t)p.k * p.n, nc = (int64_t)p.m * p.n;
  ps->a.resize(na);
  ps->b.resize(nb);
  ps->c.resize(nc);
  for (int64_t e = 0; e < na; ++e) {
    const int32_t s = p.a_sizes[e];
    ps->a[e] = EntryRef{s ? p.a_limbs + p.a_offs[e] : nullptr, s};
  }
  for (int64_t e = 0; e < nb; ++e) {
    const int32_t s = p.b_sizes[e];
    ps->b[e] = EntryRef{s ? p.b_limbs + p.b_offs[e] : nullptr, s};
  }
  for (int64_t e = 0; e < nc; ++e)
    ps->c[e] = OutRef{p.c_limbs + p.c_offs[e], p.c_caps[e], p.c_sizes + e, nullptr};
}

// All products checked (first error wins), then their references filled on
// several host threads for a large batch.
int build_specs_packed(int count, const mpzmm_product* products,
                       std::vector<ProductSpec>* specs) {
  uint64_t entries = 0;
  for (int t = 0; t < count; ++t) {
    const int st = check_product_packed(products[t]);
    if (st) return st;
    const mpzmm_product& p = products[t];
    entries += (uint64_t)p.m * p.k + (uint64_t)p.k * p.n + (uint64_t)p.m * p.n;
  }
  specs->assign((size_t)count, ProductSpec());
  parallel_chunks((size_t)count, (size_t)entries * 64, [&](size_t lo, size_t hi) {
    for (size_t t = lo; t < hi; ++t) fill_spec_packed(products[t], &(*specs)[t]);
  });
  return kOk;
}

int run_once(std::vector<ProductSpec> specs, void* stream) {
  int st = ensure_setup(-1);
  if (st) return st;
  std::lock_guard<std::mutex> lk(workspace_mutex());
  return run_batch(std::move(specs), pick_stream(stream));
}

// r x d by d x d over mpz_t arrays (src/lib/hwmpz.c:65-130)
int mpz_matmul(mpz_t* C, mpz_t* A, int r, mpz_t* B, int d) {
  if (r < 0 || d < 0) return set_error(kErrArg, "negative dimension");
  ProductSpec ps;
  ps.m = r;
  ps.k = d;
  ps.n = d;
  ps.a.resize((size_t)r * d);
  ps.b.resize((size_t)d * d);
  ps.c.resize((size_t)r * d);
  for (size_t e = 0; e < ps.a.size(); ++e)
    ps.a[e] = EntryRef{reinterpret_cast<const uint64_t*>(A[e]->_mp_d), A[e]->_mp_size};
  for (size_t e = 0; e < ps.b.size(); ++e)
    ps.b[e] = EntryRef{reinterpret_cast<const uint64_t*>(B[e]->_mp_d), B[e]->_mp_size};
  for (size_t e = 0; e < ps.c.size(); ++e) ps.c[e] = OutRef{nullptr, 0, nullptr, C[e]};
  std::vector<ProductSpec> v;
  v.push_back(std::move(ps));
  return run_once(std::move(v), nullptr);
}

}  // namespace

struct mpzmm_plan {
  Plan plan;
};

extern "C" {

void mpzmm_set_fatal_hook(mpzmm_fatal_fn fn) { g_fatal = fn ? fn : default_fatal; }

int mpzmm_setup(int device) { return ensure_setup(device); }

int mpzmm_set_option(int option, int value) {
  if (option == MPZMM_OPT_CONTRACT) {
    if (value < 0 || value > 2) return set_error(kErrArg, "contract mode must be 0, 1 or 2");
    context().contract_mode = value;
    return kOk;
  }
  if (option == MPZMM_OPT_CHUNK_LIMBS) {
    if (value < 0) return set_error(kErrArg, "chunk size must be >= 0");
    std::lock_guard<std::mutex> lk(workspace_mutex());
    context().chunk_limbs = value;
    return kOk;
  }
  if (option == MPZMM_OPT_CHECK_BOUNDS) {
    if (value < 0 || value > 1) return set_error(kErrArg, "bounds check must be 0 or 1");
    context().check_bounds = value != 0;
    return kOk;
  }
  if (option == MPZMM_OPT_TEST_STALL_TC) {
    if (value < 0) return set_error(kErrArg, "count must be >= 0");
    set_test_stall_tc(value);
    return kOk;
  }
  if (option == MPZMM_OPT_TEST_FAIL_ALLOC) {
    if (value < 0) return set_error(kErrArg, "count must be >= 0");
    set_test_fail_alloc(value);
    return kOk;
  }
  return set_error(kErrArg, "unknown option");
}

// Times the contraction stage of a representative batch per size class
// (m = n = 4, 8, 16, 32, 64 by k = 8, 16, 32, 64 terms, 2^14-bit entries,
// copies of one product until the GPU is full) on CUDA cores and on tensor
// cores, and records the faster engine for automatic mode.  ms_out (optional) receives {cuda, tc} milliseconds per
// class, k-major (40 floats).
int mpzmm_autotune(void* stream, float* ms_out) {
  int st = ensure_setup(-1);
  if (st) return st;
  cudaStream_t s = pick_stream(stream);
  const int ks[4] = {8, 16, 32, 64};
  const int mns[5] = {4, 8, 16, 32, 64};
  const int saved = context().contract_mode;
  uint64_t x = 0x9E3779B97F4A7C15ull;
  auto fail = [&](int code) {
    context().contract_mode = saved;
    return code;
  };
  for (int bk = 0; bk < 4; ++bk)
    for (int bm = 0; bm < 5; ++bm) {
      const int m = mns[bm], k = ks[bk], n = mns[bm], nl = 256;  // 2^14-bit entries
      std::vector<uint64_t> limbs((size_t)(m * k + k * n) * nl);
      for (auto& w : limbs) {
        x ^= x << 13;
        x ^= x >> 7;
        x ^= x << 17;
        w = x;
      }
      const int cap = 2 * nl + 2;
      std::vector<uint64_t> out((size_t)m * n * cap);
      // the probe runs at load: copies of the product (sharing the host
      // arrays) until either engine has about eight CTAs' work per SM -- a
      // single small product leaves most of the GPU idle and favours
      // whichever engine does more per CTA, which is not what a batch sees
      Params prm;
      if (!choose_params(64 * nl, 64 * nl, m, k, n, &prm)) return fail(kErrTooLarge);
      const int64_t ctas = (int64_t)prm.P * (((int64_t)1 << prm.lgN) + 127) / 128;
      int64_t copies = (8 * (int64_t)context().num_sms + ctas - 1) / (ctas > 0 ? ctas : 1);
      if (copies < 1) copies = 1;
      if (copies > 256) copies = 256;
      float ms[2] = {0.f, 0.f}, fc[2] = {0.f, 0.f};  // contraction; split + forward + contraction
      for (int mode = 1; mode <= 2; ++mode) {
        std::vector<ProductSpec> v;
        for (int64_t c = 0; c < copies; ++c) {
          ProductSpec ps;
          ps.m = m;
          ps.k = k;
          ps.n = n;
          for (int e = 0; e < m * k; ++e) ps.a.push_back(EntryRef{&limbs[(size_t)e * nl], nl});
          for (int e = 0; e < k * n; ++e)
            ps.b.push_back(EntryRef{&limbs[(size_t)(m * k + e) * nl], nl});
          for (int e = 0; e < m * n; ++e)
            ps.c.push_back(OutRef{&out[(size_t)e * cap], cap, nullptr, nullptr});
          v.push_back(std::move(ps));
        }
        context().contract_mode = mode;
        Plan plan;
        if ((st = plan.build(std::move(v))) || (st = plan.upload(s)) || (st = plan.execute(s)))
          return fail(st);
        // fastest of five timed executes: one slow repeat (another process
        // on the device, a clock change) must not decide the table
        plan.set_timing(true);
        float best = -1.f, best_fc = -1.f;
        for (int rep = 0; rep < 5; ++rep) {
          if ((st = plan.execute(s))) return fail(st);
          float t[Plan::kStages];
          int64_t ex = 0;  // stage_times returns (and clears) this execute's times
          if ((st = plan.stage_times(t, &ex))) return fail(st);
          if (best < 0.f || t[1] < best) best = t[1];
          if (best_fc < 0.f || t[0] + t[1] < best_fc) best_fc = t[0] + t[1];
        }
        ms[mode - 1] = best < 0.f ? 0.f : best;
        fc[mode - 1] = best_fc < 0.f ? 0.f : best_fc;
      }
      // the decision weighs split + forward with the contraction (tensor-core
      // operands are written frequency-blocked, which costs the forward a
      // little), and wants a 10 % margin (a near tie measured on a probe once
      // turned into a far slower contraction of a real batch)
      context().tc_pref[bk][bm] = fc[1] < 0.9f * fc[0] ? 1 : 0;
      if (ms_out) {
        ms_out[2 * (bk * 5 + bm)] = ms[0];
        ms_out[2 * (bk * 5 + bm) + 1] = ms[1];
      }
    }
  context().contract_mode = saved;
  return kOk;
}

int mpzmm_get_option(int option) {
  if (option == MPZMM_OPT_CONTRACT) return context().contract_mode;
  if (option == MPZMM_OPT_CHUNK_LIMBS) return (int)context().chunk_limbs;
  if (option == MPZMM_OPT_CHECK_BOUNDS) return context().check_bounds ? 1 : 0;
  if (option == MPZMM_OPT_TEST_STALL_TC) return test_stall_tc();
  if (option == MPZMM_OPT_TEST_FAIL_ALLOC) return test_fail_alloc();
  return -1;
}

int mpzmm_host_alloc(size_t bytes, void** out) { return host_alloc(bytes, out); }
int mpzmm_host_free(void* p) { return host_free(p); }
int mpzmm_host_register(void* p, size_t bytes) { return host_register(p, bytes); }
int mpzmm_host_unregister(void* p) { return host_unregister(p); }

int mpzmm_batch_stats(int64_t* ns4, int64_t* chunks, int64_t* bytes4) {
  std::lock_guard<std::mutex> lk(workspace_mutex());
  for (int i = 0; i < 4; ++i) {
    if (ns4) ns4[i] = context().batch_ns[i];
    if (bytes4) bytes4[i] = context().batch_bytes[i];
  }
  if (chunks) *chunks = context().batch_chunks;
  return kOk;
}

int mpzmm_batch_chunks(int count, const int64_t* limbs, int64_t chunk_limbs, int64_t* bounds,
                       int max_bounds, int* nchunks) {
  if (count < 0 || (count > 0 && !limbs)) return set_error(kErrArg, "bad limb counts");
  std::vector<uint64_t> l((size_t)count);
  for (int t = 0; t < count; ++t) {
    if (limbs[t] < 0) return set_error(kErrArg, "negative limb count");
    l[t] = (uint64_t)limbs[t];
  }
  std::vector<size_t> b;
  batch_chunks(l, chunk_limbs, &b);
  const int n = (int)b.size() - 1;
  if (nchunks) *nchunks = n;
  if (bounds)
    for (int i = 0; i <= n && i < max_bounds; ++i) bounds[i] = (int64_t)b[i];
  return kOk;
}

static_assert(MPZMM_TIMELINE_FIELDS == mpzmm::kTimelineFields, "timeline row size");

int mpzmm_batch_timeline(double* rows, int max_chunks, int* nchunks) {
  std::lock_guard<std::mutex> lk(workspace_mutex());
  const std::vector<double>& tl = context().timeline;
  const int n = (int)(tl.size() / kTimelineFields);
  if (nchunks) *nchunks = n;
  if (rows && max_chunks > 0) {
    const int k = n < max_chunks ? n : max_chunks;
    std::copy(tl.begin(), tl.begin() + (size_t)k * kTimelineFields, rows);
  }
  return kOk;
}

const char* mpzmm_last_error(void) { return last_error(); }

int mpzmm_device_available(void) {
  int n = 0;
  if (cudaGetDeviceCount(&n) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  return n > 0 ? 1 : 0;
}

void hw_mpz_setup(void) {
  std::lock_guard<std::mutex> lk(g_call_mu);
  int st = ensure_setup(-1);
  if (st) g_fatal(st, last_error());
}

void hw_mpz_clear(void) {
  std::lock_guard<std::mutex> lk(g_call_mu);
  teardown();
}

void mpz_rmatrix_mult_fft(mpz_t* C, mpz_t* A, int r, mpz_t* B, int d, mpz_t w) {
  (void)w;
  std::lock_guard<std::mutex> lk(g_call_mu);
  if (!context().ready) {
    g_fatal(kErrState, "mpz_rmatrix_mult_fft called before hw_mpz_setup");
    return;
  }
  int st = mpz_matmul(C, A, r, B, d);
  if (st) g_fatal(st, last_error());
}

void cu_mpz_rmatrix_mult_fft(mpz_t* C, mpz_t* A, int r, mpz_t* B, int d, mpz_t w) {
  mpz_rmatrix_mult_fft(C, A, r, B, d, w);
}

int mpz_rmatrix_gpu_fft_suitable(mpz_t* A, int r, mpz_t* B, int d) {
  if (r < 0 || d < 0) return 0;
  int64_t ab = 0, bb = 0;
  for (int64_t e = 0; e < (int64_t)r * d; ++e) {
    int64_t s = A[e]->_mp_size < 0 ? -(int64_t)A[e]->_mp_size : A[e]->_mp_size;
    if (64 * s > ab) ab = 64 * s;
  }
  for (int64_t e = 0; e < (int64_t)d * d; ++e) {
    int64_t s = B[e]->_mp_size < 0 ? -(int64_t)B[e]->_mp_size : B[e]->_mp_size;
    if (64 * s > bb) bb = 64 * s;
  }
  Params prm;
  return choose_params(ab, bb, r, d, d, &prm) ? 1 : 0;
}

int64_t mpzmm_output_limbs(int k, int64_t a_bits, int64_t b_bits) {
  return output_limbs(k, a_bits, b_bits);
}

int mpzmm_choose_params(int64_t a_bits, int64_t b_bits, int k, int* P, int* r, int* lgN) {
  Params prm;
  if (!choose_params(a_bits, b_bits, 1, k, 1, &prm))
    return set_error(kErrTooLarge, "no supported parameters");
  if (P) *P = prm.P;
  if (r) *r = prm.r;
  if (lgN) *lgN = prm.lgN;
  return kOk;
}

int mpzmm_matmul(int m, int k, int n, const uint64_t* a_limbs, const int64_t* a_offs,
                 const int32_t* a_sizes, const uint64_t* b_limbs, const int64_t* b_offs,
                 const int32_t* b_sizes, uint64_t* c_limbs, const int64_t* c_offs,
                 const int64_t* c_caps, int32_t* c_sizes, void* stream) {
  mpzmm_product p{m,      k,      n,       a_limbs, a_offs, a_sizes, b_limbs,
                  b_offs, b_sizes, c_limbs, c_offs,  c_caps, c_sizes};
  return mpzmm_matmul_batch(1, &p, stream);
}

int mpzmm_matmul_batch(int count, const mpzmm_product* products, void* stream) {
  if (count < 0 || (count > 0 && !products)) return set_error(kErrArg, "bad product list");
  std::vector<ProductSpec> specs;
  const int st = build_specs_packed(count, products, &specs);
  if (st) return st;
  return run_once(std::move(specs), stream);
}

namespace {
int64_t matrix_max_bits(const mpzmm_matrix& x) {
  int64_t bits = 0;
  for (int64_t e = 0; e < (int64_t)x.rows * x.cols; ++e) {
    const int32_t s = x.sizes[e];
    if (!s) continue;
    const EntryRef r{x.limbs + x.offs[e], s};
    const int64_t b = bit_length(r);
    if (b > bits) bits = b;
  }
  return bits;
}

int check_chain(int count, const mpzmm_matrix* mats) {
  if (count < 2 || !mats) return set_error(kErrArg, "a chain needs at least two matrices");
  for (int i = 0; i < count; ++i) {
    const mpzmm_matrix& x = mats[i];
    if (x.rows < 1 || x.cols < 1) return set_error(kErrArg, "chain matrix without entries");
    if (!x.offs || !x.sizes || !x.limbs) return set_error(kErrArg, "null array");
    if (i > 0 && x.rows != mats[i - 1].cols)
      return set_error(kErrArg, "chain matrix " + std::to_string(i) + " has " +
                                    std::to_string(x.rows) + " rows, expected " +
                                    std::to_string(mats[i - 1].cols));
  }
  return kOk;
}

// Output limb bound of every chain step (the planner's own: exact bits for
// the host operands, 64 x the previous bound for the running product).
int chain_limbs(int count, const mpzmm_matrix* mats, std::vector<int64_t>* limbs, bool* zero) {
  *zero = false;
  std::vector<int64_t> bits((size_t)count);
  for (int i = 0; i < count; ++i) {
    bits[i] = matrix_max_bits(mats[i]);
    if (!bits[i]) *zero = true;
  }
  limbs->assign((size_t)count - 1, 1);
  if (*zero) return kOk;
  int64_t a_bits = bits[0];
  for (int i = 1; i < count; ++i) {
    (*limbs)[i - 1] = output_limbs(mats[i].rows, a_bits, bits[i]);
    a_bits = 64 * (*limbs)[i - 1];
  }
  return kOk;
}
}  // namespace

int64_t mpzmm_chain_output_limbs(int count, const mpzmm_matrix* mats) {
  if (check_chain(count, mats)) return -1;
  std::vector<int64_t> lim;
  bool zero;
  chain_limbs(count, mats, &lim, &zero);
  return zero ? 1 : lim.back();
}

int mpzmm_chain(int count, const mpzmm_matrix* mats, uint64_t* c_limbs, const int64_t* c_offs,
                const int64_t* c_caps, int32_t* c_sizes, void* stream) {
  int st = check_chain(count, mats);
  if (st) return st;
  const int m = mats[0].rows, n = mats[count - 1].cols;
  if (!c_limbs || !c_offs || !c_caps || !c_sizes) return set_error(kErrArg, "null output array");
  if ((st = ensure_setup(-1))) return st;
  std::vector<int64_t> lim;
  bool zero;
  chain_limbs(count, mats, &lim, &zero);
  if (zero) {  // a zero factor: the product is zero
    for (int64_t e = 0; e < (int64_t)m * n; ++e) c_sizes[e] = 0;
    return kOk;
  }
  auto host_entries = [](const mpzmm_matrix& x, std::vector<EntryRef>* v) {
    v->resize((size_t)x.rows * x.cols);
    for (size_t e = 0; e < v->size(); ++e) {
      const int32_t s = x.sizes[e];
      (*v)[e] = EntryRef{s ? x.limbs + x.offs[e] : nullptr, s};
    }
  };
  std::vector<ProductSpec> steps((size_t)count - 1);
  for (int i = 1; i < count; ++i) {
    ProductSpec& ps = steps[(size_t)i - 1];
    ps.m = m;
    ps.k = mats[i].rows;
    ps.n = mats[i].cols;
    if (i == 1) {
      host_entries(mats[0], &ps.a);
    } else {
      ps.a.assign((size_t)ps.m * ps.k, EntryRef{nullptr, 0});  // on the device
    }
    host_entries(mats[i], &ps.b);
    ps.c.resize((size_t)ps.m * ps.n);
    for (size_t e = 0; e < ps.c.size(); ++e)
      ps.c[e] = i + 1 == count ? OutRef{c_limbs + c_offs[e], c_caps[e], c_sizes + e, nullptr}
                               : OutRef{nullptr, 0, nullptr, nullptr};
  }
  std::lock_guard<std::mutex> lk(workspace_mutex());
  return run_chain(std::move(steps), pick_stream(stream));
}

static int plan_create(mpzmm_plan** plan, int count, const mpzmm_product* products,
                       bool fixed_b, void* stream) {
  if (!plan) return set_error(kErrArg, "null plan pointer");
  *plan = nullptr;
  if (count < 0 || (count > 0 && !products)) return set_error(kErrArg, "bad product list");
  int st = ensure_setup(-1);
  if (st) return st;
  std::vector<ProductSpec> specs;
  if ((st = build_specs_packed(count, products, &specs))) return st;
  std::unique_ptr<mpzmm_plan> p(new mpzmm_plan);
  p->plan.set_fixed_b(fixed_b);
  if ((st = p->plan.build(std::move(specs)))) return st;
  if ((st = p->plan.upload(pick_stream(stream)))) return st;
  *plan = p.release();
  return kOk;
}

int mpzmm_plan_create(mpzmm_plan** plan, int count, const mpzmm_product* products,
                      void* stream) {
  return plan_create(plan, count, products, false, stream);
}

int mpzmm_plan_create_fixed_b(mpzmm_plan** plan, int count, const mpzmm_product* products,
                              void* stream) {
  return plan_create(plan, count, products, true, stream);
}

int mpzmm_plan_upload_a(mpzmm_plan* plan, void* stream) {
  if (!plan) return set_error(kErrArg, "null plan");
  return plan->plan.upload_a(pick_stream(stream));
}

int mpzmm_plan_execute(mpzmm_plan* plan, void* stream) {
  if (!plan) return set_error(kErrArg, "null plan");
  return plan->plan.execute(pick_stream(stream));
}

int mpzmm_plan_download(mpzmm_plan* plan, void* stream) {
  if (!plan) return set_error(kErrArg, "null plan");
  return plan->plan.download(pick_stream(stream));
}

int mpzmm_plan_upload(mpzmm_plan* plan, void* stream) {
  if (!plan) return set_error(kErrArg, "null plan");
  return plan->plan.upload(pick_stream(stream));
}

void mpzmm_plan_destroy(mpzmm_plan* plan) { delete plan; }

int mpzmm_plan_set_graph(mpzmm_plan* plan, int enable) {
  if (!plan) return set_error(kErrArg, "null plan");
  plan->plan.set_graph(enable != 0);
  return kOk;
}

int mpzmm_plan_set_timing(mpzmm_plan* plan, int enable) {
  if (!plan) return set_error(kErrArg, "null plan");
  plan->plan.set_timing(enable != 0);
  return kOk;
}

int mpzmm_plan_stage_times(mpzmm_plan* plan, float* ms, int64_t* launches,
                           int64_t* executes) {
  if (!plan) return set_error(kErrArg, "null plan");
  float t[Plan::kStages];
  int st = plan->plan.stage_times(t, executes);
  if (st) return st;
  int64_t l[Plan::kStages];
  plan->plan.stage_launches(l);
  for (int s = 0; s < Plan::kStages; ++s) {
    if (ms) ms[s] = t[s];
    if (launches) launches[s] = l[s];
  }
  return kOk;
}

int mpzmm_plan_info(const mpzmm_plan* plan, int64_t* launches, int64_t* bytes, int index,
                    int* P, int* r, int* lgN) {
  if (!plan) return set_error(kErrArg, "null plan");
  if (launches) *launches = plan->plan.launches_per_execute();
  if (bytes) *bytes = plan->plan.device_bytes();
  const auto& prm = plan->plan.params();
  if (index >= 0 && index < (int)prm.size()) {
    if (P) *P = prm[index].P;
    if (r) *r = prm[index].r;
    if (lgN) *lgN = prm[index].lgN;
  }
  return kOk;
}

}  // extern "C"
