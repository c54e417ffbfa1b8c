// Batch engine (see engine.h).
#include "engine.h"

#include <algorithm>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <thread>
#include <utility>

#include "../../include/mpzmm_gmp_abi.h"
#include "kernels.h"

namespace mpzmm {

namespace {
thread_local std::string g_err;
Context g_ctx;
std::mutex g_ctx_mu;

int cuda_fail(cudaError_t e, const char* what) {
  return set_error(kErrCuda, std::string(what) + ": " + cudaGetErrorString(e));
}

#define CU(call, what)                          \
  do {                                          \
    cudaError_t _e = (call);                    \
    if (_e != cudaSuccess) return cuda_fail(_e, what); \
  } while (0)

int64_t bit_length(const EntryRef& e) {
  const int64_t n = e.size < 0 ? -(int64_t)e.size : e.size;
  if (n == 0) return 0;
  uint64_t top = e.d[n - 1];
  int b = 0;
  while (top) {
    ++b;
    top >>= 1;
  }
  // a non-normalised top limb of zero is tolerated: scan down
  if (b == 0) {
    int64_t i = n - 1;
    while (i >= 0 && e.d[i] == 0) --i;
    if (i < 0) return 0;
    uint64_t t = e.d[i];
    while (t) {
      ++b;
      t >>= 1;
    }
    return 64 * i + b;
  }
  return 64 * (n - 1) + b;
}

}  // namespace

int set_error(int status, const std::string& msg) {
  g_err = msg;
  return status;
}
const char* last_error() { return g_err.c_str(); }

Context& context() { return g_ctx; }

std::mutex& workspace_mutex() {
  static std::mutex mu;
  return mu;
}

void parallel_chunks(size_t n, size_t bytes, const std::function<void(size_t, size_t)>& fn) {
  if (n == 0) return;
  unsigned hw = std::thread::hardware_concurrency();
  unsigned nt = hw ? hw : 1;
  if (nt > 16) nt = 16;
  const size_t per_thread_min = (size_t)8 << 20;  // 8 MB per thread at least
  if (bytes / per_thread_min < nt) nt = (unsigned)(bytes / per_thread_min);
  if (nt > n) nt = (unsigned)n;
  if (nt <= 1) {
    fn(0, n);
    return;
  }
  std::vector<std::thread> th;
  th.reserve(nt);
  for (unsigned i = 0; i < nt; ++i) {
    const size_t lo = n * i / nt, hi = n * (i + 1) / nt;
    th.emplace_back([&fn, lo, hi] { fn(lo, hi); });
  }
  for (auto& t : th) t.join();
}

int ensure_setup(int device) {
  std::lock_guard<std::mutex> lk(g_ctx_mu);
  if (g_ctx.ready) {
    if (device >= 0 && device != g_ctx.device)
      return set_error(kErrState, "already set up on another device");
    CU(cudaSetDevice(g_ctx.device), "cudaSetDevice");
    return kOk;
  }
  if (device < 0) {
    const char* env = std::getenv("MPZMM_DEVICE");
    device = env ? std::atoi(env) : 0;
  }
  int count = 0;
  cudaError_t e = cudaGetDeviceCount(&count);
  if (e != cudaSuccess || count <= device)
    return set_error(kErrCuda, std::string("no usable CUDA device: ") +
                                   (e != cudaSuccess ? cudaGetErrorString(e) : "index out of range"));
  CU(cudaSetDevice(device), "cudaSetDevice");
  cudaDeviceProp prop;
  CU(cudaGetDeviceProperties(&prop, device), "cudaGetDeviceProperties");
  if (prop.major < 10)
    return set_error(kErrCuda, std::string("device ") + prop.name +
                                   " is not sm_100 class; this build targets sm_100a");
  g_ctx.num_sms = prop.multiProcessorCount;
  const Moduli& M = moduli();
  CU(upload_constants(M.pc, &M.crt), "upload constants");
  CU(init_kernel_attributes(), "kernel attributes");
  const size_t tw = M.twf.size();
  CU(cudaMalloc(&g_ctx.d_twf, tw * sizeof(uint2)), "cudaMalloc twiddles");
  CU(cudaMalloc(&g_ctx.d_twi, tw * sizeof(uint2)), "cudaMalloc twiddles");
  CU(cudaMemcpy(g_ctx.d_twf, M.twf.data(), tw * sizeof(uint2), cudaMemcpyHostToDevice),
     "copy twiddles");
  CU(cudaMemcpy(g_ctx.d_twi, M.twi.data(), tw * sizeof(uint2), cudaMemcpyHostToDevice),
     "copy twiddles");
  CU(cudaStreamCreateWithFlags(&g_ctx.stream, cudaStreamNonBlocking), "cudaStreamCreate");
  g_ctx.ws = new Workspace;
  if (const char* cm = std::getenv("MPZMM_CONTRACT")) {
    const int v = std::atoi(cm);
    if (v >= 0 && v <= 2) g_ctx.contract_mode = v;
  }
  g_ctx.device = device;
  g_ctx.ready = true;
  return kOk;
}

void teardown() {
  std::lock_guard<std::mutex> lk(g_ctx_mu);
  if (!g_ctx.ready) return;
  cudaSetDevice(g_ctx.device);
  cudaStreamSynchronize(g_ctx.stream);
  cudaFree(g_ctx.d_twf);
  cudaFree(g_ctx.d_twi);
  {
    std::lock_guard<std::mutex> wl(workspace_mutex());
    delete g_ctx.ws;
  }
  cudaStreamDestroy(g_ctx.stream);
  g_ctx = Context();
}

Plan::~Plan() {
  for (cudaEvent_t e : events_) cudaEventDestroy(e);
  if (graph_exec_) cudaGraphExecDestroy(graph_exec_);
  if (graph_) cudaGraphDestroy(graph_);
}

int Workspace::reserve(size_t limbs, size_t res, size_t out_words, size_t sizes,
                       size_t desc_bytes) {
  // device: check the total growth against free memory first
  size_t grow = 0;
  if (limbs > cap_limbs) grow += limbs * 8;
  if (res > cap_res) grow += res * 4;
  if (out_words > cap_out) grow += out_words * 4;
  if (grow) {
    size_t free_b = 0, total_b = 0;
    CU(cudaMemGetInfo(&free_b, &total_b), "cudaMemGetInfo");
    size_t reclaim = (limbs > cap_limbs ? cap_limbs * 8 : 0) + (res > cap_res ? cap_res * 4 : 0) +
                     (out_words > cap_out ? cap_out * 4 : 0);
    if (grow + (64ull << 20) > free_b + reclaim)
      return set_error(kErrNoMem, "batch needs " + std::to_string(grow) +
                                      " more device bytes, " + std::to_string(free_b) +
                                      " free");
  }
  int st;
  // geometric growth: a workspace serving batches of varying size settles
  // after a few growths instead of re-allocating for every new maximum
  auto grown = [](size_t want, size_t cap) {
    const size_t g = cap + cap / 2;
    return want > g ? want : g;
  };
  auto grow_dev = [&](auto** p, size_t& cap, size_t want, size_t elem) -> int {
    if (want <= cap) return kOk;
    const size_t geo = cap ? grown(want, cap) : want;
    if (*p) {
      if (async_stream)
        cudaFreeAsync(*p, async_stream);
      else
        cudaFree(*p);
      device_bytes -= (int64_t)(cap * elem);
    }
    *p = nullptr;
    cap = 0;
    auto alloc = [&](size_t count) {
      return async_stream ? cudaMallocAsync((void**)p, count * elem, async_stream)
                          : cudaMalloc((void**)p, count * elem);
    };
    cudaError_t e = alloc(geo);
    if (e != cudaSuccess && geo != want) {  // the larger size did not fit: exact size
      cudaGetLastError();
      e = alloc(want);
    } else {
      want = geo;
    }
    if (e != cudaSuccess) {
      *p = nullptr;
      return set_error(kErrNoMem, std::string("cudaMalloc of ") + std::to_string(want * elem) +
                                      " bytes: " + cudaGetErrorString(e));
    }
    cap = want;
    device_bytes += (int64_t)(want * elem);
    return kOk;
  };
  auto grow_host = [&](auto** p, size_t& cap, size_t want, size_t elem) -> int {
    if (want <= cap) return kOk;
    if (cap) want = grown(want, cap);
    if (*p) cudaFreeHost(*p);
    *p = nullptr;
    cap = 0;
    cudaError_t e = cudaMallocHost((void**)p, want * elem);
    if (e != cudaSuccess) {
      *p = nullptr;
      return set_error(kErrNoMem, std::string("cudaMallocHost of ") +
                                      std::to_string(want * elem) + " bytes: " +
                                      cudaGetErrorString(e));
    }
    cap = want;
    return kOk;
  };
  if ((st = grow_dev(&d_limbs, cap_limbs, limbs, 8))) return st;
  if ((st = grow_dev(&d_res, cap_res, res, 4))) return st;
  if ((st = grow_dev(&d_out, cap_out, out_words, 4))) return st;
  if ((st = grow_dev(&d_sizes, cap_sizes, sizes, 4))) return st;
  if ((st = grow_dev(&d_desc, cap_desc, desc_bytes, 1))) return st;
  if (!d_status) {
    cudaError_t e = async_stream ? cudaMallocAsync((void**)&d_status, sizeof(int), async_stream)
                                 : cudaMalloc((void**)&d_status, sizeof(int));
    if (e != cudaSuccess) {
      d_status = nullptr;
      return set_error(kErrNoMem, std::string("cudaMalloc(status): ") + cudaGetErrorString(e));
    }
    device_bytes += (int64_t)sizeof(int);
  }
  if ((st = grow_host(&h_limbs, hcap_limbs, limbs, 8))) return st;
  if ((st = grow_host(&h_out, hcap_out, out_words, 4))) return st;
  if ((st = grow_host(&h_sizes, hcap_sizes, sizes, 4))) return st;
  if ((st = grow_host(&h_desc, hcap_desc, desc_bytes, 1))) return st;
  return kOk;
}

void Workspace::release_device() {
  for (void* p : {(void*)d_limbs, (void*)d_res, (void*)d_out, (void*)d_sizes, (void*)d_desc,
                  (void*)d_status}) {
    if (!p) continue;
    if (async_stream)
      cudaFreeAsync(p, async_stream);
    else
      cudaFree(p);
  }
  d_limbs = nullptr;
  d_res = d_out = nullptr;
  d_sizes = nullptr;
  d_desc = nullptr;
  d_status = nullptr;
  cap_limbs = cap_res = cap_out = cap_sizes = cap_desc = 0;
  device_bytes = 0;
}

void Workspace::release() {
  release_device();
  cudaFreeHost(h_limbs);
  cudaFreeHost(h_out);
  cudaFreeHost(h_sizes);
  cudaFreeHost(h_desc);
  h_limbs = nullptr;
  h_out = nullptr;
  h_sizes = nullptr;
  h_desc = nullptr;
  hcap_limbs = hcap_out = hcap_sizes = hcap_desc = 0;
}

int64_t estimate_device_bytes(const ProductSpec& ps) {
  int64_t a_bits = 0, b_bits = 0, limbs = 0;
  for (const auto& e : ps.a) {
    const int64_t b = bit_length(e);
    if (b > a_bits) a_bits = b;
    limbs += e.size < 0 ? -(int64_t)e.size : e.size;
  }
  for (const auto& e : ps.b) {
    const int64_t b = bit_length(e);
    if (b > b_bits) b_bits = b;
    limbs += e.size < 0 ? -(int64_t)e.size : e.size;
  }
  Params prm;
  if (!choose_params(a_bits, b_bits, ps.m, ps.k, ps.n, &prm)) return -1;
  const int64_t entries = (int64_t)ps.m * ps.k + (int64_t)ps.k * ps.n + (int64_t)ps.m * ps.n;
  const int64_t res = prm.P ? entries * prm.P * ((int64_t)1 << prm.lgN) * 4 : 0;
  const int64_t out = (int64_t)ps.m * ps.n * prm.out_limbs * 8;
  const int64_t desc = entries * 64 + 4096;
  return limbs * 8 + res + out + desc;
}

int Plan::build(std::vector<ProductSpec> prods, Workspace* ws) {
  if (built_) return set_error(kErrState, "plan already built");
  prods_ = std::move(prods);
  const int block_freqs = contract_block_freqs();
  params_.resize(prods_.size());
  zero_prod_.assign(prods_.size(), 0);

  std::map<std::pair<int, int>, Group> fwdg, invg;
  std::map<int, Group> recg;
  std::map<int, int64_t> rec_min_r;

  uint64_t out_entry = 0;
  for (size_t t = 0; t < prods_.size(); ++t) {
    ProductSpec& ps = prods_[t];
    const int m = ps.m, k = ps.k, n = ps.n;
    if (m < 0 || k < 0 || n < 0) return set_error(kErrArg, "negative dimension");
    if ((int64_t)ps.a.size() != (int64_t)m * k || (int64_t)ps.b.size() != (int64_t)k * n ||
        (int64_t)ps.c.size() != (int64_t)m * n)
      return set_error(kErrArg, "entry count does not match the dimensions");
    if (m > 65535 || k > 65535 || n > 65535) return set_error(kErrTooLarge, "dimension > 65535");
    int64_t a_bits = 0, b_bits = 0;
    for (auto& e : ps.a) {
      if (e.size != 0 && e.d == nullptr) return set_error(kErrArg, "null limb pointer");
      int64_t b = bit_length(e);
      if (b > a_bits) a_bits = b;
    }
    for (auto& e : ps.b) {
      if (e.size != 0 && e.d == nullptr) return set_error(kErrArg, "null limb pointer");
      int64_t b = bit_length(e);
      if (b > b_bits) b_bits = b;
    }
    Params prm;
    if (!choose_params(a_bits, b_bits, m, k, n, &prm))
      return set_error(kErrTooLarge, "product too large for a single transform (entries of " +
                                         std::to_string(a_bits) + " and " +
                                         std::to_string(b_bits) + " bits)");
    params_[t] = prm;
    const uint64_t first_out = out_entry;
    for (auto& c : ps.c) outs_.push_back(c);
    out_entry += ps.c.size();
    if (prm.P == 0 || m == 0 || n == 0) {
      zero_prod_[t] = 1;
      for (size_t e = 0; e < ps.c.size(); ++e) out_word_off_.push_back(-1);
      continue;
    }
    const int P = prm.P, lgN = prm.lgN, r = prm.r;
    const uint64_t N = (uint64_t)1 << lgN;
    const uint64_t poly = (uint64_t)P * N;
    // the contraction addresses a product's residues with 32-bit offsets
    if (((uint64_t)m * k + (uint64_t)k * n + (uint64_t)m * n) * poly >= (1ull << 32))
      return set_error(kErrTooLarge, "product needs more than 2^32 residue words");
    ProdDesc pd;
    pd.m = (uint16_t)m;
    pd.k = (uint16_t)k;
    pd.n = (uint16_t)n;
    pd.lgN = (uint16_t)lgN;
    pd.P = (uint16_t)P;
    pd.pad = (uint16_t)((m >= 3 ? 2 : 0) + (n >= 3 ? 1 : 0));  // contraction tile
    pd.a_res = n_res_;
    n_res_ += (uint64_t)m * k * poly;
    pd.b_res = n_res_;
    n_res_ += (uint64_t)k * n * poly;
    pd.c_res = n_res_;
    n_res_ += (uint64_t)m * n * poly;
    for (int side = 0; side < 2; ++side) {
      const auto& ents = side ? ps.b : ps.a;
      const uint64_t base = side ? pd.b_res : pd.a_res;
      for (size_t e = 0; e < ents.size(); ++e) {
        FwdDesc fd;
        const int64_t nl = ents[e].size < 0 ? -(int64_t)ents[e].size : ents[e].size;
        fd.limb_off = n_limbs_;
        n_limbs_ += (uint64_t)nl;
        fd.res_off = base + e * poly;
        fd.size = ents[e].size;
        fd.r = (uint32_t)r;
        fd.lgN = (uint16_t)lgN;
        fd.P = (uint16_t)P;
        uint64_t nc = ((uint64_t)nl * 64 + r - 1) / r;
        fd.ncoef = (uint32_t)(nc < N ? nc : N);
        auto& g = fwdg[{lgN, P * 16 + (r + 29) / 30}];
        g.P = P;
        g.lgN = lgN;
        if (r > g.max_r) g.max_r = r;
        g.idx.push_back((uint32_t)fwd_.size());
        fwd_.push_back(fd);
      }
    }
    const uint32_t prod_index = (uint32_t)pd_.size();
    pd_.push_back(pd);
    const int mode = context().contract_mode;
    const bool use_tc = contract_tc_eligible(m, k, n) &&
                        (mode == 2 || (mode == 0 && context().tc_pref[tc_bucket_k(k)][tc_bucket_mn(m, n)] == 1));
    if (use_tc) {
      if (k > tc_max_k_) tc_max_k_ = k;
      if (n > tc_max_n_) tc_max_n_ = n;
    }
    const uint64_t fstep = use_tc ? (uint64_t)kTcFreqsPerCta : (uint64_t)block_freqs;
    for (int j = 0; j < P; ++j)
      for (uint64_t h0 = 0; h0 < N; h0 += fstep) {
        ContractItem it;
        it.prod = prod_index;
        it.prime = (uint16_t)j;
        it.pad = 0;
        it.h0 = (uint32_t)h0;
        (use_tc ? tc_items_ : items_).push_back(it);
      }
    const uint64_t ncoef_c = (uint64_t)(prm.lenA + prm.lenB - 1);
    for (int e = 0; e < m * n; ++e) {
      InvDesc id;
      id.res_off = pd.c_res + (uint64_t)e * poly;
      id.out_word = n_out_words_;
      id.out_words = (uint32_t)(2 * prm.out_limbs);
      out_word_off_.push_back((int64_t)n_out_words_);
      n_out_words_ += id.out_words;
      id.r = (uint32_t)r;
      id.ncoef = (uint32_t)(ncoef_c < N ? ncoef_c : N);
      id.lgN = (uint16_t)lgN;
      id.P = (uint16_t)P;
      id.entry = (uint32_t)(first_out + e);
      const uint32_t ii = (uint32_t)inv_.size();
      inv_.push_back(id);
      auto& g = invg[{lgN, P}];
      g.P = P;
      g.lgN = lgN;
      g.idx.push_back(ii);
      auto& rg = recg[P];
      rg.P = P;
      rg.idx.push_back(ii);
      auto it = rec_min_r.find(P);
      if (it == rec_min_r.end() || r < it->second) rec_min_r[P] = r;
    }
  }
  if (out_entry > 0x7fffffffULL) return set_error(kErrTooLarge, "too many output entries");

  // launch groups and the shared index array
  // Transforms: team-sized classes (lgN >= 3) are merged into one launch per
  // digit count D, larger classes get one launch per (lgN, D); CTA work items
  // carry the class, and the largest classes come first so the long CTAs
  // start early.
  auto batch_classes = [&](std::map<std::pair<int, int>, Group>& classes, bool fwd,
                           std::vector<Group>& out) {
    std::map<std::pair<int, int>, Group> var;  // (0 = team, else lgN; D)
    for (auto& kv : classes) {
      Group& g = kv.second;
      const int D = fwd ? (g.max_r + 29) / 30 : 0;
      if (g.lgN < 3 || D > 7) {
        out.push_back(std::move(g));  // radix-2 path
        continue;
      }
      const bool team = ((int64_t)1 << g.lgN) <= (int64_t)fwd_team_points();
      // a CTA's shared memory follows the launch's largest class, so classes
      // above the team size get launches of their own
      Group& v = var[{team ? 0 : g.lgN, D}];
      v.batched = true;
      v.team = team;
      v.D = D;
      if (g.lgN > v.max_lgN) v.max_lgN = g.lgN;
      const size_t G = team ? (size_t)(fwd_team_points() >> g.lgN) : 1;
      for (size_t i = 0; i < g.idx.size(); i += G) {
        const size_t cnt = (g.idx.size() - i) < G ? (g.idx.size() - i) : G;
        CtaItem it;
        it.first = (uint32_t)idx_all_.size();
        it.count = (uint16_t)cnt;
        it.lgN = (uint8_t)g.lgN;
        it.P = (uint8_t)g.P;
        idx_all_.insert(idx_all_.end(), g.idx.begin() + i, g.idx.begin() + i + cnt);
        v.items.push_back(it);
      }
    }
    for (auto& kv : var) {
      Group& v = kv.second;
      std::stable_sort(v.items.begin(), v.items.end(),
                       [](const CtaItem& a, const CtaItem& b) { return a.lgN > b.lgN; });
      v.item_off = (uint32_t)cta_items_.size();
      cta_items_.insert(cta_items_.end(), v.items.begin(), v.items.end());
      out.push_back(std::move(v));
    }
  };
  batch_classes(fwdg, true, fwd_groups_);
  batch_classes(invg, false, inv_groups_);
  for (auto& kv : recg) {
    Group g = std::move(kv.second);
    g.max_r = (int)rec_min_r[g.P];  // narrowest r: sizes the CRT kernel's scratch
    // longest entries first (the warp that gets one works longest)
    std::stable_sort(g.idx.begin(), g.idx.end(), [&](uint32_t a, uint32_t b) {
      return inv_[a].out_words > inv_[b].out_words;
    });
    rec_groups_.push_back(std::move(g));
  }
  for (auto* gs : {&fwd_groups_, &inv_groups_, &rec_groups_})
    for (auto& g : *gs) {
      if (g.batched) continue;
      g.idx_off = (uint32_t)idx_all_.size();
      idx_all_.insert(idx_all_.end(), g.idx.begin(), g.idx.end());
    }

  // device and pinned buffers
  Context& ctx = context();
  if (!ctx.ready) return set_error(kErrState, "not set up (call hw_mpz_setup)");
  CU(cudaSetDevice(ctx.device), "cudaSetDevice");
  auto align16 = [](size_t x) { return (x + 15) & ~(size_t)15; };
  off_fwd_ = 0;
  off_inv_ = align16(off_fwd_ + fwd_.size() * sizeof(FwdDesc));
  off_pd_ = align16(off_inv_ + inv_.size() * sizeof(InvDesc));
  off_items_ = align16(off_pd_ + pd_.size() * sizeof(ProdDesc));
  off_tc_ = align16(off_items_ + items_.size() * sizeof(ContractItem));
  off_idx_ = align16(off_tc_ + tc_items_.size() * sizeof(ContractItem));
  off_cta_ = align16(off_idx_ + idx_all_.size() * sizeof(uint32_t));
  desc_bytes_ = align16(off_cta_ + cta_items_.size() * sizeof(CtaItem));
  ws_ = ws ? ws : &own_;
  int st = ws_->reserve(n_limbs_, n_res_, n_out_words_, outs_.size(), desc_bytes_);
  if (st) return st;
  uint8_t* hd = ws_->h_desc;
  if (!fwd_.empty()) std::memcpy(hd + off_fwd_, fwd_.data(), fwd_.size() * sizeof(FwdDesc));
  if (!inv_.empty()) std::memcpy(hd + off_inv_, inv_.data(), inv_.size() * sizeof(InvDesc));
  if (!pd_.empty()) std::memcpy(hd + off_pd_, pd_.data(), pd_.size() * sizeof(ProdDesc));
  if (!items_.empty())
    std::memcpy(hd + off_items_, items_.data(), items_.size() * sizeof(ContractItem));
  if (!tc_items_.empty())
    std::memcpy(hd + off_tc_, tc_items_.data(), tc_items_.size() * sizeof(ContractItem));
  if (!idx_all_.empty())
    std::memcpy(hd + off_idx_, idx_all_.data(), idx_all_.size() * sizeof(uint32_t));
  if (!cta_items_.empty())
    std::memcpy(hd + off_cta_, cta_items_.data(), cta_items_.size() * sizeof(CtaItem));
  d_fwd_ = reinterpret_cast<FwdDesc*>(ws_->d_desc + off_fwd_);
  d_inv_ = reinterpret_cast<InvDesc*>(ws_->d_desc + off_inv_);
  d_pd_ = reinterpret_cast<ProdDesc*>(ws_->d_desc + off_pd_);
  d_items_ = reinterpret_cast<ContractItem*>(ws_->d_desc + off_items_);
  d_tc_items_ = reinterpret_cast<ContractItem*>(ws_->d_desc + off_tc_);
  d_idx_ = reinterpret_cast<uint32_t*>(ws_->d_desc + off_idx_);
  d_cta_ = reinterpret_cast<CtaItem*>(ws_->d_desc + off_cta_);
  launches_ = (int64_t)fwd_groups_.size() + (items_.empty() ? 0 : 1) +
              (tc_items_.empty() ? 0 : 1) +
              (int64_t)inv_groups_.size() + (int64_t)rec_groups_.size();
  built_ = true;
  return kOk;
}

int Plan::upload(cudaStream_t st) {
  if (!built_) return set_error(kErrState, "plan not built");
  // flat list of (source, destination, limbs) to gather in parallel
  struct Copy {
    const uint64_t* src;
    uint64_t dst;
    int64_t n;
  };
  std::vector<Copy> copies;
  copies.reserve(fwd_.size());
  size_t fi = 0;
  for (size_t t = 0; t < prods_.size(); ++t) {
    if (zero_prod_[t]) continue;
    const ProductSpec& ps = prods_[t];
    for (int side = 0; side < 2; ++side) {
      const auto& ents = side ? ps.b : ps.a;
      for (const auto& e : ents) {
        const FwdDesc& fd = fwd_[fi++];
        const int64_t nl = e.size < 0 ? -(int64_t)e.size : e.size;
        if (nl != (fd.size < 0 ? -(int64_t)fd.size : fd.size) || (e.size < 0) != (fd.size < 0))
          return set_error(kErrArg, "inputs changed size or sign since the plan was built");
        if (nl) copies.push_back(Copy{e.d, fd.limb_off, nl});
      }
    }
  }
  uint64_t* hl = ws_->h_limbs;
  parallel_chunks(copies.size(), (size_t)n_limbs_ * 8, [&](size_t lo, size_t hi) {
    for (size_t i = lo; i < hi; ++i)
      std::memcpy(hl + copies[i].dst, copies[i].src, (size_t)copies[i].n * 8);
  });
  if (desc_bytes_)
    CU(cudaMemcpyAsync(ws_->d_desc, ws_->h_desc, desc_bytes_, cudaMemcpyHostToDevice, st),
       "H2D descriptors");
  CU(cudaMemsetAsync(ws_->d_status, 0, sizeof(int), st), "clear status");
  if (n_limbs_)
    CU(cudaMemcpyAsync(ws_->d_limbs, hl, n_limbs_ * 8, cudaMemcpyHostToDevice, st), "H2D limbs");
  return kOk;
}

int Plan::execute(cudaStream_t st) {
  if (!built_) return set_error(kErrState, "plan not built");
  if (!use_graph_ || timing_) return launch_all(st, timing_);
  if (!graph_exec_) {
    CU(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal), "cudaStreamBeginCapture");
    const int rc = launch_all(st, false);
    cudaGraph_t g = nullptr;
    const cudaError_t e = cudaStreamEndCapture(st, &g);
    if (rc) {
      if (g) cudaGraphDestroy(g);
      return rc;
    }
    if (e != cudaSuccess) return cuda_fail(e, "cudaStreamEndCapture");
    graph_ = g;
    CU(cudaGraphInstantiate(&graph_exec_, graph_, 0), "cudaGraphInstantiate");
  }
  CU(cudaGraphLaunch(graph_exec_, st), "cudaGraphLaunch");
  return kOk;
}

int Plan::launch_all(cudaStream_t st, bool timed) {
  const Context& ctx = context();
  cudaEvent_t ev[kStages + 1] = {};
  if (timed) {
    for (auto& e : ev) {
      CU(cudaEventCreate(&e), "cudaEventCreate");
      events_.push_back(e);
    }
    CU(cudaEventRecord(ev[0], st), "cudaEventRecord");
  }
  for (const Group& g : fwd_groups_) {
    if (g.batched)
      CU(launch_fwd_items(d_fwd_, d_idx_, d_cta_ + g.item_off, (int)g.items.size(), g.D, g.team,
                          g.max_lgN, ws_->d_limbs, ws_->d_res, ctx.d_twf, st),
         "split+forward NTT launch");
    else
      CU(launch_split_fwd(d_fwd_, d_idx_ + g.idx_off, (int)g.idx.size(), g.P, g.lgN,
                          ws_->d_limbs, ws_->d_res, ctx.d_twf, st),
         "split+forward NTT launch");
  }
  if (timed) CU(cudaEventRecord(ev[1], st), "cudaEventRecord");
  if (!items_.empty())
    CU(launch_contract(d_pd_, d_items_, (int)items_.size(), ws_->d_res, st), "contraction launch");
  if (!tc_items_.empty())
    CU(launch_contract_tc(d_pd_, d_tc_items_, (int)tc_items_.size(), ws_->d_res, kTcFreqsPerCta,
                          tc_max_k_, tc_max_n_, ws_->d_status, st),
       "tensor-core contraction launch");
  if (timed) CU(cudaEventRecord(ev[2], st), "cudaEventRecord");
  for (const Group& g : inv_groups_) {
    if (g.batched)
      CU(launch_inv_items(d_inv_, d_idx_, d_cta_ + g.item_off, (int)g.items.size(), g.team,
                          g.max_lgN, ws_->d_res, ctx.d_twi, st),
         "inverse NTT launch");
    else
      CU(launch_inv_ntt(d_inv_, d_idx_ + g.idx_off, (int)g.idx.size(), g.P, g.lgN, ws_->d_res,
                        ctx.d_twi, st),
         "inverse NTT launch");
  }
  if (timed) CU(cudaEventRecord(ev[3], st), "cudaEventRecord");
  for (const Group& g : rec_groups_)
    CU(launch_crt_recompose(d_inv_, d_idx_ + g.idx_off, (int)g.idx.size(), g.P, ws_->d_res,
                            ws_->d_out, ws_->d_sizes, g.max_r, st),
       "CRT+recompose launch");
  if (timed) CU(cudaEventRecord(ev[4], st), "cudaEventRecord");
  return kOk;
}

int Plan::stage_times(float ms[kStages], int64_t* executes) {
  for (int s = 0; s < kStages; ++s) ms[s] = 0.f;
  const size_t per = kStages + 1;
  const int64_t n = (int64_t)(events_.size() / per);
  if (executes) *executes = n;
  if (n == 0) return kOk;
  CU(cudaEventSynchronize(events_.back()), "cudaEventSynchronize");
  for (int64_t i = 0; i < n; ++i)
    for (int s = 0; s < kStages; ++s) {
      float t = 0.f;
      CU(cudaEventElapsedTime(&t, events_[i * per + s], events_[i * per + s + 1]),
         "cudaEventElapsedTime");
      ms[s] += t;
    }
  for (cudaEvent_t e : events_) cudaEventDestroy(e);
  events_.clear();
  return kOk;
}

void Plan::stage_launches(int64_t out[kStages]) const {
  out[0] = (int64_t)fwd_groups_.size();
  out[1] = (items_.empty() ? 0 : 1) + (tc_items_.empty() ? 0 : 1);
  out[2] = (int64_t)inv_groups_.size();
  out[3] = (int64_t)rec_groups_.size();
}

int Plan::download(cudaStream_t st) {
  if (!built_) return set_error(kErrState, "plan not built");
  int32_t* hs = ws_->h_sizes;
  uint32_t* ho = ws_->h_out;
  if (!outs_.empty() && !inv_.empty())
    CU(cudaMemcpyAsync(hs, ws_->d_sizes, outs_.size() * sizeof(int32_t), cudaMemcpyDeviceToHost,
                       st),
       "D2H sizes");
  if (n_out_words_)
    CU(cudaMemcpyAsync(ho, ws_->d_out, n_out_words_ * 4, cudaMemcpyDeviceToHost, st), "D2H words");
  int kstatus = 0;
  CU(cudaMemcpyAsync(&kstatus, ws_->d_status, sizeof(int), cudaMemcpyDeviceToHost, st),
     "D2H status");
  CU(cudaStreamSynchronize(st), "kernel execution");
  if (kstatus)
    return set_error(kErrTimeout, "a tensor-core contraction wait timed out; results invalid");
  // capacity check first (serial, cheap), then the copies in parallel
  int status = kOk;
  std::vector<uint8_t> ok(outs_.size(), 1);
  for (size_t e = 0; e < outs_.size(); ++e) {
    const OutRef& o = outs_[e];
    const int32_t sz = out_word_off_[e] < 0 ? 0 : hs[e];
    const int64_t nl = sz < 0 ? -(int64_t)sz : sz;
    if (o.mpz) {
      __mpz_struct* z = static_cast<__mpz_struct*>(o.mpz);
      if (z->_mp_alloc < nl) __gmpz_realloc(z, (mp_size_t)nl);  // GMP's allocator
    } else if (nl > o.cap) {
      status = set_error(kErrCapacity, "output entry " + std::to_string(e) + " needs " +
                                           std::to_string(nl) + " limbs, capacity " +
                                           std::to_string(o.cap));
      ok[e] = 0;
      if (o.size) *o.size = 0;
    }
  }
  parallel_chunks(outs_.size(), (size_t)n_out_words_ * 4, [&](size_t lo, size_t hi) {
    for (size_t e = lo; e < hi; ++e) {
      if (!ok[e]) continue;
      const OutRef& o = outs_[e];
      const int64_t woff = out_word_off_[e];
      const int32_t sz = woff < 0 ? 0 : hs[e];
      const int64_t nl = sz < 0 ? -(int64_t)sz : sz;
      const uint64_t* src = woff < 0 ? nullptr : reinterpret_cast<const uint64_t*>(ho + woff);
      if (o.mpz) {
        __mpz_struct* z = static_cast<__mpz_struct*>(o.mpz);
        if (nl) std::memcpy(z->_mp_d, src, (size_t)nl * 8);
        z->_mp_size = sz;
      } else {
        if (nl) std::memcpy(o.d, src, (size_t)nl * 8);
        if (o.size) *o.size = sz;
      }
    }
  });
  return status;
}

}  // namespace mpzmm
