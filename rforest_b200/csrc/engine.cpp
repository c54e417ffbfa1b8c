// Batch engine (see engine.h).
#include "engine.h"

#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
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

int cuda_status(cudaError_t e, const char* what) {
  return e == cudaSuccess ? kOk : cuda_fail(e, what);
}

#define CU(call, what)                          \
  do {                                          \
    cudaError_t _e = (call);                    \
    if (_e != cudaSuccess) return cuda_fail(_e, what); \
  } while (0)

}  // namespace

int64_t bit_length(const EntryRef& e) {
  int64_t i = (e.size < 0 ? -(int64_t)e.size : e.size) - 1;
  // a non-normalised top limb of zero is tolerated: scan down
  while (i >= 0 && e.d[i] == 0) --i;
  if (i < 0) return 0;
  return 64 * i + (64 - __builtin_clzll(e.d[i]));
}

namespace {

}  // namespace

int set_error(int status, const std::string& msg) {
  g_err = msg;
  return status;
}
const char* last_error() { return g_err.c_str(); }

Context& context() { return g_ctx; }

namespace {
std::atomic<int> g_test_stall_tc{0};
std::atomic<int> g_test_fail_alloc{0};
bool take_one(std::atomic<int>& c) {
  int v = c.load();
  while (v > 0)
    if (c.compare_exchange_weak(v, v - 1)) return true;
  return false;
}
}  // namespace

void set_test_stall_tc(int count) { g_test_stall_tc = count > 0 ? count : 0; }
void set_test_fail_alloc(int count) { g_test_fail_alloc = count > 0 ? count : 0; }
int test_stall_tc() { return g_test_stall_tc.load(); }
int test_fail_alloc() { return g_test_fail_alloc.load(); }
bool take_test_stall_tc() { return take_one(g_test_stall_tc); }
bool take_test_fail_alloc() { return take_one(g_test_fail_alloc); }

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

// ---- pinned host memory known to the library ----
namespace {
struct HostRange {
  size_t bytes;
  bool owned;  // allocated here (else registered)
};
std::mutex g_host_mu;
std::map<uintptr_t, HostRange> g_host;
}  // namespace

std::vector<std::pair<uintptr_t, size_t>> pinned_ranges() {
  std::lock_guard<std::mutex> lk(g_host_mu);
  std::vector<std::pair<uintptr_t, size_t>> v;
  v.reserve(g_host.size());
  for (const auto& kv : g_host) v.emplace_back(kv.first, kv.second.bytes);
  return v;  // sorted by start
}

bool in_ranges(const std::vector<std::pair<uintptr_t, size_t>>& v, const void* p, size_t bytes) {
  if (!p || !bytes || v.empty()) return false;
  const uintptr_t a = reinterpret_cast<uintptr_t>(p);
  auto it = std::upper_bound(v.begin(), v.end(), std::make_pair(a, ~(size_t)0));
  if (it == v.begin()) return false;
  --it;
  return a - it->first <= it->second && bytes <= it->second - (a - it->first);
}

uintptr_t range_end(const std::vector<std::pair<uintptr_t, size_t>>& v, const void* p,
                    size_t bytes) {
  if (!in_ranges(v, p, bytes)) return 0;
  const uintptr_t a = reinterpret_cast<uintptr_t>(p);
  auto it = std::upper_bound(v.begin(), v.end(), std::make_pair(a, ~(size_t)0));
  --it;
  return it->first + it->second;
}

bool host_range_pinned(const void* p, size_t bytes) { return in_ranges(pinned_ranges(), p, bytes); }

int host_alloc(size_t bytes, void** out) {
  if (!out) return set_error(kErrArg, "null output pointer");
  *out = nullptr;
  if (!bytes) return set_error(kErrArg, "zero-byte host allocation");
  int st = ensure_setup(-1);
  if (st) return st;
  void* p = nullptr;
  cudaError_t e = cudaHostAlloc(&p, bytes, cudaHostAllocPortable);
  if (e != cudaSuccess)
    return set_error(kErrNoMem, std::string("cudaHostAlloc of ") + std::to_string(bytes) +
                                    " bytes: " + cudaGetErrorString(e));
  std::lock_guard<std::mutex> lk(g_host_mu);
  g_host[reinterpret_cast<uintptr_t>(p)] = HostRange{bytes, true};
  *out = p;
  return kOk;
}

int host_free(void* p) {
  if (!p) return kOk;
  std::lock_guard<std::mutex> lk(g_host_mu);
  auto it = g_host.find(reinterpret_cast<uintptr_t>(p));
  if (it == g_host.end() || !it->second.owned)
    return set_error(kErrArg, "pointer was not allocated by mpzmm_host_alloc");
  g_host.erase(it);
  CU(cudaFreeHost(p), "cudaFreeHost");
  return kOk;
}

int host_register(void* p, size_t bytes) {
  if (!p || !bytes) return set_error(kErrArg, "null or empty host range");
  int st = ensure_setup(-1);
  if (st) return st;
  CU(cudaHostRegister(p, bytes, cudaHostRegisterPortable), "cudaHostRegister");
  std::lock_guard<std::mutex> lk(g_host_mu);
  g_host[reinterpret_cast<uintptr_t>(p)] = HostRange{bytes, false};
  return kOk;
}

int host_unregister(void* p) {
  std::lock_guard<std::mutex> lk(g_host_mu);
  auto it = g_host.find(reinterpret_cast<uintptr_t>(p));
  if (it == g_host.end() || it->second.owned)
    return set_error(kErrArg, "pointer was not registered by mpzmm_host_register");
  g_host.erase(it);
  CU(cudaHostUnregister(p), "cudaHostUnregister");
  return kOk;
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
  {
    const size_t nt = (size_t)kMaxPrimes * kTwistEntries;
    const size_t bytes = nt * (2 * sizeof(uint2) + 2 * sizeof(uint32_t));
    CU(cudaMalloc(&g_ctx.d_twist, bytes), "cudaMalloc twist tables");
    uint2* hf = static_cast<uint2*>(g_ctx.d_twist);
    uint2* hi = hf + nt;
    uint32_t* lf = reinterpret_cast<uint32_t*>(hi + nt);
    uint32_t* li = lf + nt;
    CU(cudaMemcpy(hf, M.twh_f.data(), nt * sizeof(uint2), cudaMemcpyHostToDevice), "copy twists");
    CU(cudaMemcpy(hi, M.twh_i.data(), nt * sizeof(uint2), cudaMemcpyHostToDevice), "copy twists");
    CU(cudaMemcpy(lf, M.twl_f.data(), nt * sizeof(uint32_t), cudaMemcpyHostToDevice),
       "copy twists");
    CU(cudaMemcpy(li, M.twl_i.data(), nt * sizeof(uint32_t), cudaMemcpyHostToDevice),
       "copy twists");
    g_ctx.twist_f = TwistTab{hf, lf};
    g_ctx.twist_i = TwistTab{hi, li};
  }
  CU(cudaStreamCreateWithFlags(&g_ctx.stream, cudaStreamNonBlocking), "cudaStreamCreate");
  g_ctx.ws = new Workspace;
  if (const char* cb = std::getenv("MPZMM_CHECK_BOUNDS")) g_ctx.check_bounds = cb[0] == '1';
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
  cudaFree(g_ctx.d_twist);
  {
    std::lock_guard<std::mutex> wl(workspace_mutex());
    for (cudaStream_t s : g_ctx.pipe_st) {
      cudaStreamSynchronize(s);
      cudaStreamDestroy(s);
    }
    for (cudaStream_t s : {g_ctx.pipe_in, g_ctx.pipe_out})
      if (s) {
        cudaStreamSynchronize(s);
        cudaStreamDestroy(s);
      }
    for (size_t i = 1; i < g_ctx.pipe_ws.size(); ++i) delete g_ctx.pipe_ws[i];
    if (g_ctx.pipe_ev) cudaEventDestroy(g_ctx.pipe_ev);
    for (auto* v : {&g_ctx.pipe_ev_in, &g_ctx.pipe_ev_exec, &g_ctx.pipe_ev_out})
      for (cudaEvent_t e : *v) cudaEventDestroy(e);
    for (cudaEvent_t e : g_ctx.tl_ev) cudaEventDestroy(e);
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
                       size_t desc_bytes, size_t stage_limbs, size_t stage_out_words) {
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
    if (take_test_fail_alloc())
      return set_error(kErrNoMem, "injected device allocation failure (test option)");
    auto alloc = [&](size_t count) {
      if (async_stream && pool)
        return cudaMallocFromPoolAsync((void**)p, count * elem, pool, async_stream);
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
    if (*p) {
      if (retire_host)
        retired_host.push_back(*p);
      else
        cudaFreeHost(*p);
    }
    *p = nullptr;
    cap = 0;
    if (take_test_fail_alloc())
      return set_error(kErrNoMem, "injected pinned-host allocation failure (test option)");
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
    cudaError_t e =
        async_stream
            ? (pool ? cudaMallocFromPoolAsync((void**)&d_status, sizeof(int), pool, async_stream)
                    : cudaMallocAsync((void**)&d_status, sizeof(int), async_stream))
            : cudaMalloc((void**)&d_status, sizeof(int));
    if (e != cudaSuccess) {
      d_status = nullptr;
      return set_error(kErrNoMem, std::string("cudaMalloc(status): ") + cudaGetErrorString(e));
    }
    device_bytes += (int64_t)sizeof(int);
  }
  if ((st = grow_host(&h_limbs, hcap_limbs, stage_limbs, 8))) return st;
  if ((st = grow_host(&h_out, hcap_out, stage_out_words, 4))) return st;
  if ((st = grow_host(&h_sizes, hcap_sizes, sizes, 4))) return st;
  if ((st = grow_host(&h_desc, hcap_desc, desc_bytes, 1))) return st;
  if (!h_status) {
    cudaError_t e = cudaMallocHost((void**)&h_status, sizeof(int));
    if (e != cudaSuccess) {
      h_status = nullptr;
      return set_error(kErrNoMem, std::string("cudaMallocHost(status): ") + cudaGetErrorString(e));
    }
  }
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

int Workspace::ensure_side() {
  if (fork_ev) return kOk;
  for (int i = 0; i < kSideStreams; ++i) {
    CU(cudaStreamCreateWithFlags(&side[i], cudaStreamNonBlocking), "cudaStreamCreate");
    CU(cudaEventCreateWithFlags(&join_ev[i], cudaEventDisableTiming), "cudaEventCreate");
  }
  CU(cudaEventCreateWithFlags(&fork_ev, cudaEventDisableTiming), "cudaEventCreate");
  return kOk;
}

void Workspace::release() {
  for (int i = 0; i < kSideStreams; ++i) {
    if (side[i]) cudaStreamDestroy(side[i]);
    if (join_ev[i]) cudaEventDestroy(join_ev[i]);
    side[i] = nullptr;
    join_ev[i] = nullptr;
  }
  if (fork_ev) cudaEventDestroy(fork_ev);
  fork_ev = nullptr;
  release_device();
  for (void* p : retired_host) cudaFreeHost(p);
  retired_host.clear();
  cudaFreeHost(h_limbs);
  cudaFreeHost(h_out);
  cudaFreeHost(h_sizes);
  cudaFreeHost(h_desc);
  cudaFreeHost(h_status);
  h_limbs = nullptr;
  h_out = nullptr;
  h_sizes = nullptr;
  h_desc = nullptr;
  h_status = nullptr;
  hcap_limbs = hcap_out = hcap_sizes = hcap_desc = 0;
}

// Largest bit length among entries: only the longest entries can hold it,
// so only their top limbs are read (each a likely cache miss) unless none of
// them is normalised.
static int64_t max_bits(const std::vector<EntryRef>& ents, int64_t* limbs) {
  int64_t max_nl = 0, bits = 0;
  for (const auto& e : ents) {
    const int64_t nl = e.size < 0 ? -(int64_t)e.size : e.size;
    *limbs += nl;
    if (nl > max_nl) max_nl = nl;
  }
  if (!max_nl) return 0;
  for (const auto& e : ents)
    if ((e.size < 0 ? -(int64_t)e.size : e.size) == max_nl) {
      const int64_t b = bit_length(e);
      if (b > bits) bits = b;
    }
  if (bits <= 64 * (max_nl - 1))
    for (const auto& e : ents) {
      const int64_t b = bit_length(e);
      if (b > bits) bits = b;
    }
  return bits;
}

int64_t estimate_device_bytes(const ProductSpec& ps, int64_t* host_bytes) {
  int64_t limbs = 0;
  const int64_t a_bits = max_bits(ps.a, &limbs);
  const int64_t b_bits = max_bits(ps.b, &limbs);
  Params prm;
  if (!choose_params(a_bits, b_bits, ps.m, ps.k, ps.n, &prm)) return -1;
  const int64_t entries = (int64_t)ps.m * ps.k + (int64_t)ps.k * ps.n + (int64_t)ps.m * ps.n;
  const int64_t res = prm.P ? entries * prm.P * ((int64_t)1 << prm.lgN) * 4 : 0;
  const int64_t out = (int64_t)ps.m * ps.n * prm.out_limbs * 8;
  const int64_t desc = entries * 64 + 4096;
  if (host_bytes) *host_bytes = limbs * 8 + out;
  return limbs * 8 + res + out + desc;
}

int Workspace::reserve_staging(size_t stage_limbs, size_t stage_out_words, size_t sizes,
                               size_t desc_bytes) {
  auto grow = [this](auto** p, size_t& cap, size_t want, size_t elem) -> int {
    if (want <= cap) return kOk;
    if (*p) {
      if (retire_host)
        retired_host.push_back(*p);
      else
        cudaFreeHost(*p);
    }
    *p = nullptr;
    cap = 0;
    if (take_test_fail_alloc())
      return set_error(kErrNoMem, "injected pinned-host allocation failure (test option)");
    const cudaError_t e = cudaMallocHost((void**)p, want * elem);
    if (e != cudaSuccess) {
      *p = nullptr;
      return set_error(kErrNoMem, std::string("cudaMallocHost of ") +
                                      std::to_string(want * elem) + " bytes: " +
                                      cudaGetErrorString(e));
    }
    cap = want;
    return kOk;
  };
  int st = grow(&h_limbs, hcap_limbs, stage_limbs, 8);
  if (!st) st = grow(&h_out, hcap_out, stage_out_words, 4);
  if (!st) st = grow(&h_sizes, hcap_sizes, sizes, 4);
  if (!st) st = grow(&h_desc, hcap_desc, desc_bytes, 1);
  return st;
}

// Checks one product, finds its operands' bit lengths and its transform
// parameters; returns a status (with the message in *msg when asked).
static int plan_product(const ProductSpec& ps, Params* prm, std::string* msg) {
  auto fail = [&](int code, const std::string& m) {
    if (msg) *msg = m;
    return code;
  };
  const int m = ps.m, k = ps.k, n = ps.n;
  if (m < 0 || k < 0 || n < 0) return fail(kErrArg, "negative dimension");
  if ((int64_t)ps.a.size() != (int64_t)m * k || (int64_t)ps.b.size() != (int64_t)k * n ||
      (int64_t)ps.c.size() != (int64_t)m * n)
    return fail(kErrArg, "entry count does not match the dimensions");
  if (m > 65535 || k > 65535 || n > 65535) return fail(kErrTooLarge, "dimension > 65535");
  int64_t a_bits = 0, b_bits = 0;
  for (int side = 0; side < 2; ++side) {
    const auto& ents = side ? ps.b : ps.a;
    int64_t& bits = side ? b_bits : a_bits;
    if (!side && ps.dev_a) {  // values on the device: plan for the bound
      bits = 64 * ps.dev_a->cap_limbs;
      continue;
    }
    // only the longest entries can hold the largest bit length: read their
    // top limbs (each read of a caller's limb is a likely cache miss, so
    // they are prefetched together first), and scan everything only when
    // none of those is normalised
    int64_t max_nl = 0;
    for (const auto& e : ents) {
      if (e.size != 0 && e.d == nullptr) return fail(kErrArg, "null limb pointer");
      const int64_t nl = e.size < 0 ? -(int64_t)e.size : e.size;
      if (nl > max_nl) max_nl = nl;
    }
    if (!max_nl) continue;
    for (const auto& e : ents)
      if ((e.size < 0 ? -(int64_t)e.size : e.size) == max_nl)
        __builtin_prefetch(e.d + max_nl - 1);
    for (const auto& e : ents) {
      if ((e.size < 0 ? -(int64_t)e.size : e.size) != max_nl) continue;
      const int64_t b = bit_length(e);
      if (b > bits) bits = b;
    }
    if (bits <= 64 * (max_nl - 1))
      for (const auto& e : ents) {
        const int64_t b = bit_length(e);
        if (b > bits) bits = b;
      }
  }
  if (!choose_params(a_bits, b_bits, m, k, n, prm))
    return fail(kErrTooLarge, "product too large for a single transform (entries of " +
                                  std::to_string(a_bits) + " and " + std::to_string(b_bits) +
                                  " bits)");
  return kOk;
}

int Plan::build(std::vector<ProductSpec> prods, Workspace* ws) {
  const int r = prepare(std::move(prods));
  return r ? r : bind(ws);
}

int Plan::prepare(std::vector<ProductSpec> prods) {
  if (built_ || prepared_) return set_error(kErrState, "plan already built");
  check_bounds_ = context().check_bounds;
  prods_ = std::move(prods);
  const int block_freqs = contract_block_freqs();
  params_.resize(prods_.size());
  zero_prod_.assign(prods_.size(), 0);

  std::map<std::pair<int, int>, Group> fwdg, invg;
  std::map<int, Group> recg;
  std::map<int, int64_t> rec_min_r;

  uint64_t out_entry = 0;
  const uint64_t* host_end = nullptr;  // end of the previous entry's host limbs
  uintptr_t run_pinned_end = 0;        // end of the pinned range of the current run (0: none)
  const auto pinned = pinned_ranges();
  in_runs_.clear();
  // pass 1, across host threads: checks, operand bit lengths, parameters
  // (independent per product); the first failing product's error is then
  // reported from this thread
  std::vector<int> bad(prods_.size(), 0);
  {
    size_t work = 0;
    for (const auto& ps : prods_) work += ps.a.size() + ps.b.size();
    parallel_chunks(prods_.size(), work * 4096, [&](size_t lo, size_t hi) {
      for (size_t t = lo; t < hi; ++t) bad[t] = plan_product(prods_[t], &params_[t], nullptr);
    });
  }
  for (size_t t = 0; t < prods_.size(); ++t)
    if (bad[t]) {
      std::string msg;
      plan_product(prods_[t], &params_[t], &msg);
      return set_error(bad[t], msg);
    }
  // pass 2, in order: offsets and descriptors
  for (size_t t = 0; t < prods_.size(); ++t) {
    ProductSpec& ps = prods_[t];
    const int m = ps.m, k = ps.k, n = ps.n;
    const Params prm = params_[t];
    const uint64_t first_out = out_entry;
    prod_first_out_.push_back((size_t)first_out);
    for (auto& c : ps.c) outs_.push_back(c);
    out_entry += ps.c.size();
    if (prm.P == 0 || m == 0 || n == 0) {
      zero_prod_[t] = 1;
      for (size_t e = 0; e < ps.c.size(); ++e) {
        out_word_off_.push_back(-1);
        out_limbs_.push_back(0);
      }
      continue;
    }
    const int P = prm.P, lgN = prm.lgN, r = prm.r;
    const uint64_t N = (uint64_t)1 << lgN;
    const uint64_t poly = (uint64_t)P * N;
    // the contraction addresses a product's residues with 32-bit offsets
    if (((uint64_t)m * k + (uint64_t)k * n + (uint64_t)m * n) * poly + 16 >= (1ull << 32))
      return set_error(kErrTooLarge, "product needs more than 2^32 residue words");
    ProdDesc pd;
    pd.m = (uint16_t)m;
    pd.k = (uint16_t)k;
    pd.n = (uint16_t)n;
    pd.lgN = (uint16_t)lgN;
    pd.P = (uint16_t)P;
    pd.pad = (uint16_t)contract_tile(m, n);
    n_res_ = (n_res_ + 7) & ~(uint64_t)7;  // 32-byte aligned polynomials (vector loads)
    pd.a_res = n_res_;
    n_res_ += (uint64_t)m * k * poly;
    n_res_ = (n_res_ + 7) & ~(uint64_t)7;  // 32-byte aligned polynomials (vector loads)
    pd.b_res = n_res_;
    n_res_ += (uint64_t)k * n * poly;
    n_res_ = (n_res_ + 7) & ~(uint64_t)7;  // 32-byte aligned polynomials (vector loads)
    pd.c_res = n_res_;
    n_res_ += (uint64_t)m * n * poly;
    // contraction engine: tensor cores where the mode or the autotuner says
    // so, for transforms of 8 .. 2^15 points (their operands are written in
    // the frequency-blocked layout by the one-CTA forward kernels)
    const int mode = context().contract_mode;
    const bool use_tc = contract_tc_eligible(m, k, n) && lgN >= 3 && lgN <= kMaxLgNOneCta &&
                        (mode == 2 || (mode == 0 && context().tc_pref[tc_bucket_k(k)]
                                                                     [tc_bucket_mn(m, n)] == 1));
    if (fixed_b_ && ps.dev_a)
      return set_error(kErrArg, "a plan that keeps B's transforms takes host operands only");
    for (int side = 0; side < 2; ++side) {
      // one class per product; operands of tensor-core products (blocked
      // layout) get launches of their own, so the plain kernels stay as
      // lean, and so do B operands whose transforms the plan keeps
      const bool b_only = fixed_b_ && side == 1;
      Group& fg =
          fwdg[{lgN, P * 16 + (r + 29) / 30 + (use_tc ? 1024 : 0) + (b_only ? 2048 : 0)}];
      fg.tiled = use_tc;
      fg.b_only = b_only;
      fg.P = P;
      fg.lgN = lgN;
      if (r > fg.max_r) fg.max_r = r;
      if (fixed_b_) host_end = nullptr;  // runs never mix the two operands
      const auto& ents = side ? ps.b : ps.a;
      const uint64_t base = side ? pd.b_res : pd.a_res;
      if (!side && ps.dev_a) {
        // the operand's limbs are copied on the device as one span (256-byte
        // aligned); its sizes are written into the descriptors on the device
        const DeviceOperand& da = *ps.dev_a;
        n_limbs_ = (n_limbs_ + 31) & ~(uint64_t)31;
        const uint64_t span0 = n_limbs_;
        dev_runs_.push_back(DevRun{da.limbs, span0, da.span_limbs});
        dev_fixes_.push_back(DevFix{da.sizes, (uint32_t)fwd_.size(), (uint32_t)ents.size()});
        n_limbs_ += da.span_limbs;
        host_end = nullptr;
        for (size_t e = 0; e < ents.size(); ++e) {
          FwdDesc fd;
          fd.limb_off = span0 + (uint64_t)da.offs[e];
          fd.res_off = base + e * poly;
          fd.size = (int32_t)da.cap_limbs;  // replaced on the device
          fd.r = (uint32_t)r;
          fd.lgN = (uint16_t)lgN;
          fd.P = (uint16_t)P;
          fd.ncoef = (uint32_t)N;  // replaced on the device
          if (use_tc) {  // the operand block, entry e of it
            fd.res_off = base;
            fd.tile_np = (uint32_t)ents.size();
            fd.tile_e = (uint32_t)e;
          }
          fg.idx.push_back((uint32_t)fwd_.size());
          fwd_.push_back(fd);
        }
        continue;
      }
      for (size_t e = 0; e < ents.size(); ++e) {
        FwdDesc fd;
        const int64_t nl = ents[e].size < 0 ? -(int64_t)ents[e].size : ents[e].size;
        if (nl) {
          // Copy runs: an entry continues the current run when it follows
          // the previous one in host memory -- directly, or, inside one
          // pinned range, after a short gap (the run then copies the gap
          // too and the device layout mirrors it).  A new run starts at the
          // same address modulo 256 bytes as its host limbs, so the copy
          // engine moves aligned bursts.
          const uint64_t* d = ents[e].d;
          const uintptr_t dend = reinterpret_cast<uintptr_t>(d + nl);
          bool join = false;
          if (host_end && (!run_pinned_end || dend <= run_pinned_end)) {
            if (d == host_end) {
              join = true;
            } else if (run_pinned_end && d > host_end && d - host_end <= kRunGapLimbs) {
              n_limbs_ += (uint64_t)(d - host_end);
              join = true;
            }
          }
          if (join) {
            in_runs_.back().n = n_limbs_ + (uint64_t)nl - in_runs_.back().dev;
          } else {
            run_pinned_end = range_end(pinned, d, (size_t)nl * 8);
            const uint64_t want = (reinterpret_cast<uintptr_t>(d) >> 3) & 31;
            n_limbs_ += (want - n_limbs_) & 31;
            in_runs_.push_back(
                Run{d, n_limbs_, (uint64_t)nl, 0, run_pinned_end != 0, 1, 0, side == 1});
          }
          host_end = d + nl;
        }
        fd.limb_off = n_limbs_;
        n_limbs_ += (uint64_t)nl;
        fd.res_off = base + e * poly;
        if (use_tc) {  // the operand block, entry e of it (frequency-blocked layout)
          fd.res_off = base;
          fd.tile_np = (uint32_t)ents.size();
          fd.tile_e = (uint32_t)e;
        }
        fd.size = ents[e].size;
        fd.r = (uint32_t)r;
        fd.lgN = (uint16_t)lgN;
        fd.P = (uint16_t)P;
        uint64_t nc = ((uint64_t)nl * 64 + r - 1) / r;
        fd.ncoef = (uint32_t)(nc < N ? nc : N);
        fg.idx.push_back((uint32_t)fwd_.size());
        fwd_.push_back(fd);
      }
    }
    const uint32_t prod_index = (uint32_t)pd_.size();
    pd_.push_back(pd);
    // tensor-core items cover blocks of at most kTcBlock rows and columns
    // of C (the launch is sized for the blocks' shapes); CUDA-core items
    // cover all of C
    const int rbs = use_tc ? (m + kTcBlock - 1) / kTcBlock : 1;
    const int cbs = use_tc ? (n + kTcBlock - 1) / kTcBlock : 1;
    if (use_tc)
      for (int rb = 0; rb < rbs; ++rb)
        for (int cb = 0; cb < cbs; ++cb) {
          const int bm = std::min(kTcBlock, m - rb * kTcBlock);
          const int bn = std::min(kTcBlock, n - cb * kTcBlock);
          bool seen = false;
          for (size_t q = 0; q < tc_shapes_.size() && !seen; q += 3)
            seen = tc_shapes_[q] == bm && tc_shapes_[q + 1] == k && tc_shapes_[q + 2] == bn;
          if (!seen) tc_shapes_.insert(tc_shapes_.end(), {bm, k, bn});
        }
    const uint64_t fstep = use_tc ? (uint64_t)kTcFreqsPerCta : (uint64_t)block_freqs;
    for (int j = 0; j < P; ++j)
      for (uint64_t h0 = 0; h0 < N; h0 += fstep)
        for (int rb = 0; rb < rbs; ++rb)
          for (int cb = 0; cb < cbs; ++cb) {
            ContractItem it;
            it.prod = prod_index;
            it.prime = (uint16_t)j;
            it.pad = (uint16_t)((rb << 8) | cb);  // block of C (tensor cores only)
            it.h0 = (uint32_t)h0;
            (use_tc ? tc_items_ : items_).push_back(it);
          }
    const uint64_t ncoef_c = (uint64_t)(prm.lenA + prm.lenB - 1);
    Group& ig = invg[{lgN, P}];
    ig.P = P;
    ig.lgN = lgN;
    Group& rg = recg[P];
    rg.P = P;
    {
      auto it = rec_min_r.find(P);
      if (it == rec_min_r.end() || r < it->second) rec_min_r[P] = r;
    }
    for (int e = 0; e < m * n; ++e) {
      InvDesc id;
      id.res_off = pd.c_res + (uint64_t)e * poly;
      id.out_word = n_out_words_;
      id.out_words = (uint32_t)(2 * prm.out_limbs);
      // the CRT kernel's bit positions are 31-bit integers
      if ((uint64_t)id.out_words * 32 + 32 * (uint64_t)P + (uint64_t)r >= (1ull << 31))
        return set_error(kErrTooLarge, "output entry above 2^31 bits");
      out_word_off_.push_back((int64_t)n_out_words_);
      out_limbs_.push_back((int32_t)prm.out_limbs);
      n_out_words_ += id.out_words;
      id.r = (uint32_t)r;
      id.ncoef = (uint32_t)(ncoef_c < N ? ncoef_c : N);
      id.lgN = (uint16_t)lgN;
      id.P = (uint16_t)P;
      id.entry = (uint32_t)(first_out + e);
      const uint32_t ii = (uint32_t)inv_.size();
      inv_.push_back(id);
      ig.idx.push_back(ii);
      rg.idx.push_back(ii);
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
      if (g.lgN < 3 || D > 7) {  // (never a blocked-layout group: lgN >= 3, r <= 192)
        out.push_back(std::move(g));  // radix-2 path
        continue;
      }
      if (g.lgN > kMaxLgNOneCta) {  // four-step transforms, a group per length
        g.large = true;
        g.D = D;
        out.push_back(std::move(g));
        continue;
      }
      const bool team = ((int64_t)1 << g.lgN) <= (int64_t)fwd_team_points();
      // a CTA's shared memory follows the launch's largest class, so classes
      // above the team size get launches of their own
      Group& v = var[{(team ? 0 : g.lgN) + (g.tiled ? 64 : 0) + (g.b_only ? 128 : 0), D}];
      v.batched = true;
      v.team = team;
      v.tiled = g.tiled;
      v.b_only = g.b_only;
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
  // CRT + recompose: the prime counts up to kCrtMixedSplit in one launch,
  // the larger ones in another, each with its narrowest coefficient width
  // per count (it sizes the kernel's scratch)
  for (int high = 0; high < 2; ++high) {
    Group g;
    g.rmin.assign(kMaxPrimes + 1, 0);
    for (auto& kv : recg) {
      if ((kv.first > kCrtMixedSplit) != (high != 0)) continue;
      g.rmin[kv.first] = (int)rec_min_r[kv.first];
      g.P = std::max(g.P, kv.first);
      g.idx.insert(g.idx.end(), kv.second.idx.begin(), kv.second.idx.end());
    }
    if (g.idx.empty()) continue;
    g.crt_high = high != 0;
    // longest entries first (the warp that gets one works longest), ties in
    // entry order: one sort of packed (longest-first key, index) integers.
    // (Grouping by prime count first, for instruction-cache locality,
    // measured no better: 11.45 against 11.29 ms on the default step.)
    std::vector<uint64_t> keys(g.idx.size());
    for (size_t i = 0; i < keys.size(); ++i)
      keys[i] = ((uint64_t)(0xffffffffu - inv_[g.idx[i]].out_words) << 32) | g.idx[i];
    std::sort(keys.begin(), keys.end());
    for (size_t i = 0; i < keys.size(); ++i) g.idx[i] = (uint32_t)keys[i];
    rec_groups_.push_back(std::move(g));
  }
  for (auto* gs : {&fwd_groups_, &inv_groups_, &rec_groups_})
    for (auto& g : *gs) {
      if (g.batched) continue;
      g.idx_off = (uint32_t)idx_all_.size();
      idx_all_.insert(idx_all_.end(), g.idx.begin(), g.idx.end());
    }
  prepared_ = true;
  return kOk;
}

int Plan::bind(Workspace* ws) {
  if (!prepared_ || built_) return set_error(kErrState, "plan not prepared, or already bound");
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
  plan_transfers();
  ws_ = ws ? ws : &own_;
  int st = ws_->reserve(n_limbs_, n_res_, n_out_words_, outs_.size(), desc_bytes_, stage_limbs_,
                        stage_out_words_);
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
  int64_t sl[kStages];
  stage_launches(sl);
  launches_ = sl[0] + sl[1] + sl[2] + sl[3];
  built_ = true;
  return kOk;
}

void Plan::plan_transfers() {
  out_runs_.clear();
  stage_limbs_ = stage_out_words_ = direct_in_limbs_ = direct_out_words_ = 0;
  // inputs: runs were formed while the limb offsets were assigned
  for (Run& r : in_runs_) {
    if (r.direct) {
      direct_in_limbs_ += r.n;
    } else {
      stage_limbs_ += (r.dev - stage_limbs_) & 31;  // same 256-byte phase as the device side
      r.stage = stage_limbs_;
      stage_limbs_ += r.n;
    }
  }
  // outputs, per product: packed destinations in pinned memory, entries at
  // a constant stride with room for every word the device writes, take the
  // device's words straight (one copy, strided when the stride exceeds the
  // device's); everything else (mpz destinations included) is staged
  const auto pinned = pinned_ranges();
  out_stage_.assign(outs_.size(), -1);
  size_t e0 = 0;
  for (size_t t = 0; t < prods_.size(); ++t) {
    const size_t cnt = prods_[t].c.size();
    const size_t first = e0;
    e0 += cnt;
    if (!cnt || zero_prod_[t] || prods_[t].device_only) continue;
    const int64_t lim = out_limbs_[first];
    const uint64_t width = 2 * (uint64_t)lim;  // words per entry on the device
    const uint64_t dev = (uint64_t)out_word_off_[first];
    bool can = true;
    int64_t stride = 0;  // limbs between consecutive destinations
    for (size_t e = first; e < first + cnt && can; ++e) {
      const OutRef& o = outs_[e];
      can = o.d && !o.mpz && o.cap >= lim;
      if (can && e > first) {
        const int64_t d = o.d - outs_[e - 1].d;
        if (e == first + 1) stride = d;
        can = d == stride && d >= lim;
      }
    }
    if (cnt == 1) stride = lim;
    if (can) {
      const size_t span = (size_t)((cnt - 1) * (uint64_t)stride + (uint64_t)lim) * 8;
      can = in_ranges(pinned, outs_[first].d, span);
    }
    if (can && stride == lim) {
      // back to back: a plain copy, merged with the previous product's when
      // both sides continue it
      if (!out_runs_.empty()) {
        Run& b = out_runs_.back();
        if (b.direct && b.rows == 1 && b.dev + b.n == dev &&
            static_cast<const uint32_t*>(b.host) + b.n ==
                reinterpret_cast<const uint32_t*>(outs_[first].d)) {
          b.n += width * cnt;
          direct_out_words_ += width * cnt;
          continue;
        }
      }
      out_runs_.push_back(Run{outs_[first].d, dev, width * cnt, 0, true, 1, 0});
      direct_out_words_ += width * cnt;
    } else if (can) {
      out_runs_.push_back(Run{outs_[first].d, dev, width, 0, true, (uint64_t)cnt,
                              2 * (uint64_t)stride});
      direct_out_words_ += width * cnt;
    } else {
      for (size_t e = first; e < first + cnt; ++e)
        out_stage_[e] = (int64_t)(stage_out_words_ + (uint64_t)out_word_off_[e] - dev);
      if (!out_runs_.empty()) {
        Run& b = out_runs_.back();
        if (!b.direct && b.dev + b.n == dev && b.stage + b.n == stage_out_words_) {
          b.n += width * cnt;
          stage_out_words_ += width * cnt;
          continue;
        }
      }
      out_runs_.push_back(Run{nullptr, dev, width * cnt, stage_out_words_, false, 1, 0});
      stage_out_words_ += width * cnt;
    }
  }
}

int Plan::upload(cudaStream_t st) {
  b_valid_ = false;  // B's limbs are read again: its transforms follow at the next execute
  return upload_sides(st, false);
}

int Plan::upload_sides(cudaStream_t st, bool a_only) {
  if (!built_) return set_error(kErrState, "plan not built");
  if (a_only && !fixed_b_) return set_error(kErrState, "the plan does not keep B's transforms");
  if (desc_bytes_)
    CU(cudaMemcpyAsync(ws_->d_desc, ws_->h_desc, desc_bytes_, cudaMemcpyHostToDevice, st),
       "H2D descriptors");
  CU(cudaMemsetAsync(ws_->d_status, 0, sizeof(int), st), "clear status");
  // operands already on the device: copy their limbs, then write their
  // sizes into the forward descriptors
  for (const DevRun& r : dev_runs_)
    if (r.n)
      CU(cudaMemcpyAsync(ws_->d_limbs + r.dst, r.src, r.n * 8, cudaMemcpyDeviceToDevice, st),
         "D2D limbs");
  for (const DevFix& f : dev_fixes_)
    CU(launch_fix_sizes(d_fwd_ + f.first_fwd, (int)f.count, f.sizes, st), "size fix-up launch");
  // a_only: B's runs stay as they are (its transforms are kept)
  auto skip = [a_only](const Run& r) { return a_only && r.b; };
  // straight copies first, so the DMA runs while the staged runs are gathered
  for (const Run& r : in_runs_)
    if (r.direct && !skip(r))
      CU(cudaMemcpyAsync(ws_->d_limbs + r.dev, r.host, r.n * 8, cudaMemcpyHostToDevice, st),
         "H2D limbs");
  if (!stage_limbs_) return kOk;
  // staged runs: gathered in pieces of at most 4 MB across host threads
  struct Piece {
    const uint64_t* src;
    uint64_t stage, n;
  };
  constexpr uint64_t kPiece = (4ull << 20) / 8;
  std::vector<Piece> pieces;
  for (const Run& r : in_runs_) {
    if (r.direct || skip(r)) continue;
    for (uint64_t o = 0; o < r.n; o += kPiece)
      pieces.push_back(Piece{static_cast<const uint64_t*>(r.host) + o, r.stage + o,
                             r.n - o < kPiece ? r.n - o : kPiece});
  }
  uint64_t* hl = ws_->h_limbs;
  parallel_chunks(pieces.size(), (size_t)stage_limbs_ * 8, [&](size_t lo, size_t hi) {
    for (size_t i = lo; i < hi; ++i)
      std::memcpy(hl + pieces[i].stage, pieces[i].src, (size_t)pieces[i].n * 8);
  });
  // consecutive staged runs go as one copy: their alignment gaps are the
  // same on both sides (staging mirrors the device's 256-byte phase), and
  // the gap words are padding nobody reads
  size_t i = 0;
  while (i < in_runs_.size()) {
    if (in_runs_[i].direct || skip(in_runs_[i])) {
      ++i;
      continue;
    }
    uint64_t dev = in_runs_[i].dev, stg = in_runs_[i].stage, n = in_runs_[i].n;
    size_t j = i + 1;
    while (j < in_runs_.size() && !in_runs_[j].direct && !skip(in_runs_[j]) &&
           in_runs_[j].dev >= dev + n &&
           in_runs_[j].dev - (dev + n) == in_runs_[j].stage - (stg + n)) {
      n = in_runs_[j].dev + in_runs_[j].n - dev;
      ++j;
    }
    CU(cudaMemcpyAsync(ws_->d_limbs + dev, hl + stg, n * 8, cudaMemcpyHostToDevice, st),
       "H2D limbs");
    i = j;
  }
  return kOk;
}

// The debug bounds check: every descriptor's extents against the
// workspace, on the device, before any other kernel of the execute runs; a
// violation is reported as MPZMM_ERR_BOUNDS and nothing else is launched.
int Plan::check_bounds(cudaStream_t st) {
  BoundsCaps caps;
  caps.limbs = ws_->cap_limbs;
  caps.res = ws_->cap_res;
  caps.out_words = ws_->cap_out;
  caps.sizes = ws_->cap_sizes;
  CU(launch_check_bounds(d_fwd_, (int)fwd_.size(), d_inv_, (int)inv_.size(), d_pd_,
                         (int)pd_.size(), caps, ws_->d_status, st),
     "bounds check launch");
  CU(cudaMemcpyAsync(ws_->h_status, ws_->d_status, sizeof(int), cudaMemcpyDeviceToHost, st),
     "D2H status");
  CU(cudaStreamSynchronize(st), "bounds check");
  if (*ws_->h_status == 2) {
    *ws_->h_status = 0;
    CU(cudaMemsetAsync(ws_->d_status, 0, sizeof(int), st), "clear status");
    return set_error(kErrBounds, "debug bounds check: a descriptor lies outside the workspace");
  }
  return kOk;
}

int Plan::execute(cudaStream_t st) {
  if (!built_) return set_error(kErrState, "plan not built");
  if (check_bounds_) {
    const int r = check_bounds(st);
    if (r) return r;
  }
  if (!use_graph_ || timing_ || fixed_b_) return launch_all(st, timing_);
  if (!graph_exec_) {
    if (ws_->fanout) {  // no stream or event creation inside the capture
      const int e0 = ws_->ensure_side();
      if (e0 != kOk) return e0;
    }
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

// Launches the n independent launches of one stage, launch(i, stream),
// round-robin over st and the workspace's side streams, forked from st and
// joined back to it, so each launch's last wave overlaps the next one's
// first.  MPZMM_FANOUT=0 keeps them all on st (tuning experiments), and so
// does a workspace with fanout off (the server's: each of its batches keeps
// the priority of its own stream).
template <class L>
static int fan_out(Workspace* ws, cudaStream_t st, int n, L launch) {
  static const bool on = [] {
    const char* e = std::getenv("MPZMM_FANOUT");
    return !(e && e[0] == '0');
  }();
  int ns = n - 1 < Workspace::kSideStreams ? n - 1 : Workspace::kSideStreams;
  if (!on || !ws->fanout || ns <= 0 || ws->ensure_side() != kOk) ns = 0;
  if (ns > 0) {
    CU(cudaEventRecord(ws->fork_ev, st), "cudaEventRecord");
    for (int i = 0; i < ns; ++i)
      CU(cudaStreamWaitEvent(ws->side[i], ws->fork_ev, 0), "cudaStreamWaitEvent");
  }
  for (int i = 0; i < n; ++i) {
    const int w = ns > 0 ? i % (ns + 1) : 0;
    const int r = launch(i, w == 0 ? st : ws->side[w - 1]);
    if (r != kOk) return r;
  }
  for (int i = 0; i < ns; ++i) {
    CU(cudaEventRecord(ws->join_ev[i], ws->side[i]), "cudaEventRecord");
    CU(cudaStreamWaitEvent(st, ws->join_ev[i], 0), "cudaStreamWaitEvent");
  }
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
  // a plan that keeps B's transforms skips B's launches while they are current
  std::vector<const Group*> fwd_run;
  for (const Group& g : fwd_groups_)
    if (!(g.b_only && b_valid_)) fwd_run.push_back(&g);
  int r = fan_out(ws_, st, (int)fwd_run.size(), [&](int i, cudaStream_t s) -> int {
    const Group& g = *fwd_run[i];
    if (g.large)
      CU(launch_large_fwd(d_fwd_, d_idx_ + g.idx_off, (int)g.idx.size(), g.lgN, g.D,
                          ws_->d_limbs, ws_->d_res, ctx.d_twf, ctx.twist_f, s),
         "split+forward NTT launch (four-step)");
    else if (g.batched)
      CU(launch_fwd_items(d_fwd_, d_idx_, d_cta_ + g.item_off, (int)g.items.size(), g.D, g.team,
                          g.max_lgN, ws_->d_limbs, ws_->d_res, ctx.d_twf, s, g.tiled),
         "split+forward NTT launch");
    else
      CU(launch_split_fwd(d_fwd_, d_idx_ + g.idx_off, (int)g.idx.size(), g.P, g.lgN,
                          ws_->d_limbs, ws_->d_res, ctx.d_twf, s),
         "split+forward NTT launch");
    return kOk;
  });
  if (r != kOk) return r;
  if (timed) CU(cudaEventRecord(ev[1], st), "cudaEventRecord");
  if (!items_.empty())
    CU(launch_contract(d_pd_, d_items_, (int)items_.size(), ws_->d_res, st), "contraction launch");
  if (!tc_items_.empty())
    CU(launch_contract_tc(d_pd_, d_tc_items_, (int)tc_items_.size(), ws_->d_res,
                          tc_shapes_.data(), (int)(tc_shapes_.size() / 3), ws_->d_status, st,
                          take_test_stall_tc() ? 1 : 0),
       "tensor-core contraction launch");
  if (timed) CU(cudaEventRecord(ev[2], st), "cudaEventRecord");
  r = fan_out(ws_, st, (int)inv_groups_.size(), [&](int i, cudaStream_t s) -> int {
    const Group& g = inv_groups_[i];
    if (g.large)
      CU(launch_large_inv(d_inv_, d_idx_ + g.idx_off, (int)g.idx.size(), g.lgN, ws_->d_res,
                          ctx.d_twi, ctx.twist_i, s),
         "inverse NTT launch (four-step)");
    else if (g.batched)
      CU(launch_inv_items(d_inv_, d_idx_, d_cta_ + g.item_off, (int)g.items.size(), g.team,
                          g.max_lgN, ws_->d_res, ctx.d_twi, s),
         "inverse NTT launch");
    else
      CU(launch_inv_ntt(d_inv_, d_idx_ + g.idx_off, (int)g.idx.size(), g.P, g.lgN, ws_->d_res,
                        ctx.d_twi, s),
         "inverse NTT launch");
    return kOk;
  });
  if (r != kOk) return r;
  if (timed) CU(cudaEventRecord(ev[3], st), "cudaEventRecord");
  r = fan_out(ws_, st, (int)rec_groups_.size(), [&](int i, cudaStream_t s) -> int {
    const Group& g = rec_groups_[i];
    CU(launch_crt_mixed(d_inv_, d_idx_ + g.idx_off, (int)g.idx.size(), g.crt_high, g.rmin.data(),
                        ws_->d_res, ws_->d_out, ws_->d_sizes, s),
       "CRT+recompose launch");
    return kOk;
  });
  if (r != kOk) return r;
  if (timed) CU(cudaEventRecord(ev[4], st), "cudaEventRecord");
  b_valid_ = fixed_b_;
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
  auto count = [](const std::vector<Group>& gs) {
    int64_t n = 0;
    for (const Group& g : gs) n += g.large ? kLargeLaunches : 1;
    return n;
  };
  out[0] = count(fwd_groups_);
  out[1] = (items_.empty() ? 0 : 1) + (tc_items_.empty() ? 0 : 1);
  out[2] = count(inv_groups_);
  out[3] = (int64_t)rec_groups_.size();
}

int Plan::download_enqueue(cudaStream_t st) {
  if (!built_) return set_error(kErrState, "plan not built");
  if (!outs_.empty() && !inv_.empty())
    CU(cudaMemcpyAsync(ws_->h_sizes, ws_->d_sizes, outs_.size() * sizeof(int32_t),
                       cudaMemcpyDeviceToHost, st),
       "D2H sizes");
  for (const Run& r : out_runs_) {
    void* dst = r.direct ? const_cast<void*>(r.host) : (void*)(ws_->h_out + r.stage);
    if (r.rows > 1)
      CU(cudaMemcpy2DAsync(dst, r.pitch * 4, ws_->d_out + r.dev, r.n * 4, r.n * 4, r.rows,
                           cudaMemcpyDeviceToHost, st),
         "D2H words (strided)");
    else
      CU(cudaMemcpyAsync(dst, ws_->d_out + r.dev, r.n * 4, cudaMemcpyDeviceToHost, st),
         "D2H words");
  }
  CU(cudaMemcpyAsync(ws_->h_status, ws_->d_status, sizeof(int), cudaMemcpyDeviceToHost, st),
     "D2H status");
  return kOk;
}

int Plan::download_finish(cudaStream_t st, cudaEvent_t done) {
  if (!built_) return set_error(kErrState, "plan not built");
  if (done)
    CU(cudaEventSynchronize(done), "kernel execution");
  else
    CU(cudaStreamSynchronize(st), "kernel execution");
  if (*ws_->h_status)
    return set_error(kErrTimeout, "a tensor-core contraction wait timed out; results invalid");
  const int32_t* hs = ws_->h_sizes;
  const uint32_t* ho = ws_->h_out;
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
  parallel_chunks(outs_.size(), (size_t)stage_out_words_ * 4, [&](size_t lo, size_t hi) {
    for (size_t e = lo; e < hi; ++e) {
      if (!ok[e]) continue;
      const OutRef& o = outs_[e];
      const int32_t sz = out_word_off_[e] < 0 ? 0 : hs[e];
      const int64_t nl = sz < 0 ? -(int64_t)sz : sz;
      const int64_t so = out_stage_[e];
      const uint64_t* src = so < 0 ? nullptr : reinterpret_cast<const uint64_t*>(ho + so);
      if (o.mpz) {
        __mpz_struct* z = static_cast<__mpz_struct*>(o.mpz);
        if (nl) std::memcpy(z->_mp_d, src, (size_t)nl * 8);
        z->_mp_size = sz;
      } else {
        if (nl && src) std::memcpy(o.d, src, (size_t)nl * 8);  // else already in place
        if (o.size) *o.size = sz;
      }
    }
  });
  return status;
}

DeviceOperand Plan::device_output(size_t product) const {
  DeviceOperand o;
  const size_t first = prod_first_out_[product];
  const size_t cnt = prods_[product].c.size();
  if (!cnt || zero_prod_[product]) return o;
  const uint64_t w0 = (uint64_t)out_word_off_[first];  // even: whole limbs
  o.limbs = reinterpret_cast<const uint64_t*>(ws_->d_out + w0);
  o.sizes = ws_->d_sizes + first;
  o.cap_limbs = out_limbs_[first];
  o.offs.resize(cnt);
  for (size_t e = 0; e < cnt; ++e) o.offs[e] = (out_word_off_[first + e] - (int64_t)w0) / 2;
  o.span_limbs = (uint64_t)o.offs[cnt - 1] + (uint64_t)o.cap_limbs;
  return o;
}

int Plan::download(cudaStream_t st) {
  int s = download_enqueue(st);
  return s ? s : download_finish(st);
}

// ---- one-shot batches ----
namespace {
int64_t now_ns() {
  return std::chrono::duration_cast<std::chrono::nanoseconds>(
             std::chrono::steady_clock::now().time_since_epoch())
      .count();
}

uint64_t input_limbs(const ProductSpec& ps) {
  uint64_t n = 0;
  for (const auto& e : ps.a) n += e.size < 0 ? (uint64_t)(-(int64_t)e.size) : (uint64_t)e.size;
  for (const auto& e : ps.b) n += e.size < 0 ? (uint64_t)(-(int64_t)e.size) : (uint64_t)e.size;
  return n;
}

int pipe_depth() {
  static const int d = [] {
    const char* e = std::getenv("MPZMM_PIPE_DEPTH");
    const int v = e ? std::atoi(e) : 0;
    return v >= 2 && v <= kPipeDepth ? v : 4;
  }();
  return d;
}

int ensure_pipeline(Context& ctx) {
  while ((int)ctx.pipe_ws.size() < kPipeDepth)
    ctx.pipe_ws.push_back(ctx.pipe_ws.empty() ? ctx.ws : new Workspace);
  while ((int)ctx.pipe_st.size() < kPipeDepth) {
    cudaStream_t s = nullptr;
    CU(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "cudaStreamCreate");
    ctx.pipe_st.push_back(s);
  }
  for (cudaStream_t* s : {&ctx.pipe_in, &ctx.pipe_out})
    if (!*s) CU(cudaStreamCreateWithFlags(s, cudaStreamNonBlocking), "cudaStreamCreate");
  if (!ctx.pipe_ev)
    CU(cudaEventCreateWithFlags(&ctx.pipe_ev, cudaEventDisableTiming), "cudaEventCreate");
  for (auto* v : {&ctx.pipe_ev_in, &ctx.pipe_ev_exec, &ctx.pipe_ev_out})
    while ((int)v->size() < kPipeDepth) {
      cudaEvent_t e = nullptr;
      CU(cudaEventCreateWithFlags(&e, cudaEventDisableTiming), "cudaEventCreate");
      v->push_back(e);
    }
  return kOk;
}

// Timing events of a batch of n chunks (the start event and four a chunk)
// and its timeline rows, zeroed.
int ensure_timeline(Context& ctx, size_t nchunks) {
  while (ctx.tl_ev.size() < 1 + 4 * nchunks) {
    cudaEvent_t e = nullptr;
    CU(cudaEventCreate(&e), "cudaEventCreate");
    ctx.tl_ev.push_back(e);
  }
  ctx.timeline.assign(nchunks * kTimelineFields, 0.0);
  return kOk;
}

// The device columns of the timeline, once every event of the batch is done.
void read_timeline(Context& ctx, size_t nchunks) {
  for (size_t c = 0; c < nchunks; ++c)
    for (int k = 0; k < 4; ++k) {
      float ms = -1.f;
      if (cudaEventElapsedTime(&ms, ctx.tl_ev[0], ctx.tl_ev[1 + 4 * c + k]) != cudaSuccess) {
        cudaGetLastError();
        ms = -1.f;
      }
      ctx.timeline[c * kTimelineFields + 4 + k] = ms;
    }
}
}  // namespace

bool batch_chunks(const std::vector<uint64_t>& limbs, int64_t chunk_option,
                  std::vector<size_t>* bounds) {
  const size_t n = limbs.size();
  uint64_t total = 0;
  for (uint64_t l : limbs) total += l;
  // automatic chunks: a 32nd of the batch, between 4 Mi and 64 Mi limbs (32
  // and 512 MB of input) -- small enough that the first results come back
  // early and both copy directions stream steadily, large enough that the
  // kernels' launch tails stay small, bounded so that the workspaces in
  // flight stay a few GB whatever the batch
  uint64_t chunk = chunk_option > 0 ? (uint64_t)chunk_option : total / 32;
  if (chunk_option <= 0) {
    if (chunk < (4ull << 20)) chunk = 4ull << 20;
    if (chunk > (64ull << 20)) chunk = 64ull << 20;
  }
  if (chunk == 0) chunk = 1;
  bounds->assign(1, 0);
  if (n < 2 || total <= chunk) {
    bounds->push_back(n);
    return false;
  }
  // chunks of consecutive whole products; the first two are a quarter and
  // a half of the others, so the first results start back sooner (the
  // device->host copies are the pipeline's longest chain),
  uint64_t acc = 0;
  for (size_t t = 0; t < n; ++t) {
    acc += limbs[t];
    const size_t c = bounds->size() - 1;
    const uint64_t target = c == 0 ? chunk / 4 : (c == 1 ? chunk / 2 : chunk);
    if (acc >= target && t + 1 < n) {
      bounds->push_back(t + 1);
      acc = 0;
    }
  }
  bounds->push_back(n);
  // and the last one is split about 2:1, so the final results come back
  // sooner after the last inputs went in
  if (bounds->size() >= 3) {
    const size_t a = (*bounds)[bounds->size() - 2], b = bounds->back();
    uint64_t tail = 0;
    for (size_t t = a; t < b; ++t) tail += limbs[t];
    if (tail > chunk / 2 && b - a >= 2) {
      uint64_t acc2 = 0;
      size_t cut = a;
      while (cut + 1 < b && 3 * (acc2 + limbs[cut]) <= 2 * tail) acc2 += limbs[cut++];
      if (cut > a) bounds->insert(bounds->end() - 1, cut);
    }
  }
  return true;
}

int run_batch(std::vector<ProductSpec> specs, cudaStream_t st) {
  Context& ctx = context();
  for (auto& v : ctx.batch_ns) v = 0;
  for (auto& v : ctx.batch_bytes) v = 0;
  auto count_bytes = [&ctx](const Plan& p) {
    ctx.batch_bytes[0] += (int64_t)p.upload_bytes();
    ctx.batch_bytes[1] += (int64_t)p.download_bytes();
    ctx.batch_bytes[2] += (int64_t)p.direct_in_bytes();
    ctx.batch_bytes[3] += (int64_t)p.direct_out_bytes();
  };
  std::vector<uint64_t> limbs(specs.size());
  for (size_t t = 0; t < specs.size(); ++t) limbs[t] = input_limbs(specs[t]);
  std::vector<size_t> bounds;
  const bool pipelined = batch_chunks(limbs, ctx.chunk_limbs, &bounds);

  if (!pipelined) {
    ctx.batch_chunks = 1;
    int s = ensure_timeline(ctx, 1);
    if (s) return s;
    double* tl = ctx.timeline.data();
    const cudaEvent_t* ev = ctx.tl_ev.data();
    const int64_t t0 = now_ns();
    s = cuda_status(cudaEventRecord(ev[0], st), "cudaEventRecord");
    Plan plan;
    if (!s) s = plan.build(std::move(specs), ctx.ws);
    if (!s) count_bytes(plan);
    const int64_t t1 = now_ns();
    if (!s) s = cuda_status(cudaEventRecord(ev[1], st), "cudaEventRecord");
    if (!s) s = plan.upload(st);
    if (!s) s = cuda_status(cudaEventRecord(ev[2], st), "cudaEventRecord");
    const int64_t t2 = now_ns();
    if (!s) s = plan.execute(st);
    if (!s) s = cuda_status(cudaEventRecord(ev[3], st), "cudaEventRecord");
    if (!s) s = plan.download_enqueue(st);
    if (!s) s = cuda_status(cudaEventRecord(ev[4], st), "cudaEventRecord");
    const int64_t t3 = now_ns();
    if (!s) s = plan.download_finish(st);
    const int64_t t4 = now_ns();
    ctx.batch_ns[0] = t1 - t0;
    ctx.batch_ns[1] = t2 - t1;
    ctx.batch_ns[2] = t3 - t2;
    ctx.batch_ns[3] = t4 - t3;
    tl[0] = 0.0;
    tl[1] = (t1 - t0) * 1e-6;
    tl[2] = tl[1];
    tl[3] = (t3 - t0) * 1e-6;
    if (!s) {
      tl[8] = (double)plan.upload_bytes();
      tl[9] = (double)plan.download_bytes();
      read_timeline(ctx, 1);
    }
    return s;
  }

  const size_t nchunks = bounds.size() - 1;
  ctx.batch_chunks = (int64_t)nchunks;
  int s = ensure_pipeline(ctx);
  if (!s) s = ensure_timeline(ctx, nchunks);
  if (s) return s;
  double* tl = ctx.timeline.data();
  const cudaEvent_t* ev = ctx.tl_ev.data();
  // the pipeline's streams start after the caller's earlier work
  CU(cudaEventRecord(ctx.pipe_ev, st), "cudaEventRecord");
  for (cudaStream_t ps : ctx.pipe_st) CU(cudaStreamWaitEvent(ps, ctx.pipe_ev, 0), "cudaStreamWaitEvent");
  CU(cudaStreamWaitEvent(ctx.pipe_in, ctx.pipe_ev, 0), "cudaStreamWaitEvent");
  CU(cudaStreamWaitEvent(ctx.pipe_out, ctx.pipe_ev, 0), "cudaStreamWaitEvent");
  const int64_t tl0 = now_ns();
  CU(cudaEventRecord(ev[0], ctx.pipe_in), "cudaEventRecord");

  // The caller's thread plans chunks and waits for finished ones; a
  // submitter thread queues each chunk's copies and kernels, because queueing
  // a copy can block the host until the copy engine takes it.
  const int depth = pipe_depth();
  std::unique_ptr<Plan> plans[kPipeDepth];
  size_t slot_chunk[kPipeDepth] = {};
  bool slot_ok[kPipeDepth] = {};
  std::mutex mu;
  std::condition_variable cv;
  std::deque<size_t> queue;
  size_t submitted = 0;  // chunks [0, submitted) have left the submitter
  bool closing = false;
  int sub_status = kOk;
  std::string sub_msg;
  int64_t sub_ns[2] = {0, 0};
  std::thread submitter([&] {
    cudaSetDevice(ctx.device);
    for (;;) {
      size_t c;
      {
        std::unique_lock<std::mutex> lk(mu);
        cv.wait(lk, [&] { return !queue.empty() || closing; });
        if (queue.empty()) return;
        c = queue.front();
        queue.pop_front();
      }
      const int w = (int)(c % depth);
      Plan* p = plans[w].get();
      cudaStream_t ps = ctx.pipe_st[w];
      const int64_t t0 = now_ns();
      const cudaEvent_t* ce = ev + 1 + 4 * c;
      // copies in each direction in chunk order on their own stream; the
      // kernels of neighbouring chunks may overlap (one chunk's tail fills
      // in beside the next)
      int r = cuda_status(cudaEventRecord(ce[0], ctx.pipe_in), "cudaEventRecord");
      if (!r) r = p->upload(ctx.pipe_in);
      if (!r) r = cuda_status(cudaEventRecord(ctx.pipe_ev_in[w], ctx.pipe_in), "cudaEventRecord");
      if (!r) r = cuda_status(cudaEventRecord(ce[1], ctx.pipe_in), "cudaEventRecord");
      const int64_t t1 = now_ns();
      if (!r) r = cuda_status(cudaStreamWaitEvent(ps, ctx.pipe_ev_in[w], 0), "wait");
      if (!r) r = p->execute(ps);
      if (!r) r = cuda_status(cudaEventRecord(ctx.pipe_ev_exec[w], ps), "cudaEventRecord");
      if (!r) r = cuda_status(cudaEventRecord(ce[2], ps), "cudaEventRecord");
      if (!r) r = cuda_status(cudaStreamWaitEvent(ctx.pipe_out, ctx.pipe_ev_exec[w], 0), "wait");
      if (!r) r = p->download_enqueue(ctx.pipe_out);
      if (!r) r = cuda_status(cudaEventRecord(ctx.pipe_ev_out[w], ctx.pipe_out), "cudaEventRecord");
      if (!r) r = cuda_status(cudaEventRecord(ce[3], ctx.pipe_out), "cudaEventRecord");
      const int64_t t2 = now_ns();
      tl[c * kTimelineFields + 2] = (t0 - tl0) * 1e-6;
      tl[c * kTimelineFields + 3] = (t2 - tl0) * 1e-6;
      std::lock_guard<std::mutex> lk(mu);
      sub_ns[0] += t1 - t0;
      sub_ns[1] += t2 - t1;
      if (r && !sub_status) {
        sub_status = r;
        sub_msg = last_error();
      }
      slot_ok[w] = r == kOk;
      submitted = c + 1;
      cv.notify_all();
    }
  });

  // first error wins; a capacity error (some output did not fit) leaves
  // every other result written, like an unchunked batch, so the chunks go on
  int status = kOk;
  bool stop = false;
  auto finish = [&](int w) {
    if (!plans[w]) return;
    bool ok;
    {
      std::unique_lock<std::mutex> lk(mu);
      cv.wait(lk, [&] { return submitted > slot_chunk[w]; });
      ok = slot_ok[w];
      if (sub_status) stop = true;
    }
    const int64_t t0 = now_ns();
    int r = kOk;
    if (ok) {
      r = plans[w]->download_finish(ctx.pipe_out, ctx.pipe_ev_out[w]);
    } else {  // wait for whatever was queued; results invalid
      cudaStreamSynchronize(ctx.pipe_in);
      cudaStreamSynchronize(ctx.pipe_st[w]);
      cudaStreamSynchronize(ctx.pipe_out);
    }
    ctx.batch_ns[3] += now_ns() - t0;
    if (r && !status) status = r;
    if (r && r != kErrCapacity) stop = true;
    plans[w].reset();
  };
  for (size_t c = 0; c < nchunks; ++c) {
    const int w = (int)(c % depth);
    // the chunk is planned before waiting for the workspace it will use, so
    // the wait (for the results of the chunk `depth` back) and the planning
    // overlap, and the chunk is queued as soon as the workspace is free
    std::vector<ProductSpec> part;
    part.reserve(bounds[c + 1] - bounds[c]);
    for (size_t t = bounds[c]; t < bounds[c + 1]; ++t) part.push_back(std::move(specs[t]));
    std::unique_ptr<Plan> np(new Plan);
    const int64_t t0 = now_ns();
    int r = np->prepare(std::move(part));
    const int64_t tp = now_ns();
    finish(w);  // the chunk that last used this workspace
    if (stop) break;
    const int64_t tb = now_ns();
    if (!r) r = np->bind(ctx.pipe_ws[w]);
    const int64_t t1 = now_ns();
    ctx.batch_ns[0] += (tp - t0) + (t1 - tb);
    if (r) {
      if (!status) status = r;
      stop = true;
      break;
    }
    plans[w] = std::move(np);
    count_bytes(*plans[w]);
    double* row = tl + c * kTimelineFields;
    row[0] = (t0 - tl0) * 1e-6;
    row[1] = (t1 - tl0) * 1e-6;
    row[8] = (double)plans[w]->upload_bytes();
    row[9] = (double)plans[w]->download_bytes();
    slot_chunk[w] = c;
    std::lock_guard<std::mutex> lk(mu);
    queue.push_back(c);
    cv.notify_all();
  }
  // drain in chunk order (every chunk in flight is waited for, also on error)
  for (size_t c = nchunks > (size_t)depth ? nchunks - depth : 0; c < nchunks; ++c)
    finish((int)(c % depth));
  {
    std::lock_guard<std::mutex> lk(mu);
    closing = true;
    cv.notify_all();
  }
  submitter.join();
  ctx.batch_ns[1] = sub_ns[0];
  ctx.batch_ns[2] = sub_ns[1];
  if (sub_status && (!status || status == kErrCapacity)) status = set_error(sub_status, sub_msg);
  if (!status) read_timeline(ctx, nchunks);
  return status;
}

int run_chain(std::vector<ProductSpec> steps, cudaStream_t st) {
  Context& ctx = context();
  if (steps.empty()) return kOk;
  int s = ensure_pipeline(ctx);
  if (s) return s;
  // two workspaces in turn: step i reads step i-1's results (device to
  // device) while step i+1 may already be planned into the other one, after
  // the copies of the step that used it last have left its host buffers
  std::unique_ptr<Plan> prev;
  for (size_t i = 0; i < steps.size(); ++i) {
    const int w = (int)(i & 1);
    ProductSpec& ps = steps[i];
    if (i > 0) {
      const DeviceOperand o = prev->device_output(0);
      if (!o.limbs) return set_error(kErrState, "chain step without device results");
      ps.dev_a = std::make_shared<DeviceOperand>(o);
    }
    ps.device_only = i + 1 < steps.size();
    CU(cudaEventSynchronize(ctx.pipe_ev_in[w]), "wait for a workspace's copies");
    std::unique_ptr<Plan> cur(new Plan);
    std::vector<ProductSpec> one;
    one.push_back(std::move(ps));
    if ((s = cur->build(std::move(one), ctx.pipe_ws[w]))) return s;
    if ((s = cur->upload(st))) return s;
    CU(cudaEventRecord(ctx.pipe_ev_in[w], st), "cudaEventRecord");
    if ((s = cur->execute(st))) return s;
    prev = std::move(cur);
  }
  return prev->download(st);
}

}  // namespace mpzmm
