// Continuous-batching request server (mpzmm_server_* in include/mpzmm_b200.h).
//
// Callers submit single products from any thread.  The server keeps up to
// `slots` batches in flight; each slot has its own host thread, CUDA stream
// and grow-only workspace.  A free slot admits queued requests in arrival
// order into a new batch while their estimated device footprint fits what
// the batches in flight leave of the device-memory budget, plans the batch
// (one launch per stage), copies its inputs, launches it, waits for it on
// its own stream and copies the results back.  So requests that arrive
// while others are on the GPU join the next batch as soon as a slot and
// memory are free, batches on different slots overlap on the device, and
// the host work of one slot (planning, copies, a workspace growing) never
// holds up the others.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstdlib>
#include <deque>
#include <memory>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/mpzmm_b200.h"
#include "engine.h"

using namespace mpzmm;

namespace {

int64_t now_ns() {
  return std::chrono::duration_cast<std::chrono::nanoseconds>(
             std::chrono::steady_clock::now().time_since_epoch())
      .count();
}

struct Ticket {
  uint64_t id = 0;
  ProductSpec spec;
  int64_t bytes = 0;
  int64_t host_bytes = 0;  // inputs + outputs across the link
  int64_t t_submit = 0, t_start = 0, t_done = 0;
  int status = -1;  // -1 pending
  std::string error;
};

// pinned result-size and descriptor staging a slot allocates at start: a
// batch needs 4 bytes an output entry and about 32 bytes an entry and 12 a
// contraction block, far below these for any batch under the host-data cap
constexpr size_t kStageSizes = (size_t)1 << 20;
constexpr size_t kStageDescBytes = (size_t)16 << 20;

struct Slot {
  cudaStream_t stream = nullptr;     // least priority: batches with much data
  cudaStream_t stream_hi = nullptr;  // greatest priority: small batches
  Workspace ws;
  std::thread thread;
  bool busy = false;
};

}  // namespace

struct mpzmm_server {
  int64_t budget = 0;
  int max_batch = 0;
  int device = 0;
  // admission window: a slot that frees up while other batches occupy the
  // GPU keeps admitting for up to this long before it launches (ns)
  int64_t window_ns = 200000;
  // host bytes (inputs + outputs) of a batch: admission stops there (a
  // larger request goes alone), and every slot's pinned staging is sized to
  // it once, so batches never allocate pinned memory
  int64_t batch_host_cap = (int64_t)256 << 20;
  // requests with at most this many host bytes are small: admission keeps
  // them in batches of their own, which run on their slot's
  // greatest-priority stream, so the block scheduler starts their CTAs ahead
  // of those of large batches already on the GPU and a small request is
  // held up neither inside nor behind a large one's batch (0: one class)
  int64_t small_batch_bytes = (int64_t)16 << 20;
  // device memory of the slots' workspaces: a stream-ordered pool of the
  // server's own that keeps freed memory, so a workspace growing or being
  // released never synchronises the device or stalls the other slots
  cudaMemPool_t pool = nullptr;
  std::vector<std::unique_ptr<Slot>> slots;
  std::mutex mu;
  std::condition_variable cv_work;  // slots wake up: new request, freed budget, stop
  std::condition_variable cv_done;  // waiters wake up
  std::deque<std::shared_ptr<Ticket>> queue;
  std::unordered_map<uint64_t, std::shared_ptr<Ticket>> tickets;
  uint64_t next_id = 1;
  bool stop = false;
  int64_t in_flight_bytes = 0;
  int64_t stat_batches = 0, stat_products = 0, stat_max_in_flight = 0;
  int64_t stat_batched_products = 0;  // products admitted into launched batches
  // slot-thread time per phase, summed over slots (ns): plan build, input
  // gather + copy, launches, wait + result copy-back + scatter
  int64_t ns_build = 0, ns_upload = 0, ns_launch = 0, ns_download = 0;
  // the longest single batch in each phase since the last read (ns)
  int64_t ns_max[4] = {0, 0, 0, 0};

  void complete(const std::shared_ptr<Ticket>& t, int status, const std::string& err) {
    t->status = status;
    t->error = err;
    t->t_done = now_ns();
  }

  // A request with at most small_batch_bytes of host data (0: none is).
  bool is_small(const Ticket& t) const {
    return small_batch_bytes > 0 && t.host_bytes <= small_batch_bytes;
  }

  // Admits queued requests for a free slot (lock held): the oldest request
  // first, then later ones of the same size class (small or large) in
  // arrival order, passing over the other class, which stays queued for
  // another slot -- so small requests never wait inside a batch for a large
  // one; at most max_batch, while the estimated footprint fits the free
  // budget; a request larger than the free budget runs once the GPU is
  // otherwise idle.
  void admit(std::vector<std::shared_ptr<Ticket>>& batch, int64_t& bytes) {
    int busy_slots = 0;
    for (auto& o : slots) busy_slots += o->busy ? 1 : 0;
    int64_t host = 0;
    for (const auto& t : batch) host += t->host_bytes;
    auto it = queue.begin();
    while (it != queue.end() && (max_batch <= 0 || (int)batch.size() < max_batch)) {
      const auto& t = *it;
      if (!batch.empty() && is_small(*t) != is_small(*batch.front())) {
        ++it;
        continue;
      }
      if (!batch.empty() && host + t->host_bytes > batch_host_cap) break;
      const bool fits = in_flight_bytes + bytes + t->bytes <= budget;
      const bool alone = batch.empty() && busy_slots == 0 && in_flight_bytes == 0 &&
                         t->bytes <= budget;
      if (!fits && !alone) break;
      bytes += t->bytes;
      host += t->host_bytes;
      batch.push_back(t);
      it = queue.erase(it);
      if (!fits) break;
    }
  }

  // One batch on a slot (slot thread, lock not held): returns its status.
  int run_batch_on(Slot& s, std::vector<std::shared_ptr<Ticket>>& batch, std::string* err) {
    std::vector<ProductSpec> specs;
    specs.reserve(batch.size());
    for (auto& t : batch) specs.push_back(t->spec);
    // a batch of small requests (admission keeps the classes apart) runs on
    // the greatest-priority stream.  The slot's batches run one after
    // another, each ending with a stream synchronisation, so switching
    // streams between batches needs no event; the workspace's stream-ordered
    // allocations follow the batch's stream.
    const cudaStream_t bs = is_small(*batch.front()) ? s.stream_hi : s.stream;
    s.ws.async_stream = bs;
    Plan plan;
    const int64_t a0 = now_ns();
    int st = plan.build(std::move(specs), &s.ws);
    const int64_t a1 = now_ns();
    if (!st) st = plan.upload(bs);
    const int64_t a2 = now_ns();
    if (!st) st = plan.execute(bs);
    const int64_t a3 = now_ns();
    {
      std::lock_guard<std::mutex> lk(mu);
      for (auto& t : batch) t->t_start = a3;
    }
    if (!st) st = plan.download(bs);
    const int64_t a4 = now_ns();
    if (st) {
      *err = last_error();
      cudaStreamSynchronize(bs);  // whatever was queued
    }
    std::lock_guard<std::mutex> lk(mu);
    ns_build += a1 - a0;
    ns_upload += a2 - a1;
    ns_launch += a3 - a2;
    ns_download += a4 - a3;
    const int64_t d[4] = {a1 - a0, a2 - a1, a3 - a2, a4 - a3};
    for (int q = 0; q < 4; ++q)
      if (d[q] > ns_max[q]) ns_max[q] = d[q];
    return st;
  }

  void slot_loop(Slot& s) {
    cudaSetDevice(device);
    // pinned staging for a full batch, once (a failure here only means the
    // first batches grow it instead)
    if (s.ws.reserve_staging((size_t)(batch_host_cap / 8), (size_t)(batch_host_cap / 4),
                             kStageSizes, kStageDescBytes))
      cudaGetLastError();
    for (;;) {
      std::vector<std::shared_ptr<Ticket>> batch;
      int64_t bytes = 0;
      {
        std::unique_lock<std::mutex> lk(mu);
        for (;;) {
          admit(batch, bytes);
          if (!batch.empty()) break;
          if (stop && queue.empty()) return;
          cv_work.wait(lk);
        }
        int others = 0;
        for (auto& o : slots) others += o->busy ? 1 : 0;
        s.busy = true;
        in_flight_bytes += bytes;
        // the GPU is busy with other batches anyway: let this batch fill for
        // a bounded window (an idle GPU gets the batch at once)
        auto full = [&] { return max_batch > 0 && (int)batch.size() >= max_batch; };
        if (others > 0 && window_ns > 0 && !full()) {
          const auto deadline =
              std::chrono::steady_clock::now() + std::chrono::nanoseconds(window_ns);
          for (;;) {
            const bool timed_out = cv_work.wait_until(lk, deadline) == std::cv_status::timeout;
            int64_t more = 0;
            admit(batch, more);
            in_flight_bytes += more;
            bytes += more;
            if (timed_out || full() || stop) break;
          }
        }
        ++stat_batches;
        stat_batched_products += (int64_t)batch.size();
        int in_flight = 0;
        for (auto& o : slots) in_flight += o->busy ? 1 : 0;
        if (in_flight > stat_max_in_flight) stat_max_in_flight = in_flight;
      }
      std::string err;
      const int st = run_batch_on(s, batch, &err);
      // workspaces are grow-only (re-growing per batch costs far more than the
      // batch); one that has grown past its share of the budget is released
      if (st || s.ws.device_bytes > budget / (int64_t)slots.size()) s.ws.release_device();
      {
        std::lock_guard<std::mutex> lk(mu);
        for (auto& t : batch) complete(t, st, err);
        stat_products += (int64_t)batch.size();
        in_flight_bytes -= bytes;
        s.busy = false;
      }
      cv_done.notify_all();
      cv_work.notify_all();  // freed budget: another slot may admit now
    }
  }
};

extern "C" {

int mpzmm_server_create(mpzmm_server** out, int64_t budget_bytes, int slots, int max_batch) {
  if (!out) return set_error(kErrArg, "null server pointer");
  *out = nullptr;
  if (slots < 1 || slots > 16) return set_error(kErrArg, "slots must be in 1..16");
  int st = ensure_setup(-1);
  if (st) return st;
  std::unique_ptr<mpzmm_server> s(new mpzmm_server);
  if (budget_bytes <= 0) {
    size_t fr = 0, tot = 0;
    const cudaError_t e = cudaMemGetInfo(&fr, &tot);
    if (e != cudaSuccess) return set_error(kErrCuda, cudaGetErrorString(e));
    budget_bytes = (int64_t)(fr / 4 * 3);
  }
  s->budget = budget_bytes;
  s->max_batch = max_batch;
  s->device = context().device;
  {
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = s->device;
    cudaError_t e = cudaMemPoolCreate(&s->pool, &props);
    if (e != cudaSuccess) return set_error(kErrCuda, std::string("cudaMemPoolCreate: ") +
                                                         cudaGetErrorString(e));
    uint64_t keep = ~(uint64_t)0;  // freed memory stays in the pool
    e = cudaMemPoolSetAttribute(s->pool, cudaMemPoolAttrReleaseThreshold, &keep);
    if (e != cudaSuccess) {
      cudaMemPoolDestroy(s->pool);
      return set_error(kErrCuda, std::string("cudaMemPoolSetAttribute: ") +
                                     cudaGetErrorString(e));
    }
    // a quarter of the budget, at most 32 GB, taken into the pool at
    // creation (allocated and freed once): slot workspaces growing later are
    // served from it without the driver mapping memory, which stalled
    // saturation runs (730 against 1,680 requests/s on the config-5 pool).
    // MPZMM_SERVER_PREWARM_GB replaces the amount (0: none).
    const int64_t prewarm = [budget_bytes] {
      const char* v = std::getenv("MPZMM_SERVER_PREWARM_GB");
      if (v) return (int64_t)std::atoi(v) << 30;
      const int64_t q = budget_bytes / 4;
      return q < ((int64_t)32 << 30) ? q : ((int64_t)32 << 30);
    }();
    if (prewarm > 0 && prewarm < budget_bytes) {
      cudaStream_t ps = nullptr;
      void* p = nullptr;
      if (cudaStreamCreateWithFlags(&ps, cudaStreamNonBlocking) == cudaSuccess) {
        if (cudaMallocFromPoolAsync(&p, (size_t)prewarm, s->pool, ps) == cudaSuccess)
          cudaFreeAsync(p, ps);
        cudaStreamSynchronize(ps);
        cudaStreamDestroy(ps);
      }
      cudaGetLastError();
    }
  }
  int least = 0, greatest = 0;
  if (cudaDeviceGetStreamPriorityRange(&least, &greatest) != cudaSuccess) {
    cudaGetLastError();
    least = greatest = 0;
  }
  static const bool prio_on = [] {
    const char* e = std::getenv("MPZMM_SERVER_PRIORITY");
    return !(e && e[0] == '0');
  }();
  if (!prio_on) s->small_batch_bytes = 0;
  for (int i = 0; i < slots; ++i) {
    std::unique_ptr<Slot> sl(new Slot);
    cudaError_t e = cudaStreamCreateWithPriority(&sl->stream, cudaStreamNonBlocking, least);
    if (e == cudaSuccess)
      e = cudaStreamCreateWithPriority(&sl->stream_hi, cudaStreamNonBlocking, greatest);
    if (e != cudaSuccess) {
      if (sl->stream) cudaStreamDestroy(sl->stream);
      for (auto& o : s->slots) {
        cudaStreamDestroy(o->stream);
        cudaStreamDestroy(o->stream_hi);
      }
      cudaMemPoolDestroy(s->pool);
      return set_error(kErrCuda, cudaGetErrorString(e));
    }
    sl->ws.async_stream = sl->stream;
    sl->ws.pool = s->pool;
    sl->ws.retire_host = true;
    sl->ws.fanout = false;  // one stream a batch: its priority holds for every launch
    s->slots.push_back(std::move(sl));
  }
  mpzmm_server* raw = s.get();
  for (auto& sl : s->slots) {
    Slot* sp = sl.get();
    sl->thread = std::thread([raw, sp] { raw->slot_loop(*sp); });
  }
  *out = s.release();
  return kOk;
}

int mpzmm_server_submit(mpzmm_server* s, const mpzmm_product* req, uint64_t* ticket) {
  if (!s || !req || !ticket) return set_error(kErrArg, "null argument");
  auto t = std::make_shared<Ticket>();
  const mpzmm_product& p = *req;
  if (p.m < 0 || p.k < 0 || p.n < 0) return set_error(kErrArg, "negative dimension");
  t->spec.m = p.m;
  t->spec.k = p.k;
  t->spec.n = p.n;
  const int64_t na = (int64_t)p.m * p.k, nb = (int64_t)p.k * p.n, nc = (int64_t)p.m * p.n;
  t->spec.a.resize(na);
  t->spec.b.resize(nb);
  t->spec.c.resize(nc);
  for (int64_t e = 0; e < na; ++e)
    t->spec.a[e] = EntryRef{p.a_sizes[e] ? p.a_limbs + p.a_offs[e] : nullptr, p.a_sizes[e]};
  for (int64_t e = 0; e < nb; ++e)
    t->spec.b[e] = EntryRef{p.b_sizes[e] ? p.b_limbs + p.b_offs[e] : nullptr, p.b_sizes[e]};
  for (int64_t e = 0; e < nc; ++e)
    t->spec.c[e] = OutRef{p.c_limbs + p.c_offs[e], p.c_caps[e], p.c_sizes + e, nullptr};
  t->bytes = estimate_device_bytes(t->spec, &t->host_bytes);
  if (t->bytes < 0) return set_error(kErrTooLarge, "product too large for a single transform");
  if (t->bytes > s->budget)
    return set_error(kErrTooLarge, "request needs " + std::to_string(t->bytes) +
                                       " device bytes, the server budget is " +
                                       std::to_string(s->budget));
  t->t_submit = now_ns();
  {
    std::lock_guard<std::mutex> lk(s->mu);
    if (s->stop) return set_error(kErrState, "server is stopping");
    t->id = s->next_id++;
    s->tickets[t->id] = t;
    s->queue.push_back(t);
  }
  s->cv_work.notify_all();
  *ticket = t->id;
  return kOk;
}

int mpzmm_server_poll(mpzmm_server* s, uint64_t ticket, int* done) {
  if (!s || !done) return set_error(kErrArg, "null argument");
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->tickets.find(ticket);
  if (it == s->tickets.end()) return set_error(kErrArg, "unknown ticket");
  *done = it->second->status >= 0 ? 1 : 0;
  return kOk;
}

int mpzmm_server_wait(mpzmm_server* s, uint64_t ticket, int64_t timeout_ms) {
  if (!s) return set_error(kErrArg, "null server");
  std::unique_lock<std::mutex> lk(s->mu);
  auto it = s->tickets.find(ticket);
  if (it == s->tickets.end()) return set_error(kErrArg, "unknown ticket");
  std::shared_ptr<Ticket> t = it->second;
  auto ready = [&] { return t->status >= 0; };
  if (timeout_ms < 0) {
    s->cv_done.wait(lk, ready);
  } else if (!s->cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), ready)) {
    return set_error(kErrTimeout, "request not finished within the time limit");
  }
  if (t->status) return set_error(t->status, t->error);
  return kOk;
}

int mpzmm_server_ticket_times(mpzmm_server* s, uint64_t ticket, int64_t* submit_ns,
                              int64_t* start_ns, int64_t* done_ns) {
  if (!s) return set_error(kErrArg, "null server");
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->tickets.find(ticket);
  if (it == s->tickets.end()) return set_error(kErrArg, "unknown ticket");
  if (submit_ns) *submit_ns = it->second->t_submit;
  if (start_ns) *start_ns = it->second->t_start;
  if (done_ns) *done_ns = it->second->t_done;
  return kOk;
}

int mpzmm_server_release(mpzmm_server* s, uint64_t ticket) {
  if (!s) return set_error(kErrArg, "null server");
  std::lock_guard<std::mutex> lk(s->mu);
  auto it = s->tickets.find(ticket);
  if (it == s->tickets.end()) return set_error(kErrArg, "unknown ticket");
  if (it->second->status < 0) return set_error(kErrState, "request still pending");
  s->tickets.erase(it);
  return kOk;
}

int mpzmm_server_phase_ns(mpzmm_server* s, int64_t* ns4) {
  if (!s || !ns4) return set_error(kErrArg, "null argument");
  std::lock_guard<std::mutex> lk(s->mu);
  ns4[0] = s->ns_build;
  ns4[1] = s->ns_upload;
  ns4[2] = s->ns_launch;
  ns4[3] = s->ns_download;
  return kOk;
}

int mpzmm_server_phase_max_ns(mpzmm_server* s, int64_t* ns4) {
  if (!s || !ns4) return set_error(kErrArg, "null argument");
  std::lock_guard<std::mutex> lk(s->mu);
  for (int q = 0; q < 4; ++q) {
    ns4[q] = s->ns_max[q];
    s->ns_max[q] = 0;
  }
  return kOk;
}

int mpzmm_server_set_admission_window(mpzmm_server* s, int64_t microseconds) {
  if (!s) return set_error(kErrArg, "null server");
  if (microseconds < 0) return set_error(kErrArg, "window must be >= 0");
  std::lock_guard<std::mutex> lk(s->mu);
  s->window_ns = microseconds * 1000;
  return kOk;
}

int mpzmm_server_stats(mpzmm_server* s, int64_t* batches, int64_t* products,
                       int64_t* max_in_flight) {
  if (!s) return set_error(kErrArg, "null server");
  std::lock_guard<std::mutex> lk(s->mu);
  if (batches) *batches = s->stat_batches;
  if (products) *products = s->stat_products;
  if (max_in_flight) *max_in_flight = s->stat_max_in_flight;
  return kOk;
}

void mpzmm_server_destroy(mpzmm_server* s) {
  if (!s) return;
  {
    std::lock_guard<std::mutex> lk(s->mu);
    s->stop = true;
  }
  s->cv_work.notify_all();
  for (auto& sl : s->slots)  // the slots drain queued and in-flight work first
    if (sl->thread.joinable()) sl->thread.join();
  for (auto& sl : s->slots) {
    cudaStreamSynchronize(sl->stream);
    cudaStreamSynchronize(sl->stream_hi);
    sl->ws.release();  // stream-ordered frees on the last batch's stream
    cudaStreamSynchronize(sl->stream);
    cudaStreamSynchronize(sl->stream_hi);
    cudaStreamDestroy(sl->stream);
    cudaStreamDestroy(sl->stream_hi);
  }
  if (s->pool) cudaMemPoolDestroy(s->pool);
  delete s;
}

}  // extern "C"
