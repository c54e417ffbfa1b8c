// Batch engine: plans a set of independent products, moves their limbs to
// the device, runs the four pipeline stages with one launch per stage and
// size class, and brings the results back.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <functional>
#include <memory>
#include <mutex>
#include <string>
#include <utility>
#include <vector>

#include "mpzmm_internal.h"
#include "planner.h"

namespace mpzmm {

// Status codes (same values as the public header).
enum Status : int {
  kOk = 0,
  kErrArg = 1,
  kErrTooLarge = 2,
  kErrCapacity = 3,
  kErrCuda = 4,
  kErrNoMem = 5,
  kErrState = 6,
  kErrTimeout = 7,
  kErrBusy = 8,
  kErrBounds = 9,
};

int set_error(int status, const std::string& msg);
const char* last_error();

// One integer operand: limb pointer and GMP-style signed size.
struct EntryRef {
  const uint64_t* d;
  int32_t size;
};

// Where one output entry goes.
struct OutRef {
  uint64_t* d;       // destination limbs (packed output) or nullptr (mpz)
  int64_t cap;       // capacity in limbs (packed output)
  int32_t* size;     // signed size destination (packed output)
  void* mpz;         // mpz_ptr destination (mpz output) or nullptr
};

// An operand already in device memory (the output of an earlier plan):
// entry e's limbs at limbs + offs[e] (at most cap_limbs of them, zero above
// the value), its signed size at sizes[e]; the sizes are read on the device.
struct DeviceOperand {
  const uint64_t* limbs = nullptr;
  const int32_t* sizes = nullptr;
  std::vector<int64_t> offs;
  int64_t cap_limbs = 0;
  uint64_t span_limbs = 0;  // limbs from limbs[0] to the end of the last entry
};

// Bit length of an entry's magnitude (0 for zero).
int64_t bit_length(const EntryRef& e);

struct ProductSpec {
  int m = 0, k = 0, n = 0;
  std::vector<EntryRef> a, b;  // m*k and k*n entries, row-major
  std::vector<OutRef> c;       // m*n entries
  // A in device memory instead of `a` (whose sizes are then ignored)
  std::shared_ptr<DeviceOperand> dev_a;
  // results stay on the device for a later plan (no host outputs)
  bool device_only = false;
};

// Device and pinned host buffers of a plan.  Grow-only, so one workspace is
// reused by every one-shot call (no per-call cudaMalloc / cudaMallocHost once
// it has reached the working size).
struct Workspace {
  uint64_t* d_limbs = nullptr;
  uint32_t* d_res = nullptr;
  uint32_t* d_out = nullptr;
  int32_t* d_sizes = nullptr;
  uint8_t* d_desc = nullptr;
  int* d_status = nullptr;  // nonzero: a kernel's bounded wait gave up
  // pinned staging: only the inputs and outputs that cannot move straight
  // between the caller's memory and the device pass through these
  uint64_t* h_limbs = nullptr;
  uint32_t* h_out = nullptr;
  int32_t* h_sizes = nullptr;
  uint8_t* h_desc = nullptr;
  int* h_status = nullptr;  // pinned copy of d_status
  size_t cap_limbs = 0, cap_res = 0, cap_out = 0, cap_sizes = 0, cap_desc = 0;
  size_t hcap_limbs = 0, hcap_out = 0, hcap_sizes = 0, hcap_desc = 0;
  int64_t device_bytes = 0;
  // With a stream set, device buffers come from a stream-ordered memory pool
  // (cudaMallocAsync / cudaFreeAsync on that stream): `pool` if set, else
  // the device's default pool.  Nothing then synchronises the device.
  cudaStream_t async_stream = nullptr;
  cudaMemPool_t pool = nullptr;
  // Pinned staging outgrown by a later batch: kept here and freed only by
  // release() when retire_host is set (cudaFreeHost synchronises the whole
  // device, which would stall every other batch in flight).
  bool retire_host = false;
  std::vector<void*> retired_host;
  // Side streams a plan spreads one stage's independent launches over (so
  // one launch's last wave overlaps the next launch's first), with the
  // events that fork them off and join them back; created on first use.
  static constexpr int kSideStreams = 2;
  bool fanout = true;  // false: every launch on the plan's own stream
  cudaStream_t side[kSideStreams] = {};
  cudaEvent_t fork_ev = nullptr;
  cudaEvent_t join_ev[kSideStreams] = {};
  int ensure_side();
  // Ensures room for the given element counts (device buffers, then the
  // pinned staging of limbs and output words); returns a status.
  int reserve(size_t limbs, size_t res, size_t out_words, size_t sizes, size_t desc_bytes,
              size_t stage_limbs, size_t stage_out_words);
  // Grows only the pinned staging (limbs, output words, result sizes,
  // descriptor bytes) to at least these counts: a long-lived workspace sized
  // once so that later batches never allocate pinned memory (cudaMallocHost
  // is slow and cudaFreeHost synchronises the device).
  int reserve_staging(size_t stage_limbs, size_t stage_out_words, size_t sizes = 0,
                      size_t desc_bytes = 0);
  void release_device();  // device buffers only (pinned host buffers stay)
  void release();
  ~Workspace() { release(); }
};

// Device bytes a batch of products will reserve (parameters, residues,
// limbs, outputs and descriptors), without building it; host_bytes (if
// given) receives the bytes its inputs and outputs move across the link.
int64_t estimate_device_bytes(const ProductSpec& ps, int64_t* host_bytes = nullptr);

// Process-wide device state: tables on the device, default stream.
struct Context {
  bool ready = false;
  int device = -1;
  cudaStream_t stream = nullptr;
  uint2* d_twf = nullptr;
  uint2* d_twi = nullptr;
  // four-step twist tables, one allocation (forward hi, inverse hi, then
  // forward lo, inverse lo)
  void* d_twist = nullptr;
  TwistTab twist_f{nullptr, nullptr}, twist_i{nullptr, nullptr};
  int num_sms = 0;
  Workspace* ws = nullptr;  // shared by one-shot calls (guarded by ws_mu)
  // contraction engine: 0 automatic (tensor cores from kTcMinK terms on),
  // 1 CUDA cores only, 2 tensor cores wherever the shape allows
  int contract_mode = 0;
  bool check_bounds = false;  // MPZMM_OPT_CHECK_BOUNDS (env MPZMM_CHECK_BOUNDS)
  // measured engine choice per size class (term-count bucket k <= 8, 16, 32,
  // 64 by row/column bucket max(m, n) <= 4, 8, 16, 32, 64) in automatic
  // mode: -1 not measured (CUDA cores), 0 CUDA cores, 1 tensor cores;
  // filled by mpzmm_autotune
  int tc_pref[4][5] = {{-1, -1, -1, -1, -1}, {-1, -1, -1, -1, -1}, {-1, -1, -1, -1, -1},
                       {-1, -1, -1, -1, -1}};
  // pipelined one-shot batches: workspaces and streams of the chunks in
  // flight (the first workspace is `ws`), created on first use
  std::vector<Workspace*> pipe_ws;
  std::vector<cudaStream_t> pipe_st;  // kernels, one stream per slot
  cudaStream_t pipe_in = nullptr;     // every chunk's host->device copies, in order
  cudaStream_t pipe_out = nullptr;    // every chunk's device->host copies, in order
  cudaEvent_t pipe_ev = nullptr;
  // per slot: its chunk's inputs on the device, its kernels done, its
  // results on the host
  std::vector<cudaEvent_t> pipe_ev_in, pipe_ev_exec, pipe_ev_out;
  int64_t chunk_limbs = 0;  // input limbs per chunk; 0 = automatic
  // last one-shot batch: host time of planning, input copies, launch
  // queueing, waiting + results (ns); chunks; bytes host->device,
  // device->host, and the parts of those that moved straight between the
  // caller's pinned memory and the device
  int64_t batch_ns[4] = {0, 0, 0, 0};
  int64_t batch_chunks = 0;
  int64_t batch_bytes[4] = {0, 0, 0, 0};
  // per-chunk timeline of the last one-shot batch, kTimelineFields values a
  // chunk (see mpzmm_batch_timeline); tl_ev: the batch's start event and
  // four per chunk, with timing
  std::vector<double> timeline;
  std::vector<cudaEvent_t> tl_ev;
};

// Values per chunk in a batch timeline: plan begin / end, submit begin /
// end (host, ms), copy-in begin / end, kernels end, copy-out end (device,
// ms), bytes in, bytes out.
constexpr int kTimelineFields = 10;

// Workspaces a pipelined one-shot batch may cycle through (chunks in
// flight); it uses MPZMM_PIPE_DEPTH of them, 2 .. kPipeDepth, default 4.
constexpr int kPipeDepth = 8;
// Largest host gap (limbs) between consecutive entries in one pinned range
// that a copy run bridges instead of starting a new copy.
constexpr int64_t kRunGapLimbs = 256;

inline int tc_bucket_k(int k) {
  int b = 0;
  while ((1 << (b + 3)) < k) ++b;
  return b < 4 ? b : 3;
}
inline int tc_bucket_mn(int m, int n) {
  const int x = m > n ? m : n;
  int b = 0;
  while ((1 << (b + 2)) < x) ++b;
  return b < 5 ? b : 4;
}

constexpr int kTcFreqsPerCta = 128;  // = contract_tc_freqs() (frequencies per tensor-core CTA)

Context& context();
std::mutex& workspace_mutex();

// Failure injection for the library's own failure-path tests (host side
// only; nothing faults a GPU): the next `count` tensor-core contraction
// launches issue no tensor work, so their bounded waits run out
// (MPZMM_ERR_TIMEOUT); the next `count` device or pinned-host allocations
// of a workspace report failure (MPZMM_ERR_NOMEM).
void set_test_stall_tc(int count);
void set_test_fail_alloc(int count);
int test_stall_tc();
int test_fail_alloc();
// consumes one pending injection (true if one was pending)
bool take_test_stall_tc();
bool take_test_fail_alloc();

// Runs fn(lo, hi) over [0, n) split across host threads when `bytes` is
// large enough to be worth it (gather/scatter of limbs).
void parallel_chunks(size_t n, size_t bytes, const std::function<void(size_t, size_t)>& fn);
int ensure_setup(int device);
void teardown();

// Pinned host memory known to the library: transfers whose host side lies
// wholly inside one such range go straight to or from the caller's memory.
int host_alloc(size_t bytes, void** out);
int host_free(void* p);
int host_register(void* p, size_t bytes);
int host_unregister(void* p);
bool host_range_pinned(const void* p, size_t bytes);
// Snapshot of the known ranges (sorted by start) and lookups in it.
std::vector<std::pair<uintptr_t, size_t>> pinned_ranges();
bool in_ranges(const std::vector<std::pair<uintptr_t, size_t>>& v, const void* p, size_t bytes);
// End address of the range holding [p, p + bytes), 0 if none does.
uintptr_t range_end(const std::vector<std::pair<uintptr_t, size_t>>& v, const void* p,
                    size_t bytes);

class Plan {
 public:
  static constexpr int kStages = 4;
  ~Plan();
  // Computes parameters, descriptors and launch groups, and reserves device
  // and pinned host buffers in `ws` (the plan's own workspace if null):
  // prepare() then bind().
  int build(std::vector<ProductSpec> prods, Workspace* ws = nullptr);
  // The host half of build(): parameters, descriptors, launch groups and
  // transfer runs; touches no workspace, so a pipeline can plan a chunk
  // while the workspace it will use is still busy with an earlier one.
  int prepare(std::vector<ProductSpec> prods);
  // The rest: reserves buffers in `ws` and writes the descriptors into its
  // pinned staging.
  int bind(Workspace* ws);
  // Copies the input limbs (and the descriptors) to the device: straight
  // from the caller's memory where it is pinned memory known to the library,
  // through the pinned staging buffer otherwise.
  int upload(cudaStream_t st);
  // Keep B's transforms (call before build): B operands get forward launches
  // of their own, which run at the first execute after an upload() and are
  // skipped by later executes; upload_a() re-reads only the A operands, so
  // their products with the same B need only A's split and transforms.
  // Such a plan takes host operands only and does not capture CUDA graphs.
  void set_fixed_b(bool on) { fixed_b_ = on; }
  int upload_a(cudaStream_t st) { return upload_sides(st, true); }
  // Runs split+fwd NTT, contraction, inverse NTT, CRT+recompose.  With
  // graph mode on (and timing off) the launches are captured into a CUDA
  // graph on the first call and replayed as one graph launch afterwards.
  int execute(cudaStream_t st);
  void set_graph(bool on) { use_graph_ = on; }
  // Copies outputs back and writes them to the output references:
  // download_enqueue queues the device->host copies, download_finish waits
  // (for `done` when given, else for the whole stream) and writes sizes and
  // staged limbs to the destinations.
  int download(cudaStream_t st);
  int download_enqueue(cudaStream_t st);
  int download_finish(cudaStream_t st, cudaEvent_t done = nullptr);
  // bytes moved per upload / download, and the parts of them that go
  // straight between pinned caller memory and the device
  uint64_t upload_bytes() const { return n_limbs_ * 8 + desc_bytes_; }
  uint64_t download_bytes() const {
    return n_out_words_ * 4 + (inv_.empty() ? 0 : outs_.size() * 4) + sizeof(int);
  }
  uint64_t direct_in_bytes() const { return direct_in_limbs_ * 8; }
  uint64_t direct_out_bytes() const { return direct_out_words_ * 4; }
  // the results on the device (valid until the workspace is reused):
  // product t's output entry e at output limb offset out_limb_offset(...)
  DeviceOperand device_output(size_t product) const;

  int64_t launches_per_execute() const { return launches_; }
  // Stage timing with CUDA events recorded on the execute stream: stages are
  // 0 split+forward NTT, 1 contraction, 2 inverse NTT, 3 CRT+recompose.
  void set_timing(bool on) { timing_ = on; }
  int stage_times(float ms[kStages], int64_t* executes);
  void stage_launches(int64_t out[kStages]) const;
  int64_t device_bytes() const { return ws_ ? ws_->device_bytes : 0; }
  const std::vector<Params>& params() const { return params_; }
  std::vector<ProductSpec>& products() { return prods_; }

 private:
  struct Group {
    int P = 0, lgN = 0;
    int max_r = 0;         // split: widest coefficient; CRT: narrowest coefficient
    uint32_t idx_off = 0;  // into the device index array
    std::vector<uint32_t> idx;
    // batched transform launch (several size classes, CTA work items)
    bool batched = false;
    bool team = false;
    bool large = false;    // four-step transform (2^lgN above one CTA)
    bool tiled = false;    // forward: operands of tensor-core products (blocked layout)
    bool b_only = false;   // forward: B operands of a plan that keeps their transforms
    int D = 0;
    int max_lgN = 0;
    std::vector<CtaItem> items;
    uint32_t item_off = 0;
    // CRT launch over several prime counts: the upper range, and the
    // narrowest coefficient width per count
    bool crt_high = false;
    std::vector<int> rmin;
  };

  std::vector<ProductSpec> prods_;
  std::vector<Params> params_;
  std::vector<FwdDesc> fwd_;
  std::vector<InvDesc> inv_;
  std::vector<ProdDesc> pd_;
  std::vector<ContractItem> items_;     // CUDA-core contraction work
  std::vector<ContractItem> tc_items_;  // tensor-core contraction work
  std::vector<int> tc_shapes_;  // distinct (m, k, n) of the tensor-core products
  std::vector<Group> fwd_groups_, inv_groups_, rec_groups_;
  std::vector<uint32_t> idx_all_;
  std::vector<CtaItem> cta_items_;
  std::vector<OutRef> outs_;          // flattened output references
  std::vector<int64_t> out_word_off_; // per output entry (words)
  std::vector<int32_t> out_limbs_;    // per output entry: limbs the device writes
  // host<->device transfer runs: `rows` rows of `n` elements (limbs in,
  // words out) between host address `host` (rows `pitch` elements apart)
  // and device element offset `dev` (rows back to back); staged runs go
  // through the pinned staging buffer at element offset `stage`
  struct Run {
    const void* host;
    uint64_t dev, n, stage;
    bool direct;
    uint64_t rows, pitch;
    bool b = false;  // input run of B operands (plans that keep B's transforms)
  };
  std::vector<Run> in_runs_, out_runs_;
  // device-resident operands: limb spans copied on the device, and the
  // forward descriptors whose sizes come from device memory
  struct DevRun {
    const uint64_t* src;
    uint64_t dst, n;
  };
  std::vector<DevRun> dev_runs_;
  struct DevFix {
    const int32_t* sizes;  // device array of the operand
    uint32_t first_fwd;    // descriptors first_fwd .. + count - 1
    uint32_t count;
  };
  std::vector<DevFix> dev_fixes_;
  std::vector<size_t> prod_first_out_;  // first output entry of each product
  std::vector<int64_t> out_stage_;    // per output entry: staging word offset, -1 if direct
  uint64_t stage_limbs_ = 0, stage_out_words_ = 0;
  uint64_t direct_in_limbs_ = 0, direct_out_words_ = 0;
  void plan_transfers();
  std::vector<uint8_t> zero_prod_;    // product is identically zero

  uint64_t n_limbs_ = 0, n_res_ = 0, n_out_words_ = 0;
  int64_t launches_ = 0;

  Workspace own_;
  Workspace* ws_ = nullptr;
  // descriptor blob: offsets of each section (bytes) and its size
  size_t off_fwd_ = 0, off_inv_ = 0, off_pd_ = 0, off_items_ = 0, off_idx_ = 0, off_cta_ = 0,
         desc_bytes_ = 0;
  CtaItem* d_cta_ = nullptr;
  FwdDesc* d_fwd_ = nullptr;
  InvDesc* d_inv_ = nullptr;
  ProdDesc* d_pd_ = nullptr;
  ContractItem* d_items_ = nullptr;
  ContractItem* d_tc_items_ = nullptr;
  size_t off_tc_ = 0;
  uint32_t* d_idx_ = nullptr;
  bool built_ = false;
  bool prepared_ = false;
  bool timing_ = false;
  std::vector<cudaEvent_t> events_;  // kStages + 1 per timed execute
  bool use_graph_ = false;
  bool fixed_b_ = false;
  bool check_bounds_ = false;  // the debug bounds check runs before every execute
  int check_bounds(cudaStream_t st);
  bool b_valid_ = false;  // B's transforms in device memory match its limbs
  int upload_sides(cudaStream_t st, bool a_only);
  cudaGraph_t graph_ = nullptr;
  cudaGraphExec_t graph_exec_ = nullptr;
  int launch_all(cudaStream_t st, bool timed);
};

// One-shot batch on the shared workspace: build, upload, execute, download.
// Batches with more input than one chunk are split into chunks of whole
// products that run as a pipeline over kPipeDepth workspaces: all chunks'
// host->device copies go in order on one stream, all device->host copies on
// another, and each chunk's kernels on its slot's stream between the two,
// so one chunk's inputs move in while earlier chunks compute and return
// their results (two copy streams also keep the copy directions on
// separate copy queues).  Returns when every result is written.
int run_batch(std::vector<ProductSpec> specs, cudaStream_t st);
// How run_batch splits a batch whose products have `limbs` input limbs each
// (chunk_option: MPZMM_OPT_CHUNK_LIMBS, 0 automatic): product-index bounds
// (first 0, last the count); false when it runs as one unchunked pass.
bool batch_chunks(const std::vector<uint64_t>& limbs, int64_t chunk_option,
                  std::vector<size_t>* bounds);

// Chain of products, each step's A being the previous step's result kept in
// device memory (steps[0] is an ordinary product; steps[i > 0] give B and
// the dimensions, their `a` entries are placeholders); only the last step's
// results are copied back to its outputs.  Returns when they are written.
int run_chain(std::vector<ProductSpec> steps, cudaStream_t st);

}  // namespace mpzmm
