// mpzmm_matmul_noalloc: the exact product for callers that cannot allocate
// device memory.
//
// Who needs it: code whose device memory is owned entirely by a host
// framework's pool (a caching allocator that has reserved the GPU's memory,
// or a process run under a fixed memory budget), where a raw cudaMalloc
// fails or escapes the pool's accounting, and latency-sensitive callers that
// cannot afford cudaMalloc/cudaFree, whose calls may synchronise the whole
// device.  They hand in device buffers for the operands and results; this
// entry point brings nothing of its own but a fixed scratch area compiled
// into the library.
//
// The scratch (residues and descriptors) is the file-scope array
// g_noalloc_scratch below: kNoAllocScratchBytes (16 MiB) on every GPU that
// loads the library, held until the process exits.  The transform tables for
// this path live in two more static arrays (g_noalloc_twf / g_noalloc_twi,
// 4 MiB each, transforms up to 2^15 points).  Host code only sees
// the arrays' names as host-side stand-ins, never device addresses, so the
// first call on each device (with that device current) fetches their device
// addresses with cudaGetSymbolAddress and uploads the tables and constants
// with plain copies; that first call should come before any stream capture.
// Every call shares the one scratch array and leaves the last call's data in
// it: calls whose GPU work overlaps (two streams, two host threads) race and
// must be serialised by the caller.  It calls no cudaMalloc, cudaFree or
// other allocating routine.

#include <cuda_runtime.h>

#include <cstring>
#include <mutex>
#include <string>

#include "../../include/mpzmm_b200.h"
#include "engine.h"
#include "kernels.h"
#include "planner.h"

namespace mpzmm {
namespace {

constexpr size_t kNoAllocScratchBytes = (size_t)16 << 20;
constexpr int kNoAllocLgN = kTwiddleLg;             // largest transform: 2^15 points
constexpr int kNoAllocTwEntries = 1 << kTwiddleLg;  // same table layout as the batch path
constexpr size_t kNoAllocDescBytes = (size_t)1 << 20;  // part of the scratch
constexpr int kMaxDevices = 64;

static __device__ __align__(256) uint8_t g_noalloc_scratch[kNoAllocScratchBytes];
static __device__ __align__(256) uint2 g_noalloc_twf[kMaxPrimes * kNoAllocTwEntries];
static __device__ __align__(256) uint2 g_noalloc_twi[kMaxPrimes * kNoAllocTwEntries];

struct DeviceState {
  bool ready = false;
  uint8_t* scratch = nullptr;
  uint2* twf = nullptr;
  uint2* twi = nullptr;
};
DeviceState g_dev[kMaxDevices];
std::mutex g_mu;                                   // serialises the host side
alignas(64) uint8_t g_host_desc[kNoAllocDescBytes];  // descriptor staging (pageable)

int cufail(cudaError_t e, const char* what) {
  return set_error(kErrCuda, std::string(what) + ": " + cudaGetErrorString(e));
}

// Once per device, with that device current.
int setup_device(int dev, DeviceState** out) {
  if (dev < 0 || dev >= kMaxDevices) return set_error(kErrArg, "device index out of range");
  DeviceState& s = g_dev[dev];
  if (!s.ready) {
    cudaError_t e;
    if ((e = cudaGetSymbolAddress((void**)&s.scratch, g_noalloc_scratch)) != cudaSuccess)
      return cufail(e, "cudaGetSymbolAddress(scratch)");
    if ((e = cudaGetSymbolAddress((void**)&s.twf, g_noalloc_twf)) != cudaSuccess)
      return cufail(e, "cudaGetSymbolAddress(twiddles)");
    if ((e = cudaGetSymbolAddress((void**)&s.twi, g_noalloc_twi)) != cudaSuccess)
      return cufail(e, "cudaGetSymbolAddress(twiddles)");
    const Moduli& M = moduli();
    if ((e = upload_constants(M.pc, &M.crt)) != cudaSuccess) return cufail(e, "constants");
    if ((e = init_kernel_attributes()) != cudaSuccess) return cufail(e, "kernel attributes");
    if ((e = cudaMemcpy(s.twf, M.twf.data(), sizeof(uint2) * M.twf.size(),
                        cudaMemcpyHostToDevice)) != cudaSuccess ||
        (e = cudaMemcpy(s.twi, M.twi.data(), sizeof(uint2) * M.twi.size(),
                        cudaMemcpyHostToDevice)) != cudaSuccess)
      return cufail(e, "twiddle upload");
    s.ready = true;
  }
  *out = &s;
  return kOk;
}

size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

}  // namespace
}  // namespace mpzmm

using namespace mpzmm;

extern "C" int mpzmm_matmul_noalloc(int m, int k, int n, const uint64_t* d_a_limbs,
                                    const int64_t* a_offs, const int32_t* a_sizes,
                                    const uint64_t* d_b_limbs, const int64_t* b_offs,
                                    const int32_t* b_sizes, uint64_t* d_c_limbs,
                                    const int64_t* c_offs, const int64_t* c_caps,
                                    int32_t* d_c_sizes, void* stream) {
  std::lock_guard<std::mutex> lk(g_mu);
  if (m <= 0 || k < 0 || n <= 0) return set_error(kErrArg, "dimensions must be m, n > 0, k >= 0");
  const int64_t na = (int64_t)m * k, nb = (int64_t)k * n, nc = (int64_t)m * n;
  if ((na && (!a_offs || !a_sizes || !d_a_limbs)) || (nb && (!b_offs || !b_sizes || !d_b_limbs)) ||
      !c_offs || !c_caps || !d_c_sizes || !d_c_limbs)
    return set_error(kErrArg, "null array");
  // the product descriptor holds the dimensions in 16 bits
  if (m > 65535 || k > 65535 || n > 65535)
    return set_error(kErrTooLarge, "mpzmm_matmul_noalloc: dimension > 65535");
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  // the descriptors go up from one pageable host buffer that the next call
  // overwrites, so a call captured into a CUDA graph would replay stale ones
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  cudaError_t e = cudaStreamIsCapturing(s, &cap);
  if (e != cudaSuccess) return cufail(e, "cudaStreamIsCapturing");
  if (cap != cudaStreamCaptureStatusNone)
    return set_error(kErrArg, "mpzmm_matmul_noalloc: the stream is capturing (calls cannot be "
                              "captured into a CUDA graph)");
  int dev = 0;
  e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return cufail(e, "cudaGetDevice");
  DeviceState* ds = nullptr;
  int st = setup_device(dev, &ds);
  if (st) return st;

  // operand bit lengths bounded from the limb counts (the limbs are on the device)
  int64_t a_bits = 0, b_bits = 0;
  for (int64_t i = 0; i < na; ++i) {
    const int64_t l = a_sizes[i] < 0 ? -(int64_t)a_sizes[i] : a_sizes[i];
    if (64 * l > a_bits) a_bits = 64 * l;
  }
  for (int64_t i = 0; i < nb; ++i) {
    const int64_t l = b_sizes[i] < 0 ? -(int64_t)b_sizes[i] : b_sizes[i];
    if (64 * l > b_bits) b_bits = 64 * l;
  }
  Params prm;
  if (!choose_params(a_bits, b_bits, m, k, n, &prm))
    return set_error(kErrTooLarge, "mpzmm_matmul_noalloc: product too large");
  if (prm.P == 0) {  // identically zero: every result size is 0
    if ((e = cudaMemsetAsync(d_c_sizes, 0, sizeof(int32_t) * (size_t)nc, s)) != cudaSuccess)
      return cufail(e, "cudaMemsetAsync(sizes)");
    return kOk;
  }
  if (prm.lgN > kNoAllocLgN)
    return set_error(kErrTooLarge, "mpzmm_matmul_noalloc: transform of 2^" +
                                       std::to_string(prm.lgN) + " points exceeds the 2^" +
                                       std::to_string(kNoAllocLgN) + " limit of this entry point");
  for (int64_t i = 0; i < nc; ++i)
    if (c_caps[i] < prm.out_limbs)
      return set_error(kErrCapacity, "mpzmm_matmul_noalloc: output entry " + std::to_string(i) +
                                         " needs a capacity of " + std::to_string(prm.out_limbs) +
                                         " limbs");

  const int P = prm.P, lgN = prm.lgN, r = prm.r;
  const uint64_t N = (uint64_t)1 << lgN, poly = (uint64_t)P * N;
  const int bf = contract_block_freqs();
  const int64_t nitems = (int64_t)P * (int64_t)((N + bf - 1) / bf);
  // descriptor blob: fwd (A then B), inv, prod, items, index lists
  const size_t off_fwd = 0;
  const size_t off_inv = align256(off_fwd + sizeof(FwdDesc) * (size_t)(na + nb));
  const size_t off_pd = align256(off_inv + sizeof(InvDesc) * (size_t)nc);
  const size_t off_items = align256(off_pd + sizeof(ProdDesc));
  const size_t off_idx = align256(off_items + sizeof(ContractItem) * (size_t)nitems);
  const size_t desc_bytes = align256(off_idx + sizeof(uint32_t) * (size_t)(na + nb + nc));
  const size_t res_bytes = sizeof(uint32_t) * (size_t)(na + nb + nc) * poly;
  if (desc_bytes > kNoAllocDescBytes || desc_bytes + res_bytes > kNoAllocScratchBytes)
    return set_error(kErrTooLarge,
                     "mpzmm_matmul_noalloc: needs " + std::to_string(desc_bytes + res_bytes) +
                         " scratch bytes, the static scratch holds " +
                         std::to_string(kNoAllocScratchBytes));

  uint8_t* hd = g_host_desc;
  FwdDesc* fwd = reinterpret_cast<FwdDesc*>(hd + off_fwd);
  InvDesc* inv = reinterpret_cast<InvDesc*>(hd + off_inv);
  ProdDesc* pd = reinterpret_cast<ProdDesc*>(hd + off_pd);
  ContractItem* items = reinterpret_cast<ContractItem*>(hd + off_items);
  uint32_t* idx = reinterpret_cast<uint32_t*>(hd + off_idx);
  pd->m = (uint16_t)m;
  pd->k = (uint16_t)k;
  pd->n = (uint16_t)n;
  pd->lgN = (uint16_t)lgN;
  pd->P = (uint16_t)P;
  pd->pad = (uint16_t)contract_tile(m, n);  // contraction tile
  pd->a_res = 0;
  pd->b_res = (uint64_t)na * poly;
  pd->c_res = (uint64_t)(na + nb) * poly;
  for (int64_t i = 0; i < na + nb; ++i) {
    const bool isb = i >= na;
    const int64_t e2 = isb ? i - na : i;
    const int32_t sz = isb ? b_sizes[e2] : a_sizes[e2];
    const int64_t nl = sz < 0 ? -(int64_t)sz : sz;
    FwdDesc& f = fwd[i];
    f.limb_off = nl ? (uint64_t)(isb ? b_offs[e2] : a_offs[e2]) : 0;
    f.res_off = (isb ? pd->b_res : pd->a_res) + (uint64_t)e2 * poly;
    f.size = sz;
    f.r = (uint32_t)r;
    f.lgN = (uint16_t)lgN;
    f.P = (uint16_t)P;
    const uint64_t nco = ((uint64_t)nl * 64 + r - 1) / r;
    f.ncoef = (uint32_t)(nco < N ? nco : N);
    f.tile_np = 0;  // plain layout (this entry point contracts on CUDA cores)
    f.tile_e = 0;
    idx[i] = (uint32_t)i;
  }
  int64_t it = 0;
  for (int j = 0; j < P; ++j)
    for (uint64_t h0 = 0; h0 < N; h0 += (uint64_t)bf) {
      items[it].prod = 0;
      items[it].prime = (uint16_t)j;
      items[it].pad = 0;
      items[it].h0 = (uint32_t)h0;
      ++it;
    }
  const uint64_t ncoef_c = (uint64_t)(prm.lenA + prm.lenB - 1);
  for (int64_t i = 0; i < nc; ++i) {
    InvDesc& d = inv[i];
    d.res_off = pd->c_res + (uint64_t)i * poly;
    d.out_word = 2 * (uint64_t)c_offs[i];
    d.out_words = (uint32_t)(2 * prm.out_limbs);
    d.r = (uint32_t)r;
    d.ncoef = (uint32_t)(ncoef_c < N ? ncoef_c : N);
    d.lgN = (uint16_t)lgN;
    d.P = (uint16_t)P;
    d.entry = (uint32_t)i;
    idx[na + nb + i] = (uint32_t)i;
  }
  uint8_t* dd = ds->scratch;
  uint32_t* dres = reinterpret_cast<uint32_t*>(ds->scratch + desc_bytes);
  // every check has passed: only now is anything of the caller's touched.
  // Results start cleared: every size is rewritten by the CRT kernel or
  // stays 0.
  if ((e = cudaMemsetAsync(d_c_sizes, 0, sizeof(int32_t) * (size_t)nc, s)) != cudaSuccess)
    return cufail(e, "cudaMemsetAsync(sizes)");
  // a copy from pageable memory: it returns once the descriptors are staged,
  // so the next call may reuse g_host_desc
  if ((e = cudaMemcpyAsync(dd, hd, desc_bytes, cudaMemcpyHostToDevice, s)) != cudaSuccess)
    return cufail(e, "descriptor upload");
  const FwdDesc* dfwd = reinterpret_cast<const FwdDesc*>(dd + off_fwd);
  const InvDesc* dinv = reinterpret_cast<const InvDesc*>(dd + off_inv);
  const ProdDesc* dpd = reinterpret_cast<const ProdDesc*>(dd + off_pd);
  const ContractItem* ditems = reinterpret_cast<const ContractItem*>(dd + off_items);
  const uint32_t* didx = reinterpret_cast<const uint32_t*>(dd + off_idx);

  if ((e = launch_split_fwd(dfwd, didx, (int)na, P, lgN, d_a_limbs, dres, ds->twf, s)) !=
          cudaSuccess ||
      (e = launch_split_fwd(dfwd, didx + na, (int)nb, P, lgN, d_b_limbs, dres, ds->twf, s)) !=
          cudaSuccess ||
      (e = launch_contract(dpd, ditems, (int)nitems, dres, s)) != cudaSuccess ||
      (e = launch_inv_ntt(dinv, didx + na + nb, (int)nc, P, lgN, dres, ds->twi, s)) !=
          cudaSuccess ||
      (e = launch_crt_recompose(dinv, didx + na + nb, (int)nc, P, dres,
                                reinterpret_cast<uint32_t*>(d_c_limbs), d_c_sizes, r, s)) !=
          cudaSuccess)
    return cufail(e, "mpzmm_matmul_noalloc launch");
  return kOk;
}
