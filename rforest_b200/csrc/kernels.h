// Host-side launchers of the sm_100a kernels (kernels.cu).
#pragma once

#include <cuda_runtime.h>

#include "mpzmm_internal.h"

namespace mpzmm {

cudaError_t upload_constants(const PrimeConst* primes, const CrtConst* crt);
// Sets every kernel's dynamic shared-memory limit on the current device.
cudaError_t init_kernel_attributes();

// Radix-2 split + forward NTT / inverse NTT, one CTA per (entry, prime),
// for `count` entries of one class (any lgN >= 1; used for lgN < 3).
cudaError_t launch_split_fwd(const FwdDesc* descs, const uint32_t* idx, int count, int P,
                             int lgN, const uint64_t* limbs, uint32_t* res,
                             const uint2* twf, cudaStream_t st);
cudaError_t launch_inv_ntt(const InvDesc* descs, const uint32_t* idx, int count, int P,
                           int lgN, uint32_t* res, const uint2* twi, cudaStream_t st);

// Register-blocked transforms (lgN >= 3) over CTA work items of mixed size
// classes in ONE launch.  team: every item has 2^lgN <= fwd_team_points()
// (several entries per CTA); otherwise one entry per CTA and max_lgN sizes
// the shared memory.  D = digits of 30 bits of the widest coefficient.
int fwd_team_points();
// tiled: the launch's entries are operands of tensor-core products, written
// in the frequency-blocked layout (FwdDesc::tile_np); else the plain layout.
cudaError_t launch_fwd_items(const FwdDesc* descs, const uint32_t* idx, const CtaItem* items,
                             int nitems, int D, bool team, int max_lgN, const uint64_t* limbs,
                             uint32_t* res, const uint2* twf, cudaStream_t st,
                             bool tiled = false);
cudaError_t launch_inv_items(const InvDesc* descs, const uint32_t* idx, const CtaItem* items,
                             int nitems, bool team, int max_lgN, uint32_t* res,
                             const uint2* twi, cudaStream_t st);

// Transforms of 2^16 .. 2^20 points (four-step: column transforms, twist,
// block transforms), `count` entries of one length 2^lgN in one group (idx
// lists their descriptors).  Forward: split of D-digit coefficients + the
// transform; inverse: the transform back to natural order, ready for the
// CRT.  Two launches each.  tt: the twist tables of the direction.
cudaError_t launch_large_fwd(const FwdDesc* descs, const uint32_t* idx, int count, int lgN, int D,
                             const uint64_t* limbs, uint32_t* res, const uint2* twf,
                             const TwistTab& tt, cudaStream_t st);
cudaError_t launch_large_inv(const InvDesc* descs, const uint32_t* idx, int count, int lgN,
                             uint32_t* res, const uint2* twi, const TwistTab& tt,
                             cudaStream_t st);
constexpr int kLargeLaunches = 2;  // kernel launches per direction of a four-step group

// CUDA-core contraction over `count` work items.
cudaError_t launch_contract(const ProdDesc* prods, const ContractItem* items, int count,
                            uint32_t* res, cudaStream_t st);
int contract_block_freqs();
// writes the device-held signed sizes (and coefficient counts) of `count`
// forward descriptors
cudaError_t launch_fix_sizes(FwdDesc* descs, int count, const int32_t* sizes, cudaStream_t st);
// modular reduction helpers: sizes of operands viewed `shift` limbs up, and
// the final step of x mod d (see mod.cpp)
cudaError_t launch_shift_sizes(const int32_t* in, int32_t* out, int count, int shift,
                               cudaStream_t st);
cudaError_t launch_mod_finish(int count, int n, const uint64_t* xl, const int64_t* xo,
                              const int32_t* xs, const uint64_t* sl, int64_t s_stride,
                              const int32_t* ss, const uint64_t* d, uint64_t* rbuf, int32_t* rs,
                              cudaStream_t st);

// Tensor-core contraction (tcgen05 kind::i8) for products with m <= 128,
// k <= 64, n <= 64; shapes: the launch's distinct (m, k, n), nshapes triples
// (they size its shared memory); each work item covers contract_tc_freqs()
// consecutive frequencies.  *status is set to 1 if a bounded wait gave up.
// stall != 0 (failure-path tests only) issues no tensor work, so every CTA's
// wait runs out.
// Debug check (MPZMM_OPT_CHECK_BOUNDS): every forward, inverse and product
// descriptor's extents against the workspace capacities (limbs, residue
// words, output words, result sizes); a thread that finds one outside sets
// *status to 2 and touches nothing else.
struct BoundsCaps {
  uint64_t limbs, res, out_words, sizes;
};
cudaError_t launch_check_bounds(const FwdDesc* fwd, int nfwd, const InvDesc* inv, int ninv,
                                const ProdDesc* prods, int nprods, BoundsCaps caps, int* status,
                                cudaStream_t st);
bool contract_tc_eligible(int m, int k, int n);
int contract_tc_freqs();
int tc_smem_bytes(int m, int k, int n, int F);
cudaError_t launch_contract_tc(const ProdDesc* prods, const ContractItem* items, int count,
                               uint32_t* res, const int* shapes, int nshapes, int* status,
                               cudaStream_t st, int stall = 0);

// CRT + recompose + sign for `count` output entries with P primes; rmin is
// the narrowest coefficient width among them (it sizes the shared scratch).
cudaError_t launch_crt_recompose(const InvDesc* descs, const uint32_t* idx, int count, int P,
                                 const uint32_t* res, uint32_t* out, int32_t* sizes, int rmin,
                                 cudaStream_t st);

// The same over several prime counts in one launch: high = false takes the
// entries with 2..kCrtMixedSplit primes, high = true those with more (each
// launch's entries in idx, longest first); rmin[P] is the narrowest
// coefficient width among the entries with P primes (0: none).
constexpr int kCrtMixedSplit = 10;
struct CrtScratch {
  int cmax[kMaxPrimes + 1];  // tile coefficients per prime count
  int warp_words;            // scratch words of one warp
};
cudaError_t launch_crt_mixed(const InvDesc* descs, const uint32_t* idx, int count, bool high,
                             const int* rmin, const uint32_t* res, uint32_t* out, int32_t* sizes,
                             cudaStream_t st);

}  // namespace mpzmm
