// Host-side launchers of the sm_100a kernels (kernels.cu).
#pragma once

#include <cuda_runtime.h>

#include "mpzmm_internal.h"

namespace mpzmm {

cudaError_t upload_constants(const PrimeConst* primes, const CrtConst* crt);

// Split + forward NTT for `count` entries (descriptor indices idx[0..count)),
// all with transform length 2^lgN and P primes.
// max_r: the widest coefficient (bits) among the launch's entries.
cudaError_t launch_split_fwd(const FwdDesc* descs, const uint32_t* idx, int count, int P,
                             int lgN, const uint64_t* limbs, uint32_t* res,
                             const uint2* twf, cudaStream_t st, int max_r);

// Inverse NTT, in place, for `count` output entries of length 2^lgN.
cudaError_t launch_inv_ntt(const InvDesc* descs, const uint32_t* idx, int count, int P,
                           int lgN, uint32_t* res, const uint2* twi, cudaStream_t st);

// CUDA-core contraction over `count` work items.
cudaError_t launch_contract(const ProdDesc* prods, const ContractItem* items, int count,
                            uint32_t* res, cudaStream_t st);
int contract_block_freqs();

// CRT + recompose + sign for `count` output entries with P primes; rmin is
// the narrowest coefficient width among them (it sizes the shared scratch).
cudaError_t launch_crt_recompose(const InvDesc* descs, const uint32_t* idx, int count, int P,
                                 const uint32_t* res, uint32_t* out, int32_t* sizes, int rmin,
                                 cudaStream_t st);

}  // namespace mpzmm
