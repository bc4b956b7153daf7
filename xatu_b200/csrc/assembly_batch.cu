// Batched persistent assembly of many systems (mixed precision); the tile body is assemble_tile
// (assembly_tile.cuh).
#include <algorithm>

#include "assembly_tile.cuh"
#include "kernels.h"

// Persistent batched assembly (mixed precision) over the tiles of many systems
// of one band-window class: each CTA takes (system, tile) items from a device
// work list through an atomic counter until the list is exhausted; the
// system's parameters are copied to shared memory once per item.
template <int NV, int NC, int NA, int TK>
__global__ void __launch_bounds__(TK * TK)
bse_assemble_batch_kernel(const AsmBatchMember* __restrict__ members, const int2* __restrict__ work, int nwork,
                          int* __restrict__ counter) {
  __shared__ AsmBatchMember sm;
  __shared__ int s_item;
  for (;;) {
    if (threadIdx.x == 0) s_item = atomicAdd(counter, 1);
    __syncthreads();
    const int it = s_item;
    if (it >= nwork) break;
    const int2 w = work[it];
    {
      const int* src = reinterpret_cast<const int*>(members + w.x);
      int* dst = reinterpret_cast<int*>(&sm);
      for (int q = threadIdx.x; q < (int)(sizeof(AsmBatchMember) / sizeof(int)); q += blockDim.x) dst[q] = src[q];
    }
    __syncthreads();
    assemble_tile<float, NV, NC, NA, true, TK>(sm.p, sm.in, sm.out, sm.nblk, w.y);
    __syncthreads();
  }
}

size_t xatu_assembly_batch_smem(int nv, int nc, int na, int tk, int norb, int exchange) {
  const int tr = tk * nv * nc;
  return (2 * (size_t)(nv + nc) * norb * (tk + 1) + (size_t)tr * (tr + 1) + (exchange ? 2 * (size_t)tr * na : 0)) *
         sizeof(cplx<float>);
}

template <int NV, int NC, int NA, int TK>
static cudaError_t launch_batch_t(const AsmBatchMember* members, const int2* work, int nwork, int* counter,
                                  size_t smem, int num_sms, bool set_attr, cudaStream_t s) {
  auto kern = bse_assemble_batch_kernel<NV, NC, NA, TK>;
  if (set_attr) {
    cudaError_t e = xatu_raise_smem_limit((const void*)kern, smem);
    if (e != cudaSuccess) return e;
  }
  int per_sm = 0;
  cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, TK * TK, smem);
  if (e != cudaSuccess) return e;
  if (per_sm < 1) return cudaErrorInvalidConfiguration;
  const int grid = std::max(1, std::min(nwork, per_sm * num_sms));
  kern<<<grid, TK * TK, smem, s>>>(members, work, nwork, counter);
  return cudaGetLastError();
}

template <int NV, int NC, int NA>
static cudaError_t launch_batch_tk(int tk, const AsmBatchMember* members, const int2* work, int nwork, int* counter,
                                   size_t smem, int num_sms, bool set_attr, cudaStream_t s) {
  if (tk == 8) return launch_batch_t<NV, NC, NA, 8>(members, work, nwork, counter, smem, num_sms, set_attr, s);
  if (tk == 16) return launch_batch_t<NV, NC, NA, 16>(members, work, nwork, counter, smem, num_sms, set_attr, s);
  return cudaErrorInvalidValue;
}

template <int NV, int NC>
static cudaError_t launch_batch_na(int na, int tk, const AsmBatchMember* members, const int2* work, int nwork,
                                   int* counter, size_t smem, int num_sms, bool set_attr, cudaStream_t s) {
  if (na == 2) return launch_batch_tk<NV, NC, 2>(tk, members, work, nwork, counter, smem, num_sms, set_attr, s);
  if (na == 3) return launch_batch_tk<NV, NC, 3>(tk, members, work, nwork, counter, smem, num_sms, set_attr, s);
  return cudaErrorInvalidValue;
}

bool xatu_assembly_batch_supported(int nv, int nc, int na) {
  return nv >= 1 && nv <= 3 && nc >= 1 && nc <= 3 && (na == 2 || na == 3);
}

cudaError_t xatu_launch_assembly_batch(int nv, int nc, int na, int tk, const AsmBatchMember* members,
                                       const int2* work, int nwork, int* counter, size_t smem, int num_sms,
                                       bool set_attr, cudaStream_t s) {
#define XATU_BCASE(NVv, NCv) \
  if (nv == NVv && nc == NCv) return launch_batch_na<NVv, NCv>(na, tk, members, work, nwork, counter, smem, num_sms, set_attr, s);
  XATU_BCASE(1, 1)
  XATU_BCASE(1, 2)
  XATU_BCASE(1, 3)
  XATU_BCASE(2, 1)
  XATU_BCASE(2, 2)
  XATU_BCASE(2, 3)
  XATU_BCASE(3, 1)
  XATU_BCASE(3, 2)
  XATU_BCASE(3, 3)
#undef XATU_BCASE
  return cudaErrorInvalidValue;
}

