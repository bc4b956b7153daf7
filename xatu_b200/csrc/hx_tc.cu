// Y = K X on the 5th-generation tensor cores (tcgen05, sm_100a).
//
// K is the mixed-precision BSE interaction kernel, stored as two BF16 planes
// (K = K_hi + K_lo, complex interleaved, row pitch ldk complex elements).  Read
// as a real matrix it is A = N x 2N (row i = Re K_i0, Im K_i0, Re K_i1, ...).
// The complex block X (N x b) enters through the real operand
//   Bt (2b x 2N, K-major):  Bt[s][2j] = Re X_js,  Bt[s][2j+1] = -Im X_js,
//                           Bt[b+s][2j] = Im X_js, Bt[b+s][2j+1] = Re X_js,
// so that (A Bt^T)[i][s] = Re (K X)_is and (A Bt^T)[i][b+s] = Im (K X)_is.
// Split-BF16 products: A_hi Bt_hi + A_hi Bt_lo + A_lo Bt_hi, FP32 accumulation
// in tensor memory (the lo*lo term is below FP32 rounding of the result).
//
// Kernel structure (one CTA per SM, persistent, split-K):
//   * the 128-row x 64-column (128 B) tiles of A are enumerated m-block-major and
//     cut into equal contiguous ranges, one per CTA; a range spans at most
//     XHX_NACC m-blocks, each with its own TMEM accumulator;
//   * warp 0: TMA producer (128B-swizzled tiles of A_hi, A_lo, Bt_hi, Bt_lo into an
//     XHX_STAGES-deep ring, mbarrier expect-tx);
//   * warp 1: one elected thread issues tcgen05.mma (M = 128, N = 2b, K = 16) and
//     tcgen05.commit to free ring slots and to publish finished accumulators;
//   * warps 4-7: epilogue, tcgen05.ld of the accumulator rows and FP32 atomic adds
//     into Y (column-major N x 2b, zeroed by the caller);
//   * every mbarrier wait is bounded; on timeout the CTA records an error word,
//     drains its tensor-core work (bounded) and frees its tensor memory.
#include <cuda.h>
#include <cudaTypedefs.h>

#include "engine.h"

#define XHX_BM 128
#define XHX_BK 64             // bf16 elements per K tile = 128 bytes
#define XHX_STAGES 4
#define XHX_NACC 4
#define XHX_THREADS 256
#define XHX_SPIN_LIMIT (1u << 26)

struct HxTcParams {
  int mblocks;        // ceil(N / 128)
  int ktiles;         // ceil(2N / 64)
  long long tiles;    // mblocks * ktiles
  int ng;             // 2b, multiple of 16, <= 64
  int nrows;          // N
  int* status;        // device error word
  const int* active;  // NULL, or a device word: 0 = skip this product (a converged system of a batch)
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

// Bounded wait for the phase with the given parity; false on timeout.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, volatile int* abort_flag) {
  const uint32_t addr = smem_u32(bar);
  for (uint32_t it = 0; it < XHX_SPIN_LIMIT; it++) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(addr), "r"(parity)
        : "memory");
    if (done) return true;
    if (abort_flag && *abort_flag) return false;
  }
  return false;
}

__device__ __forceinline__ void tma_load_2d(const CUtensorMap* map, uint64_t* bar, void* dst, int x, int y) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];" ::"r"(
          smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(x), "r"(y)
      : "memory");
}

// Shared-memory matrix descriptor: K-major, 128-byte swizzle, 8-row groups 1024 B apart.
__device__ __forceinline__ uint64_t umma_desc_sw128(const void* base) {
  const uint64_t addr = smem_u32(base);
  uint64_t d = 0;
  d |= (addr >> 4) & 0x3FFFull;           // start address
  d |= (uint64_t)1 << 16;                 // leading byte offset (unused for swizzled K-major)
  d |= (uint64_t)(1024 >> 4) << 32;       // stride byte offset
  d |= (uint64_t)1 << 46;                 // descriptor version (sm_100)
  d |= (uint64_t)2 << 61;                 // SWIZZLE_128B
  return d;
}

// Instruction descriptor, kind::f16: BF16 x BF16 -> FP32, both K-major, M = 128, N = ng.
__host__ __device__ constexpr uint32_t umma_idesc_bf16(int ng) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(ng >> 3) << 17) | ((uint32_t)(XHX_BM >> 4) << 24);
}

__device__ __forceinline__ void umma_bf16(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                          uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
}

__device__ __forceinline__ void umma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

struct HxTcSmem {
  uint64_t full[XHX_STAGES];
  uint64_t empty[XHX_STAGES];
  uint64_t acc_full[XHX_NACC];
  uint64_t drain;
  uint32_t tmem_base;
  int abort_flag;
  int nseg;
  long long issued;     // tiles whose loads the producer issued
  long long consumed;   // tiles whose MMAs were issued
};

extern "C" __global__ void __launch_bounds__(XHX_THREADS, 1)
hx_tcgen05_kernel(const __grid_constant__ CUtensorMap tm_ahi, const __grid_constant__ CUtensorMap tm_alo,
                  const __grid_constant__ CUtensorMap tm_bhi, const __grid_constant__ CUtensorMap tm_blo,
                  HxTcParams p, float* __restrict__ Y) {
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  // 1024-byte aligned ring of stages: A_hi | A_lo | B_hi | B_lo
  unsigned char* ring = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  const uint32_t a_bytes = XHX_BM * XHX_BK * 2;     // 16 KB
  const uint32_t b_bytes = p.ng * XHX_BK * 2;       // ng * 128 B
  const uint32_t stage_bytes = 2 * a_bytes + 2 * ((b_bytes + 1023) & ~1023u);
  HxTcSmem* sh = reinterpret_cast<HxTcSmem*>(ring + XHX_STAGES * stage_bytes);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  // the same word for every thread of the grid, read before any barrier or TMEM allocation
  if (p.active && *p.active == 0) return;

  // this CTA's tile range
  const long long t0 = (p.tiles * blockIdx.x) / gridDim.x;
  const long long t1 = (p.tiles * (blockIdx.x + 1)) / gridDim.x;
  const int m_first = (int)(t0 / p.ktiles);
  const int m_last = (t1 > t0) ? (int)((t1 - 1) / p.ktiles) : m_first - 1;
  const int nseg = m_last - m_first + 1;

  if (threadIdx.x == 0) {
    for (int s = 0; s < XHX_STAGES; s++) {
      mbar_init(&sh->full[s], 1);
      mbar_init(&sh->empty[s], 1);
    }
    for (int a = 0; a < XHX_NACC; a++) mbar_init(&sh->acc_full[a], 1);
    mbar_init(&sh->drain, 1);
    sh->abort_flag = 0;
    sh->nseg = nseg;
    sh->issued = 0;
    sh->consumed = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncwarp();
  if (warp == 0) {
    // tensor memory: XHX_NACC accumulators of ng FP32 columns
    const uint32_t ncols = 256;
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&sh->tmem_base)),
                 "r"(ncols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  const uint32_t tmem = sh->tmem_base;
  volatile int* abort_flag = &sh->abort_flag;

  if (nseg > XHX_NACC) {
    if (threadIdx.x == 0) atomicOr(p.status, XATU_DEVERR_INDEX);
  } else if (warp == 0) {
    if (lane == 0) {
      // ---------------- TMA producer
      for (long long t = t0; t < t1; t++) {
        const long long li = t - t0;
        const int s = (int)(li % XHX_STAGES);
        const uint32_t ph = (uint32_t)((li / XHX_STAGES) & 1);
        if (!mbar_wait(&sh->empty[s], ph ^ 1, abort_flag)) {
          atomicOr(p.status, XATU_DEVERR_NOCONV);
          *abort_flag = 1;
          break;
        }
        const int m = (int)(t / p.ktiles);
        const int kt = (int)(t - (long long)m * p.ktiles);
        unsigned char* st = ring + s * stage_bytes;
        const uint32_t bpad = (b_bytes + 1023) & ~1023u;
        mbar_expect_tx(&sh->full[s], 2 * a_bytes + 2 * b_bytes);
        tma_load_2d(&tm_ahi, &sh->full[s], st, kt * XHX_BK, m * XHX_BM);
        tma_load_2d(&tm_alo, &sh->full[s], st + a_bytes, kt * XHX_BK, m * XHX_BM);
        tma_load_2d(&tm_bhi, &sh->full[s], st + 2 * a_bytes, kt * XHX_BK, 0);
        tma_load_2d(&tm_blo, &sh->full[s], st + 2 * a_bytes + bpad, kt * XHX_BK, 0);
        sh->issued = li + 1;
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {
      // ---------------- MMA issuer
      const uint32_t idesc = umma_idesc_bf16(p.ng);
      const uint32_t bpad = (b_bytes + 1023) & ~1023u;
      int seg = 0;
      bool fresh = true;
      for (long long t = t0; t < t1; t++) {
        const long long li = t - t0;
        const int s = (int)(li % XHX_STAGES);
        const uint32_t ph = (uint32_t)((li / XHX_STAGES) & 1);
        if (!mbar_wait(&sh->full[s], ph, abort_flag)) {
          atomicOr(p.status, XATU_DEVERR_NOCONV);
          *abort_flag = 1;
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;");
        const int m = (int)(t / p.ktiles);
        seg = m - m_first;
        const uint32_t d_tmem = tmem + (uint32_t)(seg * p.ng);
        unsigned char* st = ring + s * stage_bytes;
        const uint64_t ahi = umma_desc_sw128(st), alo = umma_desc_sw128(st + a_bytes);
        const uint64_t bhi = umma_desc_sw128(st + 2 * a_bytes), blo = umma_desc_sw128(st + 2 * a_bytes + bpad);
#pragma unroll
        for (int k = 0; k < XHX_BK / 16; k++) {
          const uint64_t adv = (uint64_t)((k * 32) >> 4);   // 16 bf16 = 32 bytes along K
          umma_bf16(d_tmem, ahi + adv, bhi + adv, idesc, (fresh && k == 0) ? 0u : 1u);
          umma_bf16(d_tmem, ahi + adv, blo + adv, idesc, 1u);
          umma_bf16(d_tmem, alo + adv, bhi + adv, idesc, 1u);
        }
        fresh = false;
        sh->consumed = li + 1;
        umma_commit(&sh->empty[s]);           // ring slot free once these MMAs complete
        const bool last_of_block = ((t + 1) % p.ktiles == 0) || (t + 1 == t1);
        if (last_of_block) {
          umma_commit(&sh->acc_full[seg]);
          fresh = true;
        }
      }
      // drain: every MMA issued so far has completed once this commit arrives
      umma_commit(&sh->drain);
      mbar_wait(&sh->drain, 0, nullptr);
    }
  } else if (warp >= 4) {
    // ---------------- epilogue: TMEM -> registers -> atomics into Y (column-major N x ng)
    const int ew = warp - 4;                    // TMEM lanes [32*ew, 32*ew + 32)
    for (int seg = 0; seg < nseg; seg++) {
      const bool ok = __all_sync(0xffffffffu, mbar_wait(&sh->acc_full[seg], 0, abort_flag));
      if (!ok) {
        if (lane == 0) atomicOr(p.status, XATU_DEVERR_NOCONV);
        *abort_flag = 1;
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;");
      const int row = (m_first + seg) * XHX_BM + ew * 32 + lane;
      for (int c0 = 0; c0 < p.ng; c0 += 16) {
        uint32_t r[16];
        const uint32_t taddr = tmem + ((uint32_t)(ew * 32) << 16) + (uint32_t)(seg * p.ng + c0);
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
            : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
              "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
            : "r"(taddr));
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        if (row < p.nrows) {
#pragma unroll
          for (int j = 0; j < 16; j++) atomicAdd(&Y[(long long)(c0 + j) * p.nrows + row], __uint_as_float(r[j]));
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  if (threadIdx.x == 0 && sh->abort_flag) {
    // loads issued but never consumed must land before the CTA's shared memory goes away
    for (long long li = sh->consumed; li < sh->issued; li++)
      mbar_wait(&sh->full[li % XHX_STAGES], (uint32_t)((li / XHX_STAGES) & 1), nullptr);
  }
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(256u));
  }
}

// ------------------------------------------------------------------ host side
static PFN_cuTensorMapEncodeTiled_v12000 get_encode() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  if (!fn) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
  }
  return fn;
}

// 2-D bf16 tensor map: inner extent `inner` elements, `outer` rows, row pitch `pitch_bytes`.
static bool make_map(CUtensorMap* map, const void* base, uint64_t inner, uint64_t outer, uint64_t pitch_bytes,
                     uint32_t box_inner, uint32_t box_outer) {
  auto enc = get_encode();
  if (!enc) return false;
  if ((reinterpret_cast<uintptr_t>(base) & 15) || (pitch_bytes & 15)) return false;
  cuuint64_t dims[2] = {inner, outer};
  cuuint64_t strides[1] = {pitch_bytes};
  cuuint32_t box[2] = {box_inner, box_outer};
  cuuint32_t estr[2] = {1, 1};
  CUresult r = enc(map, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(base), dims, strides, box, estr,
                   CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                   CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

size_t xatu_hx_tc_smem(int ng) {
  const size_t a_bytes = XHX_BM * XHX_BK * 2;
  const size_t b_bytes = ((size_t)ng * XHX_BK * 2 + 1023) & ~(size_t)1023;
  return 1024 + XHX_STAGES * (2 * a_bytes + 2 * b_bytes) + sizeof(HxTcSmem);
}

// Khi/Klo: N x ldk complex bf16 (ldk % 4 == 0).  Bhi/Blo: ng x ldb bf16 (ldb % 8 == 0).
// Y: column-major N x ng FP32, zeroed here.
cudaError_t xatu_launch_hx_tc(const void* Khi, const void* Klo, long long N, long long ldk, const void* Bhi,
                              const void* Blo, long long ldb, int ng, float* Y, int* status, int num_sms,
                              cudaStream_t s, const int* active) {
  if (ng % 16 != 0 || ng < 16 || ng > 64 || (ldk % 4) != 0 || (ldb % 8) != 0) return cudaErrorInvalidValue;
  CUtensorMap ahi, alo, bhi, blo;
  const uint64_t kdim = 2ull * N;
  if (!make_map(&ahi, Khi, kdim, N, ldk * 4, XHX_BK, XHX_BM) || !make_map(&alo, Klo, kdim, N, ldk * 4, XHX_BK, XHX_BM) ||
      !make_map(&bhi, Bhi, kdim, ng, ldb * 2, XHX_BK, ng) || !make_map(&blo, Blo, kdim, ng, ldb * 2, XHX_BK, ng))
    return cudaErrorInvalidValue;
  HxTcParams p;
  p.mblocks = (int)((N + XHX_BM - 1) / XHX_BM);
  p.ktiles = (int)((kdim + XHX_BK - 1) / XHX_BK);
  p.tiles = (long long)p.mblocks * p.ktiles;
  p.ng = ng;
  p.nrows = (int)N;
  p.status = status;
  p.active = active;
  int grid = (int)std::min<long long>(num_sms, p.tiles);
  // a CTA's range must not span more than XHX_NACC m-blocks
  while (grid < p.tiles && (p.tiles + grid - 1) / grid > (long long)(XHX_NACC - 1) * p.ktiles) grid++;
  cudaError_t e = cudaMemsetAsync(Y, 0, sizeof(float) * (size_t)N * ng, s);
  if (e != cudaSuccess) return e;
  const size_t smem = xatu_hx_tc_smem(ng);
  e = xatu_raise_smem_limit((const void*)hx_tcgen05_kernel, smem);
  if (e != cudaSuccess) return e;
  hx_tcgen05_kernel<<<grid, XHX_THREADS, smem, s>>>(ahi, alo, bhi, blo, p, Y);
  return cudaGetLastError();
}
