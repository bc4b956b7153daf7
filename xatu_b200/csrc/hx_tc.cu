// Y = K X on the 5th-generation tensor cores (tcgen05, sm_100a), reading the Hermitian K once.
//
// K is the mixed-precision BSE interaction kernel, a Hermitian matrix stored as two BF16 planes
// (K = K_hi + K_lo, complex interleaved, row pitch ldk complex elements).  Only its upper block triangle is
// stored: with blocks of XATU_KBLOCK x XATU_KBLOCK, block (I, J) is valid for J >= I, the diagonal blocks in
// full.  Read as a real matrix, row i of K is A[i][2j + p] = (Re, Im) K_ij.
//
// Tiles: 128 rows (row block I) x 64 complex columns (column tile t, inside block J = t / 2 >= I), 32 KB
// per plane, loaded once.  Each tile feeds two products:
//   direct      Y_I += K_It X_t    -- the tile K-major (K along the interleaved column), operand Bt of X_t;
//   transposed  Y_t += K_It^H X_I  -- the same shared-memory tile read MN-major (M along the interleaved
//               column, K along the rows), operand Bu of X_I; skipped in the diagonal blocks (stored in full).
// Operands (split BF16, hi + lo; rows s < bp hold the real block, rows bp + s the imaginary one; ng = 2 bp):
//   Bt[s][2j] = Re x_js, Bt[s][2j+1] = -Im x_js, Bt[bp+s][2j] = Im x_js, Bt[bp+s][2j+1] = Re x_js
//     -> D[i][s] = Re (K x)_is,  D[i][bp+s] = Im (K x)_is;
//   Bu[s][i] = Re x_is, Bu[bp+s][i] = Im x_is
//     -> D'[2j+p][s'] = sum_i A[i][2j+p] Bu[s'][i], and
//        Re (K^H x)_js = D'[2j][s] + D'[2j+1][bp+s],   Im (K^H x)_js = D'[2j][bp+s] - D'[2j+1][s]
//        (tensor-memory lanes 2j and 2j+1 belong to one warp: one shuffle combines them).
// Split-BF16 products A_hi B_hi + A_hi B_lo + A_lo B_hi, FP32 accumulation in tensor memory (the lo*lo term
// is below FP32 rounding of the result).
//
// Kernel structure (one CTA per SM, persistent): the tiles of the upper block triangle, enumerated row block
// by row block, are cut into equal contiguous ranges, one per CTA.
//   * warp 0: TMA producer, an XHH_STAGES-deep ring of stages (A_hi, A_lo, Bt_hi, Bt_lo, Bu_hi, Bu_lo);
//   * warps 1 and 2: one thread each issues tcgen05.mma (M = 128, N = ng, K = 16), warp 1 the direct products,
//     warp 2 the transposed ones; a ring stage is free once both have committed it.  The direct accumulator of a
//     row block (a segment of the range) takes a slot of a ring of two in tensor memory, the transposed accumulator of a
//     tile one of a ring of XHH_TSLOTS; tcgen05.commit frees ring stages and publishes finished accumulators;
//   * warps 4-7: epilogue, tcgen05.ld of the accumulator lanes, FP32 vector atomics into Y (row-major N x ng),
//     then an arrive that frees the accumulator slot;
//   * every wait is bounded; on timeout the CTA records an error word, drains its tensor-core work (bounded)
//     and frees its tensor memory.
// The host caches the six tensor maps of recent launches (a Davidson solve repeats the same product).
#include <cuda.h>
#include <cudaTypedefs.h>

#include <mutex>

#include "engine.h"

#define XHH_BM 128            // rows of a tile (one row block)
#define XHH_BOX 64            // bf16 per TMA box row: 128 bytes, the swizzle width
#define XHH_STAGES 2
#define XHH_TSLOTS 4          // transposed accumulators in tensor memory (the epilogue drains while the MMA runs on)
#define XHH_THREADS 256
#define XHH_TMEM_COLS 512     // 2 direct + XHH_TSLOTS transposed slots of ng <= 48 columns
#define XHH_SPIN_LIMIT (1u << 26)

static_assert(XATU_KBLOCK == 2 * 64 && XHH_BM == XATU_KBLOCK, "tile geometry assumes 128-blocks of 64-column tiles");

struct HxTcParams {
  int nb;             // row blocks: ceil(N / 128)
  int nt;             // column tiles: ceil(N / 64)
  long long tiles;    // tiles of the upper block triangle
  int nrows;          // N
  int* status;        // device error word
  const int* active;  // NULL, or a device word: 0 = skip this product (a converged system of a batch)
};

// first tile of row block I in the enumeration: row block I holds the column tiles [2 I, nt)
__host__ __device__ __forceinline__ long long hxh_row_start(long long I, int nt) { return I * nt - I * (I - 1); }

__device__ __forceinline__ void hxh_tile_pos(long long g, int nb, int nt, int& I, int& t) {
  const double b = nt + 1.0;
  int r = (int)floor(0.5 * (b - sqrt(fmax(b * b - 4.0 * (double)g, 0.0))));
  r = max(0, min(r, nb - 1));
  while (r > 0 && hxh_row_start(r, nt) > g) r--;
  while (r + 1 < nb && hxh_row_start(r + 1, nt) <= g) r++;
  I = r;
  t = 2 * r + (int)(g - hxh_row_start(r, nt));
}

__device__ __forceinline__ void hxh_advance(int& I, int& t, int nt) {
  if (++t == nt) {
    I++;
    t = 2 * I;
  }
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

// Bounded wait for the phase with the given parity; false on timeout or when another role aborted.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity, volatile int* abort_flag) {
  const uint32_t addr = smem_u32(bar);
  for (uint32_t it = 0; it < XHH_SPIN_LIMIT; it++) {
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

// Shared-memory matrix descriptor, 128-byte swizzle (sm_100 form).  K-major: 8-row groups 1024 B apart (SBO),
// the leading offset unused.  MN-major: 64-element chunks along M/N `lbo` bytes apart, 8-row groups along K
// 1024 B apart.
__device__ __forceinline__ uint64_t umma_desc_sw128(const void* base, uint32_t lbo_bytes) {
  const uint64_t addr = smem_u32(base);
  uint64_t d = 0;
  d |= (addr >> 4) & 0x3FFFull;                        // start address
  d |= (uint64_t)((lbo_bytes >> 4) & 0x3FFF) << 16;    // leading byte offset
  d |= (uint64_t)(1024 >> 4) << 32;                    // stride byte offset
  d |= (uint64_t)1 << 46;                              // descriptor version (sm_100)
  d |= (uint64_t)2 << 61;                              // SWIZZLE_128B
  return d;
}

// Instruction descriptor, kind::f16: BF16 x BF16 -> FP32, B K-major, A K-major (a_mn = 0) or MN-major (1),
// M = 128, N = ng.
__host__ __device__ constexpr uint32_t umma_idesc_bf16(int ng, int a_mn) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)a_mn << 15) | ((uint32_t)(ng >> 3) << 17) |
         ((uint32_t)(XHH_BM >> 4) << 24);
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

// 16 consecutive accumulator columns of this warp's 32 lanes
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float* v) {
  uint32_t r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr));
#pragma unroll
  for (int j = 0; j < 16; j++) v[j] = __uint_as_float(r[j]);
}

struct HxTcSmem {
  uint64_t full[XHH_STAGES];
  uint64_t empty[XHH_STAGES];
  uint64_t dfull[2], dempty[2];   // direct accumulator slots
  uint64_t tfull[XHH_TSLOTS], tempty[XHH_TSLOTS];   // transposed accumulator slots
  uint64_t drain;
  uint32_t tmem_base;
  int abort_flag;
  long long issued;     // tiles whose loads the producer issued
  long long consumed;   // tiles whose MMAs were issued
};

template <int NG>
__global__ void __launch_bounds__(XHH_THREADS, 1)
hx_herm_tcgen05_kernel(const __grid_constant__ CUtensorMap tm_ahi, const __grid_constant__ CUtensorMap tm_alo,
                       const __grid_constant__ CUtensorMap tm_bhi, const __grid_constant__ CUtensorMap tm_blo,
                       const __grid_constant__ CUtensorMap tm_uhi, const __grid_constant__ CUtensorMap tm_ulo,
                       HxTcParams p, float* __restrict__ Y) {
  constexpr int BP = NG / 2;
  constexpr uint32_t A_BOX = XHH_BM * XHH_BOX * 2;   // 16 KB: 128 rows x 128 B
  constexpr uint32_t A_PLANE = 2 * A_BOX;            // a tile holds 128 bf16 per row: two boxes
  constexpr uint32_t B_BOX = NG * XHH_BOX * 2;       // ng rows x 128 B
  constexpr uint32_t B_PLANE = 2 * B_BOX;
  constexpr uint32_t OFF_BT = 2 * A_PLANE;           // Bt_hi, Bt_lo, Bu_hi, Bu_lo follow the A planes
  constexpr uint32_t OFF_BU = OFF_BT + 2 * B_PLANE;
  constexpr uint32_t STAGE = OFF_BU + 2 * B_PLANE;
  extern __shared__ __align__(1024) unsigned char smem_raw[];
  unsigned char* ring = reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  HxTcSmem* sh = reinterpret_cast<HxTcSmem*>(ring + XHH_STAGES * STAGE);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  // the same word for every thread of the grid, read before any barrier or tensor-memory allocation
  if (p.active && *p.active == 0) return;

  const long long t0 = (p.tiles * blockIdx.x) / gridDim.x;
  const long long t1 = (p.tiles * (blockIdx.x + 1)) / gridDim.x;

  if (threadIdx.x == 0) {
    for (int s = 0; s < XHH_STAGES; s++) {
      mbar_init(&sh->full[s], 1);
      mbar_init(&sh->empty[s], 2);   // one commit from each MMA issuer
    }
    for (int a = 0; a < 2; a++) {
      mbar_init(&sh->dfull[a], 1);
      mbar_init(&sh->dempty[a], 4);
    }
    for (int a = 0; a < XHH_TSLOTS; a++) {
      mbar_init(&sh->tfull[a], 1);
      mbar_init(&sh->tempty[a], 4);
    }
    mbar_init(&sh->drain, 2);
    sh->abort_flag = 0;
    sh->issued = 0;
    sh->consumed = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncwarp();
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&sh->tmem_base)),
                 "r"((uint32_t)XHH_TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  const uint32_t tmem = sh->tmem_base;
  volatile int* abort_flag = &sh->abort_flag;

  if (warp == 0) {
    if (lane == 0 && t1 > t0) {
      // ---------------- TMA producer
      int I, t;
      hxh_tile_pos(t0, p.nb, p.nt, I, t);
      for (long long g = t0; g < t1; g++, hxh_advance(I, t, p.nt)) {
        const long long li = g - t0;
        const int s = (int)(li % XHH_STAGES);
        const uint32_t ph = (uint32_t)((li / XHH_STAGES) & 1);
        if (!mbar_wait(&sh->empty[s], ph ^ 1, abort_flag)) {
          atomicOr(p.status, XATU_DEVERR_NOCONV);
          *abort_flag = 1;
          break;
        }
        const bool diag = (t >> 1) == I;
        unsigned char* st = ring + s * STAGE;
        mbar_expect_tx(&sh->full[s], 2 * A_PLANE + 2 * B_PLANE + (diag ? 0u : 2 * B_PLANE));
        const int xa = t * 2 * XHH_BOX, ya = I * XHH_BM;
        tma_load_2d(&tm_ahi, &sh->full[s], st, xa, ya);
        tma_load_2d(&tm_ahi, &sh->full[s], st + A_BOX, xa + XHH_BOX, ya);
        tma_load_2d(&tm_alo, &sh->full[s], st + A_PLANE, xa, ya);
        tma_load_2d(&tm_alo, &sh->full[s], st + A_PLANE + A_BOX, xa + XHH_BOX, ya);
        tma_load_2d(&tm_bhi, &sh->full[s], st + OFF_BT, xa, 0);
        tma_load_2d(&tm_bhi, &sh->full[s], st + OFF_BT + B_BOX, xa + XHH_BOX, 0);
        tma_load_2d(&tm_blo, &sh->full[s], st + OFF_BT + B_PLANE, xa, 0);
        tma_load_2d(&tm_blo, &sh->full[s], st + OFF_BT + B_PLANE + B_BOX, xa + XHH_BOX, 0);
        if (!diag) {
          const int xu = I * XHH_BM;
          tma_load_2d(&tm_uhi, &sh->full[s], st + OFF_BU, xu, 0);
          tma_load_2d(&tm_uhi, &sh->full[s], st + OFF_BU + B_BOX, xu + XHH_BOX, 0);
          tma_load_2d(&tm_ulo, &sh->full[s], st + OFF_BU + B_PLANE, xu, 0);
          tma_load_2d(&tm_ulo, &sh->full[s], st + OFF_BU + B_PLANE + B_BOX, xu + XHH_BOX, 0);
        }
        sh->issued = li + 1;
      }
    }
  } else if (warp == 1 || warp == 2) {
    if (lane == 0 && t1 > t0) {
      // ---------------- MMA issuers: warp 1 the direct products, warp 2 the transposed ones (two threads on different
      // SM sub-partitions issue side by side; a ring stage is free once both have committed it)
      const bool direct = warp == 1;
      constexpr uint32_t idesc_d = umma_idesc_bf16(NG, 0);
      constexpr uint32_t idesc_t = umma_idesc_bf16(NG, 1);
      int I, t;
      hxh_tile_pos(t0, p.nb, p.nt, I, t);
      int seg = -1, curI = -1, tcount = 0;
      bool dfresh = true;
      uint32_t dslot = 0;
      for (long long g = t0; g < t1; g++, hxh_advance(I, t, p.nt)) {
        const long long li = g - t0;
        const int s = (int)(li % XHH_STAGES);
        const uint32_t ph = (uint32_t)((li / XHH_STAGES) & 1);
        if (!mbar_wait(&sh->full[s], ph, abort_flag)) {
          atomicOr(p.status, XATU_DEVERR_NOCONV);
          *abort_flag = 1;
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;");
        const bool diag = (t >> 1) == I;
        const unsigned char* st = ring + s * STAGE;
        if (direct) {
          if (I != curI) {   // a new row block: the next direct slot, once the epilogue has emptied it
            seg++;
            curI = I;
            dslot = (uint32_t)(seg & 1);
            if (seg >= 2 && !mbar_wait(&sh->dempty[dslot], (uint32_t)(((seg >> 1) - 1) & 1), abort_flag)) {
              atomicOr(p.status, XATU_DEVERR_NOCONV);
              *abort_flag = 1;
              break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;");
            dfresh = true;
          }
          const uint32_t dtm = tmem + dslot * NG;
#pragma unroll
          for (int kk = 0; kk < 2 * XHH_BOX / 16; kk++) {
            const uint32_t ao = (kk >> 2) * A_BOX + (kk & 3) * 32, bo = (kk >> 2) * B_BOX + (kk & 3) * 32;
            const uint64_t ahi = umma_desc_sw128(st + ao, 0), alo = umma_desc_sw128(st + A_PLANE + ao, 0);
            const uint64_t bhi = umma_desc_sw128(st + OFF_BT + bo, 0);
            const uint64_t blo = umma_desc_sw128(st + OFF_BT + B_PLANE + bo, 0);
            umma_bf16(dtm, ahi, bhi, idesc_d, (dfresh && kk == 0) ? 0u : 1u);
            umma_bf16(dtm, ahi, blo, idesc_d, 1u);
            umma_bf16(dtm, alo, bhi, idesc_d, 1u);
          }
          dfresh = false;
          sh->consumed = li + 1;
          umma_commit(&sh->empty[s]);           // ring stage free once both issuers' MMAs complete
          if (t + 1 == p.nt || g + 1 == t1) umma_commit(&sh->dfull[dslot]);
        } else {
          if (!diag) {
            const uint32_t tslot = (uint32_t)(tcount % XHH_TSLOTS);
            const int tuse = tcount / XHH_TSLOTS;
            if (tuse >= 1 && !mbar_wait(&sh->tempty[tslot], (uint32_t)((tuse - 1) & 1), abort_flag)) {
              atomicOr(p.status, XATU_DEVERR_NOCONV);
              *abort_flag = 1;
              break;
            }
            asm volatile("tcgen05.fence::after_thread_sync;");
            const uint32_t ttm = tmem + (2 + tslot) * NG;
#pragma unroll
            for (int kk = 0; kk < XHH_BM / 16; kk++) {
              // K step: 16 rows of the tile = two 8-row groups (2048 B); M: the two 64-column boxes, A_BOX apart
              const uint32_t ao = kk * 2048, bo = (kk >> 2) * B_BOX + (kk & 3) * 32;
              const uint64_t ahi = umma_desc_sw128(st + ao, A_BOX), alo = umma_desc_sw128(st + A_PLANE + ao, A_BOX);
              const uint64_t uhi = umma_desc_sw128(st + OFF_BU + bo, 0);
              const uint64_t ulo = umma_desc_sw128(st + OFF_BU + B_PLANE + bo, 0);
              umma_bf16(ttm, ahi, uhi, idesc_t, kk == 0 ? 0u : 1u);
              umma_bf16(ttm, ahi, ulo, idesc_t, 1u);
              umma_bf16(ttm, alo, uhi, idesc_t, 1u);
            }
            umma_commit(&sh->tfull[tslot]);
            tcount++;
          }
          umma_commit(&sh->empty[s]);
        }
      }
      // drain: every MMA either issuer issued has completed once both commits arrive
      umma_commit(&sh->drain);
      mbar_wait(&sh->drain, 0, nullptr);
    }
  } else if (warp >= 4 && t1 > t0) {
    // ---------------- epilogue: tensor memory -> registers -> vector atomics into Y (row-major N x ng)
    const int ew = warp - 4;                    // tensor-memory lanes [32 ew, 32 ew + 32)
    const uint32_t lane_base = (uint32_t)(ew * 32) << 16;
    int I, t;
    hxh_tile_pos(t0, p.nb, p.nt, I, t);
    int seg = -1, curI = -1, tcount = 0;
    for (long long g = t0; g < t1; g++, hxh_advance(I, t, p.nt)) {
      if (I != curI) {
        seg++;
        curI = I;
      }
      if ((t >> 1) != I) {
        const uint32_t tslot = (uint32_t)(tcount % XHH_TSLOTS);
        const bool ok = __all_sync(0xffffffffu, mbar_wait(&sh->tfull[tslot], (uint32_t)((tcount / XHH_TSLOTS) & 1),
                                                          abort_flag));
        if (!ok) {
          if (lane == 0) atomicOr(p.status, XATU_DEVERR_NOCONV);
          *abort_flag = 1;
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;");
        float v[NG];
#pragma unroll
        for (int c0 = 0; c0 < NG; c0 += 16) tmem_ld16(tmem + lane_base + (2 + tslot) * NG + c0, v + c0);
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        // lanes 2j (p = 0) and 2j + 1 (p = 1): Re and Im of row j of K^H x
        const int par = lane & 1;
        float out[BP];
#pragma unroll
        for (int s = 0; s < BP; s++) {
          const float other = __shfl_xor_sync(0xffffffffu, v[BP + s], 1);
          out[s] = par ? other - v[s] : v[s] + other;
        }
        const long long row = (long long)t * 64 + ((ew * 32 + lane) >> 1);
        if (row < p.nrows) {
          float4* y = reinterpret_cast<float4*>(Y + row * NG + par * BP);
#pragma unroll
          for (int q = 0; q < BP / 4; q++)
            atomicAdd(y + q, make_float4(out[4 * q], out[4 * q + 1], out[4 * q + 2], out[4 * q + 3]));
        }
        asm volatile("tcgen05.fence::before_thread_sync;");
        __syncwarp();
        if (lane == 0) mbar_arrive(&sh->tempty[tslot]);
        tcount++;
      }
      if (t + 1 == p.nt || g + 1 == t1) {
        const uint32_t dslot = (uint32_t)(seg & 1);
        const bool ok = __all_sync(0xffffffffu, mbar_wait(&sh->dfull[dslot], (uint32_t)((seg >> 1) & 1), abort_flag));
        if (!ok) {
          if (lane == 0) atomicOr(p.status, XATU_DEVERR_NOCONV);
          *abort_flag = 1;
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;");
        float v[NG];
#pragma unroll
        for (int c0 = 0; c0 < NG; c0 += 16) tmem_ld16(tmem + lane_base + dslot * NG + c0, v + c0);
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        const long long row = (long long)I * XHH_BM + ew * 32 + lane;
        if (row < p.nrows) {
          float4* y = reinterpret_cast<float4*>(Y + row * NG);
#pragma unroll
          for (int q = 0; q < NG / 4; q++)
            atomicAdd(y + q, make_float4(v[4 * q], v[4 * q + 1], v[4 * q + 2], v[4 * q + 3]));
        }
        asm volatile("tcgen05.fence::before_thread_sync;");
        __syncwarp();
        if (lane == 0) mbar_arrive(&sh->dempty[dslot]);
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  if (threadIdx.x == 0 && sh->abort_flag) {
    // loads issued but never consumed must land before the CTA's shared memory goes away
    for (long long li = sh->consumed; li < sh->issued; li++)
      mbar_wait(&sh->full[li % XHH_STAGES], (uint32_t)((li / XHH_STAGES) & 1), nullptr);
  }
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"((uint32_t)XHH_TMEM_COLS));
  }
}

// Operand planes of a K.X product from the columns x_s = X[s * ldx ...] (complex FP64, s < b), split BF16:
// Bt (ng x ldb) and Bu (ng x ldu) as laid out in the kernel's header comment; rows of padding vectors
// (b <= s < bp) are zero.
__global__ void hx_operand_kernel(const cd* __restrict__ X, long long ldx, long long N, int b, int bp, long long ldb,
                                  long long ldu, __nv_bfloat16* __restrict__ Bhi, __nv_bfloat16* __restrict__ Blo,
                                  __nv_bfloat16* __restrict__ Uhi, __nv_bfloat16* __restrict__ Ulo) {
  xatu_grid_chain();
  const long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (t >= N * bp) return;
  const int s = (int)(t / N);
  const long long j = t - (long long)s * N;
  float re = 0.f, im = 0.f;
  if (s < b) {
    const cd v = X[(long long)s * ldx + j];
    re = (float)v.x;
    im = (float)v.y;
  }
  const float vals[6] = {re, -im, im, re, re, im};
  const long long off[6] = {(long long)s * ldb + 2 * j, (long long)s * ldb + 2 * j + 1,
                            (long long)(bp + s) * ldb + 2 * j, (long long)(bp + s) * ldb + 2 * j + 1,
                            (long long)s * ldu + j, (long long)(bp + s) * ldu + j};
#pragma unroll
  for (int q = 0; q < 6; q++) {
    const __nv_bfloat16 h = __float2bfloat16_rn(vals[q]);
    const __nv_bfloat16 l = __float2bfloat16_rn(vals[q] - __bfloat162float(h));
    if (q < 4) {
      Bhi[off[q]] = h;
      Blo[off[q]] = l;
    } else {
      Uhi[off[q]] = h;
      Ulo[off[q]] = l;
    }
  }
}

cudaError_t xatu_launch_hx_operands(const cd* X, long long ldx, long long N, int b, int bp, void* Bhi, void* Blo,
                                    long long ldb, void* Uhi, void* Ulo, long long ldu, cudaStream_t s) {
  if (b > bp || ldb < 2 * N || ldu < N) return cudaErrorInvalidValue;
  const long long tot = N * bp;
  return xatu_launch_chained(hx_operand_kernel, dim3((unsigned)((tot + 255) / 256)), dim3(256), 0, s, X, ldx, N, b, bp,
                             ldb, ldu, static_cast<__nv_bfloat16*>(Bhi), static_cast<__nv_bfloat16*>(Blo),
                             static_cast<__nv_bfloat16*>(Uhi), static_cast<__nv_bfloat16*>(Ulo));
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
  const size_t stage = (size_t)4 * XHH_BM * XHH_BOX * 2 + (size_t)8 * ng * XHH_BOX * 2;
  return 1024 + XHH_STAGES * stage + sizeof(HxTcSmem);
}

template <int NG>
static cudaError_t launch_ng(const CUtensorMap* m, const HxTcParams& p, float* Y, int grid, cudaStream_t s) {
  const size_t smem = xatu_hx_tc_smem(NG);
  cudaError_t e = xatu_raise_smem_limit((const void*)hx_herm_tcgen05_kernel<NG>, smem);
  if (e != cudaSuccess) return e;
  hx_herm_tcgen05_kernel<NG><<<grid, XHH_THREADS, smem, s>>>(m[0], m[1], m[2], m[3], m[4], m[5], p, Y);
  return cudaGetLastError();
}

namespace {
// Tensor maps of recent launches: encoding six maps costs host time that a Davidson step would otherwise
// wait for between its kernels.  Keyed by every argument the maps depend on.
struct MapKey {
  const void* ptr[6];
  long long N, ldk, ldb, ldu;
  int ng, dev;
  bool operator==(const MapKey& o) const {
    for (int i = 0; i < 6; i++)
      if (ptr[i] != o.ptr[i]) return false;
    return N == o.N && ldk == o.ldk && ldb == o.ldb && ldu == o.ldu && ng == o.ng && dev == o.dev;
  }
};
struct MapEntry {
  MapKey key;
  CUtensorMap maps[6];
  bool used = false;
};
std::mutex g_map_mu;
MapEntry g_maps[16];
int g_map_next = 0;
}  // namespace

cudaError_t xatu_launch_hx_tc(const void* Khi, const void* Klo, long long N, long long ldk, const void* Bhi,
                              const void* Blo, long long ldb, const void* Uhi, const void* Ulo, long long ldu, int ng,
                              float* Y, int* status, int num_sms, cudaStream_t s, const int* active) {
  if ((ng != 16 && ng != 32 && ng != 48) || (ldk % 4) != 0 || (ldb % 8) != 0 || (ldu % 8) != 0 || N < 1)
    return cudaErrorInvalidValue;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  MapKey key{{Khi, Klo, Bhi, Blo, Uhi, Ulo}, N, ldk, ldb, ldu, ng, dev};
  CUtensorMap m[6];
  {
    std::lock_guard<std::mutex> lock(g_map_mu);
    int hit = -1;
    for (int i = 0; i < 16; i++)
      if (g_maps[i].used && g_maps[i].key == key) hit = i;
    if (hit < 0) {
      MapEntry& en = g_maps[g_map_next];
      const uint64_t kdim = 2ull * N;
      if (!make_map(&en.maps[0], Khi, kdim, N, ldk * 4, XHH_BOX, XHH_BM) ||
          !make_map(&en.maps[1], Klo, kdim, N, ldk * 4, XHH_BOX, XHH_BM) ||
          !make_map(&en.maps[2], Bhi, kdim, ng, ldb * 2, XHH_BOX, ng) ||
          !make_map(&en.maps[3], Blo, kdim, ng, ldb * 2, XHH_BOX, ng) ||
          !make_map(&en.maps[4], Uhi, N, ng, ldu * 2, XHH_BOX, ng) ||
          !make_map(&en.maps[5], Ulo, N, ng, ldu * 2, XHH_BOX, ng)) {
        en.used = false;
        return cudaErrorInvalidValue;
      }
      en.key = key;
      en.used = true;
      hit = g_map_next;
      g_map_next = (g_map_next + 1) % 16;
    }
    for (int i = 0; i < 6; i++) m[i] = g_maps[hit].maps[i];
  }
  HxTcParams p;
  p.nb = (int)((N + XHH_BM - 1) / XHH_BM);
  p.nt = (int)((N + 63) / 64);
  p.tiles = hxh_row_start(p.nb, p.nt);
  p.nrows = (int)N;
  p.status = status;
  p.active = active;
  const int grid = (int)std::min<long long>(num_sms, p.tiles);
  e = cudaMemsetAsync(Y, 0, sizeof(float) * (size_t)N * ng, s);
  if (e != cudaSuccess) return e;
  if (ng == 16) return launch_ng<16>(m, p, Y, grid, s);
  if (ng == 32) return launch_ng<32>(m, p, Y, grid, s);
  return launch_ng<48>(m, p, Y, grid, s);
}
