// Mixed-precision tile assembly with the band overlaps on the tensor cores (ExcitonTB::BShamiltonian,
// ExcitonTB.cpp:840-921; realSpaceInteractionTerm :520-548; reciprocal and exchange terms as in
// assembly_tile.cuh).
//
// For a TK x TK tile of (k, k') pairs the per-atom band overlaps are small complex GEMMs over the orbitals of
// one atom:
//   rho1_a[(k,c),(k',c')] = sum_{o in a} conj(CQ_k[c]_o) CQ_k'[c']_o
//   rho2_b[(k,v),(k',v')] = sum_{o in b} conj(C_k'[v']_o) C_k[v]_o
// They run as tcgen05.mma (kind::f16, M = 128, FP32 accumulation in tensor memory):
//   A (128 x KP, K-major): rows (atom, k', band') from the k' side, each row holding [Re, Im] of the orbital
//     coefficients of its atom only (zeros elsewhere), so one product gives every atom's sum; the product also
//     reads the rows after the NA * TK * nband valid ones (whatever follows in shared memory), and those
//     accumulator rows are never used;
//   B (2 TK nband x KP, K-major): rows (k, band) from the k side in two forms, [Re, Im] and the form whose
//     product is the imaginary part ([-Im, Re] for rho1, [Im, -Re] for rho2);
//   D[(a, k', band')][(k, band)] = Re, D[...][TK nband + (k, band)] = Im.
// KP = 2 norb rounded up to 16.  Operands are split FP16 (x = hi + lo, 22 significant bits: |C| <= 1 keeps
// them in range) and each overlap is hi*hi + hi*lo + lo*hi, so rho carries FP32-level accuracy.
// Shared-memory operands use the no-swizzle K-major layout of 8-row x 16-byte core matrices.  Both operand
// kinds of every k block are formatted once per build (asm_tc_format_kernel) into images in global memory
// laid out exactly as the tile needs them in shared memory, so a tile stages its operands with four bulk
// copies (cp.async.bulk, completion on an mbarrier) and no conversion work.
//
// The accumulators are moved to shared memory (k side first, so that the per-pair reads below are contiguous
// across the threads of a warp; the block has at least 128 threads, one warp per tensor-memory sub-partition),
// and one thread per (k, k') pair forms
//   T_a(v', v) = sum_b V_ab rho2_b(v', v),   D(c v, c' v') = sum_a rho1_a(c, c') T_a(v', v)
// minus the exchange term, exactly as the CUDA-core tile (assembly_tile.cuh) does after its own overlaps.
// The output stage (packed split-BF16 staging tile, 16-byte stores, mirror block next to the diagonal) is
// the same as there.
#pragma once
#include "assembly_tile.cuh"

#define XATU_ASM_TC_KPMAX 128   // 2 norb rounded up to 16; larger orbital bases take the CUDA-core tile

// threads of a tensor-core tile: one per (k, k') pair, at least four warps
__host__ __device__ constexpr int asm_tc_threads(int tk) { return tk * tk < 128 ? 128 : tk * tk; }
#define XATU_ASM_TC_SPIN (1u << 24)

struct AsmTcGeom {
  int KP;            // K of the overlap GEMMs (2 norb rounded up to 16)
  int sbo;           // core-matrix row-group stride of the operands, bytes (KP * 16)
  size_t opA1_plane, opA2_plane;   // bytes of one FP16 plane of an A operand (its valid rows)
  size_t opB1_plane, opB2_plane;
  size_t off_A1, off_A2, off_B1, off_B2;  // operand planes: hi at off, lo at off + plane
  size_t off_r1, off_r2, off_tile, off_ex;
  size_t bytes;
};

// Staging tile of a tensor-core tile kept apart from the overlaps (windows of more than 4 e-h pairs per k);
// smaller windows hold a pair's values in registers while the overlaps are read, and reuse their space.
template <int NV, int NC>
__host__ __device__ constexpr bool asm_tc_tile_apart() { return NV * NC > 4; }

template <int NV, int NC, int NA, int TK>
__host__ __device__ inline AsmTcGeom asm_tc_geom(int norb) {
  constexpr int NCV = NV * NC;
  constexpr int TR = TK * NCV;
  constexpr bool SWZ = (TR % 16) == 0;
  constexpr int LDT = SWZ ? TR : TR + 1;
  AsmTcGeom g;
  g.KP = ((2 * norb + 15) / 16) * 16;
  g.sbo = g.KP * 16;
  // an A plane holds its NA TK nband valid rows only: the M = 128 product also reads the rows after them
  // (the next planes, or the padding at the end), and those accumulator rows are never used
  g.opA1_plane = (size_t)NA * TK * NC * g.KP * 2;
  g.opA2_plane = (size_t)NA * TK * NV * g.KP * 2;
  g.opB1_plane = (size_t)2 * TK * NC * g.KP * 2;
  g.opB2_plane = (size_t)2 * TK * NV * g.KP * 2;
  auto al = [](size_t x) { return (x + 127) & ~(size_t)127; };
  g.off_A1 = 0;
  g.off_A2 = al(g.off_A1 + 2 * g.opA1_plane);
  g.off_B1 = al(g.off_A2 + 2 * g.opA2_plane);
  g.off_B2 = al(g.off_B1 + 2 * g.opB1_plane);
  size_t ops_end = al(g.off_B2 + 2 * g.opB2_plane);
  const size_t read_end = g.off_A2 + g.opA2_plane + (size_t)128 * g.KP * 2;   // 128 rows from the last A plane
  if (read_end > ops_end) ops_end = al(read_end);
  // after the products: the overlaps (FP32 complex) reuse the operand space, then the staging tile
  g.off_r1 = 0;
  g.off_r2 = al(g.off_r1 + (size_t)NA * (TK * NC) * (TK * NC) * 8);
  const size_t rho_end = al(g.off_r2 + (size_t)NA * (TK * NV) * (TK * NV) * 8);
  g.off_tile = asm_tc_tile_apart<NV, NC>() ? rho_end : 0;
  const size_t tile_end = al(g.off_tile + (size_t)TR * LDT * 8);
  size_t end = ops_end > rho_end ? ops_end : rho_end;
  if (tile_end > end) end = tile_end;
  g.off_ex = end;
  g.bytes = g.off_ex + (size_t)2 * TR * NA * 8;
  return g;
}

// Operand images of one k block in global memory: A1 (hi, lo planes), A2, B1, B2, the same bytes as the
// tile's shared-memory planes (the A images built from the block's k points as the k' side, the B images as
// the k side).
struct AsmTcImage {
  size_t A1, A2, B1, B2;   // byte offsets inside a block's image
  size_t block;            // bytes per k block
};

template <int NV, int NC, int NA, int TK>
__host__ __device__ inline AsmTcImage asm_tc_image(const AsmTcGeom& g) {
  AsmTcImage im;
  im.A1 = 0;
  im.A2 = im.A1 + 2 * g.opA1_plane;
  im.B1 = im.A2 + 2 * g.opA2_plane;
  im.B2 = im.B1 + 2 * g.opB1_plane;
  im.block = (im.B2 + 2 * g.opB2_plane + 127) & ~(size_t)127;
  return im;
}

__device__ __forceinline__ uint32_t asm_smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

// Shared-memory descriptor, no swizzle, K-major: core matrices of 8 rows x 16 B, adjacent along K 128 B apart
// (leading byte offset), 8-row groups `sbo` bytes apart.
__device__ __forceinline__ uint64_t asm_desc_noswz(const void* base, uint32_t sbo) {
  const uint64_t addr = asm_smem_u32(base);
  uint64_t d = 0;
  d |= (addr >> 4) & 0x3FFFull;
  d |= (uint64_t)(128 >> 4) << 16;
  d |= (uint64_t)((sbo >> 4) & 0x3FFF) << 32;
  d |= (uint64_t)1 << 46;   // descriptor version (sm_100); layout type 0 = no swizzle
  return d;
}

// kind::f16 instruction descriptor: FP16 x FP16 -> FP32, both K-major, M = 128, N = n.
__host__ __device__ constexpr uint32_t asm_idesc_f16(int n) {
  return (1u << 4) | ((uint32_t)(n >> 3) << 17) | ((uint32_t)(128 >> 4) << 24);
}

__device__ __forceinline__ void asm_umma(uint32_t tmem_d, uint64_t adesc, uint64_t bdesc, uint32_t idesc,
                                         uint32_t accumulate) {
  asm volatile(
      "{\n\t.reg .pred p;\n\t"
      "setp.ne.b32 p, %4, 0;\n\t"
      "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}" ::"r"(tmem_d),
      "l"(adesc), "l"(bdesc), "r"(idesc), "r"(accumulate));
}

__device__ __forceinline__ bool asm_mbar_wait(uint64_t* bar, uint32_t parity) {
  const uint32_t addr = asm_smem_u32(bar);
  for (uint32_t it = 0; it < XATU_ASM_TC_SPIN; it++) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.b32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(addr), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

// 8 consecutive FP32 accumulator columns of this warp's 32 tensor-memory lanes
__device__ __forceinline__ void asm_tmem_ld8(uint32_t taddr, float* v) {
  uint32_t r[8];
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
               : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
               : "r"(taddr));
#pragma unroll
  for (int j = 0; j < 8; j++) v[j] = __uint_as_float(r[j]);
}

// (x, y) = hi + lo in FP16, each part packed as one 32-bit word (x in the low half)
__device__ __forceinline__ void asm_split_f16x2(float x, float y, uint32_t& hi, uint32_t& lo) {
  const __half hx = __float2half_rn(x), hy = __float2half_rn(y);
  const __half lx = __float2half_rn(x - __half2float(hx)), ly = __float2half_rn(y - __half2float(hy));
  const __half2 h = __halves2half2(hx, hy), l = __halves2half2(lx, ly);
  hi = *reinterpret_cast<const uint32_t*>(&h);
  lo = *reinterpret_cast<const uint32_t*>(&l);
}

// Byte offset of element (row r, K index k) in a no-swizzle K-major operand plane.
__device__ __forceinline__ uint32_t asm_op_off(int r, int k, int sbo) {
  return (uint32_t)((r >> 3) * sbo + (k >> 3) * 128 + (r & 7) * 16 + (k & 7) * 2);
}

// Operand images of every k block (one thread per group of 4 orbitals of one band at one k): the A form
// (atom-masked rows (atom, k, band), [Re, Im]) and the two B forms (rows (k, band): [Re, Im] and the
// imaginary-part form, [-Im, Re] for conduction bands (rho1), [Im, -Re] for valence bands (rho2)).
template <int NV, int NC, int NA, int TK>
__global__ void asm_tc_format_kernel(AsmParams p, AsmInputs in, int nblk) {
  constexpr int NB = NV + NC;
  constexpr int TKC = TK * NC, TKV = TK * NV;
  const AsmTcGeom G = asm_tc_geom<NV, NC, NA, TK>(p.norb);
  const AsmTcImage IM = asm_tc_image<NV, NC, NA, TK>(G);
  const int norb = p.norb, NQ = G.KP / 8;
  const long long total = (long long)nblk * TK * NB * NQ;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    const int q = (int)(t % NQ);
    const long long r = t / NQ;
    const int band = (int)(r % NB);
    const int kq = (int)((r / NB) % TK);
    const int blk = (int)(r / (NB * TK));
    const int kg = blk * TK + kq;
    float re[4], im[4];
#pragma unroll
    for (int j = 0; j < 4; j++) {
      re[j] = 0.f;
      im[j] = 0.f;
      const int o = 4 * q + j;
      if (kg < p.nk && o < norb) {
        const cd c = (band < NV ? in.eigvec : in.eigvecQ)[((int64_t)kg * p.nb + band) * norb + o];
        re[j] = (float)c.x;
        im[j] = (float)c.y;
      }
    }
    const bool cond = band >= NV;
    const int bb = cond ? band - NV : band;
    unsigned char* img = in.tc_ops + (size_t)blk * IM.block;
    uint32_t h[4], l[4];
#pragma unroll
    for (int j = 0; j < 4; j++) asm_split_f16x2(re[j], im[j], h[j], l[j]);
    {
      // A form, one row per atom
      unsigned char* base = img + (cond ? IM.A1 : IM.A2);
      const size_t plane = cond ? G.opA1_plane : G.opA2_plane;
      const int nbw = cond ? NC : NV;
#pragma unroll
      for (int a = 0; a < NA; a++) {
        uint32_t hm[4], lm[4];
#pragma unroll
        for (int j = 0; j < 4; j++) {
          const int o = 4 * q + j;
          const bool own = o >= p.orb_off[a] && o < p.orb_off[a + 1];
          hm[j] = own ? h[j] : 0u;
          lm[j] = own ? l[j] : 0u;
        }
        const uint32_t off = asm_op_off((a * TK + kq) * nbw + bb, 8 * q, G.sbo);
        *reinterpret_cast<uint4*>(base + off) = make_uint4(hm[0], hm[1], hm[2], hm[3]);
        *reinterpret_cast<uint4*>(base + plane + off) = make_uint4(lm[0], lm[1], lm[2], lm[3]);
      }
    }
    {
      // B forms
      unsigned char* base = img + (cond ? IM.B1 : IM.B2);
      const size_t plane = cond ? G.opB1_plane : G.opB2_plane;
      const int row = kq * (cond ? NC : NV) + bb;
      uint32_t off = asm_op_off(row, 8 * q, G.sbo);
      *reinterpret_cast<uint4*>(base + off) = make_uint4(h[0], h[1], h[2], h[3]);
      *reinterpret_cast<uint4*>(base + plane + off) = make_uint4(l[0], l[1], l[2], l[3]);
#pragma unroll
      for (int j = 0; j < 4; j++) asm_split_f16x2(cond ? -im[j] : im[j], cond ? re[j] : -re[j], h[j], l[j]);
      off = asm_op_off(row + (cond ? TKC : TKV), 8 * q, G.sbo);
      *reinterpret_cast<uint4*>(base + off) = make_uint4(h[0], h[1], h[2], h[3]);
      *reinterpret_cast<uint4*>(base + plane + off) = make_uint4(l[0], l[1], l[2], l[3]);
    }
  }
}

__device__ __forceinline__ void asm_bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   asm_smem_u32(dst)),
               "l"(reinterpret_cast<uint64_t>(src)), "r"(bytes), "r"(asm_smem_u32(bar))
               : "memory");
}

template <int NV, int NC, int NA, int TK>
__device__ __forceinline__ void assemble_tile_tc(const AsmParams& p, const AsmInputs& in, const AsmOutputs& out,
                                                 int nblk, int tile) {
  constexpr int NB = NV + NC;
  constexpr int NCV = NV * NC;
  constexpr int TR = TK * NCV;
  constexpr int TKC = TK * NC, TKV = TK * NV;
  constexpr int N1 = 2 * TKC, N2 = 2 * TKV;
  constexpr int TMEM_COLS = (N1 + N2) <= 32 ? 32 : (N1 + N2) <= 64 ? 64 : (N1 + N2) <= 128 ? 128 : 256;
  static_assert(NA * TKC <= 128 && NA * TKV <= 128, "overlap rows must fit one M = 128 product");
  static_assert(N1 % 16 == 0 && N2 % 16 == 0 && N1 + N2 <= 256, "product widths");
  constexpr bool SWZ = (TR % 16) == 0;
  constexpr int LDT = SWZ ? TR : TR + 1;
#define TIDX(r, c) ((r) * LDT + (SWZ ? ((c) ^ (((r) >> 2) & 15)) : (c)))
  using E = cplx<float>;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  __shared__ uint64_t s_mma_done, s_ops_done;
  __shared__ uint32_t s_tmem;
  const AsmTcGeom G = asm_tc_geom<NV, NC, NA, TK>(p.norb);
  int kb, kb2;
  tile_of(tile, nblk, kb, kb2);
  const int tid = threadIdx.x;
  const int warp = tid >> 5, lane = tid & 31;
  const int kk = tid / TK, kk2 = tid % TK;
  const int k = kb * TK + kk, k2 = kb2 * TK + kk2;
  // one thread per pair; a block of fewer than 128 pairs has spare threads (all four tensor-memory
  // sub-partitions need a warp for the accumulator read-out)
  const bool active = tid < TK * TK && (k < p.nk) && (k2 < p.nk) && !(kb == kb2 && k > k2);
  const int norb = p.norb;

  // the pair's interaction-table row goes to registers first, so its latency overlaps the staging
  E Vr[NA][NA];
  if (active) {
    const cd* Vt = interaction_ptr(p, in, k, k2);
#pragma unroll
    for (int a = 0; a < NA; a++)
#pragma unroll
      for (int b = 0; b < NA; b++) {
        const cd v = Vt[a * NA + b];
        Vr[a][b] = {(float)v.x, (float)v.y};
      }
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(asm_smem_u32(&s_tmem)),
                 "r"((uint32_t)TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(asm_smem_u32(&s_mma_done)), "r"(1));
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(asm_smem_u32(&s_ops_done)), "r"(1));
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }

  // ---- operands: the A images of block kb2 (the k' side) and the B images of block kb (the k side), four bulk
  //      copies into the planes of the shared-memory layout; only the thread that issues the products waits
  if (tid == 0) {
    const AsmTcImage IM = asm_tc_image<NV, NC, NA, TK>(G);
    const unsigned char* ia = in.tc_ops + (size_t)kb2 * IM.block;
    const unsigned char* ib = in.tc_ops + (size_t)kb * IM.block;
    const uint32_t bA1 = (uint32_t)(2 * G.opA1_plane), bA2 = (uint32_t)(2 * G.opA2_plane);
    const uint32_t bB1 = (uint32_t)(2 * G.opB1_plane), bB2 = (uint32_t)(2 * G.opB2_plane);
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(asm_smem_u32(&s_ops_done)),
                 "r"(bA1 + bA2 + bB1 + bB2)
                 : "memory");
    asm_bulk_load(smem_raw + G.off_A1, ia + IM.A1, bA1, &s_ops_done);
    asm_bulk_load(smem_raw + G.off_A2, ia + IM.A2, bA2, &s_ops_done);
    asm_bulk_load(smem_raw + G.off_B1, ib + IM.B1, bB1, &s_ops_done);
    asm_bulk_load(smem_raw + G.off_B2, ib + IM.B2, bB2, &s_ops_done);
  }
  // exchange factors of the tile's rows and columns
  const int64_t row0 = (int64_t)kb * TR, col0 = (int64_t)kb2 * TR;
  E* sL = reinterpret_cast<E*>(smem_raw + G.off_ex);
  E* sR = sL + TR * NA;
  if (p.exchange) {
    for (int t = tid; t < TR * NA; t += blockDim.x) {
      const int r = t / NA, a = t - r * NA;
      E l = {0.f, 0.f}, rr = {0.f, 0.f};
      if (row0 + r < p.N) {
        const cd x = in.exL[(row0 + r) * NA + a];
        l = {(float)x.x, (float)x.y};
      }
      if (col0 + r < p.N) {
        const cd x = in.exR[(col0 + r) * NA + a];
        rr = {(float)x.x, (float)x.y};
      }
      sL[t] = l;
      sR[t] = rr;
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  const uint32_t tmem = s_tmem;

  // ---- the two overlap products, issued by one thread once the operand copies have landed
  bool ops_ok = true;
  if (tid == 0) {
    ops_ok = asm_mbar_wait(&s_ops_done, 0);
    // copies still in flight must land before this block's shared memory is released
    if (!ops_ok) asm_mbar_wait(&s_ops_done, 0);
  }
  if (tid == 0 && ops_ok) {
    constexpr uint32_t id1 = asm_idesc_f16(N1), id2 = asm_idesc_f16(N2);
    const uint32_t d1 = tmem, d2 = tmem + N1;
    const unsigned char* A1 = smem_raw + G.off_A1;
    const unsigned char* B1 = smem_raw + G.off_B1;
    const unsigned char* A2 = smem_raw + G.off_A2;
    const unsigned char* B2 = smem_raw + G.off_B2;
    for (int s = 0; s < G.KP / 16; s++) {
      const uint32_t ko = s * 256;   // 16 K values = two core matrices along K
      const uint64_t a1h = asm_desc_noswz(A1 + ko, G.sbo), a1l = asm_desc_noswz(A1 + G.opA1_plane + ko, G.sbo);
      const uint64_t b1h = asm_desc_noswz(B1 + ko, G.sbo), b1l = asm_desc_noswz(B1 + G.opB1_plane + ko, G.sbo);
      const uint64_t a2h = asm_desc_noswz(A2 + ko, G.sbo), a2l = asm_desc_noswz(A2 + G.opA2_plane + ko, G.sbo);
      const uint64_t b2h = asm_desc_noswz(B2 + ko, G.sbo), b2l = asm_desc_noswz(B2 + G.opB2_plane + ko, G.sbo);
      asm_umma(d1, a1h, b1h, id1, s > 0 ? 1u : 0u);
      asm_umma(d1, a1h, b1l, id1, 1u);
      asm_umma(d1, a1l, b1h, id1, 1u);
      asm_umma(d2, a2h, b2h, id2, s > 0 ? 1u : 0u);
      asm_umma(d2, a2h, b2l, id2, 1u);
      asm_umma(d2, a2l, b2h, id2, 1u);
    }
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     asm_smem_u32(&s_mma_done))
                 : "memory");
  }
  // (on a failed operand wait no product was issued and nothing will arrive: skip the wait)
  const bool mma_ok = __syncthreads_and(ops_ok ? 1 : 0) && __syncthreads_and(asm_mbar_wait(&s_mma_done, 0) ? 1 : 0);
  asm volatile("tcgen05.fence::after_thread_sync;");
  if (!mma_ok) {
    if (tid == 0) atomicOr(in.status, XATU_DEVERR_NOCONV);
  } else {
    // ---- accumulators -> shared memory, k side first: r1[a][(k, c)][(k', c')], r2[b][(k, v)][(k', v')] as
    //      complex FP32.  Warp w reads sub-partition w mod 4 (accumulator rows 32 (w mod 4) ...) and every
    //      (nwarps / 4)-th group of 8 columns of the real block together with the same columns of the
    //      imaginary block.
    float2* r1 = reinterpret_cast<float2*>(smem_raw + G.off_r1);
    float2* r2 = reinterpret_cast<float2*>(smem_raw + G.off_r2);
    const int sub = warp & 3, part = warp >> 2, nparts = (int)(blockDim.x >> 7);
    const int m = sub * 32 + lane;   // accumulator row of this thread
    const uint32_t lane_base = (uint32_t)(sub * 32) << 16;
    for (int c0 = part * 8; c0 < TKC; c0 += 8 * nparts) {
      float re[8], im[8];
      asm_tmem_ld8(tmem + lane_base + c0, re);
      asm_tmem_ld8(tmem + lane_base + TKC + c0, im);
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      if (m < NA * TKC) {
        const int a = m / TKC, col = m % TKC;   // col = (k', c'), column n = (k, c)
#pragma unroll
        for (int j = 0; j < 8; j++) r1[((size_t)a * TKC + c0 + j) * TKC + col] = make_float2(re[j], im[j]);
      }
    }
    for (int c0 = part * 8; c0 < TKV; c0 += 8 * nparts) {
      float re[8], im[8];
      asm_tmem_ld8(tmem + lane_base + N1 + c0, re);
      asm_tmem_ld8(tmem + lane_base + N1 + TKV + c0, im);
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      if (m < NA * TKV) {
        const int b = m / TKV, col = m % TKV;   // col = (k', v'), column n = (k, v)
#pragma unroll
        for (int j = 0; j < 8; j++) r2[((size_t)b * TKV + c0 + j) * TKV + col] = make_float2(re[j], im[j]);
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  if (warp == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"((uint32_t)TMEM_COLS));
  }
  if (!mma_ok) return;

  // ---- per pair: T_a = sum_b V_ab rho2_b, D = sum_a rho1_a T_a, minus exchange; packed split-BF16 words into
  //      the staging tile (for windows of up to 4 e-h pairs per k the tile reuses the overlaps' space: the
  //      pair's words wait in registers until every thread has read its overlaps)
  constexpr bool APART = asm_tc_tile_apart<NV, NC>();
  uint2* sT2 = reinterpret_cast<uint2*>(smem_raw + G.off_tile);
  uint2 held[APART ? 1 : NCV * NCV];
  if (active) {
    const E* r1 = reinterpret_cast<const E*>(smem_raw + G.off_r1);
    const E* r2 = reinterpret_cast<const E*>(smem_raw + G.off_r2);
    E Tm[NA][NV][NV];
#pragma unroll
    for (int a = 0; a < NA; a++)
#pragma unroll
      for (int v2 = 0; v2 < NV; v2++)
#pragma unroll
        for (int v = 0; v < NV; v++) Tm[a][v2][v] = {0.f, 0.f};
#pragma unroll
    for (int b = 0; b < NA; b++) {
      E rho2[NV][NV];   // rho2_b(v', v) of this pair
#pragma unroll
      for (int v = 0; v < NV; v++) {
        const E* src = r2 + ((size_t)b * TKV + kk * NV + v) * TKV + kk2 * NV;
        if constexpr (NV == 2) {   // the pair's two v' values are one 16-byte word
          const float4 w = *reinterpret_cast<const float4*>(src);
          rho2[0][v] = {w.x, w.y};
          rho2[1][v] = {w.z, w.w};
        } else {
#pragma unroll
          for (int v2 = 0; v2 < NV; v2++) rho2[v2][v] = src[v2];
        }
      }
#pragma unroll
      for (int a = 0; a < NA; a++)
#pragma unroll
        for (int v2 = 0; v2 < NV; v2++)
#pragma unroll
          for (int v = 0; v < NV; v++) cfma(Tm[a][v2][v], Vr[a][b], rho2[v2][v]);
    }
    // rho1_a(c, c') of this pair (for two conduction bands the pair's two c' values are one 16-byte word)
    E rho1c[NA][NC][NC];
#pragma unroll
    for (int a = 0; a < NA; a++)
#pragma unroll
      for (int c = 0; c < NC; c++) {
        const E* src = r1 + ((size_t)a * TKC + kk * NC + c) * TKC + kk2 * NC;
        if constexpr (NC == 2) {
          const float4 w = *reinterpret_cast<const float4*>(src);
          rho1c[a][c][0] = {w.x, w.y};
          rho1c[a][c][1] = {w.z, w.w};
        } else {
#pragma unroll
          for (int c2 = 0; c2 < NC; c2++) rho1c[a][c][c2] = src[c2];
        }
      }
#pragma unroll
    for (int c = 0; c < NC; c++) {
#pragma unroll
      for (int c2 = 0; c2 < NC; c2++) {
        E rho1[NA];
#pragma unroll
        for (int a = 0; a < NA; a++) rho1[a] = rho1c[a][c][c2];
#pragma unroll
        for (int v = 0; v < NV; v++) {
#pragma unroll
          for (int v2 = 0; v2 < NV; v2++) {
            const int pi = c * NV + v, pj = c2 * NV + v2;
            E d = {0.f, 0.f};
#pragma unroll
            for (int a = 0; a < NA; a++) cfma(d, rho1[a], Tm[a][v2][v]);
            const int r = kk * NCV + pi, cc = kk2 * NCV + pj;
            if (p.exchange) {
#pragma unroll
              for (int a = 0; a < NA; a++) {
                const E l = sL[r * NA + a], rr = sR[cc * NA + a];
                d.x -= l.x * rr.x - l.y * rr.y;
                d.y -= l.x * rr.y + l.y * rr.x;
              }
            }
            E val;
            if (k == k2 && pi == pj) {
              const double ec = in.eigvalQ[(int64_t)k * p.nb + NV + c];
              const double ev = in.eigval[(int64_t)k * p.nb + v];
              val.x = -d.x;
              val.y = 0.f;
              out.diag[row0 + r] = p.scissor + ec - ev;
            } else {
              val.x = -d.x;
              val.y = -d.y;
            }
            // on a diagonal pair the lower triangle is filled from the upper one below
            if (APART) {
              if (!(k == k2 && pj < pi)) sT2[TIDX(r, cc)] = split_pack(val.x, val.y);
            } else {
              held[APART ? 0 : pi * NCV + pj] = split_pack(val.x, val.y);
            }
          }
        }
      }
    }
  }
  if (!APART) {
    __syncthreads();   // every thread has read its overlaps: the staging tile may overwrite them
    if (active) {
#pragma unroll
      for (int pi = 0; pi < NCV; pi++) {
        if constexpr (NCV % 2 != 0) {
#pragma unroll
          for (int pj = 0; pj < NCV; pj++)
            if (!(k == k2 && pj < pi)) sT2[TIDX(kk * NCV + pi, kk2 * NCV + pj)] = held[APART ? 0 : pi * NCV + pj];
        } else {
          // two neighbouring columns per 16-byte store where the swizzle keeps them adjacent (XOR of a
          // multiple of 4 with an even column moves both together)
#pragma unroll
          for (int pj = 0; pj < NCV; pj += 2) {
            const int r = kk * NCV + pi, c0 = kk2 * NCV + pj;
            const uint2 u0 = held[APART ? 0 : pi * NCV + pj], u1 = held[APART ? 0 : pi * NCV + pj + 1];
            const bool w0 = !(k == k2 && pj < pi), w1 = !(k == k2 && pj + 1 < pi);
            if (w0 && w1 && ((TIDX(r, c0) & 1) == 0) && TIDX(r, c0 + 1) == TIDX(r, c0) + 1) {
              *reinterpret_cast<uint4*>(&sT2[TIDX(r, c0)]) = make_uint4(u0.x, u0.y, u1.x, u1.y);
            } else {
              if (w0) sT2[TIDX(r, c0)] = u0;
              if (w1) sT2[TIDX(r, c0 + 1)] = u1;
            }
          }
        }
      }
    }
  }
  __syncthreads();
  const int rows = (int)min((int64_t)TR, p.N - row0);
  const int cols = (int)min((int64_t)TR, p.N - col0);
  if (kb == kb2) {
    // lower triangle of a diagonal tile = conjugate of its upper triangle
    for (int t = tid; t < TR * TR; t += blockDim.x) {
      const int r = t / TR, c = t - r * TR;
      if (r > c && r < rows) sT2[TIDX(r, c)] = split_conj(sT2[TIDX(c, r)]);
    }
    __syncthreads();
  }
  unsigned* Kh = reinterpret_cast<unsigned*>(out.Khi);
  unsigned* Kl = reinterpret_cast<unsigned*>(out.Klo);
  constexpr int VEC = 4;                  // complex elements per 16-byte store
  constexpr int CV = (TR + VEC - 1) / VEC;
  for (int t = tid; t < TR * CV; t += blockDim.x) {
    const int r = t / CV, c = (t - r * CV) * VEC;
    if (r >= rows || c >= cols) continue;
    const int64_t o = (row0 + r) * p.ldk + col0 + c;
    if (c + VEC <= cols && (o & 3) == 0) {
      uint2 u[VEC];
#pragma unroll
      for (int q = 0; q < VEC; q++) u[q] = sT2[TIDX(r, c + q)];
      *reinterpret_cast<uint4*>(Kh + o) = make_uint4(u[0].x, u[1].x, u[2].x, u[3].x);
      *reinterpret_cast<uint4*>(Kl + o) = make_uint4(u[0].y, u[1].y, u[2].y, u[3].y);
    } else {
      for (int q = 0; q < VEC && c + q < cols; q++) {
        const uint2 u = sT2[TIDX(r, c + q)];
        Kh[o + q] = u.x;
        Kl[o + q] = u.y;
      }
    }
  }
  // mirror block (rows col0 + c, columns row0 + r, conjugate transpose): only where it reaches the stored upper
  // block triangle of the kernel planes (xatu_kstored), next to the diagonal
  if (kb != kb2 && (row0 + rows - 1) / XATU_KBLOCK >= col0 / XATU_KBLOCK) {
    constexpr int RV = (TR + VEC - 1) / VEC;
    for (int t = tid; t < TR * RV; t += blockDim.x) {
      const int c = t / RV, r = (t - c * RV) * VEC;
      if (c >= cols || r >= rows) continue;
      const int64_t o = (col0 + c) * p.ldk + row0 + r;
      if (r + VEC <= rows && (o & 3) == 0) {
        uint2 u[VEC];
#pragma unroll
        for (int q = 0; q < VEC; q++) u[q] = split_conj(sT2[TIDX(r + q, c)]);
        *reinterpret_cast<uint4*>(Kh + o) = make_uint4(u[0].x, u[1].x, u[2].x, u[3].x);
        *reinterpret_cast<uint4*>(Kl + o) = make_uint4(u[0].y, u[1].y, u[2].y, u[3].y);
      } else {
        for (int q = 0; q < VEC && r + q < rows; q++) {
          const uint2 u = split_conj(sT2[TIDX(r + q, c)]);
          Kh[o + q] = u.x;
          Kl[o + q] = u.y;
        }
      }
    }
  }
#undef TIDX
}
