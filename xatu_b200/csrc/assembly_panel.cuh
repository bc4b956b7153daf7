// Mixed-precision assembly by row panels, persistent and pipelined (ExcitonTB::BShamiltonian,
// ExcitonTB.cpp:840-921; realSpaceInteractionTerm :520-548; reciprocal and exchange terms :562-621, :897,
// :905, as in assembly_tile.cuh).
//
// Work unit: a row panel of TKR k points (the 128 rows of one tcgen05 product, rows (k, band)) against a
// column tile of TKC = 8 k' points.  For every (k, k') pair the per-atom band overlaps
//   rho1_a[(k,c),(k',c')] = sum_{o in a} conj(CQ_k[c]_o) CQ_k'[c']_o
//   rho2_b[(k',v'),(k,v)] = sum_{o in b} conj(C_k'[v']_o) C_k[v]_o
// are products with M = 128 rows (k, band) of the panel and N columns (k', band', form) of the tile, one
// product per atom over that atom's orbitals only:
//   A (128 x KPT, K-major): row (k, beta) holds [Re, Im] of the coefficients of band beta at k, the orbitals
//     of every atom in a block of its own along K (2 norb_a values rounded up to 16);
//   B_a (16 nband x K_a per atom, K-major): rows (k', band', form) in a real-part form [Re, Im] and the form
//     whose product is the imaginary part ([Im, -Re] for rho1, [-Im, Re] for rho2).
// FP16 hi/lo operands (x = hi + lo, 22 significant bits; |C| <= 1 keeps them in range), three products per
// overlap (hi.hi + hi.lo + lo.hi), FP32 accumulation in tensor memory.
//
// Tensor memory lane m is row m of the panel, so the thread of lane (k, beta) reads its own overlaps
// straight from tensor memory and forms, for each k' of its column group,
//   T_a(v', beta) = sum_b V_ab rho2_b(v', beta)          (the lanes of one k swap their T by a shuffle)
//   D(beta v, c' v') = sum_a rho1_a(beta, c') T_a(v', v) - sum_a L_a(i) R_a(j)
// and writes -(D - X) as split-BF16 words (hi, lo) into a staging buffer shared by the four warps of its
// tensor-memory sub-partition, which then store whole 128-byte row segments of it.
//
// Pipeline, one CTA per SM: each CTA takes an equal contiguous range of the (panel, tile) pairs that reach the
// stored upper block triangle (xatu_kstored).  One thread stages the operand images with bulk copies (the
// panel's A once per panel, each tile's B into a ring of three stages), three more issue the products into one
// of two tensor-memory slots; sixteen consumer warps (four per sub-partition, two k' each) read a slot, release it
// and combine while the next tile's products run.  The warpgroup of the copy and product threads hands
// registers to the consumers (setmaxnreg).  Every wait is bounded; on a timeout the CTA records
// XATU_DEVERR_NOCONV, waits (bounded) for its own copies and products and frees its tensor memory.
//
// The lower triangles of the diagonal 128 x 128 blocks are rewritten afterwards as the conjugate transpose of
// the upper ones (asm_diag_mirror_kernel), so the stored kernel is exactly Hermitian.
#pragma once
#include "assembly_tc.cuh"

#define XATU_PANEL_TKC 8                                  // k' points per column tile
#define XATU_PANEL_NCW 16                                 // consumer warps (four warpgroups)
#define XATU_PANEL_THREADS (XATU_PANEL_NCW * 32 + 128)   // + one warpgroup: the copy warp and three product warps
// Registers per thread after the split: the block is launched with 96 per thread (640 threads, one block per SM);
// the copy/product warpgroup gives back down to 32, the consumer warpgroups take 112: 128 x 32 + 512 x 112 = 640 x 96.
#define XATU_PANEL_REGS_LAUNCH 96
#define XATU_PANEL_REGS_PRODUCER 32
#define XATU_PANEL_REGS_CONSUMER 112
#define XATU_PANEL_NBS 3                                  // operand stages of the column tiles
#define XATU_PANEL_KPT_MAX 128                            // K of the A operand (shared-memory budget)
#define XATU_PANEL_SMEM_MAX (225 * 1024)

template <int NV, int NC, int NA>
struct PanelShape {
  static constexpr int NBW = NV > NC ? NV : NC;             // lanes per k point
  static constexpr int NCV = NV * NC;                       // e-h pairs per k point
  static constexpr int KPW = 32 / NBW;                      // k points per sub-partition
  static constexpr int TKR = 4 * KPW;                       // k points per panel
  static constexpr int N1 = 2 * XATU_PANEL_TKC * NC;        // product columns per atom: rho1 ...
  static constexpr int N2 = 2 * XATU_PANEL_TKC * NV;        // ... and rho2
  static constexpr int SLOT = NA * (N1 + N2);               // accumulator columns of one tile
  static constexpr int SLOT_STRIDE = SLOT <= 32 ? 32 : SLOT <= 64 ? 64 : SLOT <= 128 ? 128 : SLOT <= 256 ? 256 : 512;
  static constexpr int NSLOT = SLOT_STRIDE <= 256 ? 2 : 1;
  static constexpr int TMEM_COLS = NSLOT * SLOT_STRIDE;
  static constexpr int GROWS = KPW * NCV;                   // staging rows of a sub-partition group
  static constexpr int GCOLS = XATU_PANEL_TKC * NCV;        // columns of a tile
  static constexpr int CPR = GCOLS / 4;                     // 16-byte chunks per staging row and plane
  static constexpr int PITCH = GCOLS * 4;                   // staging row pitch, bytes
  static constexpr bool SUPPORTED = NV <= 2 && NC <= 2 && NA <= 4 && SLOT <= 512;
};

struct AsmPanelGeom {
  int KPT;                                   // K of the A operand
  int koff[XATU_MAX_ATOMS + 1];              // K offset of each atom's block (koff[na] = KPT)
  int npanel, ntile, total;                  // row panels, column tiles, stored (panel, tile) pairs
  int vstride;                               // float2 per entry of the FP32 table (packed upper triangle)
  int nstg;                                  // staging buffers per sub-partition group (2: one barrier per tile)
  uint32_t a_plane, a_bytes;                 // one FP16 plane of an A operand (128 x KPT); A image of a panel
  uint32_t b_off[2][XATU_MAX_ATOMS];         // B image of a tile: product, atom -> hi plane (lo plane follows)
  uint32_t b_plane[2][XATU_MAX_ATOMS];       // bytes of one plane
  uint32_t b_bytes;                          // B image of a column tile
  uint32_t s_B, s_stage, stage_bytes, smem;  // shared memory: A at 0, the B ring, the staging buffers; total
  size_t img_A, img_B, img_V, img_U, img_F;  // scratch: A images, B images, FP32 table, scaled reduced k
                                             // coordinates, flag word (set when their differences are not integral)
  size_t bytes;
};

// First column tile of panel i that reaches the stored upper block triangle.
template <class S>
__host__ __device__ __forceinline__ int panel_jmin(int i) {
  const long long r0 = (long long)i * S::TKR * S::NCV;
  const long long cmin = (r0 / XATU_KBLOCK) * XATU_KBLOCK;
  return (int)(cmin / ((long long)S::NCV * XATU_PANEL_TKC));
}

template <int NV, int NC, int NA>
inline bool asm_panel_geom(const AsmParams& p, AsmPanelGeom& g) {
  using S = PanelShape<NV, NC, NA>;
  if (!S::SUPPORTED || p.na != NA || p.nk <= 0) return false;
  memset(&g, 0, sizeof(g));
  int kk = 0;
  for (int a = 0; a < NA; a++) {
    g.koff[a] = kk;
    kk += ((2 * (p.orb_off[a + 1] - p.orb_off[a]) + 15) / 16) * 16;
  }
  g.koff[NA] = kk;
  g.KPT = kk;
  if (kk <= 0 || kk > XATU_PANEL_KPT_MAX) return false;
  g.npanel = (p.nk + S::TKR - 1) / S::TKR;
  g.ntile = (p.nk + XATU_PANEL_TKC - 1) / XATU_PANEL_TKC;
  long long tot = 0;
  for (int i = 0; i < g.npanel; i++) tot += g.ntile - panel_jmin<S>(i);
  if (tot <= 0 || tot > (1LL << 30)) return false;
  g.total = (int)tot;
  g.vstride = (NA * (NA + 1) / 2 + 1) & ~1;
  g.a_plane = 128u * g.KPT * 2u;
  g.a_bytes = 4u * g.a_plane;
  uint32_t off = 0;
  for (int pr = 0; pr < 2; pr++)
    for (int a = 0; a < NA; a++) {
      const uint32_t rows = pr == 0 ? S::N1 : S::N2;
      g.b_off[pr][a] = off;
      g.b_plane[pr][a] = rows * (uint32_t)(g.koff[a + 1] - g.koff[a]) * 2u;
      off += 2u * g.b_plane[pr][a];
    }
  g.b_bytes = off;
  auto al = [](size_t x) { return (x + 1023) & ~(size_t)1023; };
  g.s_B = (uint32_t)al(g.a_bytes);
  g.s_stage = (uint32_t)al(g.s_B + (size_t)XATU_PANEL_NBS * g.b_bytes);
  g.stage_bytes = 2u * S::GROWS * S::PITCH;
  g.nstg = 2;
  g.smem = g.s_stage + 4u * g.nstg * g.stage_bytes;
  if (g.smem > XATU_PANEL_SMEM_MAX) {
    g.nstg = 1;
    g.smem = g.s_stage + 4u * g.stage_bytes;
  }
  if (g.smem > XATU_PANEL_SMEM_MAX) return false;
  auto al256 = [](size_t x) { return (x + 255) & ~(size_t)255; };
  g.img_A = 0;
  g.img_B = al256((size_t)g.npanel * g.a_bytes);
  g.img_V = al256(g.img_B + (size_t)g.ntile * g.b_bytes);
  g.img_U = al256(g.img_V + (size_t)p.nentries * g.vstride * 8);
  g.img_F = al256(g.img_U + (size_t)p.nk * 3 * 8);
  g.bytes = g.img_F + 256;
  return true;
}

// ----------------------------------------------------------------- operand images, FP32 table, k coordinates
// One thread per 8 K values of one operand row (A: panel, product, row; B: tile, product, atom, row), then one
// per value of the FP32 table (the packed upper triangle of each entry), then one per k point: 2n inv(B B^T) B k,
// the reduced coordinates of k scaled as findEquivalentPointBZ scales a difference (Lattice.cpp:251-279), so
// that k' - k needs one subtraction.
template <int NV, int NC, int NA>
__global__ void asm_panel_format_kernel(AsmParams p, AsmInputs in, AsmPanelGeom g) {
  using S = PanelShape<NV, NC, NA>;
  constexpr int NBW = S::NBW, KPW = S::KPW, TKR = S::TKR;
  const int KC = g.KPT / 8;
  const long long nA = (long long)g.npanel * 2 * 128 * KC;
  int bchunks = 0;   // K chunks of all B rows of one tile
  for (int pr = 0; pr < 2; pr++)
    for (int a = 0; a < NA; a++) bchunks += (pr == 0 ? S::N1 : S::N2) * ((g.koff[a + 1] - g.koff[a]) / 8);
  const long long nB = (long long)g.ntile * bchunks;
  const long long nV = p.nentries * g.vstride;
  const long long total = nA + nB + nV + p.nk;
  for (long long t = blockIdx.x * (long long)blockDim.x + threadIdx.x; t < total;
       t += (long long)gridDim.x * blockDim.x) {
    if (t < nA) {
      const int kc = (int)(t % KC);
      const int r = (int)((t / KC) % 128);
      const int pr = (int)((t / (KC * 128)) % 2);
      const int i = (int)(t / (KC * 256));
      const int sp = r >> 5, l = r & 31, kw = l / NBW, beta = l - kw * NBW;
      const int k = i * TKR + sp * KPW + kw;
      const cd* C = nullptr;
      if (kw < KPW && k < p.nk) {
        if (pr == 0 && beta < NC) C = in.eigvecQ + ((int64_t)k * p.nb + NV + beta) * p.norb;
        if (pr == 1 && beta < NV) C = in.eigvec + ((int64_t)k * p.nb + beta) * p.norb;
      }
      float v[8];
#pragma unroll
      for (int x = 0; x < 8; x++) {
        const int kk = 8 * kc + x;
        v[x] = 0.f;
        if (C) {
          int a = 0;
          while (a + 1 < NA && kk >= g.koff[a + 1]) a++;
          const int loc = kk - g.koff[a];
          const int o = p.orb_off[a] + (loc >> 1);
          if (o < p.orb_off[a + 1]) v[x] = (loc & 1) ? (float)C[o].y : (float)C[o].x;
        }
      }
      uint32_t h[4], lo[4];
#pragma unroll
      for (int x = 0; x < 4; x++) asm_split_f16x2(v[2 * x], v[2 * x + 1], h[x], lo[x]);
      unsigned char* base = in.tc_ops + g.img_A + (size_t)i * g.a_bytes + (size_t)pr * 2 * g.a_plane;
      const uint32_t off = asm_op_off(r, 8 * kc, g.KPT * 16);
      *reinterpret_cast<uint4*>(base + off) = make_uint4(h[0], h[1], h[2], h[3]);
      *reinterpret_cast<uint4*>(base + g.a_plane + off) = make_uint4(lo[0], lo[1], lo[2], lo[3]);
    } else if (t < nA + nB) {
      long long u = t - nA;
      const int j = (int)(u / bchunks);
      int rem = (int)(u % bchunks);
      int pr = 0, a = 0;
      for (;;) {
        const int c = (pr == 0 ? S::N1 : S::N2) * ((g.koff[a + 1] - g.koff[a]) / 8);
        if (rem < c) break;
        rem -= c;
        if (++a == NA) {
          a = 0;
          pr++;
        }
      }
      const int Ka = g.koff[a + 1] - g.koff[a];
      const int kc = rem % (Ka / 8), r = rem / (Ka / 8);
      const int nbp = pr == 0 ? NC : NV;
      const int kq = r / (2 * nbp), band = (r % (2 * nbp)) >> 1, form = r & 1;
      const int kp = j * XATU_PANEL_TKC + kq;
      float v[8];
#pragma unroll
      for (int x = 0; x < 8; x++) {
        const int kk = 8 * kc + x;
        const int o = p.orb_off[a] + (kk >> 1);
        v[x] = 0.f;
        if (kp < p.nk && o < p.orb_off[a + 1]) {
          const cd y = pr == 0 ? in.eigvecQ[((int64_t)kp * p.nb + NV + band) * p.norb + o]
                               : in.eigvec[((int64_t)kp * p.nb + band) * p.norb + o];
          const float yr = (float)y.x, yi = (float)y.y;
          if (form == 0) v[x] = (kk & 1) ? yi : yr;
          else if (pr == 0) v[x] = (kk & 1) ? -yr : yi;   // rho1: [Im, -Re]
          else v[x] = (kk & 1) ? yr : -yi;                // rho2: [-Im, Re]
        }
      }
      uint32_t h[4], lo[4];
#pragma unroll
      for (int x = 0; x < 4; x++) asm_split_f16x2(v[2 * x], v[2 * x + 1], h[x], lo[x]);
      unsigned char* base = in.tc_ops + g.img_B + (size_t)j * g.b_bytes + g.b_off[pr][a];
      const uint32_t off = asm_op_off(r, 8 * kc, Ka * 16);
      *reinterpret_cast<uint4*>(base + off) = make_uint4(h[0], h[1], h[2], h[3]);
      *reinterpret_cast<uint4*>(base + g.b_plane[pr][a] + off) = make_uint4(lo[0], lo[1], lo[2], lo[3]);
    } else if (t < nA + nB + nV) {
      // packed upper triangle -V_ab, a <= b (the tables are Hermitian in the atom pair), zero padding; stored
      // negated: the combination then yields -(D - X) without a sign flip
      const long long u = t - nA - nB;
      const long long e = u / g.vstride;
      const int x = (int)(u % g.vstride);
      int a = 0, b = -1;
      for (int r = 0, q = 0; r < NA && b < 0; r++)
        for (int c = r; c < NA; c++, q++)
          if (q == x) {
            a = r;
            b = c;
            break;
          }
      float2 val = make_float2(0.f, 0.f);
      if (b >= 0) {
        const cd y = in.table[e * NA * NA + a * NA + b];
        val = make_float2((float)-y.x, (float)-y.y);
      }
      reinterpret_cast<float2*>(in.tc_ops + g.img_V)[u] = val;
    } else {
      const int k = (int)(t - nA - nB - nV);
      double* U = reinterpret_cast<double*>(in.tc_ops + g.img_U);
      const EquivMap& m = p.emap;
      double u[3], u0[3];
      for (int pass = 0; pass < 2; pass++) {
        const int kk = pass == 0 ? k : 0;
        double ind[3] = {0., 0., 0.};
        for (int i = 0; i < m.ndim; i++)
          ind[i] = m.B[3 * i] * in.kpoints[3 * kk] + m.B[3 * i + 1] * in.kpoints[3 * kk + 1] +
                   m.B[3 * i + 2] * in.kpoints[3 * kk + 2];
        for (int i = 0; i < 3; i++) {
          double c = 0.0;
          if (i < m.ndim)
            for (int jj = 0; jj < m.ndim; jj++) c += m.inv[i * m.ndim + jj] * ind[jj];
          (pass == 0 ? u : u0)[i] = c * (2.0 * m.n);
        }
      }
      bool integral = true;
      for (int i = 0; i < 3; i++) {
        U[3 * k + i] = u[i];
        const double d = u[i] - u0[i];
        if (fabs(d - rint(d)) > 1e-6) integral = false;
      }
      // differences of the scaled coordinates are integers on Monkhorst-Pack meshes (shifted or not): the
      // consumers then locate table rows with integer arithmetic
      if (!integral) atomicOr(reinterpret_cast<int*>(in.tc_ops + g.img_F), 1);
    }
  }
}

__device__ __forceinline__ uint64_t panel_clock_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

// Bounded mbarrier wait (one second) that gives up early once another role of the CTA has aborted.  The
// waiting thread is suspended by the hardware until the phase completes (or 0.2 ms pass).  The barrier is
// tested first, so a phase that has completed is seen by every waiter even after an abort.
__device__ __forceinline__ bool panel_wait(uint64_t* bar, uint32_t parity, const volatile int* abort) {
  const uint32_t addr = asm_smem_u32(bar);
  uint64_t start = 0;
  for (;;) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2, %3;\n\t"
        "selp.b32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(addr), "r"(parity), "r"(200000u)
        : "memory");
    if (done) return true;
    if (*abort) return false;
    const uint64_t now = panel_clock_ns();
    if (start == 0) start = now;
    else if (now - start > 1000000000ull) return false;
  }
}

__device__ __forceinline__ void panel_expect(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(asm_smem_u32(bar)), "r"(bytes)
               : "memory");
}

__device__ __forceinline__ void panel_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(asm_smem_u32(bar))
               : "memory");
}

template <int NCOL>
__device__ __forceinline__ void panel_tmem_ld(uint32_t taddr, float* v) {
  uint32_t r[NCOL];
  if constexpr (NCOL == 2) {
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x2.b32 {%0,%1}, [%2];" : "=r"(r[0]), "=r"(r[1]) : "r"(taddr));
  } else if constexpr (NCOL == 4) {
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x4.b32 {%0,%1,%2,%3}, [%4];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3])
                 : "r"(taddr));
  } else {
    static_assert(NCOL == 8, "tensor-memory load width");
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7])
                 : "r"(taddr));
  }
#pragma unroll
  for (int j = 0; j < NCOL; j++) v[j] = __uint_as_float(r[j]);
}

struct PanelIter {
  int i, j;
};

template <class S>
__device__ __forceinline__ PanelIter panel_locate(int t, int npanel, int ntile) {
  int i = 0;
  for (; i < npanel - 1; i++) {
    const int n = ntile - panel_jmin<S>(i);
    if (t < n) break;
    t -= n;
  }
  return {i, panel_jmin<S>(i) + t};
}

template <class S>
__device__ __forceinline__ void panel_next(PanelIter& it, int ntile) {
  if (++it.j == ntile) {
    it.i++;
    it.j = panel_jmin<S>(it.i);
  }
}

// Completion barriers of the tiles' products: a ring of XATU_PANEL_NDONE (a multiple of both the operand stages
// and the tensor-memory slots), tile t -> done[t mod NDONE], phase t / NDONE; every product thread commits to it.
#define XATU_PANEL_NDONE 6
#define XATU_PANEL_NISSUE 3   // product-issuing threads (warps NCW + 1 ...)
static_assert(XATU_PANEL_NISSUE >= 1 && XATU_PANEL_NISSUE <= 3, "the issuers share the fifth warpgroup with the copier");

// The thread that stages the operands: the panel's A image once per panel (after every product of the previous
// panel has completed), each tile's B image into the ring of NBS stages (after the products of the tile that
// used the stage before).
template <int NV, int NC, int NA>
__device__ __forceinline__ void panel_copier(const AsmPanelGeom& g, const unsigned char* __restrict__ img,
                                             unsigned char* smem, uint64_t* full, uint64_t* done, uint64_t* afull,
                                             int t0, int nt, int* status, volatile int* abort) {
  using S = PanelShape<NV, NC, NA>;
  constexpr int NBS = XATU_PANEL_NBS, ND = XATU_PANEL_NDONE;
  static_assert(ND % NBS == 0, "done ring");
  PanelIter it = panel_locate<S>(t0, g.npanel, g.ntile);
  int cur = -1, nA = 0, u = 0;
  bool ok = true;
  for (; u < nt; u++, panel_next<S>(it, g.ntile)) {
    const int st = u % NBS;
    if (u >= NBS && !(ok = panel_wait(&done[(u - NBS) % ND], ((u - NBS) / ND) & 1, abort))) break;
    if (it.i != cur) {
      if (u > 0 && !(ok = panel_wait(&done[(u - 1) % ND], ((u - 1) / ND) & 1, abort))) break;
      panel_expect(afull, g.a_bytes);
      const unsigned char* src = img + g.img_A + (size_t)it.i * g.a_bytes;
#pragma unroll
      for (int q = 0; q < 4; q++)
        asm_bulk_load(smem + (size_t)q * g.a_plane, src + (size_t)q * g.a_plane, g.a_plane, afull);
      nA++;
      cur = it.i;
    }
    panel_expect(&full[st], g.b_bytes);
    asm_bulk_load(smem + g.s_B + (size_t)st * g.b_bytes, img + g.img_B + (size_t)it.j * g.b_bytes, g.b_bytes,
                  &full[st]);
  }
  if (!ok) {
    atomicOr(status, XATU_DEVERR_NOCONV);
    *abort = 1;
  }
  // copies in flight land before the CTA's shared memory is released
  for (int st = 0; st < NBS; st++) {
    const int f = u - 1 - ((u - 1 - st) % NBS + NBS) % NBS;   // last copy issued into stage st
    if (f >= 0 && f < u) asm_mbar_wait(&full[st], (f / NBS) & 1);
  }
  if (nA > 0) asm_mbar_wait(afull, (nA - 1) & 1);
}

// Threads that issue the products of each tile into its tensor-memory slot: the (product, atom) chains c = pr NA + a
// (pr = 0: rho1, 1: rho2), chain c by issuer c mod XATU_PANEL_NISSUE, the issuers in different warps (different SM
// sub-partitions) side by side.  The shared-memory descriptors of an issuer's chains are formed once, for stage 0,
// in a small table: a tile adds its stage offset to the B descriptors, each further K step of an atom 256 bytes to
// both.  One commit per issuer and tile to the tile's done barrier.
template <int NV, int NC, int NA>
__device__ __forceinline__ void panel_mma(const AsmPanelGeom& g, unsigned char* smem, uint64_t* full, uint64_t* done,
                                          uint64_t* afull, uint64_t* tfree, uint64_t* desc, uint32_t tmem, int t0,
                                          int nt, int issuer, int* status, volatile int* abort) {
  using S = PanelShape<NV, NC, NA>;
  constexpr int NBS = XATU_PANEL_NBS, NSLOT = S::NSLOT, ND = XATU_PANEL_NDONE, NI = XATU_PANEL_NISSUE;
  constexpr int NCH = (2 * NA + NI - 1) / NI;   // chains per issuer (at most)
  static_assert(ND % NSLOT == 0, "done ring");
  // desc[5 x + {0, 1, 2, 3}] = A hi, A lo, B hi, B lo (stage 0) of the issuer's chain x, desc[5 x + 4] = K steps
#pragma unroll
  for (int x = 0; x < NCH; x++) {
    const int c = issuer + x * NI;
    if (c >= 2 * NA) break;
    const int pr = c / NA, a = c - pr * NA;
    const int Ka = g.koff[a + 1] - g.koff[a];
    const unsigned char* A = smem + (size_t)pr * 2 * g.a_plane + (uint32_t)(g.koff[a] / 8) * 128;
    const unsigned char* B = smem + g.s_B + g.b_off[pr][a];
    uint64_t* d = desc + 5 * x;
    d[0] = asm_desc_noswz(A, g.KPT * 16);
    d[1] = asm_desc_noswz(A + g.a_plane, g.KPT * 16);
    d[2] = asm_desc_noswz(B, Ka * 16);
    d[3] = asm_desc_noswz(B + g.b_plane[pr][a], Ka * 16);
    d[4] = (uint64_t)(Ka / 16);
  }
  PanelIter it = panel_locate<S>(t0, g.npanel, g.ntile);
  int cur = -1, nA = 0, last = -1;
  bool ok = true;
  for (int t = 0; t < nt; t++, panel_next<S>(it, g.ntile)) {
    const int st = t % NBS, slot = t % NSLOT;
    if (it.i != cur) {
      nA++;
      cur = it.i;
      if (!(ok = panel_wait(afull, (nA - 1) & 1, abort))) break;
    }
    if (!(ok = panel_wait(&full[st], (t / NBS) & 1, abort))) break;
    if (t >= NSLOT && !(ok = panel_wait(&tfree[slot], ((t / NSLOT) - 1) & 1, abort))) break;
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    const uint32_t dbase = tmem + (uint32_t)(slot * S::SLOT_STRIDE);
    const uint64_t boff = (uint64_t)((st * g.b_bytes) >> 4);
#pragma unroll
    for (int x = 0; x < NCH; x++) {
      const int c = issuer + x * NI;
      if (c >= 2 * NA) break;
      const int pr = c / NA, a = c - pr * NA;
      const uint64_t* d5 = desc + 5 * x;
      const uint64_t ah = d5[0], al = d5[1], bh = d5[2] + boff, bl = d5[3] + boff;
      const int steps = (int)d5[4];
      const uint32_t dcol = dbase + (pr == 0 ? a * S::N1 : NA * S::N1 + a * S::N2);
      const uint32_t id = pr == 0 ? asm_idesc_f16(S::N1) : asm_idesc_f16(S::N2);
      for (int k = 0; k < steps; k++) {
        const uint64_t o = (uint64_t)(16 * k);   // 256 bytes along K
        asm_umma(dcol, ah + o, bh + o, id, k > 0 ? 1u : 0u);
        asm_umma(dcol, ah + o, bl + o, id, 1u);
        asm_umma(dcol, al + o, bh + o, id, 1u);
      }
    }
    panel_commit(&done[t % ND]);
    last = t;
  }
  if (!ok) {
    atomicOr(status, XATU_DEVERR_NOCONV);
    *abort = 1;
  }
  // products in flight complete before the CTA's shared and tensor memory are released (the commit tracks this
  // thread's products; the barrier's phase also needs the other issuers', so the wait is bounded)
  if (last >= 0) asm_mbar_wait(&done[last % ND], (last / ND) & 1);
}

// Coordinates of k point k for panel_entry_c: real space the scaled reduced coordinates (format kernel),
// reciprocal space the integer grid offsets.
__device__ __forceinline__ void panel_coords(const AsmParams& p, const double* __restrict__ U,
                                             const int* __restrict__ kgrid, int k, double* u) {
#pragma unroll
  for (int d = 0; d < 3; d++) u[d] = p.mode == 0 ? U[3 * k + d] : (double)kgrid[3 * k + d];
}

// Row of the interaction table for the pair (k, k') from their coordinates: real space the mesh point
// equivalent to k' - k (the rounding, wrapping and halving of equivalent_index), reciprocal space the grid offset
// k - k'.  integral: the coordinate differences are integers, and the same steps run in integer arithmetic
// (the halving of equivalent_index then truncates a non-negative sum: a shift).  -1 when the entry falls outside
// the table.
__device__ __forceinline__ int panel_entry_c(const AsmParams& p, const double* uk, const double* ukp, bool integral) {
  int64_t e = 0;
  if (p.mode == 0) {
    const int n = p.emap.n;
    if (integral) {
      int sum = 0, stride = 1;
#pragma unroll
      for (int d = 0; d < 3; d++) {
        if (d < p.emap.ndim) {
          int c = __double2int_rn(ukp[d] - uk[d]) - (n & 1);
          if (c >= n) c -= 2 * n;
          else if (c < -n) c += 2 * n;
          sum += (c + n) * stride;
          stride *= n;
        }
      }
      e = sum >> 1;
    } else {
      double acc = 0.0, stride = 1.0;
#pragma unroll
      for (int d = 0; d < 3; d++) {
        if (d < p.emap.ndim) {
          double c = ukp[d] - uk[d];
          if (n & 1) c -= 1;
          c = round(c);
          if (c >= n) c -= 2 * n;
          else if (c < -n) c += 2 * n;
          c += n;
          c /= 2;
          acc += c * stride;
          stride *= n;
        }
      }
      e = (int64_t)acc;
    }
  } else {
    int sum = 0, stride = 1;
#pragma unroll
    for (int d = 0; d < 3; d++) {
      if (d < p.rt_ndim) {
        const int off = __double2int_rn(uk[d] - ukp[d]);
        sum += (off + p.rt_span[d]) * stride;
        stride *= p.rt_len[d];
      }
    }
    e = sum;
  }
  return (e < 0 || e >= p.nentries) ? -1 : (int)e;
}

// Packed upper triangle (a <= b) of the Hermitian atom-pair matrix of one table entry.
__host__ __device__ constexpr int panel_vidx(int a, int b, int na) { return a * na - a * (a - 1) / 2 + (b - a); }

// Consumer warps: sub-partition sp = warp mod 4 (tensor-memory lanes 32 sp ...), column group cg = warp / 4
// (k' points 2 cg, 2 cg + 1 of every tile).  The table rows of the next tile are prefetched: their k
// coordinates at the start of a tile, the rows themselves into the registers of each k' as soon as it is done.
// Every address that does not change from tile to tile (tensor-memory columns, staging offsets) is formed once.
template <int NV, int NC, int NA>
__device__ __forceinline__ void panel_consumer(const AsmParams& p, const AsmInputs& in, const AsmOutputs& out,
                                               const AsmPanelGeom& g, unsigned char* smem, uint64_t* done,
                                               uint64_t* tfree, uint32_t tmem, int t0, int nt, int warp, int lane,
                                               volatile int* abort) {
  using S = PanelShape<NV, NC, NA>;
  constexpr int TKC = XATU_PANEL_TKC;
  constexpr int NBW = S::NBW, NCV = S::NCV, KPW = S::KPW, TKR = S::TKR, NSLOT = S::NSLOT;
  constexpr int VU = NA * (NA + 1) / 2;       // complex values of a packed table row
  constexpr int VQ = (VU + 1) / 2;            // 16-byte loads per row
  constexpr int NQE = NBW == 2 ? 1 : 2;       // table rows this lane locates per tile
  constexpr int CPR = S::CPR, PITCH = S::PITCH, GROWS = S::GROWS;
  constexpr int RSTEP = 128 / CPR;            // staging rows per store pass of the group
  constexpr int NPASS = (GROWS + RSTEP - 1) / RSTEP;
  static_assert((RSTEP / 2) % CPR == 0, "the staging swizzle of a thread's rows is the same in every pass");
  const int sp = warp & 3, cg = warp >> 2;
  const int kw = lane / NBW, beta = lane - kw * NBW;
  const int k_local = sp * KPW + kw;
  const int N = (int)p.N, nk = p.nk;
  const uint32_t tl = tmem + ((uint32_t)(sp * 32) << 16);
  unsigned char* stage0 = smem + g.s_stage + (size_t)sp * g.nstg * g.stage_bytes;
  const float4* __restrict__ V4 = reinterpret_cast<const float4*>(in.tc_ops + g.img_V);
  const double* __restrict__ U = reinterpret_cast<const double*>(in.tc_ops + g.img_U);
  const bool integral = *reinterpret_cast<const volatile int*>(in.tc_ops + g.img_F) == 0;
  // rows of this lane (conduction band beta): valence band v_r, staging offsets of the row at each k' of the warp
  int vr[NV];
  uint32_t so[NV][2];
#pragma unroll
  for (int r = 0; r < NV; r++) {
    vr[r] = (NBW == 2 && NV == 2) ? (r == 0 ? beta : 1 - beta) : 0;
    const int lr = kw * NCV + beta * NV + vr[r];
#pragma unroll
    for (int q = 0; q < 2; q++) {
      const int col = (2 * cg + q) * NCV, ch = col >> 2;
      so[r][q] = (uint32_t)(lr * PITCH + (ch ^ ((lr >> 1) & (CPR - 1))) * 16 + (col & 3) * 4);
    }
  }
  // store map inside the group: chunk sch of rows slr0 + RSTEP x
  const int gt = cg * 32 + lane;
  const int sch = gt % CPR, slr0 = gt / CPR;
  const size_t pass_stride = (size_t)RSTEP * p.ldk;

  auto kclamp = [&](const PanelIter& at) { return min(at.i * TKR + k_local, nk - 1); };
  auto kpmine = [&](const PanelIter& at, int qe) {
    return min(at.j * TKC + 2 * cg + (NBW == 2 ? beta : qe), nk - 1);
  };
  double uk[3], ukp[NQE][3];
  auto entries = [&](int* e) {
    if constexpr (NBW == 2) {
      int em = panel_entry_c(p, uk, ukp[0], integral);
      if (em < 0) {
        atomicOr(in.status, XATU_DEVERR_INDEX);
        em = 0;
      }
      e[0] = __shfl_sync(0xffffffffu, em, lane & ~1);
      e[1] = __shfl_sync(0xffffffffu, em, lane | 1);
    } else {
#pragma unroll
      for (int q = 0; q < 2; q++) {
        e[q] = panel_entry_c(p, uk, ukp[q], integral);
        if (e[q] < 0) {
          atomicOr(in.status, XATU_DEVERR_INDEX);
          e[q] = 0;
        }
      }
    }
  };
  float2 Vr[2][2 * VQ];
  auto load_v = [&](int q, int e) {
    const float4* src = V4 + (size_t)e * VQ;
#pragma unroll
    for (int x = 0; x < VQ; x++) {
      const float4 w = __ldg(src + x);
      Vr[q][2 * x] = make_float2(w.x, w.y);
      Vr[q][2 * x + 1] = make_float2(w.z, w.w);
    }
  };

  PanelIter it = panel_locate<S>(t0, g.npanel, g.ntile), itn = it;
  panel_next<S>(itn, g.ntile);
  {
    panel_coords(p, U, in.kgrid, kclamp(it), uk);
#pragma unroll
    for (int qe = 0; qe < NQE; qe++) panel_coords(p, U, in.kgrid, kpmine(it, qe), ukp[qe]);
    int e[2];
    entries(e);
    load_v(0, e[0]);
    load_v(1, e[1]);
  }
  for (int t = 0; t < nt; t++) {
    const int slot = NSLOT == 2 ? (t & 1) : 0;
    const bool has_next = t + 1 < nt;
    const int k = it.i * TKR + k_local;
    // coordinates of the next tile's k and k' points (used in the middle of this tile)
    if (has_next) {
      panel_coords(p, U, in.kgrid, kclamp(itn), uk);
#pragma unroll
      for (int qe = 0; qe < NQE; qe++) panel_coords(p, U, in.kgrid, kpmine(itn, qe), ukp[qe]);
    }
    if (!panel_wait(&done[t % XATU_PANEL_NDONE], (t / XATU_PANEL_NDONE) & 1, abort)) {
      if (lane == 0) {
        atomicOr(in.status, XATU_DEVERR_NOCONV);
        *abort = 1;
      }
      break;
    }
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (g.nstg == 1 && t > 0) asm volatile("bar.sync %0, 128;" ::"r"(1 + sp) : "memory");
    const int sb = g.nstg == 2 ? (t & 1) : 0;
    unsigned char* stg = stage0 + sb * g.stage_bytes;
    const uint32_t cbase = tl + (uint32_t)(slot * S::SLOT_STRIDE);
    const int kp0 = it.j * TKC + 2 * cg;
    int en[2] = {0, 0};
    // overlaps of both k' points of the warp, then the slot is free for the products of a later tile
    float r2q[2][NA][2 * NV], r1q[2][NA][2 * NC];
#pragma unroll
    for (int q = 0; q < 2; q++) {
      const int kq = 2 * cg + q;
#pragma unroll
      for (int b = 0; b < NA; b++) panel_tmem_ld<2 * NV>(cbase + NA * S::N1 + b * S::N2 + kq * 2 * NV, r2q[q][b]);
#pragma unroll
      for (int a = 0; a < NA; a++) panel_tmem_ld<2 * NC>(cbase + a * S::N1 + kq * 2 * NC, r1q[q][a]);
    }
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncwarp();
    if (lane == 0) asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(asm_smem_u32(&tfree[slot])) : "memory");
#pragma unroll
    for (int q = 0; q < 2; q++) {
      const int kq = 2 * cg + q;   // k' of the tile
      const int kp = kp0 + q;
      float (&r2)[NA][2 * NV] = r2q[q];
      float (&r1)[NA][2 * NC] = r1q[q];
      // T_a(v', beta) = sum_b (-V_ab) rho2_b(v', beta), V_ba = conj(V_ab)
      float2 T[NA][NV];
#pragma unroll
      for (int a = 0; a < NA; a++)
#pragma unroll
        for (int v2 = 0; v2 < NV; v2++) {
          float sx = 0.f, sy = 0.f;
#pragma unroll
          for (int b = 0; b < NA; b++) {
            const float2 vv = a <= b ? Vr[q][panel_vidx(a, b, NA)] : Vr[q][panel_vidx(b, a, NA)];
            const float vy = a <= b ? vv.y : -vv.y;
            const float rr = r2[b][2 * v2], ri = r2[b][2 * v2 + 1];
            sx = fmaf(vv.x, rr, fmaf(-vy, ri, sx));
            sy = fmaf(vv.x, ri, fmaf(vy, rr, sy));
          }
          T[a][v2] = make_float2(sx, sy);
        }
      // the rows of this lane's conduction band beta: v = own band (T), then the partner lane's band (its T, by a
      // shuffle once this lane's own row is done)
#pragma unroll
      for (int r = 0; r < NV; r++) {
        if constexpr (NBW == 2) {
#pragma unroll
          for (int a = 0; a < NA; a++)
#pragma unroll
            for (int v2 = 0; v2 < NV; v2++) {
              if (NV == 2 && r == 1) {
                T[a][v2].x = __shfl_xor_sync(0xffffffffu, T[a][v2].x, 1);
                T[a][v2].y = __shfl_xor_sync(0xffffffffu, T[a][v2].y, 1);
              } else if (NV == 1) {
                T[a][v2].x = __shfl_sync(0xffffffffu, T[a][v2].x, lane & ~1);
                T[a][v2].y = __shfl_sync(0xffffffffu, T[a][v2].y, lane & ~1);
              }
            }
        }
        if (NC < NBW && beta >= NC) continue;
        // -(D - X)(beta v, c' v') = sum_a rho1_a(beta, c') T_a(v', v) + sum_a L_a(i) R_a(j)
        float2 d[NC][NV];
#pragma unroll
        for (int c2 = 0; c2 < NC; c2++)
#pragma unroll
          for (int v2 = 0; v2 < NV; v2++) {
            float dx = 0.f, dy = 0.f;
#pragma unroll
            for (int a = 0; a < NA; a++) {
              const float rr = r1[a][2 * c2], ri = r1[a][2 * c2 + 1];
              const float2 tt = T[a][v2];
              dx = fmaf(rr, tt.x, fmaf(-ri, tt.y, dx));
              dy = fmaf(rr, tt.y, fmaf(ri, tt.x, dy));
            }
            d[c2][v2] = make_float2(dx, dy);
          }
        if (p.exchange) {
          const int v = vr[r];
          const int64_t ic = (int64_t)min(k, nk - 1) * NCV + beta * NV + v;
          const int64_t jc = (int64_t)min(kp, nk - 1) * NCV;
#pragma unroll
          for (int a = 0; a < NA; a++) {
            const cd l = in.exL[ic * NA + a];
            const float lx = (float)l.x, ly = (float)l.y;
#pragma unroll
            for (int c2 = 0; c2 < NC; c2++)
#pragma unroll
              for (int v2 = 0; v2 < NV; v2++) {
                const cd y = in.exR[(jc + c2 * NV + v2) * NA + a];
                const float yr = (float)y.x, yi = (float)y.y;
                d[c2][v2].x += lx * yr - ly * yi;
                d[c2][v2].y += lx * yi + ly * yr;
              }
          }
        }
        if (k == kp) {
          // diagonal element (c' v') = (beta v): real; the band energies go to the FP64 diagonal
          const int v = vr[r];
#pragma unroll
          for (int c2 = 0; c2 < NC; c2++)
#pragma unroll
            for (int v2 = 0; v2 < NV; v2++)
              if (c2 == beta && v2 == v) {
                d[c2][v2].y = 0.f;
                if (k < nk) {
                  const double ec = in.eigvalQ[(int64_t)k * p.nb + NV + beta];
                  const double ev = in.eigval[(int64_t)k * p.nb + v];
                  out.diag[(int64_t)k * NCV + beta * NV + v] = p.scissor + ec - ev;
                }
              }
        }
        uint32_t hw[NCV], lw[NCV];
#pragma unroll
        for (int c2 = 0; c2 < NC; c2++)
#pragma unroll
          for (int v2 = 0; v2 < NV; v2++) {
            const uint2 w = split_pack(d[c2][v2].x, d[c2][v2].y);
            hw[c2 * NV + v2] = w.x;
            lw[c2 * NV + v2] = w.y;
          }
        // staging: row (kw, beta, v) of the group, the NCV columns of k'
        unsigned char* s0 = stg + so[r][q];
        unsigned char* s1 = s0 + GROWS * PITCH;
        if constexpr (NCV == 4) {
          *reinterpret_cast<uint4*>(s0) = make_uint4(hw[0], hw[1], hw[2], hw[3]);
          *reinterpret_cast<uint4*>(s1) = make_uint4(lw[0], lw[1], lw[2], lw[3]);
        } else if constexpr (NCV == 2) {
          *reinterpret_cast<uint2*>(s0) = make_uint2(hw[0], hw[1]);
          *reinterpret_cast<uint2*>(s1) = make_uint2(lw[0], lw[1]);
        } else {
          *reinterpret_cast<uint32_t*>(s0) = hw[0];
          *reinterpret_cast<uint32_t*>(s1) = lw[0];
        }
      }
      // table rows of the next tile: located once this tile's first k' is done, loaded into the registers of the
      // k' just finished
      if (has_next) {
        if (q == 0) entries(en);
        load_v(q, en[q]);
      }
    }
    asm volatile("bar.sync %0, 128;" ::"r"(1 + sp) : "memory");
    // the group's rows: 16-byte chunks of whole row segments of the tile, both planes
    {
      const int row0 = it.i * TKR * NCV + sp * GROWS + slr0;
      const int col = it.j * TKC * NCV + 4 * sch;
      const int cblk = col / XATU_KBLOCK;
      const size_t base = (size_t)row0 * p.ldk + col;
      unsigned* dh = reinterpret_cast<unsigned*>(out.Khi) + base;
      unsigned* dl = reinterpret_cast<unsigned*>(out.Klo) + base;
      if (col < N) {
#pragma unroll
        for (int x = 0; x < NPASS; x++) {
          const int lr = slr0 + x * RSTEP;
          const int row = row0 + x * RSTEP;
          if (lr < GROWS && row < N && cblk >= row / XATU_KBLOCK) {
            const uint32_t o = (uint32_t)(lr * PITCH + (sch ^ ((lr >> 1) & (CPR - 1))) * 16);
            const uint4 wh = *reinterpret_cast<const uint4*>(stg + o);
            const uint4 wl = *reinterpret_cast<const uint4*>(stg + GROWS * PITCH + o);
            unsigned* ph = dh + x * pass_stride;
            unsigned* pl = dl + x * pass_stride;
            if (col + 4 <= N) {
              *reinterpret_cast<uint4*>(ph) = wh;
              *reinterpret_cast<uint4*>(pl) = wl;
            } else {
              ph[0] = wh.x;
              pl[0] = wl.x;
              if (col + 1 < N) {
                ph[1] = wh.y;
                pl[1] = wl.y;
              }
              if (col + 2 < N) {
                ph[2] = wh.z;
                pl[2] = wl.z;
              }
            }
          }
        }
      }
    }
    it = itn;
    panel_next<S>(itn, g.ntile);
  }
}

template <int NV, int NC, int NA>
__global__ void __launch_bounds__(XATU_PANEL_THREADS, 1)
bse_assemble_panel_kernel(AsmParams p, AsmInputs in, AsmOutputs out, AsmPanelGeom g) {
  using S = PanelShape<NV, NC, NA>;
  constexpr int NBS = XATU_PANEL_NBS;
  extern __shared__ __align__(1024) unsigned char smem[];
  __shared__ uint64_t s_full[NBS], s_done[XATU_PANEL_NDONE], s_afull, s_tfree[2];
  __shared__ uint64_t s_desc[XATU_PANEL_NISSUE][5 * ((2 * NA + XATU_PANEL_NISSUE - 1) / XATU_PANEL_NISSUE)];
  __shared__ uint32_t s_tmem;
  __shared__ int s_abort;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int t0 = (int)((long long)blockIdx.x * g.total / gridDim.x);
  const int nt = (int)((long long)(blockIdx.x + 1) * g.total / gridDim.x) - t0;

  if (warp == XATU_PANEL_NCW) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(asm_smem_u32(&s_tmem)),
                 "r"((uint32_t)S::TMEM_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    for (int st = 0; st < NBS; st++)
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(asm_smem_u32(&s_full[st])), "r"(1));
    for (int d = 0; d < XATU_PANEL_NDONE; d++)   // one commit from each product thread
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(asm_smem_u32(&s_done[d])), "r"(XATU_PANEL_NISSUE));
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(asm_smem_u32(&s_afull)), "r"(1));
    for (int s = 0; s < 2; s++)
      asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(asm_smem_u32(&s_tfree[s])), "r"(XATU_PANEL_NCW));
    s_abort = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = s_tmem;
  volatile int* abort = &s_abort;
  // launched chained to the operand formatting: the set-up above overlaps its tail; no global memory is read
  // before this point
  xatu_grid_chain();

  if (warp >= XATU_PANEL_NCW) {
    asm volatile("setmaxnreg.dec.sync.aligned.u32 %0;" ::"n"(XATU_PANEL_REGS_PRODUCER));
    if (warp == XATU_PANEL_NCW && lane == 0 && nt > 0)
      panel_copier<NV, NC, NA>(g, in.tc_ops, smem, s_full, s_done, &s_afull, t0, nt, in.status, abort);
    const int issuer = warp - XATU_PANEL_NCW - 1;
    if (issuer >= 0 && issuer < XATU_PANEL_NISSUE && lane == 0 && nt > 0)
      panel_mma<NV, NC, NA>(g, smem, s_full, s_done, &s_afull, s_tfree, s_desc[issuer], tmem, t0, nt, issuer,
                            in.status, abort);
  } else {
    asm volatile("setmaxnreg.inc.sync.aligned.u32 %0;" ::"n"(XATU_PANEL_REGS_CONSUMER));
    panel_consumer<NV, NC, NA>(p, in, out, g, smem, s_done, s_tfree, tmem, t0, nt, warp, lane, abort);
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == XATU_PANEL_NCW) {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"((uint32_t)S::TMEM_COLS));
  }
}

// Lower triangles of the diagonal XATU_KBLOCK blocks of the kernel planes := conjugate transpose of the upper
// ones (the split-BF16 words of a conjugate differ in the sign bits of their imaginary halves only).
// Grid: (diagonal blocks, 10 sub-tile pairs (si >= sj) of 32 x 32), block 32 x 8.
__global__ void asm_diag_mirror_kernel(unsigned* __restrict__ Kh, unsigned* __restrict__ Kl, long long N,
                                       long long ldk) {
  __shared__ unsigned th[32][33], tlo[32][33];
  xatu_grid_chain();
  int q = blockIdx.y, si = 0;
  while (q > si) {
    q -= si + 1;
    si++;
  }
  const int sj = q;
  const long long base = (long long)blockIdx.x * XATU_KBLOCK;
  const int tx = threadIdx.x, ty = threadIdx.y;
  for (int yy = ty; yy < 32; yy += 8) {
    const long long r = base + 32 * sj + yy, c = base + 32 * si + tx;
    if (r < N && c < N) {
      th[yy][tx] = Kh[r * ldk + c];
      tlo[yy][tx] = Kl[r * ldk + c];
    }
  }
  __syncthreads();
  for (int yy = ty; yy < 32; yy += 8) {
    const long long r = base + 32 * si + yy, c = base + 32 * sj + tx;
    if (r > c && r < N && c < N) {
      Kh[r * ldk + c] = th[tx][yy] ^ 0x80000000u;
      Kl[r * ldk + c] = tlo[tx][yy] ^ 0x80000000u;
    }
  }
}
